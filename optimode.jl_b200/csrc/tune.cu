// Autotuner for the FP32 operator passes (the analogue of the reference's FFTW PATIENT
// planning, lib/MaxwellEigenmodes/src/maxwell.jl:940-943): per (device, Nx, Ny) it times
// the row-tile × column-tile × wave-size variants and the one-kernel cluster apply of an M̂ application on
// device-resident data and keeps the fastest.  Choices live in a process-wide table keyed by
// the device name and grid, persisted as text lines
// "<device>|<Nx>|<Ny>|<row>|<col>|<seconds>|<wave>" in a cache file (OMB_TUNE_CACHE, else
// $XDG_CACHE_HOME/omb200/tiles.txt, else ~/.cache/omb200/tiles.txt).
#include <sys/stat.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <random>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "context.h"
#include "ops.h"

namespace omb {

constexpr int TUNE_UNITS = 64;  // units of the timed applications (above L2 for ≥ 128² grids)

namespace {
struct TuneEntry {
  int row = 1, col = 1;
  double seconds = 0;
  int wave = 0;
};
using TuneKey = std::tuple<std::string, int, int>;
std::mutex g_tune_mu;
std::map<TuneKey, TuneEntry> g_tune;
bool g_tune_loaded = false;
std::map<int, std::string> g_dev_names;  // device ordinal → name (guarded by g_tune_mu)

std::string default_cache_path() {
  if (const char* p = std::getenv("OMB_TUNE_CACHE")) return p;
  std::string base;
  if (const char* x = std::getenv("XDG_CACHE_HOME")) base = x;
  else if (const char* h = std::getenv("HOME")) base = std::string(h) + "/.cache";
  else return "";
  return base + "/omb200/tiles.txt";
}

bool parse_line(const std::string& line, TuneKey& k, TuneEntry& e) {
  std::vector<std::string> f;
  std::stringstream ss(line);
  std::string item;
  while (std::getline(ss, item, '|')) f.push_back(item);
  if ((f.size() != 6 && f.size() != 7) || f[0].empty()) return false;
  try {
    const int nx = std::stoi(f[1]), ny = std::stoi(f[2]), r = std::stoi(f[3]), c = std::stoi(f[4]);
    const double s = std::stod(f[5]);
    const int w = f.size() == 7 ? std::stoi(f[6]) : 0;
    if (nx <= 0 || ny <= 0 || r < 0 || r >= ROW_VARIANTS || c < 0 || c >= COL_VARIANTS || w < 0 ||
        w >= WAVE_VARIANTS || !(s >= 0))
      return false;
    k = TuneKey{f[0], nx, ny};
    e = TuneEntry{r, c, s, w};
    return true;
  } catch (...) {
    return false;
  }
}

int load_locked(const std::string& path) {
  std::ifstream in(path);
  if (!in) return 0;
  std::string line;
  int n = 0;
  while (std::getline(in, line)) {
    TuneKey k;
    TuneEntry e;
    if (parse_line(line, k, e)) { g_tune[k] = e; ++n; }
  }
  return n;
}

int save_locked(const std::string& path) {
  if (path.empty()) return fail(OMB_ERR_INVALID_ARG, "no tuning cache path");
  // create the parent directories
  for (size_t i = 1; i < path.size(); ++i)
    if (path[i] == '/') mkdir(path.substr(0, i).c_str(), 0755);
  const std::string tmp = path + ".tmp";
  {
    std::ofstream out(tmp, std::ios::trunc);
    if (!out) return fail(OMB_ERR_INVALID_ARG, "cannot write the tuning cache " + tmp);
    for (const auto& kv : g_tune)
      out << std::get<0>(kv.first) << '|' << std::get<1>(kv.first) << '|' << std::get<2>(kv.first) << '|'
          << kv.second.row << '|' << kv.second.col << '|' << kv.second.seconds << '|' << kv.second.wave << '\n';
  }
  if (std::rename(tmp.c_str(), path.c_str()) != 0) return fail(OMB_ERR_INVALID_ARG, "cannot replace " + path);
  return OMB_OK;
}

void ensure_loaded_locked() {
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  const std::string p = default_cache_path();
  if (!p.empty()) load_locked(p);
}

std::string device_name(int dev) {
  cudaDeviceProp pr{};
  if (cudaGetDeviceProperties(&pr, dev) != cudaSuccess) return "unknown";
  std::string s = pr.name;
  for (char& c : s)
    if (c == '|' || c == '\n') c = '_';
  return s;
}
}  // namespace

static std::string current_device_name_locked() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return "unknown";
  auto it = g_dev_names.find(dev);
  if (it != g_dev_names.end()) return it->second;
  return g_dev_names[dev] = device_name(dev);
}

TileChoice tiles_for(int Nx, int Ny) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  ensure_loaded_locked();
  auto it = g_tune.find(TuneKey{current_device_name_locked(), Nx, Ny});
  TileChoice t;
  if (it != g_tune.end()) { t.row = it->second.row; t.col = it->second.col; t.wave = it->second.wave; }
  return t;
}

bool tune_known(int dev, int Nx, int Ny) {
  const std::string name = device_name(dev);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  ensure_loaded_locked();
  return g_tune.count(TuneKey{name, Nx, Ny}) > 0;
}

// Times the tile × wave variants (168 slots; each cluster apply once) of one FP32 M̂ application to `ncol` columns on `units`
// copies of a uniform cell and records the fastest.
int autotune_grid(omb_ctx* ctx, const omb_grid* g, int ncol, int units, TileChoice* best, double* times) {
  int rc = check_grid(g);
  if (rc) return rc;
  if (ncol < 1 || ncol > 64 || units < 1 || units > 64) return fail(OMB_ERR_INVALID_ARG, "autotune: ncol/units");
  cudaStream_t st = ctx->stream;
  const size_t N = (size_t)g->Nx * g->Ny;
  std::vector<double> ei(9 * N, 0.0);
  for (size_t p = 0; p < N; ++p) ei[9 * p] = ei[9 * p + 4] = ei[9 * p + 8] = 0.4 + 0.2 * ((p * 7919) % 11) / 11.0;
  Problem P;
  rc = upload_problem(ctx, g, ei.data(), P);
  if (rc) return rc;
  DevBuf<float2> hin, hout, scr;
  const size_t ncolt = (size_t)ncol * units;
  OMB_CU(hin.alloc(2 * N * ncolt, st));
  OMB_CU(hout.alloc(2 * N * ncolt, st));
  OMB_CU(scr.alloc(3 * N * ncolt, st));
  OMB_CU(cudaMemsetAsync(hin.p, 0, 2 * N * ncolt * sizeof(float2), st));
  DevBuf<double> kd;
  OMB_CU(kd.alloc(1, st));
  const double k = 1.0;
  OMB_CU(cudaMemcpyAsync(kd.p, &k, sizeof(double), cudaMemcpyHostToDevice, st));
  std::vector<OpUnit<float>> hu(units);
  for (int i = 0; i < units; ++i) {
    OpUnit<float> u = make_unit<float>(P);
    u.in = hin.p + 2 * N * ncol * i; u.out = hout.p + 2 * N * ncol * i; u.scr = scr.p + 3 * N * ncol * i;
    u.k_dev = kd.p;
    u.in_cs = u.out_cs = (long long)(2 * N); u.scr_cs = (long long)(3 * N); u.ncol = ncol;
    hu[i] = u;
  }
  DevBuf<OpUnit<float>> du;
  OMB_CU(du.alloc(units, st));
  OMB_CU(cudaMemcpyAsync(du.p, hu.data(), units * sizeof(OpUnit<float>), cudaMemcpyHostToDevice, st));
  cudaEvent_t e0, e1;
  OMB_CU(cudaEventCreate(&e0));
  OMB_CU(cudaEventCreate(&e1));
  const std::string name = device_name(ctx->device);
  double best_s = 1e30;
  TileChoice bt;
  int vi = 0;
  rc = OMB_OK;
  for (int r = 0; r < ROW_VARIANTS && !rc; ++r)
    for (int c = 0; c < COL_VARIANTS && !rc; ++c)
      for (int wv = 0; wv < WAVE_VARIANTS && !rc; ++wv, ++vi) {
      if ((r == ROW_CLUSTER || r == ROW_CLUSTER16) && (c != 1 || wv != 0 || !cluster_apply_available(g->Nx, g->Ny))) {
        if (times) times[vi] = -1.0;  // one kernel whatever the column and wave choices: timed once
        continue;
      }
      {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        ensure_loaded_locked();
        g_tune[TuneKey{name, g->Nx, g->Ny}] = TuneEntry{r, c, 0.0, wv};
      }
      cudaError_t e = cudaSuccess;
      for (int w = 0; w < 2 && e == cudaSuccess; ++w) e = launch_op<float>(OP_M, du.p, units, g->Nx, g->Ny, ncol, ctx->tw, st);
      if (e == cudaSuccess) e = cudaEventRecord(e0, st);
      const int reps = 5;
      for (int w = 0; w < reps && e == cudaSuccess; ++w) e = launch_op<float>(OP_M, du.p, units, g->Nx, g->Ny, ncol, ctx->tw, st);
      if (e == cudaSuccess) e = cudaEventRecord(e1, st);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float ms = 0;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e != cudaSuccess) { rc = cuda_fail(e, "autotune"); break; }
      const double s = ms * 1e-3 / reps;
      if (times) times[vi] = s;
      if (s < best_s) { best_s = s; bt.row = r; bt.col = c; bt.wave = wv; }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (rc) g_tune.erase(TuneKey{name, g->Nx, g->Ny});
    else {
      g_tune[TuneKey{name, g->Nx, g->Ny}] = TuneEntry{bt.row, bt.col, best_s, bt.wave};
      const std::string p = default_cache_path();
      if (!p.empty()) save_locked(p);  // best effort: a read-only home only loses persistence
    }
  }
  if (rc) return rc;
  if (best) *best = bt;
  return OMB_OK;
}

}  // namespace omb

using namespace omb;

extern "C" {

int omb_autotune(omb_ctx* ctx, const omb_grid* grid, int32_t ncol, int32_t* row_variant, int32_t* col_variant,
                 int32_t* wave_variant, double* seconds) {
  if (!ctx || !grid) return fail(OMB_ERR_INVALID_ARG, "NULL argument");
  OMB_CU(cudaSetDevice(ctx->device));
  TileChoice t;
  const int rc = autotune_grid(ctx, grid, ncol, TUNE_UNITS, &t, seconds);
  if (rc) return rc;
  if (row_variant) *row_variant = t.row;
  if (col_variant) *col_variant = t.col;
  if (wave_variant) *wave_variant = t.wave;
  return OMB_OK;
}

int omb_ctx_set_autotune(omb_ctx* ctx, int32_t enabled) {
  if (!ctx) return fail(OMB_ERR_INVALID_ARG, "ctx is NULL");
  ctx->autotune = enabled ? 1 : 0;
  return OMB_OK;
}

int omb_tune_set(const char* device_name, int32_t Nx, int32_t Ny, int32_t row_variant, int32_t col_variant,
                 int32_t wave_variant) {
  if (!device_name || !*device_name || Nx <= 0 || Ny <= 0 || row_variant < 0 || row_variant >= ROW_VARIANTS ||
      col_variant < 0 || col_variant >= COL_VARIANTS || wave_variant < 0 || wave_variant >= WAVE_VARIANTS)
    return fail(OMB_ERR_INVALID_ARG, "omb_tune_set: bad key or variant (rows 0..6, columns 0..5, wave 0..3)");
  std::string n = device_name;
  for (char& c : n)
    if (c == '|' || c == '\n') c = '_';
  std::lock_guard<std::mutex> lk(g_tune_mu);
  ensure_loaded_locked();
  g_tune[TuneKey{n, Nx, Ny}] = TuneEntry{row_variant, col_variant, 0.0, wave_variant};
  return OMB_OK;
}

int omb_tune_get(const char* device_name, int32_t Nx, int32_t Ny, int32_t* row_variant, int32_t* col_variant,
                 int32_t* wave_variant) {
  if (!device_name) return fail(OMB_ERR_INVALID_ARG, "device_name is NULL");
  std::lock_guard<std::mutex> lk(g_tune_mu);
  ensure_loaded_locked();
  auto it = g_tune.find(TuneKey{device_name, Nx, Ny});
  if (it == g_tune.end()) return fail(OMB_ERR_INVALID_ARG, "no tuned tiles for this device and grid");
  if (row_variant) *row_variant = it->second.row;
  if (col_variant) *col_variant = it->second.col;
  if (wave_variant) *wave_variant = it->second.wave;
  return OMB_OK;
}

int omb_tune_clear(void) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune.clear();
  g_tune_loaded = true;  // a cleared table does not reload the cache file by itself
  return OMB_OK;
}

int omb_tune_save(const char* path) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  return save_locked(path ? std::string(path) : default_cache_path());
}

int omb_tune_load(const char* path, int32_t* entries) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_loaded = true;
  const int n = load_locked(path ? std::string(path) : default_cache_path());
  if (entries) *entries = n;
  return OMB_OK;
}

}  // extern "C"

// Stand-alone run of the LOBPCG Gram kernel on caller blocks (omb_gram_blocks): the
// streaming G = ZᴴZ, S = ZᴴAZ products of one track, in FP32 (compensated) or FP64, so their
// accuracy can be checked against an exact product of the same blocks.
#include <algorithm>
#include <vector>

#include "context.h"
#include "lobpcg.cuh"
#include "vec.cuh"

using namespace omb;

namespace {

template <typename T>
int gram_blocks(omb_ctx* ctx, long long n2, int n, const double* Z, const double* AZ, double* G, double* S) {
  cudaStream_t st = ctx->stream;
  const size_t tot = (size_t)n2 * n;
  DevBuf<double2> z64, az64;
  OMB_CU(z64.alloc(tot, st));
  OMB_CU(az64.alloc(tot, st));
  OMB_CU(cudaMemcpyAsync(z64.p, Z, tot * sizeof(double2), cudaMemcpyHostToDevice, st));
  OMB_CU(cudaMemcpyAsync(az64.p, AZ, tot * sizeof(double2), cudaMemcpyHostToDevice, st));
  DevBuf<cplx<T>> z, az;
  if constexpr (std::is_same<T, double>::value) {
    z = std::move(z64);
    az = std::move(az64);
  } else {
    OMB_CU(z.alloc(tot, st));
    OMB_CU(az.alloc(tot, st));
    const int nb = (int)std::min<size_t>((tot + 255) / 256, 65535 * 8);
    k_c64_to_c32<<<nb, 256, 0, st>>>(z64.p, z.p, tot);
    k_c64_to_c32<<<nb, 256, 0, st>>>(az64.p, az.p, tot);
    OMB_CU(cudaGetLastError());
  }
  TrackState hs{};
  hs.M = n; hs.need = n; hs.status = TS_RUNNING;
  DevBuf<TrackState> ds;
  OMB_CU(ds.alloc(1, st));
  OMB_CU(cudaMemcpyAsync(ds.p, &hs, sizeof(hs), cudaMemcpyHostToDevice, st));
  DevBuf<double2> acc;
  OMB_CU(acc.alloc(2 * (size_t)NMAX * NMAX, st));
  OMB_CU(acc.zero());
  TrackDesc<T> d{};
  d.Y[0] = d.Y[1] = z.p;
  d.AY[0] = d.AY[1] = az.p;
  d.st = ds.p;
  d.gram_acc = acc.p;
  d.n2 = n2;
  d.M = n;
  DevBuf<TrackDesc<T>> dd;
  OMB_CU(dd.alloc(1, st));
  OMB_CU(cudaMemcpyAsync(dd.p, &d, sizeof(d), cudaMemcpyHostToDevice, st));
  const int nmax = n;
  const int rg = GramCfg<T>::rows(nmax);
  const int tiles = (int)((n2 + rg - 1) / rg);
  const int hpre[2] = {0, tiles};
  DevBuf<int> pre, err;
  OMB_CU(pre.alloc(2, st));
  OMB_CU(cudaMemcpyAsync(pre.p, hpre, sizeof(hpre), cudaMemcpyHostToDevice, st));
  OMB_CU(err.alloc(1, st));
  OMB_CU(err.zero());
  const size_t gstage = GramCfg<T>::stage_elems(nmax, rg) * sizeof(cplx<T>);
  const size_t gred = GramCfg<T>::red_entries(nmax) * sizeof(double2);
  const int gstages = (int)std::max<size_t>(2, std::min<size_t>(8, (200 * 1024 - 128 - gred) / gstage));
  const size_t sm = 128 + gstages * gstage + gred;
  OMB_CU(ensure_smem(reinterpret_cast<const void*>(k_gram<T>), sm));
  const int grid = std::min(tiles, ctx->num_sms);
  k_gram<T><<<grid, GramCfg<T>::NT, sm, st>>>(dd.p, pre.p, nullptr, 1, 0, nmax, rg, gstages, err.p, ctx->wait_ns);
  OMB_CU(cudaGetLastError());
  std::vector<double2> h(2 * (size_t)NMAX * NMAX);
  int herr = 0;
  OMB_CU(cudaMemcpyAsync(h.data(), acc.p, h.size() * sizeof(double2), cudaMemcpyDeviceToHost, st));
  OMB_CU(cudaMemcpyAsync(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  OMB_CU(cudaStreamSynchronize(st));
  if (herr) return fail(OMB_ERR_TIMEOUT, "Gram pipeline wait ran out (code " + std::to_string(herr) + ")");
  for (int w = 0; w < 2; ++w) {
    double* out = w ? S : G;
    for (int a = 0; a < n; ++a)
      for (int b = 0; b < n; ++b) {
        const double2 v = a <= b ? h[(size_t)w * NMAX * NMAX + (size_t)a * NMAX + b]
                                 : h[(size_t)w * NMAX * NMAX + (size_t)b * NMAX + a];
        // column-major n×n complex; the lower triangle is the conjugate of the upper
        out[2 * (a + (size_t)n * b)] = v.x;
        out[2 * (a + (size_t)n * b) + 1] = a <= b ? v.y : -v.y;
      }
  }
  return OMB_OK;
}

}  // namespace

extern "C" int omb_gram_blocks(omb_ctx* ctx, int precision, int64_t n2, int32_t n, const double* Z, const double* AZ,
                               double* G, double* S) {
  if (!ctx || !Z || !AZ || !G || !S) return fail(OMB_ERR_INVALID_ARG, "NULL argument");
  if (n < 1 || n > NMAX || n2 < 2 || n2 % 2)
    return fail(OMB_ERR_INVALID_ARG, "need 1 <= n <= 36 columns and an even number n2 >= 2 of rows");
  if (precision != OMB_PREC_FP32 && precision != OMB_PREC_FP64) return fail(OMB_ERR_INVALID_ARG, "precision");
  OMB_CU(cudaSetDevice(ctx->device));
  return precision == OMB_PREC_FP32 ? gram_blocks<float>(ctx, n2, n, Z, AZ, G, S)
                                    : gram_blocks<double>(ctx, n2, n, Z, AZ, G, S);
}

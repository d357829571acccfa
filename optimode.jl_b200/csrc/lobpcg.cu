// Rayleigh–Ritz, control and Newton kernels of the device LOBPCG (FP64, precision-agnostic).
#include "lobpcg.cuh"

namespace omb {

__global__ void k_live_prefix(TrackState* const* __restrict__ states, const long long* __restrict__ n2,
                              int ntracks, int rg, int ru, int* __restrict__ pre_g, int* __restrict__ pre_u,
                              long long* __restrict__ wpre_g, long long* __restrict__ wpre_u) {
  // one CTA of 1024 threads: inclusive scans of the live tracks' tile counts and tile costs
  __shared__ int sg[1024], su[1024];
  __shared__ long long wg[1024], wu[1024];
  __shared__ int carry[2];
  __shared__ long long wcarry[2];
  const int tid = threadIdx.x;
  if (tid == 0) {
    carry[0] = carry[1] = 0; pre_g[0] = 0; pre_u[0] = 0;
    wcarry[0] = wcarry[1] = 0; wpre_g[0] = 0; wpre_u[0] = 0;
  }
  __syncthreads();
  for (int base = 0; base < ntracks; base += 1024) {
    const int t = base + tid;
    int vg = 0, vu = 0;
    long long xg = 0, xu = 0;
    if (t < ntracks && !states[t]->done) {
      const TrackState& s = *states[t];
      const int n = s.M + s.nWa + s.nP;
      vg = (int)((n2[t] + rg - 1) / rg);
      vu = (int)((n2[t] + ru - 1) / ru);
      xg = vg * gram_tile_cost(n) + GRAM_TRACK_COST;
      xu = vu * update_tile_cost(n, s.M);
    }
    sg[tid] = vg; su[tid] = vu; wg[tid] = xg; wu[tid] = xu;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
      const int ag = tid >= off ? sg[tid - off] : 0, au = tid >= off ? su[tid - off] : 0;
      const long long bg = tid >= off ? wg[tid - off] : 0, bu = tid >= off ? wu[tid - off] : 0;
      __syncthreads();
      sg[tid] += ag; su[tid] += au; wg[tid] += bg; wu[tid] += bu;
      __syncthreads();
    }
    if (t < ntracks) {
      pre_g[t + 1] = carry[0] + sg[tid]; pre_u[t + 1] = carry[1] + su[tid];
      wpre_g[t + 1] = wcarry[0] + wg[tid]; wpre_u[t + 1] = wcarry[1] + wu[tid];
    }
    __syncthreads();
    if (tid == 1023) { carry[0] += sg[1023]; carry[1] += su[1023]; wcarry[0] += wg[1023]; wcarry[1] += wu[1023]; }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(RR_NT) k_rr(TrackState* const* __restrict__ states,
                                               double2* const* __restrict__ gram_accs,
                                               double2* const* __restrict__ coefs,
                                               float2* const* __restrict__ coefs32, int ntracks,
                                               IterParams prm) {
  const int t = blockIdx.x;
  if (t >= ntracks) return;
  TrackState& s = *states[t];
  if (s.done) return;
  const int M = s.M;
  const int n = M + s.nWa + s.nP;
  const double jtol2 = prm.jacobi_tol2;
  constexpr int ld = NMAX;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* G = reinterpret_cast<double2*>(smem_raw);
  double2* S = G + NMAX * NMAX;
  double2* V = S + NMAX * NMAX;
  double2* B = V + NMAX * NMAX;
  __shared__ RotIdx ri[NMAX];
  __shared__ double red[64];
  __shared__ int order[NMAX];
  __shared__ double dsc[NMAX];
  __shared__ double theta[NMAX];
  __shared__ int keep[NMAX];
  __shared__ int rank;
  const int tid = threadIdx.x, nt = blockDim.x;
  double2* acc = gram_accs[t];
  // 1. the summed Gram matrices (upper triangles), mirrored; then clear the accumulators
  for (int e = tid; e < 2 * n * n; e += nt) {
    const int which = e / (n * n), ab = e % (n * n), a = ab / n, b = ab % n;
    if (a > b) continue;
    double2 g = acc[which * NMAX * NMAX + a * NMAX + b];
    double2* Mx = which ? S : G;
    if (a == b) g.y = 0;
    Mx[a * ld + b] = g;
    Mx[b * ld + a] = make_double2(g.x, -g.y);
  }
  __syncthreads();
  for (int e = tid; e < 2 * n * n; e += nt) {
    const int which = e / (n * n), ab = e % (n * n), a = ab / n, b = ab % n;
    if (a <= b) acc[which * NMAX * NMAX + a * NMAX + b] = make_double2(0, 0);
  }
  // 2. unit-diagonal scaling
  for (int a = tid; a < n; a += nt) {
    const double g = G[a * ld + a].x;
    dsc[a] = (g > 0 && isfinite(g)) ? 1.0 / sqrt(g) : 0.0;
  }
  __syncthreads();
  for (int e = tid; e < n * n; e += nt) {
    const int a = e / n, b = e % n;
    const double f = dsc[a] * dsc[b];
    G[a * ld + b].x *= f; G[a * ld + b].y *= f;
    S[a * ld + b].x *= f; S[a * ld + b].y *= f;
    B[a * ld + b] = G[a * ld + b];  // the SVQB path needs it after the Cholesky attempt
  }
  __syncthreads();
  // 3. Basis of the Gram metric.  Fast path: Cholesky Gs = L Lᴴ, then the projected
  //    problem L⁻¹ Ss L⁻ᴴ u = λu and C = D L⁻ᴴ u.  When a pivot falls below the floor
  //    (near-dependent directions) the SVQB path below drops them instead.
  __shared__ int chol_ok;
  if (tid == 0) chol_ok = 1;
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    const double piv = G[j * ld + j].x;
    if (!(piv > prm.gram_drop)) { chol_ok = 0; break; }  // uniform across the block
    const double ljj = sqrt(piv);
    for (int i = j + 1 + tid; i < n; i += nt) {
      const double2 g = G[i * ld + j];
      G[i * ld + j] = make_double2(g.x / ljj, g.y / ljj);
    }
    __syncthreads();
    if (tid == 0) G[j * ld + j] = make_double2(ljj, 0.0);
    const int w = n - j - 1;
    for (int e = tid; e < w * w; e += nt) {
      const int i = j + 1 + e / w, k = j + 1 + e % w;
      if (k <= i) {
        const double2 li = G[i * ld + j], lk = G[k * ld + j];
        G[i * ld + k].x -= li.x * lk.x + li.y * lk.y;  // L_ij·conj(L_kj)
        G[i * ld + k].y -= li.y * lk.x - li.x * lk.y;
      }
    }
    __syncthreads();
  }
  __syncthreads();
  int r;
  double2* Ev;  // eigenvectors of the projected problem (columns), n_eff × n_eff
  double2* Av;  // the projected matrix, eigenvalues on its diagonal after Jacobi
  if (chol_ok) {
    r = n;
    // V ← L⁻¹ Ss (column-parallel forward substitution)
    for (int c = tid; c < n; c += nt) {
      for (int i = 0; i < n; ++i) {
        double2 t = S[i * ld + c];
        for (int k = 0; k < i; ++k) {
          const double2 l = G[i * ld + k], v = V[k * ld + c];
          t.x -= l.x * v.x - l.y * v.y;
          t.y -= l.x * v.y + l.y * v.x;
        }
        const double d = G[i * ld + i].x;
        V[i * ld + c] = make_double2(t.x / d, t.y / d);
      }
    }
    __syncthreads();
    // B ← L⁻¹ Vᴴ = L⁻¹ Ss L⁻ᴴ
    for (int c = tid; c < n; c += nt) {
      for (int i = 0; i < n; ++i) {
        const double2 vc = V[c * ld + i];
        double2 t = make_double2(vc.x, -vc.y);
        for (int k = 0; k < i; ++k) {
          const double2 l = G[i * ld + k], v = B[k * ld + c];
          t.x -= l.x * v.x - l.y * v.y;
          t.y -= l.x * v.y + l.y * v.x;
        }
        const double d = G[i * ld + i].x;
        B[i * ld + c] = make_double2(t.x / d, t.y / d);
      }
    }
    __syncthreads();
    for (int e = tid; e < n * n; e += nt) {  // Hermitian part
      const int i = e / n, j = e % n;
      if (i < j) {
        const double2 x = B[i * ld + j], y = B[j * ld + i];
        const double2 h = make_double2(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
        B[i * ld + j] = h;
        B[j * ld + i] = make_double2(h.x, -h.y);
      } else if (i == j) {
        B[i * ld + i].y = 0;
      }
    }
    __syncthreads();
    jacobi_eigh(B, V, r, ld, S, ri, red, jtol2);  // S is free once B = L⁻¹ S L⁻ᴴ
    Ev = V;
    Av = B;
  } else {
    // SVQB: restore the scaled Gram matrix (the Cholesky attempt overwrote it)
    for (int e = tid; e < n * n; e += nt) {
      const int a = e / n, b = e % n;
      G[a * ld + b] = B[a * ld + b];
    }
    __syncthreads();
    jacobi_eigh(G, V, n, ld, B, ri, red, jtol2);  // B's copy of G is back in G
    if (tid == 0) {
      double tmax = 0;
      for (int i = 0; i < n; ++i) { theta[i] = G[i * ld + i].x; tmax = fmax(tmax, theta[i]); }
      int rr = 0;
      for (int i = 0; i < n; ++i)
        if (theta[i] > prm.gram_drop * tmax) keep[rr++] = i;
      rank = rr;
    }
    __syncthreads();
    r = rank;
    if (r < M) {
      if (tid == 0) {
        s.status = TS_ORTHO; s.done = 1; s.op_ncol = 0; s.pw_ncol = 0; s.hmkh_ncol = 0;
        s.rr_n = n; s.rr_rank = r;
      }
      return;
    }
    // B = V_keep Θ^{-1/2}   (n × r)
    for (int e = tid; e < n * r; e += nt) {
      const int l = e / r, j = e % r;
      const double f = 1.0 / sqrt(theta[keep[j]]);
      const double2 v = V[l * ld + keep[j]];
      B[l * ld + j] = make_double2(v.x * f, v.y * f);
    }
    __syncthreads();
    // V ← S B (n × r), then G ← Bᴴ V (r × r)
    for (int e = tid; e < n * r; e += nt) {
      const int l = e / r, j = e % r;
      double2 acc = make_double2(0, 0);
      for (int m = 0; m < n; ++m) {
        const double2 a = S[l * ld + m], b = B[m * ld + j];
        acc.x += a.x * b.x - a.y * b.y;
        acc.y += a.x * b.y + a.y * b.x;
      }
      V[l * ld + j] = acc;
    }
    __syncthreads();
    for (int e = tid; e < r * r; e += nt) {
      const int i = e / r, j = e % r;
      double2 acc = make_double2(0, 0);
      for (int l = 0; l < n; ++l) {
        const double2 a = B[l * ld + i], b = V[l * ld + j];
        acc.x += a.x * b.x + a.y * b.y;  // conj(a)·b
        acc.y += a.x * b.y - a.y * b.x;
      }
      G[i * ld + j] = acc;
    }
    __syncthreads();
    jacobi_eigh(G, V, r, ld, S, ri, red, jtol2);  // S is folded into G = Bᴴ S B
    Ev = V;
    Av = G;
  }
  sort_diag(Av, r, ld, order);
  // 5. coefficients of the new X in the Z columns, Ritz values
  double2* coef = coefs[t];
  float2* coef32 = coefs32[t];
  if (chol_ok) {
    // C = D L⁻ᴴ U[:, order[:M]] (column-parallel back substitution; S is free scratch)
    for (int m = tid; m < M; m += nt) {
      const int um = order[m];
      for (int i = n - 1; i >= 0; --i) {
        double2 y = Ev[i * ld + um];
        for (int k = i + 1; k < n; ++k) {
          const double2 l = G[k * ld + i], v = S[k * ld + m];  // conj(L_ki)·y_k
          y.x -= l.x * v.x + l.y * v.y;
          y.y -= l.x * v.y - l.y * v.x;
        }
        const double d = G[i * ld + i].x;
        S[i * ld + m] = make_double2(y.x / d, y.y / d);
      }
      for (int i = 0; i < n; ++i) {
        const double2 y = S[i * ld + m];
        coef[i * MMAX + m] = make_double2(y.x * dsc[i], y.y * dsc[i]);
        coef32[i * MMAX + m] = make_float2((float)(y.x * dsc[i]), (float)(y.y * dsc[i]));
      }
    }
  } else {
    for (int e = tid; e < n * M; e += nt) {
      const int l = e / M, m = e % M;
      const int um = order[m];
      double2 acc = make_double2(0, 0);
      for (int j = 0; j < r; ++j) {
        const double2 a = B[l * ld + j], b = Ev[j * ld + um];
        acc.x += a.x * b.x - a.y * b.y;
        acc.y += a.x * b.y + a.y * b.x;
      }
      coef[l * MMAX + m] = make_double2(acc.x * dsc[l], acc.y * dsc[l]);
      coef32[l * MMAX + m] = make_float2((float)(acc.x * dsc[l]), (float)(acc.y * dsc[l]));
    }
  }
  for (int m = tid; m < M; m += nt) s.lam[m] = Av[order[m] * ld + order[m]].x;
  __syncthreads();
  // 6. P coefficients for the active columns: the W and P parts of the Ritz vectors
  const int nPn = (s.nWa + s.nP > 0) ? (M - s.nlocked) : 0;
  for (int e = tid; e < n * nPn; e += nt) {
    const int l = e / nPn, mp = e % nPn;
    const double2 c = (l < M) ? make_double2(0, 0) : coef[l * MMAX + (s.nlocked + mp)];
    coef[NMAX * MMAX + l * MMAX + mp] = c;
    coef32[NMAX * MMAX + l * MMAX + mp] = make_float2((float)c.x, (float)c.y);
  }
  if (tid == 0) { s.nP_next = nPn; s.rr_n = n; s.rr_rank = r; }
}

__device__ __forceinline__ void finish(TrackState& s, int status) {
  s.status = status;
  s.done = 1;
  s.op_ncol = 0; s.pw_ncol = 0; s.hmkh_ncol = 0;
}

__global__ void k_control(TrackState* const* __restrict__ states, double* const* __restrict__ res_accs,
                          int ntracks, IterParams prm) {
  const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= ntracks) return;
  TrackState& s = *states[t];
  if (s.done) return;
  if (lane != 0) return;
  const int M = s.M;
  // ‖R‖² summed by k_update; cleared for the next iteration
  double* ra = res_accs[t];
  double rs[MMAX];
  for (int m = 0; m < M; ++m) { rs[m] = ra[m]; ra[m] = 0.0; }
  bool bad = false;
  for (int m = 0; m < M; ++m) {
    s.resid[m] = sqrt(rs[m]);
    if (!isfinite(s.resid[m]) || !isfinite(s.lam[m])) bad = true;
  }
  s.nP = s.nP_next;
  s.iter++; s.iter_phase++; s.since_newton++;
  if (bad || !isfinite(s.k)) { finish(s, TS_NAN); return; }
  const int need = s.need;
  double maxres = 0;
  for (int i = 0; i < need; ++i) maxres = fmax(maxres, s.resid[i]);
  if (maxres < 0.9 * s.resid_best) { s.resid_best = maxres; s.stall = 0; } else { s.stall++; }
  while (s.nlocked < need && s.resid[s.nlocked] < prm.lock_tol) s.nlocked++;
  const bool last = prm.last_phase != 0;
  s.hmkh_ncol = 0;
  if (s.mode == MODE_OMEGA2) {
    if (maxres < prm.tau_phase) { finish(s, last ? TS_CONVERGED : TS_PHASE_DONE); return; }
    if (!last && s.stall >= 8) { finish(s, TS_PHASE_DONE); return; }
  } else if (s.mode == MODE_NEWTON_INNER) {
    const double dw2 = s.lam[s.band] - s.omega2;
    if (last) {
      // final steps from converged eigenpairs; earlier ones while the k mismatch dominates
      // the eigen-residual, plus at most one early step per phase near the tolerance.  The
      // track returns band `band` only, and that Ritz pair's own residual bounds its error,
      // so the polish watches it alone; the lower bands (resolved to the FP32 floor before
      // the hand-over, which keeps the Ritz ordering) keep iterating beside it.
      const double rb = s.resid[s.band];
      if (rb < prm.tol) s.hmkh_ncol = 1;
      else if (s.since_newton >= 2 && rb < 0.1 * fabs(dw2)) s.hmkh_ncol = 1;
      else if (s.since_newton >= 2 && s.newton_phase == 0 && rb < 100 * prm.tol) s.hmkh_ncol = 1;
    } else {
      if (s.newton_steps > 0 && maxres < prm.tau_phase && fabs(s.dk_last) < prm.dk_phase) {
        finish(s, TS_PHASE_DONE); return;
      }
      // stalled at the FP32 floor: the FP64 phase takes over, with or without a Newton step
      // here (a warm start can give a k so close that λ_b − ω² never dominates the
      // residual); plateaus far above the floor keep iterating in FP32
      const bool at_floor = maxres < 4.0 * prm.tau_phase;
      if (at_floor && s.stall >= 8) { finish(s, TS_PHASE_DONE); return; }
      if (s.newton_steps > 0 && s.stall >= 8) { finish(s, TS_PHASE_DONE); return; }
      if (s.since_newton >= 2 && (maxres < fmax(0.1 * fabs(dw2), prm.tau_phase) || (at_floor && s.stall >= 4)))
        s.hmkh_ncol = 1;
    }
  } else {  // MODE_NEWTON_OUTER: the reference loop, a step after each converged eigensolve
    if (maxres < prm.tol) s.hmkh_ncol = 1;
  }
  if (s.iter_phase >= prm.maxiter && s.hmkh_ncol == 0) { finish(s, last ? TS_MAXITER : TS_PHASE_DONE); return; }
  s.nWa = M - s.nlocked;
  s.op_col0 = M + s.nlocked;
  s.op_ncol = s.nWa;
  s.pw_col0 = s.nlocked;
  s.pw_ncol = s.nWa;
}

__global__ void k_newton(TrackState* const* __restrict__ states, double* const* __restrict__ hmkh_parts,
                         const int* __restrict__ hmkh_nb, int ntracks, IterParams prm) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntracks) return;
  TrackState& s = *states[t];
  if (s.done || s.hmkh_ncol == 0) return;
  const double* hp = hmkh_parts[t];
  double re = 0;
  for (int b = 0; b < hmkh_nb[t]; ++b) re += hp[2 * b];
  const double h = -re;
  const double dw2dk = 2.0 * h;
  const int j = s.band;
  const double dk = (s.lam[j] - s.omega2) / dw2dk;
  s.hmkh_ncol = 0;
  if (!(dw2dk > 0) || !isfinite(dk)) { finish(s, TS_NAN); return; }
  s.k_eig = s.k;
  s.hmkh = h;
  s.k -= dk;
  s.dk_last = dk;
  s.newton_steps++;
  s.newton_phase++;
  s.since_newton = 0;
  if (s.mode == MODE_NEWTON_OUTER) s.iter_phase = 0;  // the reference budgets each eigensolve
  double maxres = 0;
  for (int i = 0; i < s.need; ++i) maxres = fmax(maxres, s.resid[i]);
  if (s.mode == MODE_NEWTON_INNER) maxres = s.resid[j];  // the returned band (see k_control)
  if (!(s.k > 0)) { finish(s, TS_NAN); return; }
  if (prm.last_phase && maxres < prm.tol && fabs(dk) < prm.k_tol) { finish(s, TS_CONVERGED); return; }
  if (s.newton_steps >= prm.max_newton) { finish(s, prm.last_phase ? TS_MAXITER : TS_PHASE_DONE); return; }
  // k moved: recompute AX, AW and AP at the new k (keeping the P direction keeps LOBPCG's
  // momentum across Newton steps) and restart locking
  const int M = s.M;
  s.nlocked = 0;
  s.nWa = M;
  s.op_col0 = 0;
  s.op_ncol = 2 * M + s.nP;
  s.pw_ncol = 0;
  s.resid_best = 1e300;
  s.stall = 0;
}

}  // namespace omb

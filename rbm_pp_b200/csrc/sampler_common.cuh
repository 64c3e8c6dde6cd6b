// sampler_common.cuh -- walker-level routines shared by the two sampler kernels (sampler.cu: immediate
// rank-2 updates; sampler_stream.cu: TMA-streamed projections with deferred updates).
#pragma once
#include "tma.cuh"
#include "walker_ops.cuh"

namespace {

struct SCtx {
  const DevDims& d;
  const DevTables& t;
  const DevParams& p;
  const DevWalkers& W;
  int w;
  const WS& s;  // pointer table kept in shared memory
  double* Yw;   // this walker's Y
  // Optional: par_ntile >= 2 tiles of Np x (Np + 1) doubles at par_tiles let one warp per tile invert
  // projections in parallel during from-scratch recomputes (the streaming sampler's stage area).
  double* par_tiles;
  int par_ntile;
};

__device__ __forceinline__ int& status(const SCtx& c) { return c.s.iflag[F_STATUS]; }

// Scratch inverse of every projection, one warp per projection on its own tile (warps 1..par_ntile):
// the same results as the CTA-wide path below, which inverts one projection at a time.
template <int KPL, int NP>
__device__ __forceinline__ void warp_scratch_all(const SCtx& c, const int* idx, double* pf_out, bool write_y,
                                                 bool diff) {
  const DevDims& d = c.d;
  const WS& s = c.s;
  const int Np = NP > 0 ? NP : d.Np, ld = Np + 1, N = d.N;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, wk = warp - 1;
  double wratio = -1.0;
  bool sing_any = false;
  if (wk >= 0 && wk < c.par_ntile) {
    double* T = c.par_tiles + (size_t)wk * Np * ld;
    int* perm = (int*)(s.wS + (size_t)warp * Np);
    for (int qp = wk; qp < d.n_qp && !sing_any; qp += c.par_ntile) {
      warp_gather_tile<KPL, NP, 8>(T, c.p.XF + (size_t)qp * N * N, idx, Np, N);
      bool sing;
      const double det = warp_gj<KPL, NP, 4>(T, Np, perm, sing);
      if (sing) {
        sing_any = true;
        break;
      }
      double* Yq = c.Yw + (size_t)qp * Np * Np;
      if (diff) {  // make_sample.f90:106-113
        // the stored Y comes from HBM: a batch of RB rows is loaded before any is compared
        constexpr int RB = 10;
        double mx = 0.0, md = 0.0;
        for (int a0 = 0; a0 < Np; a0 += RB) {
          double yv[RB][KPL];
#pragma unroll
          for (int r = 0; r < RB; r++)
#pragma unroll
            for (int q = 0; q < KPL; q++) {
              const int a = a0 + r, b = lane + 32 * q;
              yv[r][q] = (a < Np && b < Np) ? Yq[a * Np + b] : 0.0;
            }
#pragma unroll
          for (int r = 0; r < RB; r++)
#pragma unroll
            for (int q = 0; q < KPL; q++) {
              const int a = a0 + r, b = lane + 32 * q;
              if (a < Np && b < Np) {
                const double nv = T[a * ld + perm[b]];
                mx = fmax(mx, fabs(nv));
                md = fmax(md, fabs(yv[r][q] - nv));
              }
            }
        }
        mx = warp_max(mx);
        md = warp_max(md);
        wratio = fmax(wratio, md / mx);
      }
      if (write_y)
        for (int a = 0; a < Np; a++)
          for (int b = lane; b < Np; b += 32) Yq[a * Np + b] = T[a * ld + perm[b]];
      if (lane == 0) pf_out[qp] = (double)d.pf_sign * det;
      __syncwarp();
    }
  }
  if (lane == 0) {
    s.red[warp] = wratio;
    s.red[32 + warp] = sing_any ? 1.0 : 0.0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double di = -1.0;
    bool sg = false;
    for (int w = 1; w <= c.par_ntile; w++) {
      di = fmax(di, s.red[w]);
      if (s.red[32 + w] != 0.0) sg = true;
    }
    if (sg) status(c) = ST_SINGULAR;
    s.dsc[D_DIFFINV] = di;
  }
  // generic writes of Y / of the shared tiles before later bulk (async-proxy) copies touch them
  if (write_y) fence_proxy_async_global();
  fence_proxy_async_smem();
  __syncthreads();
}

// Scratch inverse of every projection for labelling idx: writes Y (when write_y) and pf_out.
// When diff is requested, also computes the reference's drift measures against the stored Y / pf.
// KPL > 0 selects the warp-parallel path when the context provides tiles for it.
template <int KPL = 0, int NP = 0>
__device__ __forceinline__ void cta_scratch_all(const SCtx& c, const int* idx, double* pf_out, bool write_y, bool diff) {
  if constexpr (KPL > 0) {
    if (c.par_ntile >= 2) {
      warp_scratch_all<KPL, NP>(c, idx, pf_out, write_y, diff);
      return;
    }
  }
  const DevDims& d = c.d;
  const WS& s = c.s;
  const int Np = d.Np, ld = Np + 1, tid = threadIdx.x;
  double diff_inv = -1.0;
  for (int qp = 0; qp < d.n_qp; qp++) {
    cta_build_x(d, c.p, qp, idx, s.tile);
    __syncthreads();
    cta_gauss_jordan(d, s);
    if (s.iflag[F_SINGULAR]) {
      if (tid == 0) status(c) = ST_SINGULAR;
      __syncthreads();
      return;
    }
    double* Yq = c.Yw + (size_t)qp * Np * Np;
    if (diff) {  // make_sample.f90:106-113
      double mx = 0.0, md = 0.0;
      for (int a = tid >> 5; a < Np; a += blockDim.x >> 5)
        for (int b = tid & 31; b < Np; b += 32) {
          const double nv = s.tile[a * ld + s.perm[b]];
          mx = fmax(mx, fabs(nv));
          md = fmax(md, fabs(Yq[a * Np + b] - nv));
        }
      mx = warp_max(mx);
      md = warp_max(md);
      if ((tid & 31) == 0) {
        s.red[tid >> 5] = mx;
        s.red[32 + (tid >> 5)] = md;
      }
      __syncthreads();
      if (tid == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) {
          a = fmax(a, s.red[k]);
          b = fmax(b, s.red[32 + k]);
        }
        diff_inv = fmax(diff_inv, b / a);
      }
    }
    if (write_y)
      for (int a = tid >> 5; a < Np; a += blockDim.x >> 5)
        for (int b = tid & 31; b < Np; b += 32) Yq[a * Np + b] = s.tile[a * ld + s.perm[b]];
    if (tid == 0) pf_out[qp] = (double)d.pf_sign * s.dsc[D_DET];
    __syncthreads();
  }
  if (tid == 0) s.dsc[D_DIFFINV] = diff_inv;
  // generic writes of Y / of the shared tile before later bulk (async-proxy) copies touch them
  if (write_y) fence_proxy_async_global();
  fence_proxy_async_smem();
  __syncthreads();
}

// The from-scratch Pfaffians and inverses of every projection (calculate_MAll) as a policy of the walker
// routines below: the block form's, or the full skew form's (skew.cu).
template <int KPL, int NP>
struct BlockScratch {
  static __device__ __forceinline__ void run(const SCtx& c, const int* idx, double* pf_out, bool write_y, bool diff) {
    cta_scratch_all<KPL, NP>(c, idx, pf_out, write_y, diff);
  }
};

// calc_theta, x_to_Ele_Idx, calculate_MAll, sign_PP, calc_amplitude (make_sample.f90:54-60 / :345-350)
template <int KPL = 0, int NP = 0, class F = BlockScratch<KPL, NP>>
__device__ __forceinline__ void full_state(const SCtx& c) {
  const WS& s = c.s;
  cta_calc_theta(c.d, c.t, c.p, s.x, s.th);
  if (threadIdx.x == 0) {
    int e = x_to_ele(c.d, s.x, s.idx, s.cfg);
    if (e) status(c) = e;
  }
  __syncthreads();
  if (status(c)) return;
  F::run(c, s.idx, s.pf, true, false);
  if (status(c)) return;
  cta_sign_pp(c.d, c.t, s, s.idx, s.sgn);
  __syncthreads();
  if (threadIdx.x == 0)
    for (int mp = 1; mp < c.d.n_mp; mp++)
      if (s.pb[mp] != s.pb[0]) status(c) = ST_SIGN;
  __syncthreads();
  if (status(c)) return;
  cta_amplitude(c.d, c.t, s, s.th, s.pf, s.sgn, s.psi, D_PSI0R);
}

// make_initial_x make_sample.f90:298-362
template <int KPL = 0, int NP = 0, class F = BlockScratch<KPL, NP>>
__device__ __forceinline__ void make_initial_x(const SCtx& c) {
  const WS& s = c.s;
  for (int it1 = 0; it1 < 1000000; it1++) {
    if (threadIdx.x == 0) {
      for (int i = 0; i < c.d.N; i++) s.x[i] = -1;
      int i3 = 0, ok = 0;
      for (int it2 = 0; it2 < 1000000; it2++) {
        int i = nran(s.mt, c.d.N) - 1;
        if (s.x[i] == -1) {
          i3++;
          s.x[i] = 1;
        }
        if (i3 == c.d.N / 2) {
          ok = 1;
          break;
        }
      }
      if (!ok) status(c) = ST_INITX;
    }
    __syncthreads();
    if (status(c)) return;
    full_state<KPL, NP, F>(c);
    if (status(c)) return;
    if (hypot(s.dsc[D_PSI0R], s.dsc[D_PSI0I]) > 1e-300) return;
  }
  if (threadIdx.x == 0) status(c) = ST_INITX;
  __syncthreads();
}

// One record of the optional chain trace (thread 0 only; see DevWalkers::trace).
__device__ __forceinline__ void trace_rec(const SCtx& c, int type, double a, double b, double x, double u, double e) {
  const int k = c.s.iflag[F_EV_TRACE]++;
  if (c.W.trace && k < c.d.trace_max) {
    double* r = c.W.trace + ((size_t)c.w * c.d.trace_max + k) * 6;
    r[0] = (double)type;
    r[1] = a;
    r[2] = b;
    r[3] = x;
    r[4] = u;
    r[5] = e;
  }
}

// Nfastup checkpoint make_sample.f90:74-128.  i0 (sweep) only labels the trace record.
template <int KPL = 0, int NP = 0, class F = BlockScratch<KPL, NP>>
__device__ __forceinline__ void checkpoint(const SCtx& c, int& nfastup, int i0) {
  const DevDims& d = c.d;
  const WS& s = c.s;
  for (int j = threadIdx.x; j < d.Mr + 2 * d.Mc; j += blockDim.x) s.thp[j] = s.th[j];
  for (int mp = threadIdx.x; mp < d.n_mp; mp += blockDim.x) s.sgnp[mp] = s.sgn[mp];
  __syncthreads();
  cta_calc_theta(d, c.t, c.p, s.x, s.th);
  if (threadIdx.x == 0) {
    int e = check_ele(d, s.x, s.idx, s.cfg);
    if (e) status(c) = e;
  }
  __syncthreads();
  if (status(c)) return;
  cta_sign_pp(d, c.t, s, s.idx, s.sgn);
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int mp = 1; mp < d.n_mp; mp++)
      if (s.pb[mp] != s.pb[0]) status(c) = ST_SIGN;
    for (int mp = 0; mp < d.n_mp; mp++)
      if (s.sgnp[mp] != s.sgn[mp]) status(c) = ST_SIGN;
  }
  for (int j = threadIdx.x; j < d.Mr; j += blockDim.x)
    if (fabs(s.th[j] - s.thp[j]) > 1.0e-5) status(c) = ST_THETA;
  for (int j = threadIdx.x; j < d.Mc; j += blockDim.x)  // make_sample.f90:84-86
    if (hypot(s.th[d.Mr + 2 * j] - s.thp[d.Mr + 2 * j], s.th[d.Mr + 2 * j + 1] - s.thp[d.Mr + 2 * j + 1]) > 1.0e-5)
      status(c) = ST_THETA;
  __syncthreads();
  if (status(c)) return;
  // old Pf kept in pfp for the drift measure
  for (int qp = threadIdx.x; qp < d.n_qp; qp += blockDim.x) s.pfp[qp] = s.pf[qp];
  __syncthreads();
  F::run(c, s.idx, s.pf, true, true);
  if (status(c)) return;
  cta_amplitude(d, c.t, s, s.th, s.pf, s.sgn, s.psi, D_PSI0R);
  if (threadIdx.x == 0) {
    double r2 = 0.0;
    for (int qp = 0; qp < d.n_qp; qp++) r2 = r2 + fabs(s.pf[qp]);
    r2 = r2 / (double)d.n_qp;
    double dpf = -1.0;
    for (int qp = 0; qp < d.n_qp; qp++) dpf = fmax(dpf, fabs(s.pfp[qp] - s.pf[qp]) / r2);
    double dinv = s.dsc[D_DIFFINV];
    const int nf0 = nfastup;
    const int k = s.iflag[F_EV_CKPT]++;
    (void)grnd(s.mt);  // make_sample.f90:116
    if (c.W.replay && k < d.replay_max) {
      // verification replay: the decision of this checkpoint is given (Nfastup after, extra draw)
      const int* rp = c.W.replay + ((size_t)c.w * d.replay_max + k) * 2;
      nfastup = rp[0];
      if (rp[1]) (void)grnd(s.mt);
    } else if (dinv > 1.0e-5 || dpf > 1.0e-5) {
      nfastup = max(1, (int)floor((double)nfastup / 1.2 + 0.5));
      if (dinv > 10.0 && dpf > 10.0) (void)grnd(s.mt);  // make_sample.f90:122
    } else {
      nfastup = min(100, (int)floor((double)nfastup * 1.1 + 0.5));
    }
    s.iflag[F_AUX] = nfastup;
    if (c.W.trace) trace_rec(c, 1, (double)i0, dinv, dpf, (double)nf0, (double)nfastup);
  }
  __syncthreads();
  nfastup = s.iflag[F_AUX];
}

// Global spin flip make_sample.f90:135-158 (RNG check already drawn by the caller).
template <int KPL = 0, int NP = 0, class F = BlockScratch<KPL, NP>>
__device__ __forceinline__ void global_flip(const SCtx& c) {
  const DevDims& d = c.d;
  const WS& s = c.s;
  for (int i = threadIdx.x; i < d.N; i += blockDim.x) s.x2[i] = -s.x[i];
  __syncthreads();
  cta_calc_theta(d, c.t, c.p, s.x2, s.thp);
  if (threadIdx.x == 0) {
    int e = x_to_ele(d, s.x2, s.idx2, s.cfg2);
    if (e) status(c) = e;
  }
  __syncthreads();
  if (status(c)) return;
  F::run(c, s.idx2, s.pfp, false, false);  // Pf of the flipped configuration
  if (status(c)) return;
  cta_sign_pp(d, c.t, s, s.idx2, s.sgnp);
  __syncthreads();
  if (threadIdx.x == 0)
    for (int mp = 1; mp < d.n_mp; mp++)
      if (s.pb[mp] != s.pb[0]) status(c) = ST_SIGN;
  __syncthreads();
  if (status(c)) return;
  cta_amplitude(d, c.t, s, s.thp, s.pfp, s.sgnp, s.psip, D_PSIPR);
  if (threadIdx.x == 0) {
    double r1 = (hypot(s.dsc[D_PSIPR], s.dsc[D_PSIPI]) + d.shift) / (hypot(s.dsc[D_PSI0R], s.dsc[D_PSI0I]) + d.shift);
    const double u = grnd(s.mt);
    const int acc = u < r1 * r1;
    if (c.W.trace) trace_rec(c, 2, 0.0, 0.0, r1 * r1, u, (double)acc);
    if (acc) (void)grnd(s.mt);  // make_sample.f90:146
    s.iflag[F_ACCEPT] = acc;
    s.iflag[F_EV_FLIPACC] += acc;
  }
  __syncthreads();
  if (!s.iflag[F_ACCEPT]) return;
  for (int i = threadIdx.x; i < d.N; i += blockDim.x) {
    s.x[i] = s.x2[i];
    s.idx[i] = s.idx2[i];
    s.cfg[i] = s.cfg2[i];
  }
  for (int j = threadIdx.x; j < d.Mr + 2 * d.Mc; j += blockDim.x) s.th[j] = s.thp[j];
  for (int mp = threadIdx.x; mp < d.n_mp; mp += blockDim.x) s.sgn[mp] = s.sgnp[mp];
  for (int qp = threadIdx.x; qp < d.n_qp; qp += blockDim.x) {
    s.psi[2 * qp] = s.psip[2 * qp];
    s.psi[2 * qp + 1] = s.psip[2 * qp + 1];
  }
  if (threadIdx.x == 0) {
    s.dsc[D_PSI0R] = s.dsc[D_PSIPR];
    s.dsc[D_PSI0I] = s.dsc[D_PSIPI];
  }
  __syncthreads();
  F::run(c, s.idx, s.pf, true, false);  // Tmp_Inv_M of the accepted flipped state
}


// event counters of one make_sample: reset at its start (thread 0), stored with the walker state at its end
__device__ __forceinline__ void events_reset(const WS& s) {
  s.iflag[F_EV_FLIP] = s.iflag[F_EV_FLIPACC] = s.iflag[F_EV_RESEED] = s.iflag[F_EV_CKPT] = s.iflag[F_EV_TRACE] = 0;
}
__device__ __forceinline__ void events_store(const SCtx& c) {
  if (c.W.events) {
    int* e = c.W.events + (size_t)c.w * 5;
    e[0] = c.s.iflag[F_EV_FLIP];
    e[1] = c.s.iflag[F_EV_FLIPACC];
    e[2] = c.s.iflag[F_EV_RESEED];
    e[3] = c.s.iflag[F_EV_CKPT];
    e[4] = c.s.iflag[F_EV_TRACE];
  }
}

// make_spin_flip_candidate make_sample.f90:244-294 (thread 0): writes F_I1/F_I2 or sets ST_CANDIDATE
__device__ __forceinline__ void candidate_search(const SCtx& c) {
  const WS& s = c.s;
  const int L = c.d.L, N = c.d.N;
  int dist_max = nran(s.mt, L - 1) + 1, ok = 0;
  for (int it = 0; it < 1000000; it++) {
    int i1 = nran(s.mt, N);
    int ix = (i1 - 1) / L, iy = (i1 - 1) - ix * L;
    ix = ix + nran(s.mt, dist_max) - 1;
    iy = iy + nran(s.mt, dist_max) - 1;
    if (ix >= L) ix -= L;
    if (iy >= L) iy -= L;
    int i2 = ix * L + iy + 1;
    if (s.x[i1 - 1] != s.x[i2 - 1]) {
      s.iflag[F_I1] = i1 - 1;
      s.iflag[F_I2] = i2 - 1;
      ok = 1;
      break;
    }
  }
  if (!ok || dist_max <= 1) status(c) = ST_CANDIDATE;
}

}  // namespace

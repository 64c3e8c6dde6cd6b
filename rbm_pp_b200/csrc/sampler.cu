// sampler.cu -- persistent Metropolis sampler: one CTA per walker runs the whole make_sample call
// (make_sample.f90:4-240): warm-up + Nsample sweeps of Nupdate exchange proposals, Nfastup-scheduled
// scratch recomputation with the drift check, rare global spin flips, sample storage.
//
// RNG draws happen on thread 0 in exactly the reference's order, so spin configurations and
// accept/reject sequences are bit-identical to a rank of the reference (ties of the acceptance
// test within rounding excepted).
//
// Per proposal and projection qp one warp gathers the new row u and column v of X from XF/XFT,
// streams Y = X^{-1} (coalesced, lane <-> column) and evaluates the determinant ratio
//     R = (u^T Y)_ua (Y v)_db - Y(db,ua) (u^T Y v - c)      (= Pf'/Pf, pfupdate_two.f90:27-88)
// An accepted move applies the rank-2 Sherman-Morrison update of Y (pfupdate_two.f90:113-224).
#include "sampler_common.cuh"

namespace {

// ---- per-warp determinant ratio for projection qp; result valid on all lanes ----
template <int KPL>
__device__ __forceinline__ double warp_ratio(const DevDims& d, const DevParams& p, const double* Yq, int qp, const int* idx,
                                    int ua, int db, int s_up, int s_dn, double* u, double* v) {
  const int lane = threadIdx.x & 31, Np = d.Np, N = d.N;
  const double* XFq = p.XF + (size_t)qp * N * N;
  const double* XFTq = p.XFT + (size_t)qp * N * N;
  const double c = XFq[(size_t)s_dn * N + s_up];
  for (int j = lane; j < Np; j += 32) {
    u[j] = (j == db) ? c : XFq[(size_t)s_dn * N + idx[Np + j]];
    v[j] = (j == ua) ? c : XFTq[(size_t)s_up * N + idx[j]];
  }
  __syncwarp();
  double acc[KPL];
#pragma unroll
  for (int m = 0; m < KPL; m++) acc[m] = 0.0;
  int j = 0;
  for (; j + 4 <= Np; j += 4) {
    double y[4][KPL];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
      for (int m = 0; m < KPL; m++) {
        int k = lane + 32 * m;
        y[r][m] = (k < Np) ? __ldg(Yq + (size_t)(j + r) * Np + k) : 0.0;
      }
#pragma unroll
    for (int r = 0; r < 4; r++) {
      double uj = u[j + r];
#pragma unroll
      for (int m = 0; m < KPL; m++) acc[m] = fma(uj, y[r][m], acc[m]);
    }
  }
  for (; j < Np; j++) {
    double uj = u[j];
#pragma unroll
    for (int m = 0; m < KPL; m++) {
      int k = lane + 32 * m;
      if (k < Np) acc[m] = fma(uj, __ldg(Yq + (size_t)j * Np + k), acc[m]);
    }
  }
  double wv = 0.0, sb = 0.0, ra = 0.0, ydbua = 0.0;
#pragma unroll
  for (int m = 0; m < KPL; m++) {
    int k = lane + 32 * m;
    if (k < Np) {
      double rho = __ldg(Yq + (size_t)db * Np + k);
      wv = fma(acc[m], v[k], wv);
      sb = fma(rho, v[k], sb);
      if (k == ua) {
        ra = acc[m];
        ydbua = rho;
      }
    }
  }
  wv = warp_sum(wv);
  sb = warp_sum(sb);
  ra = warp_sum(ra);
  ydbua = warp_sum(ydbua);
  __syncwarp();
  return ra * sb - ydbua * (wv - c);
}

// ---- per-warp rank-2 update of Y after an accepted exchange (u, v from warp_ratio) ----
template <int KPL>
__device__ __forceinline__ void warp_update(const DevDims& d, double* Yq, int ua, int db, double c, const double* u,
                                   const double* v, double* A, double* S) {
  const int lane = threadIdx.x & 31, Np = d.Np;
  double acc[KPL];
#pragma unroll
  for (int m = 0; m < KPL; m++) acc[m] = 0.0;
  for (int j = 0; j < Np; j++) {
    double uj = u[j], part = 0.0;
#pragma unroll
    for (int m = 0; m < KPL; m++) {
      int k = lane + 32 * m;
      if (k < Np) {
        double y = Yq[(size_t)j * Np + k];
        acc[m] = fma(uj, y, acc[m]);
        part = fma(y, v[k], part);
        if (k == ua) A[j] = y;
      }
    }
    part = warp_sum(part);
    if (lane == 0) S[j] = part;
  }
  double rho[KPL];
  double wv = 0.0, ra = 0.0, ydbua = 0.0;
#pragma unroll
  for (int m = 0; m < KPL; m++) {
    int k = lane + 32 * m;
    rho[m] = 0.0;
    if (k < Np) {
      rho[m] = Yq[(size_t)db * Np + k];
      wv = fma(acc[m], v[k], wv);
      if (k == ua) {
        ra = acc[m];
        ydbua = rho[m];
      }
    }
  }
  wv = warp_sum(wv);
  ra = warp_sum(ra);
  ydbua = warp_sum(ydbua);
  __syncwarp();
  const double sb = S[db];
  const double R1 = ra;
  const double R = ra * sb - ydbua * (wv - c);
  const double inv_r1 = 1.0 / R1, r1_over_r = R1 / R, wc = (wv - c) * inv_r1;
  double bk[KPL], tk[KPL];
#pragma unroll
  for (int m = 0; m < KPL; m++) {
    int k = lane + 32 * m;
    double B = acc[m] - (k == ua ? 1.0 : 0.0);
    bk[m] = B * inv_r1;
    tk[m] = (rho[m] - ydbua * B * inv_r1) * r1_over_r;
  }
  for (int j = 0; j < Np; j++) {
    double Aj = A[j];
    double s1 = S[j] - Aj * wc - (j == db ? 1.0 : 0.0);
#pragma unroll
    for (int m = 0; m < KPL; m++) {
      int k = lane + 32 * m;
      if (k < Np) {
        double* py = Yq + (size_t)j * Np + k;
        *py = *py - Aj * bk[m] - s1 * tk[m];
      }
    }
  }
  __syncwarp();
}

// make_sample for walker w of one context, by the whole CTA
template <int KPL>
__device__ __forceinline__ void sampler_body(const DevDims& d, const DevTables& t, const DevParams& p,
                                             const DevWalkers& W, const int w, const int first) {
  extern __shared__ __align__(16) char smem[];
  __shared__ WS ws;
  if (threadIdx.x == 0) {
    ws_layout(d, blockDim.x >> 5, smem, &ws);
    if (d.gj_global) ws.tile = W.gj + (size_t)w * d.Np * (d.Np + 1);
  }
  __syncthreads();
  const SCtx c{d, t, p, W, w, ws, W.Y + (size_t)w * d.n_qp * d.Np * d.Np};
  const WS& s = ws;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nwarps = blockDim.x >> 5;
  const int N = d.N, Np = d.Np;

  for (int k = tid; k < 625; k += blockDim.x) s.mt[k] = W.mt[(size_t)w * 625 + k];
  if (tid == 0) {
    status(c) = 0;
    events_reset(s);
  }
  __syncthreads();
  int nfastup = W.nfastup[w];

  if (first) {
    make_initial_x(c);
  } else {
    for (int i = tid; i < N; i += blockDim.x) s.x[i] = W.xs[((size_t)w * d.ns + (d.ns - 1)) * N + i];
    __syncthreads();
    full_state(c);
    if (!status(c)) {
      if (tid == 0) {
        s.iflag[F_AUX] = grnd(s.mt) < 0.05;  // make_sample.f90:61
        s.iflag[F_EV_RESEED] += s.iflag[F_AUX];
        if (s.iflag[F_AUX] && W.trace) trace_rec(c, 3, 0.0, 0.0, 0.0, 0.0, 0.0);
      }
      __syncthreads();
      if (s.iflag[F_AUX]) make_initial_x(c);
    }
  }

  int naccept = 0, nacc_tmp = 0, nacc_all = 0;
  for (int i0 = -d.nwarm; i0 <= d.ns && !status(c); i0++) {
    if (nacc_tmp > nfastup) {
      checkpoint(c, nfastup, i0);
      if (status(c)) break;
      nacc_tmp = 0;
    }
    for (int iu = 0; iu < d.nupdate; iu++) {
      if (tid == 0) {
        s.iflag[F_FLIP] = grnd(s.mt) < 3.0e-4;  // make_sample.f90:135
        s.iflag[F_EV_FLIP] += s.iflag[F_FLIP];
      }
      __syncthreads();
      if (s.iflag[F_FLIP]) {
        global_flip(c);
        if (status(c)) break;
      }
      if (tid == 0) candidate_search(c);
      __syncthreads();
      if (status(c)) break;
      const int i1 = s.iflag[F_I1], i2 = s.iflag[F_I2];
      const int x1 = s.x[i1];
      const int i3 = s.cfg[i1], i4 = s.cfg[i2];
      int ua, db, s_up, s_dn;
      if (x1 == 1) {
        ua = i3;
        db = i4 - Np;
        s_up = i1;
        s_dn = i2;
      } else {
        ua = i4;
        db = i3 - Np;
        s_up = i2;
        s_dn = i1;
      }
      cta_update_theta(d, t, p, s.x, i1, i2, s.th, s.thp);
      const int flipsign = (t.subB[i1] ? -1 : 1) * (t.subB[i2] ? -1 : 1);
      for (int mp = tid; mp < d.n_mp; mp += blockDim.x) s.sgnp[mp] = -s.sgn[mp] * flipsign;
      __syncthreads();
      cta_rbm_factors(d, s.thp, s.rbm, s.rbmc);
      __syncthreads();
      double* u = s.wu + (size_t)warp * Np;
      double* v = s.wv + (size_t)warp * Np;
      double pre = 0.0, pim = 0.0;
      for (int qp = warp; qp < d.n_qp; qp += nwarps) {
        double R = warp_ratio<KPL>(d, p, c.Yw + (size_t)qp * Np * Np, qp, s.idx, ua, db, s_up, s_dn, u, v);
        if (lane == 0) {
          double pfn = R * s.pf[qp];
          s.pfp[qp] = pfn;
          cplx cw = psi_wo_pf_s(d, t, s, s.sgnp[qp >> 1], qp);
          s.psip[2 * qp] = cw.re * pfn;
          s.psip[2 * qp + 1] = cw.im * pfn;
          pre += cw.re * pfn;
          pim += cw.im * pfn;
        }
      }
      if (lane == 0) {
        s.red[warp] = pre;
        s.red[32 + warp] = pim;
      }
      __syncthreads();
      if (tid == 0) {
        double re = 0.0, im = 0.0;
        for (int k = 0; k < nwarps; k++) {
          re += s.red[k];
          im += s.red[32 + k];
        }
        s.dsc[D_PSIPR] = re;
        s.dsc[D_PSIPI] = im;
        (void)grnd(s.mt);  // sub.f90:72
        double r1 = (hypot(re, im) + d.shift) / (hypot(s.dsc[D_PSI0R], s.dsc[D_PSI0I]) + d.shift);
        const double u = grnd(s.mt);
        s.iflag[F_ACCEPT] = u < r1 * r1;  // make_sample.f90:203-204
        if (W.trace) trace_rec(c, 0, (double)i1, (double)i2, r1 * r1, u, (double)s.iflag[F_ACCEPT]);
      }
      __syncthreads();
      if (s.iflag[F_ACCEPT]) {  // make_sample.f90:205-219
        for (int qp = warp; qp < d.n_qp; qp += nwarps) {
          // rebuild u, v for this projection (same gathers as the ratio)
          const double* XFq = p.XF + (size_t)qp * N * N;
          const double* XFTq = p.XFT + (size_t)qp * N * N;
          const double cc = XFq[(size_t)s_dn * N + s_up];
          for (int j = lane; j < Np; j += 32) {
            u[j] = (j == db) ? cc : XFq[(size_t)s_dn * N + s.idx[Np + j]];
            v[j] = (j == ua) ? cc : XFTq[(size_t)s_up * N + s.idx[j]];
          }
          __syncwarp();
          warp_update<KPL>(d, c.Yw + (size_t)qp * Np * Np, ua, db, cc, u, v, s.wA + (size_t)warp * Np,
                           s.wS + (size_t)warp * Np);
        }
        for (int j = tid; j < d.Mr + 2 * d.Mc; j += blockDim.x) s.th[j] = s.thp[j];
        for (int mp = tid; mp < d.n_mp; mp += blockDim.x) s.sgn[mp] = s.sgnp[mp];
        for (int qp = tid; qp < d.n_qp; qp += blockDim.x) {
          s.pf[qp] = s.pfp[qp];
          s.psi[2 * qp] = s.psip[2 * qp];
          s.psi[2 * qp + 1] = s.psip[2 * qp + 1];
        }
        __syncthreads();
        if (tid == 0) {
          s.x[i1] = -s.x[i1];
          s.x[i2] = -s.x[i2];
          s.cfg[i1] = i4;
          s.cfg[i2] = i3;
          s.idx[i3] = i2;
          s.idx[i4] = i1;
          s.dsc[D_PSI0R] = s.dsc[D_PSIPR];
          s.dsc[D_PSI0I] = s.dsc[D_PSIPI];
        }
        __syncthreads();
        if (i0 > 0) naccept++;
        nacc_tmp++;
        nacc_all++;
      }
    }
    if (status(c)) break;
    if (i0 > 0) {  // make_sample.f90:228-232
      size_t sidx = (size_t)w * d.ns + (i0 - 1);
      for (int i = tid; i < N; i += blockDim.x) W.xs[sidx * N + i] = (int8_t)s.x[i];
      for (int qp = tid; qp < d.n_qp; qp += blockDim.x) W.pfs[sidx * d.n_qp + qp] = s.pf[qp];
      double* ps = W.psis + sidx * (size_t)(d.n_qp + 1) * 2;
      for (int k = tid; k < d.n_qp; k += blockDim.x) {
        ps[2 * (k + 1)] = s.psi[2 * k];
        ps[2 * (k + 1) + 1] = s.psi[2 * k + 1];
      }
      if (tid == 0) {
        ps[0] = s.dsc[D_PSI0R];
        ps[1] = s.dsc[D_PSI0I];
      }
    }
    __syncthreads();
  }
  // persist walker state
  for (int k = tid; k < 625; k += blockDim.x) W.mt[(size_t)w * 625 + k] = s.mt[k];
  for (int i = tid; i < N; i += blockDim.x) {
    W.x[(size_t)w * N + i] = (int8_t)s.x[i];
    W.idx[(size_t)w * N + i] = (int16_t)s.idx[i];
    W.cfg[(size_t)w * N + i] = (int16_t)s.cfg[i];
  }
  if (tid == 0) {
    W.nfastup[w] = nfastup;
    W.naccept[w] = naccept;
    W.nacc_all[w] = nacc_all;
    W.status[w] = status(c);
    events_store(c);
  }
}

template <int KPL>
__global__ void __launch_bounds__(256, 1)
    sampler_kernel(const __grid_constant__ DevDims d, const __grid_constant__ DevTables t,
                   const __grid_constant__ DevParams p, const __grid_constant__ DevWalkers W, int first) {
  sampler_body<KPL>(d, t, p, W, (int)blockIdx.x, first);
}

}  // namespace

// ---- one launch over the walkers of several contexts ----------------------------------------------
// Block b runs walker sched[b].y of context sched[b].x, with that context's dimensions, tables,
// parameters and walker arrays copied to shared memory first.
namespace {

template <int KPL, int THREADS>
__global__ void __launch_bounds__(THREADS, 1)
    sampler_batch_kernel(const BatchInst* __restrict__ inst, const int2* __restrict__ sched, int first,
                         long long* __restrict__ cycles) {
  __shared__ BatchInst bi;
  const int2 job = sched[blockIdx.x];
  if (threadIdx.x == 0) bi = inst[job.x];
  __syncthreads();
  const long long c0 = clock64();
  sampler_body<KPL>(bi.d, bi.t, bi.p, bi.W, job.y, first);
  if (cycles && threadIdx.x == 0) cycles[blockIdx.x] = clock64() - c0;
}

}  // namespace

// Host launchers -----------------------------------------------------------------------------------
// sched: n_blocks (context, walker) pairs; kpl: columns per lane covering the largest block size;
// threads: 128, 256 or 512; smem: dynamic shared memory for the largest context; cycles: per-block
// SM cycles (nullable).
cudaError_t rbmpp_launch_sampler_batch(const BatchInst* inst, const int2* sched, int n_blocks, int first, int kpl,
                                       int threads, size_t smem, long long* cycles, cudaStream_t st) {
#define BLAUNCH(K, TH)                                                                                      \
  do {                                                                                                      \
    cudaError_t e = cudaFuncSetAttribute(sampler_batch_kernel<K, TH>,                                       \
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);           \
    if (e != cudaSuccess) return e;                                                                         \
    rbmpp_note_launch();                                                                                    \
    sampler_batch_kernel<K, TH><<<n_blocks, TH, smem, st>>>(inst, sched, first, cycles);                    \
    return cudaGetLastError();                                                                              \
  } while (0)
#define BTHREADS(K)                     \
  do {                                  \
    if (threads == 128) BLAUNCH(K, 128); \
    if (threads == 256) BLAUNCH(K, 256); \
    if (threads == 512) BLAUNCH(K, 512); \
  } while (0)
  if (kpl <= 1) BTHREADS(1);
  if (kpl <= 2) BTHREADS(2);
  if (kpl <= 4) BTHREADS(4);
  if (kpl <= 8) BTHREADS(8);
#undef BTHREADS
#undef BLAUNCH
  return cudaErrorInvalidValue;
}

size_t rbmpp_sampler_smem(const DevDims& d, int threads) { return ws_layout(d, threads / 32, nullptr, nullptr); }

cudaError_t rbmpp_launch_sampler(const DevDims& d, const DevTables& t, const DevParams& p, const DevWalkers& W,
                                 int first, cudaStream_t st) {
  const int threads = 256;
  size_t smem = rbmpp_sampler_smem(d, threads);
  int kpl = (d.Np + 31) / 32;
#define LAUNCH(K)                                                                                        \
  do {                                                                                                   \
    cudaError_t e = cudaFuncSetAttribute(sampler_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                         (int)smem);                                                     \
    if (e != cudaSuccess) return e;                                                                      \
    rbmpp_note_launch(); sampler_kernel<K><<<d.nw, threads, smem, st>>>(d, t, p, W, first);                                   \
    return cudaGetLastError();                                                                           \
  } while (0)
  if (kpl <= 1) LAUNCH(1);
  if (kpl <= 2) LAUNCH(2);
  if (kpl <= 4) LAUNCH(4);
  if (kpl <= 8) LAUNCH(8);
#undef LAUNCH
  return cudaErrorInvalidValue;
}

// Resident blocks per SM of the batched sampler for a launch shape (0 if it cannot launch).
int rbmpp_batch_occupancy(int kpl, int threads, size_t smem) {
  int nb = 0;
  cudaError_t e = cudaErrorInvalidValue;
#define BOCC(K, TH)                                                                                              \
  do {                                                                                                           \
    if (cudaFuncSetAttribute(sampler_batch_kernel<K, TH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) \
        != cudaSuccess)                                                                                          \
      return 0;                                                                                                  \
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, sampler_batch_kernel<K, TH>, TH, smem);             \
    return e == cudaSuccess ? nb : 0;                                                                            \
  } while (0)
#define BOT(K)                          \
  do {                                  \
    if (threads == 128) BOCC(K, 128);   \
    if (threads == 256) BOCC(K, 256);   \
    if (threads == 512) BOCC(K, 512);   \
  } while (0)
  if (kpl <= 1) BOT(1);
  if (kpl <= 2) BOT(2);
  if (kpl <= 4) BOT(4);
  if (kpl <= 8) BOT(8);
#undef BOT
#undef BOCC
  (void)e;
  return 0;
}

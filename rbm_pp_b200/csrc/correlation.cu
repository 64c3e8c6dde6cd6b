// correlation.cu -- spin-correlation measurement of the Calc_Correlation program
// (Calc_Correlation/calc_phys_quantity.f90:264-344 calc_phys_quantity_after_opt, :348-424
// calc_local_energy_correlation, :477-550 calc_local_correlation): one CTA per stored sample.
//
// Every up electron ua and down electron db form an antiparallel site pair, so the exchanged amplitudes
// psi(x') of all N/2 x N/2 pairs are needed per sample.  A round of up to eight projections is inverted
// first (one warp-level Gauss-Jordan per projection, as in the estimator).  Then warp w takes the up
// electrons ua = w, w + 8, ... over every projection of the round: one mat-vec W = Y v_ua per (ua, qp), and
// for each chunk of eight down electrons their rows u are gathered together, the sixteen dot products
// u.Y(:,ua) and u.W are reduced in one transposed butterfly, and lane t forms the block-form ratio of
// pair (ua, db_t).  Then one lane per pair applies the cosh product of the exchanged spins' theta' and the
// projection weight.  psi(x') of pair (ua, db) accumulates in shared memory, written only by the warp that
// owns ua, in projection order, so the sums are deterministic.
//
// Per sample the CTA then writes, for a deterministic reduction over samples afterwards:
//   row[i0]            = w^2 psi(0) x_i1 x_i2 psi(0)                 (Chi_sp(1, i0) term)
//   row[Nchi + i0]     = w^2 psi(0) Chi_loc(2, i0)                  (Chi_sp(2, i0) term)
//   row[2 Nchi]        = psi(0) / |psi(0)|                          (wf_sgn term)
//   sdr[t N + i1]      = w SdotS(i1, t)                              (Chi_vbs is sum_s sdr sdr^T per t)
// with i0 = i2 (i2 + 1) / 2 + i1 for sites i1 <= i2 (0-based), w = 1 / (|psi(0)| + shift).  psi(0), the
// reweighted local energy and the antiparallel-bond count go to the estimator's outputs so the energy
// scalars and the RNG advance reuse the estimator's host path.
#include "walker_ops.cuh"

namespace {

constexpr int kCorThreads = 256;
constexpr int kCorWarps = kCorThreads / 32;

struct Cor {
  double* pfw;    // [n_qp] Pf per projection
  double* psx;    // [Np][Np] psi(x') of the exchange of up electron ua and down electron db
  int* perm;      // [kCorWarps][Np] column map of each projection's inverse
  double* vp;     // [kCorWarps][Np] v_ua at the tile's column positions
  double* rb;     // [kCorWarps][Np] ratios of one up electron's pairs, one projection
  double* bsum;   // [4N] J_t SdotS of every bond (unweighted), summed in bond order by thread 0
  double* tiles;  // [nqw][Np*(Np+1)]
  int nqw;
};

// Shared-memory layout of one correlation block.  With gbuf the nqw tiles and the pair table psx live in a
// per-block slice of a global scratch buffer (block sizes whose tiles do not fit one block's shared memory).
__host__ __device__ __forceinline__ size_t cor_layout(const DevDims& d, int nqw, char* base, WS* w, Cor* e,
                                                      bool gbuf = false) {
  size_t off = 0;
  auto take = [&](size_t bytes) -> char* {
    char* p = base ? base + off : nullptr;
    off = align16(off + bytes);
    return p;
  };
  const int N = d.N, Np = d.Np;
  WS t;
  t.mt = nullptr;
  t.x = (int*)take(N * 4);
  t.idx = (int*)take(N * 4);
  t.cfg = (int*)take(N * 4);
  t.x2 = t.idx2 = t.cfg2 = nullptr;
  t.th = (double*)take((size_t)d.Mr * 8);
  t.thp = nullptr;
  t.sgn = (int*)take(d.n_mp * 4);
  t.sgnp = nullptr;
  t.pb = (int*)take(d.n_mp * 4);
  t.pf = nullptr;
  t.pfp = nullptr;
  t.psi = (double*)take((size_t)d.n_qp * 16);
  t.psip = nullptr;
  t.rbm = (double*)take((size_t)d.n_qp * 8);
  t.colbuf = t.rowbuf = nullptr;
  t.perm = nullptr;
  t.wA = t.wS = nullptr;
  t.red = (double*)take(64 * 8);
  t.iflag = (int*)take(32 * 4);
  t.dsc = (double*)take(32 * 8);
  Cor x;
  x.pfw = (double*)take((size_t)d.n_qp * 8);
  x.psx = gbuf ? nullptr : (double*)take((size_t)Np * Np * 8);
  x.perm = (int*)take((size_t)kCorWarps * Np * 4);
  x.vp = (double*)take((size_t)kCorWarps * Np * 8);
  x.rb = (double*)take((size_t)kCorWarps * Np * 8);
  x.bsum = (double*)take((size_t)4 * N * 8);
  const size_t tile = (size_t)Np * (Np + 1) * 8;
  const size_t signbuf = (size_t)kCorWarps * N * 4;
  if (gbuf) {
    x.tiles = nullptr;
    t.wu = (double*)take(signbuf);  // per-warp N-int buffers of cta_sign_pp
  } else {
    size_t tiles_bytes = (size_t)nqw * tile;
    if (tiles_bytes < signbuf) tiles_bytes = signbuf;  // sign_PP scratch reuses the tile area
    x.tiles = (double*)take(tiles_bytes);
    t.wu = x.tiles;
  }
  x.nqw = nqw;
  t.tile = x.tiles;
  t.wv = nullptr;
  if (w) *w = t;
  if (e) *e = x;
  return off;
}

template <int KPL, int NP>
__device__ __forceinline__ void correlation_config(const DevDims& d, const DevTables& t, const DevParams& p,
                                                   const int8_t* xs, int n, double* out_psi, double* out_hpsi,
                                                   double* rows, double* sdr, int* out_nap, int* out_status,
                                                   const WS& s, const Cor& e, int cfgi) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int N = d.N, Np = NP > 0 ? NP : d.Np, ld = Np + 1, NB = 4 * N;

  for (int i = tid; i < N; i += blockDim.x) s.x[i] = (int)xs[(size_t)cfgi * N + i];
  for (int k = tid; k < Np * Np; k += blockDim.x) e.psx[k] = 0.0;
  if (tid == 0) {
    s.iflag[F_STATUS] = 0;
    s.iflag[F_SINGULAR] = 0;
  }
  __syncthreads();
  if (tid == 0) {
    const int st = x_to_ele(d, s.x, s.idx, s.cfg);
    if (st) s.iflag[F_STATUS] = st;
  }
  __syncthreads();
  if (s.iflag[F_STATUS]) {
    if (tid == 0 && out_status) out_status[cfgi] = s.iflag[F_STATUS];
    return;
  }
  cta_calc_theta(d, t, p, s.x, s.th);
  cta_sign_pp(d, t, s, s.idx, s.sgn);
  __syncthreads();
  if (tid == 0)
    for (int mp = 1; mp < d.n_mp; mp++)
      if (s.pb[mp] != s.pb[0]) s.iflag[F_STATUS] = ST_SIGN;
  cta_rbm_factors(d, s.th, s.rbm);
  __syncthreads();
  if (s.iflag[F_STATUS]) {
    if (tid == 0 && out_status) out_status[cfgi] = s.iflag[F_STATUS];
    return;
  }
  int jc[KPL], dsite[KPL];
#pragma unroll
  for (int q = 0; q < KPL; q++) {
    const int j = lane + 32 * q;
    jc[q] = j < Np ? j : Np - 1;  // in-tile index for every lane
    dsite[q] = s.idx[Np + jc[q]];
  }
  double* vp = e.vp + (size_t)warp * Np;
  double* rb = e.rb + (size_t)warp * Np;
  for (int q0 = 0; q0 < d.n_qp; q0 += e.nqw) {
    // inversions of this round's projections, one warp each
    if (warp < e.nqw && q0 + warp < d.n_qp) {
      const int qp = q0 + warp, mp = qp >> 1;
      double* T = e.tiles + (size_t)warp * Np * ld;
      warp_gather_tile<KPL, NP, 8>(T, p.XF + (size_t)qp * N * N, s.idx, Np, N);
      bool sing;
      const double det = warp_gj<KPL, NP, (KPL <= 2 ? 16 : (KPL <= 4 ? 8 : 4))>(T, Np, e.perm + (size_t)warp * Np, sing);
      const double pfq = (double)d.pf_sign * det;
      const cplx cw = psi_wo_pf(d, t, s.rbm[qp], s.sgn[mp], qp);
      if (lane == 0) {
        if (sing) s.iflag[F_SINGULAR] = 1;
        e.pfw[qp] = pfq;
        s.psi[2 * qp] = cw.re * pfq;
        s.psi[2 * qp + 1] = cw.im * pfq;
      }
    }
    __syncthreads();
    if (s.iflag[F_SINGULAR]) break;
    // exchanged amplitudes of every pair: warp w owns up electrons w, w + 8, ...
    for (int ua = warp; ua < Np; ua += kCorWarps) {
      const int s_up = s.idx[ua];
      const double x_up = (double)s.x[s_up];
      for (int pp = 0; pp < e.nqw && q0 + pp < d.n_qp; pp++) {
        const int qp = q0 + pp, mp = qp >> 1, sp = qp & 1;
        const double* T = e.tiles + (size_t)pp * Np * ld;
        const int* src = e.perm + (size_t)pp * Np;
        const double* XFq = p.XF + (size_t)qp * N * N;
        const double* XFTq = p.XFT + (size_t)qp * N * N;
        const int* wm = t.wmap + (size_t)mp * N;
        const double pfq = e.pfw[qp];
        const double s_sign = sp == 0 ? 1.0 : -1.0;
        const int cu = src[ua];
        double vv[KPL];
#pragma unroll
        for (int q = 0; q < KPL; q++) vv[q] = XFTq[(size_t)s_up * N + s.idx[jc[q]]];
        const double xfuu = XFq[(size_t)s_up * N + s_up];
        const int iwu = wm[s_up];
        // v_ua(i) = XF(u_i, s_up) at the tile's column positions, W = Y v_ua (lane <-> row)
#pragma unroll
        for (int q = 0; q < KPL; q++)
          if (lane + 32 * q < Np) vp[src[lane + 32 * q]] = vv[q];
        __syncwarp();
        double wv[KPL], tj[KPL];
#pragma unroll
        for (int q = 0; q < KPL; q++) {
          double a0 = 0.0, a1 = 0.0;
          const double* Tr = T + jc[q] * ld;
#pragma unroll 5
          for (int k = 0; k + 1 < Np; k += 2) {
            a0 = fma(Tr[k], vp[k], a0);
            a1 = fma(Tr[k + 1], vp[k + 1], a1);
          }
          if (Np & 1) a0 = fma(Tr[Np - 1], vp[Np - 1], a0);
          wv[q] = a0 + a1;
          tj[q] = Tr[cu];
        }
        constexpr int MB = KPL <= 2 ? 8 : (KPL <= 4 ? 4 : 2);
        constexpr int NV = 2 * MB, SH = MB == 8 ? 1 : (MB == 4 ? 2 : 3);  // value v ends in lane v << SH
        for (int c0 = 0; c0 < Np; c0 += MB) {
          const int m = Np - c0 < MB ? Np - c0 : MB;
          // down electron db = c0 + t in lane t: its site and X'(ua, db) = XF(s_dn, s_up)
          int db_l = 0, sdn_l = 0;
          double c_l = 0.0;
          if (lane < m) {
            db_l = c0 + lane;
            sdn_l = s.idx[Np + db_l];
            c_l = XFq[(size_t)sdn_l * N + s_up];
          }
          double uu[MB][KPL], cb[MB];
          int dbv[MB];
#pragma unroll
          for (int t2 = 0; t2 < MB; t2++) {
            dbv[t2] = -1;
            cb[t2] = 0.0;
#pragma unroll
            for (int q = 0; q < KPL; q++) uu[t2][q] = 0.0;
            if (t2 < m) {
              const int sdn = __shfl_sync(0xffffffffu, sdn_l, t2);
              dbv[t2] = c0 + t2;
              const double* urow = XFq + (size_t)sdn * N;
#pragma unroll
              for (int q = 0; q < KPL; q++) uu[t2][q] = urow[dsite[q]];
            }
          }
#pragma unroll
          for (int t2 = 0; t2 < MB; t2++)
            if (t2 < m) cb[t2] = __shfl_sync(0xffffffffu, c_l, t2);
          double val[NV];
#pragma unroll
          for (int t2 = 0; t2 < MB; t2++) {
            val[t2] = 0.0;
            val[MB + t2] = 0.0;
#pragma unroll
            for (int q = 0; q < KPL; q++)
              if (lane + 32 * q < Np) {
                const double uj = (lane + 32 * q == dbv[t2]) ? cb[t2] : uu[t2][q];
                val[t2] = fma(uj, tj[q], val[t2]);
                val[MB + t2] = fma(uj, wv[q], val[MB + t2]);
              }
          }
          const double tot = warp_transpose_sum<NV>(val, lane);
          const double ra = __shfl_sync(0xffffffffu, tot, (lane << SH) & 31);
          const double uw = __shfl_sync(0xffffffffu, tot, ((MB + lane) << SH) & 31);
          double y = 0.0, wdb = 0.0;
#pragma unroll
          for (int q = 0; q < KPL; q++) {
            const double a = __shfl_sync(0xffffffffu, tj[q], db_l & 31);  // Y(db, ua)
            const double b = __shfl_sync(0xffffffffu, wv[q], db_l & 31);  // W(db)
            if (q == (db_l >> 5)) {
              y = a;
              wdb = b;
            }
          }
          if (lane < m) {
            const double dv = c_l - xfuu;
            const double sb = wdb + dv * y;
            const double wvv = uw + dv * ra;
            rb[db_l] = ra * sb - y * (wvv - c_l);
          }
        }
        __syncwarp();
        // weights of the exchanged configurations, one pair per lane: the cosh product of theta' on the
        // sites (min, max) (update_theta, RBM.f90:95-148) for this projection, the sign and projection factor
        for (int db = lane; db < Np; db += 32) {
          const int sdn = s.idx[Np + db];
          const int i1 = s_up < sdn ? s_up : sdn, i2 = s_up < sdn ? sdn : s_up;
          const int iw1 = s_up < sdn ? iwu : wm[sdn], iw2 = s_up < sdn ? wm[sdn] : iwu;
          const double x1 = s_up < sdn ? x_up : -x_up, x2 = -x1;
          double ch = 1.0;
          for (int f = 0; f < d.alphar; f++) {
            double th = s.th[qp * d.alphar + f];
            th = th - 2.0 * p.Wr[(size_t)f * N + iw1] * x1 * s_sign;
            th = th - 2.0 * p.Wr[(size_t)f * N + iw2] * x2 * s_sign;
            ch = ch * cosh(th);
          }
          const int sg = -s.sgn[mp] * (t.subB[i1] ? -1 : 1) * (t.subB[i2] ? -1 : 1);
          const cplx cbw = psi_wo_pf(d, t, ch, sg, qp);
          double& acc = e.psx[(size_t)ua * Np + db];
          acc = acc + cbw.re * (rb[db] * pfq);
        }
        __syncwarp();  // vp is rewritten for the next projection
      }
    }
    __syncthreads();  // the next round rewrites the tiles
  }
  __syncthreads();
  if (s.iflag[F_SINGULAR]) {
    if (tid == 0 && out_status) out_status[cfgi] = ST_SINGULAR;
    return;
  }
  if (tid == 0) {
    double re = 0.0, im = 0.0;
    for (int qp = 0; qp < d.n_qp; qp++) {
      re += s.psi[2 * qp];
      im += s.psi[2 * qp + 1];
    }
    s.dsc[D_PSI0R] = re;
    s.dsc[D_PSI0I] = im;
  }
  __syncthreads();
  const double psi0 = s.dsc[D_PSI0R];
  const double apsi = hypot(s.dsc[D_PSI0R], s.dsc[D_PSI0I]);
  const double w = 1.0 / (apsi + d.shift);
  // psi(x') of the antiparallel pair on sites a, b
  auto pair_psi = [&](int a, int b) -> double {
    const int up = s.x[a] == 1 ? a : b, dn = s.x[a] == 1 ? b : a;
    return e.psx[(size_t)s.cfg[up] * Np + (s.cfg[dn] - Np)];
  };
  // bonds in bond_map order (calc_local_energy_correlation :364-421): SdotS and the local energy
  for (int b = tid; b < NB; b += blockDim.x) {
    const int i1 = t.bonds[2 * b], i2 = t.bonds[2 * b + 1], typ = b / N;
    const double J = typ < 2 ? d.J1 : d.J2, sg = typ < 2 ? -1.0 : 1.0;
    double sd = (double)s.x[i1] * (double)s.x[i2] * psi0;
    if (s.x[i1] != s.x[i2]) sd = sd + 2.0 * sg * pair_psi(i1, i2);
    e.bsum[b] = J * sd;
    sdr[(size_t)cfgi * NB + b] = sd * w;
  }
  // pairs i1 <= i2 (calc_local_correlation :495-547), premultiplied by w^2 psi(0)
  const size_t nchi = (size_t)N * (N + 1) / 2;
  double* row = rows + (size_t)cfgi * (2 * nchi + 1);
  const double w2p = w * w * psi0;
  for (int i2 = 0; i2 < N; i2++)
    for (int i1 = tid; i1 <= i2; i1 += blockDim.x) {
      const size_t i0 = (size_t)i2 * (i2 + 1) / 2 + i1;
      double c2 = 0.0;
      if (i1 == i2) {
        c2 = psi0;
      } else if (s.x[i1] != s.x[i2]) {
        const double sgs = (t.subB[i1] ? -1.0 : 1.0) * (t.subB[i2] ? -1.0 : 1.0);
        c2 = sgs * pair_psi(i1, i2);
      }
      row[i0] = w2p * ((double)s.x[i1] * (double)s.x[i2] * psi0);
      row[nchi + i0] = w2p * c2;
    }
  __syncthreads();
  if (tid == 0) {
    double h = 0.0;
    int nap = 0;
    for (int b = 0; b < NB; b++) {
      h += e.bsum[b];
      if (s.x[t.bonds[2 * b]] != s.x[t.bonds[2 * b + 1]]) nap++;
    }
    row[2 * nchi] = psi0 / apsi;
    if (out_psi) {
      double* ps = out_psi + (size_t)cfgi * (d.n_qp + 1) * 2;
      ps[0] = s.dsc[D_PSI0R];
      ps[1] = s.dsc[D_PSI0I];
      for (int qp = 0; qp < d.n_qp; qp++) {
        ps[2 * (qp + 1)] = s.psi[2 * qp];
        ps[2 * (qp + 1) + 1] = s.psi[2 * qp + 1];
      }
    }
    if (out_hpsi) {
      out_hpsi[2 * (size_t)cfgi] = h * w;
      out_hpsi[2 * (size_t)cfgi + 1] = 0.0;
    }
    if (out_nap) out_nap[cfgi] = nap;
    if (out_status) out_status[cfgi] = 0;
  }
}

__global__ void fill_kernel(double* a, long long n, double v) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    a[i] = v;
}

template <int KPL, int NP>
__global__ void __launch_bounds__(kCorThreads, 1)
    correlation_kernel(const __grid_constant__ DevDims d, const __grid_constant__ DevTables t,
                       const __grid_constant__ DevParams p, const int8_t* xs, int n, double* out_psi,
                       double* out_hpsi, double* rows, double* sdr, int* out_nap, int* out_status, int nqw,
                       double* gbuf) {
  extern __shared__ __align__(16) char smem[];
  __shared__ WS s;
  __shared__ Cor e;
  const int Np = NP > 0 ? NP : d.Np, ld = Np + 1;
  if (threadIdx.x == 0) {
    cor_layout(d, nqw, smem, &s, &e, gbuf != nullptr);
    if (gbuf) {
      e.tiles = gbuf + (size_t)blockIdx.x * ((size_t)nqw * Np * ld + (size_t)Np * Np);
      e.psx = e.tiles + (size_t)nqw * Np * ld;
      s.tile = e.tiles;
    }
  }
  __syncthreads();
  // one sample per block, or (global scratch) the samples blockIdx.x, blockIdx.x + gridDim.x, ...
  for (int cfgi = blockIdx.x; cfgi < n; cfgi += gridDim.x) {
    __syncthreads();
    correlation_config<KPL, NP>(d, t, p, xs, n, out_psi, out_hpsi, rows, sdr, out_nap, out_status, s, e, cfgi);
  }
}

int cor_tile_warps(const DevDims& d, int max_smem) {
  for (int q = kCorWarps; q >= 1; q--)
    if ((long long)cor_layout(d, q, nullptr, nullptr, nullptr) <= max_smem) return q;
  return 0;
}

}  // namespace

// Projections inverted together per round, 0 when one block's shared memory cannot hold the workspace.
// 1 when the correlation kernel can run at this shape (tiles in shared memory, or in global scratch when the
// rest of its workspace fits), else 0.
int rbmpp_correlation_fits(const DevDims& d, int max_smem) {
  if (cor_tile_warps(d, max_smem) >= 1) return 1;
  return (long long)cor_layout(d, kCorWarps, nullptr, nullptr, nullptr, true) <= max_smem ? 1 : 0;
}

cudaError_t rbmpp_launch_correlation(const DevDims& d, const DevTables& t, const DevParams& p, const int8_t* xs, int n,
                                     double* out_psi, double* out_hpsi, double* rows, double* sdr, int* out_nap,
                                     int* out_status, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  int dev = 0, maxsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  int nqw = cor_tile_warps(d, maxsm);
  size_t smem = 0;
  double* gbuf = nullptr;
  int grid = n;
  if (nqw >= 1) {
    smem = cor_layout(d, nqw, nullptr, nullptr, nullptr);
  } else {
    // tiles and pair table beyond one block's shared memory (N/2 beyond about 100): one block per SM loops over
    // the samples with a stream-ordered scratch slice of global memory
    nqw = kCorWarps;
    smem = cor_layout(d, nqw, nullptr, nullptr, nullptr, true);
    if ((long long)smem > maxsm) return cudaErrorInvalidValue;
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    grid = n < nsm ? n : nsm;
    const size_t per = (size_t)nqw * d.Np * (d.Np + 1) + (size_t)d.Np * d.Np;
    cudaError_t e = cudaMallocAsync((void**)&gbuf, (size_t)grid * per * sizeof(double), st);
    if (e != cudaSuccess) return e;
  }
  const int kpl = (d.Np + 31) / 32;
  cudaError_t rc = cudaErrorInvalidValue;
#define LAUNCH(K, NPC)                                                                                          \
  do {                                                                                                          \
    rc = cudaFuncSetAttribute(correlation_kernel<K, NPC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
    if (rc == cudaSuccess) {                                                                                    \
      rbmpp_note_launch();                                                                                      \
      correlation_kernel<K, NPC><<<grid, kCorThreads, smem, st>>>(d, t, p, xs, n, out_psi, out_hpsi, rows, sdr,  \
                                                                   out_nap, out_status, nqw, gbuf);              \
      rc = cudaGetLastError();                                                                                  \
    }                                                                                                           \
    if (gbuf) cudaFreeAsync(gbuf, st);                                                                          \
    return rc;                                                                                                  \
  } while (0)
  switch (d.Np) {
    case 8: LAUNCH(1, 8);
    case 18: LAUNCH(1, 18);
    case 32: LAUNCH(1, 32);
    case 50: LAUNCH(2, 50);
    default: break;
  }
  if (kpl <= 1) LAUNCH(1, 0);
  if (kpl <= 2) LAUNCH(2, 0);
  if (kpl <= 4) LAUNCH(4, 0);
  if (kpl <= 8) LAUNCH(8, 0);
#undef LAUNCH
  if (gbuf) cudaFreeAsync(gbuf, st);
  return rc;
}

cudaError_t rbmpp_fill(double* a, long long n, double v, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  rbmpp_note_launch();
  fill_kernel<<<(unsigned)((n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184), 256, 0, st>>>(a, n, v);
  return cudaGetLastError();
}

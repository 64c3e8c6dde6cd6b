// walker_ops.cuh -- CTA-collective building blocks for one walker / one configuration.
// Each routine cites the reference subroutine it restates.
#pragma once
#include "common.cuh"

// Shared-memory workspace of one CTA (one walker or one configuration).
struct WS {
  uint32_t* mt;  // [625]
  int* x;        // [N]   spins
  int* idx;      // [N]   Ele_Idx (0-based sites)
  int* cfg;      // [N]   Ele_Cfg
  int* x2;       // [N]   global-flip candidate
  int* idx2;
  int* cfg2;
  double* th;    // [Mr]
  double* thp;   // [Mr]
  int* sgn;      // [n_mp]
  int* sgnp;     // [n_mp]
  int* pb;       // [n_mp] sublattice parity per projection (sign_PP consistency)
  double* pf;    // [n_qp]
  double* pfp;   // [n_qp]
  double* psi;   // [n_qp][2]
  double* psip;  // [n_qp][2]
  double* rbm;   // [n_qp] cosh products
  double* rbmc;  // [n_qp][2] complex factor 0.5^alphac prod cosh(thetac) (null without complex units)
  double* tile;  // [Np][Np+1]
  double* colbuf;  // [Np]
  double* rowbuf;  // [Np]
  int* perm;       // [Np]
  double* wu;  // [nwarps][Np]
  double* wv;  // [nwarps][Np]
  double* wA;  // [nwarps][Np]
  double* wS;  // [nwarps][Np]
  double* red;     // [64]
  int* iflag;      // [32]
  double* dsc;     // [32]
};

// shared int slots
#define F_STATUS 0
#define F_I1 1
#define F_I2 2
#define F_ACCEPT 3
#define F_FLIP 4
#define F_PIV 5
#define F_SINGULAR 6
#define F_AUX 7
// per-walker event counters of one make_sample (written to DevWalkers::events)
#define F_EV_FLIP 8
#define F_EV_FLIPACC 9
#define F_EV_RESEED 10
#define F_EV_CKPT 11
#define F_EV_TRACE 12
// shared double slots
#define D_DET 0
#define D_PVAL 1
#define D_PSI0R 2
#define D_PSI0I 3
#define D_PSIPR 4
#define D_PSIPI 5
#define D_DIFFINV 6
#define D_DIFFPF 7
#define D_PIVOT 8

__host__ __device__ __forceinline__ size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

// Carve the workspace; returns total bytes.  Same code on host (sizing) and device (pointers).
__host__ __device__ __forceinline__ size_t ws_layout(const DevDims& d, int nwarps, char* base, WS* w,
                                                     bool own_tile = true) {
  size_t off = 0;
  auto take = [&](size_t bytes) -> char* {
    char* p = base ? base + off : nullptr;
    off = align16(off + bytes);
    return p;
  };
  const int N = d.N, Np = d.Np;
  WS t;
  t.mt = (uint32_t*)take(625 * 4);
  t.x = (int*)take(N * 4);
  t.idx = (int*)take(N * 4);
  t.cfg = (int*)take(N * 4);
  t.x2 = (int*)take(N * 4);
  t.idx2 = (int*)take(N * 4);
  t.cfg2 = (int*)take(N * 4);
  t.th = (double*)take((size_t)(d.Mr + 2 * d.Mc) * 8);
  t.thp = (double*)take((size_t)(d.Mr + 2 * d.Mc) * 8);
  t.sgn = (int*)take(d.n_mp * 4);
  t.sgnp = (int*)take(d.n_mp * 4);
  t.pb = (int*)take(d.n_mp * 4);
  t.pf = (double*)take(d.n_qp * 8);
  t.pfp = (double*)take(d.n_qp * 8);
  t.psi = (double*)take(d.n_qp * 16);
  t.psip = (double*)take(d.n_qp * 16);
  t.rbm = (double*)take(d.n_qp * 8);
  t.rbmc = d.alphac ? (double*)take((size_t)d.n_qp * 16) : nullptr;
  t.tile = (own_tile && !d.gj_global) ? (double*)take((size_t)Np * (Np + 1) * 8) : nullptr;
  t.colbuf = (double*)take(Np * 8);
  t.rowbuf = (double*)take(Np * 8);
  t.perm = (int*)take(Np * 4);
  t.wu = (double*)take((size_t)nwarps * Np * 8);
  t.wv = (double*)take((size_t)nwarps * Np * 8);
  t.wA = (double*)take((size_t)nwarps * Np * 8);
  t.wS = (double*)take((size_t)nwarps * Np * 8);
  t.red = (double*)take(64 * 8);
  t.iflag = (int*)take(32 * 4);
  t.dsc = (double*)take(32 * 8);
  if (w) *w = t;
  return off;
}

// calc_theta RBM.f90:31-91: th[j], j = mp*2*alphar + (s==+1 ? 0 : alphar) + f, then thetac as (re, im) pairs
// at th[Mr + 2 j'] with the same index pattern over alphac
__device__ __forceinline__ void cta_calc_theta(const DevDims& d, const DevTables& t, const DevParams& p, const int* x,
                                      double* th) {
  const int A2 = 2 * d.alphar;
  for (int j = threadIdx.x; j < d.Mr; j += blockDim.x) {
    int mp = j / A2, rem = j - mp * A2;
    double s = rem < d.alphar ? 1.0 : -1.0;
    int f = rem < d.alphar ? rem : rem - d.alphar;
    const int* wm = t.wmap + (size_t)mp * d.N;
    const double* Wf = p.Wr + (size_t)f * d.N;
    double acc = p.br[f];
    for (int i = 0; i < d.N; i++) acc = acc + Wf[wm[i]] * (double)x[i] * s;
    th[j] = acc;
  }
  const int C2 = 2 * d.alphac;
  for (int j = threadIdx.x; j < d.Mc; j += blockDim.x) {
    int mp = j / C2, rem = j - mp * C2;
    double s = rem < d.alphac ? 1.0 : -1.0;
    int f = rem < d.alphac ? rem : rem - d.alphac;
    const int* wm = t.wmap + (size_t)mp * d.N;
    const double* Wf = p.Wc + (size_t)f * d.N * 2;
    double ar = p.bc[2 * f], ai = p.bc[2 * f + 1];
    for (int i = 0; i < d.N; i++) {
      const double xs = (double)x[i] * s;
      ar = ar + Wf[2 * wm[i]] * xs;
      ai = ai + Wf[2 * wm[i] + 1] * xs;
    }
    th[d.Mr + 2 * j] = ar;
    th[d.Mr + 2 * j + 1] = ai;
  }
}

// update_theta RBM.f90:95-148 (x is the spin configuration BEFORE the exchange), real and complex angles
__device__ __forceinline__ void cta_update_theta(const DevDims& d, const DevTables& t, const DevParams& p, const int* x, int i1,
                                        int i2, const double* th, double* thp) {
  const int A2 = 2 * d.alphar;
  const double x1 = (double)x[i1], x2 = (double)x[i2];
  for (int j = threadIdx.x; j < d.Mr; j += blockDim.x) {
    int mp = j / A2, rem = j - mp * A2;
    double s = rem < d.alphar ? 1.0 : -1.0;
    int f = rem < d.alphar ? rem : rem - d.alphar;
    const double* Wf = p.Wr + (size_t)f * d.N;
    int iw1 = t.wmap[(size_t)mp * d.N + i1], iw2 = t.wmap[(size_t)mp * d.N + i2];
    double v = th[j];
    v = v - 2.0 * Wf[iw1] * x1 * s;
    v = v - 2.0 * Wf[iw2] * x2 * s;
    thp[j] = v;
  }
  const int C2 = 2 * d.alphac;
  for (int j = threadIdx.x; j < d.Mc; j += blockDim.x) {
    int mp = j / C2, rem = j - mp * C2;
    double s = rem < d.alphac ? 1.0 : -1.0;
    int f = rem < d.alphac ? rem : rem - d.alphac;
    const double* Wf = p.Wc + (size_t)f * d.N * 2;
    int iw1 = t.wmap[(size_t)mp * d.N + i1], iw2 = t.wmap[(size_t)mp * d.N + i2];
    double vr = th[d.Mr + 2 * j], vi = th[d.Mr + 2 * j + 1];
    vr = vr - 2.0 * Wf[2 * iw1] * x1 * s;
    vi = vi - 2.0 * Wf[2 * iw1 + 1] * x1 * s;
    vr = vr - 2.0 * Wf[2 * iw2] * x2 * s;
    vi = vi - 2.0 * Wf[2 * iw2 + 1] * x2 * s;
    thp[d.Mr + 2 * j] = vr;
    thp[d.Mr + 2 * j + 1] = vi;
  }
}

// x_to_Ele_Idx_Ele_Cfg interface_for_PP.f90:5-33 (thread 0); returns 0 or ST_CONFIG
__device__ __forceinline__ int x_to_ele(const DevDims& d, const int* x, int* idx, int* cfg) {
  int i1 = 0, i2 = d.Np;
  for (int i = 0; i < d.N; i++) {
    if (x[i] == 1) {
      if (i1 >= d.Np) return ST_CONFIG;
      idx[i1] = i;
      cfg[i] = i1++;
    } else if (x[i] == -1) {
      if (i2 >= d.N) return ST_CONFIG;
      idx[i2] = i;
      cfg[i] = i2++;
    } else
      return ST_CONFIG;
  }
  return (i1 == d.Np && i2 == d.N) ? 0 : ST_CONFIG;
}

// check_Ele_Idx_Ele_Cfg interface_for_PP.f90:37-65 (thread 0)
__device__ __forceinline__ int check_ele(const DevDims& d, const int* x, const int* idx, const int* cfg) {
  unsigned seen[(RBMPP_MAX_N + 31) / 32];
  for (int k = 0; k < (d.N + 31) / 32; k++) seen[k] = 0u;
  for (int i = 0; i < d.N; i++) {
    int s = idx[i];
    if (s < 0 || s >= d.N) return ST_CONFIG;
    if (cfg[s] != i) return ST_CONFIG;
    if (x[s] != (i < d.Np ? 1 : -1)) return ST_CONFIG;
    seen[s >> 5] |= 1u << (s & 31);
  }
  for (int s = 0; s < d.N; s++)
    if (!(seen[s >> 5] & (1u << (s & 31)))) return ST_CONFIG;
  return 0;
}

// sign_PP interface_for_PP.f90:71-106: warp per projection; the per-warp buffer wu holds the
// translated positions.  Writes sgn[mp] and pb[mp] (parity of down electrons on sublattice B).
__device__ __forceinline__ void cta_sign_pp(const DevDims& d, const DevTables& t, const WS& s, const int* idx, int* sgn) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  int* tb = (int*)(s.wu + (size_t)warp * d.Np);  // Np doubles = N ints
  for (int mp = warp; mp < d.n_mp; mp += nwarps) {
    const int* wm = t.wmap + (size_t)mp * d.N;
    for (int i = lane; i < d.N; i += 32) tb[i] = wm[idx[i]];
    __syncwarp();
    unsigned par = 0, parB = 0;
    for (int i1 = 1 + lane; i1 < d.N; i1 += 32) {
      int t1 = tb[i1];
      if (i1 >= d.Np && t.subB[t1]) parB ^= 1u;
      for (int i2 = 0; i2 < i1; i2++)
        if (tb[i2] > t1) par ^= 1u;
    }
    par = __reduce_xor_sync(0xffffffffu, par);
    parB = __reduce_xor_sync(0xffffffffu, parB);
    if (lane == 0) {
      sgn[mp] = ((par ^ parB) & 1u) ? -1 : 1;
      s.pb[mp] = (int)parB;
    }
    __syncwarp();
  }
}

// X(i, j) = XF(u_i, d_j) for the current labelling into the padded tile (rows: up electrons).
__device__ __forceinline__ void cta_build_x(const DevDims& d, const DevParams& p, int qp, const int* idx, double* tile) {
  const int Np = d.Np, ld = Np + 1, warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const double* XFq = p.XF + (size_t)qp * d.N * d.N;
  for (int i = warp; i < Np; i += nwarps) {
    const double* row = XFq + (size_t)idx[i] * d.N;
    for (int j = lane; j < Np; j += 32) tile[i * ld + j] = row[idx[Np + j]];
  }
}

// In-place Gauss-Jordan inverse with partial pivoting of the Np x Np tile (the role of
// dgetrf/dgetri, matrix.f90:155-177) and its determinant (-> Pf through the block identity; the role
// of dskpfa, matrix.f90:133-151).  After the call column b of Y = X^{-1} is column s.perm[b] of the
// tile (the row interchanges are not undone in place); dsc[D_DET] = det(X).  Sets iflag[F_SINGULAR]
// when a zero pivot is met.  All threads of the CTA must call it.
__device__ __forceinline__ void cta_gauss_jordan(const DevDims& d, const WS& s) {
  const int n = d.Np, ld = n + 1;
  double* T = s.tile;
  const int tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5, lane = tid & 31, nwarps = nt >> 5;
  if (tid == 0) {
    s.dsc[D_DET] = 1.0;
    s.iflag[F_SINGULAR] = 0;
  }
  for (int k = 0; k < n; k++) {
    if (warp == 0) {
      double best = -1.0;
      int bi = k;
      for (int i = k + lane; i < n; i += 32) {
        double v = fabs(T[i * ld + k]);
        if (v > best) {
          best = v;
          bi = i;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        double ob = __shfl_xor_sync(0xffffffffu, best, o);
        int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (lane == 0) {
        s.iflag[F_PIV] = bi;
        s.dsc[D_PVAL] = best;
        s.dsc[D_PIVOT] = T[bi * ld + k];
        s.perm[k] = bi;
      }
    }
    __syncthreads();
    const int piv = s.iflag[F_PIV];
    if (!(s.dsc[D_PVAL] > 0.0)) {
      if (tid == 0) {
        s.iflag[F_SINGULAR] = 1;
        s.dsc[D_DET] = 0.0;
      }
      __syncthreads();
      return;
    }
    // pivot row (after the interchange) scaled, pivot column saved
    const double pivot = s.dsc[D_PIVOT];
    for (int j = tid; j < n; j += nt) {
      const double rk = T[piv * ld + j], ck = T[j * ld + k];
      if (piv != k) T[piv * ld + j] = T[k * ld + j];  // interchange rows k and piv
      s.rowbuf[j] = rk / pivot;
      s.colbuf[j] = (j == piv) ? T[k * ld + k] : ck;  // column k after the interchange
    }
    if (tid == 0) s.dsc[D_DET] = (piv != k ? -s.dsc[D_DET] : s.dsc[D_DET]) * pivot;
    __syncthreads();
    for (int i = warp; i < n; i += nwarps) {
      const double ci = s.colbuf[i];
      for (int j = lane; j < n; j += 32) {
        double v;
        if (i == k) v = (j == k) ? 1.0 / pivot : s.rowbuf[j];
        else if (j == k) v = -ci / pivot;
        else v = T[i * ld + j] - ci * s.rowbuf[j];
        T[i * ld + j] = v;
      }
    }
    __syncthreads();
  }
  // column b of the inverse is column src(b) of the tile: compose the interchanges in reverse order
  if (tid == 0) {
    int src[RBMPP_MAX_N / 2];
    for (int b = 0; b < n; b++) src[b] = b;
    for (int k = n - 1; k >= 0; k--) {
      const int pk = s.perm[k];
      const int a = src[k];
      src[k] = src[pk];
      src[pk] = a;
    }
    for (int b = 0; b < n; b++) s.perm[b] = src[b];
  }
  __syncthreads();
}

// cosh of a complex angle as sub.f90:40 writes it: (cosh a cos b, sinh a sin b)
__device__ __forceinline__ cplx ccosh_(double a, double b) { return {cosh(a) * cos(b), sinh(a) * sin(b)}; }

// 0.5^alphac prod_f cosh(thetac(qp, f)) (sub.f90:37-41) for the complex angles stored after the Mr real ones
__device__ __forceinline__ cplx complex_factor(const DevDims& d, const double* th, int qp) {
  cplx c = {1.0, 0.0};
  for (int f = 0; f < d.alphac; f++) {
    const int j = d.Mr + 2 * (qp * d.alphac + f);
    c = cscale(cmul(c, ccosh_(th[j], th[j + 1])), 0.5);
  }
  return c;
}

// RBM cosh products per projection for theta vector th (sub.f90:37-46): the real product into rbm and, with
// complex units, the complex factor into rbmc
__device__ __forceinline__ void cta_rbm_factors(const DevDims& d, const double* th, double* rbm, double* rbmc = nullptr) {
  for (int qp = threadIdx.x; qp < d.n_qp; qp += blockDim.x) {
    double r = 1.0;
    for (int f = 0; f < d.alphar; f++) r = r * cosh(th[qp * d.alphar + f]);
    rbm[qp] = r;
    if (d.alphac && rbmc) {
      const cplx c = complex_factor(d, th, qp);
      rbmc[2 * qp] = c.re;
      rbmc[2 * qp + 1] = c.im;
    }
  }
}

// psi_wo_pf(qp) = rbm * sgn(mp) * para_mp(mp) * para_spin_proj(sp)  (sub.f90:47)
__device__ __forceinline__ cplx psi_wo_pf(const DevDims& d, const DevTables& t, double rbm, int sgn_mp, int qp) {
  int mp = qp >> 1, sp = qp & 1;
  cplx c = {rbm * (double)sgn_mp, 0.0};
  cplx pm = {t.para_mp[2 * mp], t.para_mp[2 * mp + 1]};
  c = cmul(c, pm);
  return cscale(c, d.para_sp[sp]);
}

// psi_wo_pf with the complex factor of the workspace's current angles (rbmc) when there are complex units
__device__ __forceinline__ cplx psi_wo_pf_s(const DevDims& d, const DevTables& t, const WS& s, int sgn_mp, int qp) {
  cplx c = psi_wo_pf(d, t, s.rbm[qp], sgn_mp, qp);
  if (d.alphac) c = cmul(c, cplx{s.rbmc[2 * qp], s.rbmc[2 * qp + 1]});
  return c;
}

// calc_amplitude_RBM_PP sub.f90:4-89 for the current (th, pf, sgn): psi[qp], D_PSI0; one draw.
__device__ __forceinline__ void cta_amplitude(const DevDims& d, const DevTables& t, const WS& s, const double* th,
                                     const double* pf, const int* sgn, double* psi, int psi0_slot) {
  cta_rbm_factors(d, th, s.rbm, s.rbmc);
  __syncthreads();
  for (int qp = threadIdx.x; qp < d.n_qp; qp += blockDim.x) {
    cplx c = psi_wo_pf_s(d, t, s, sgn[qp >> 1], qp);
    psi[2 * qp] = c.re * pf[qp];
    psi[2 * qp + 1] = c.im * pf[qp];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double re = 0.0, im = 0.0;
    for (int qp = 0; qp < d.n_qp; qp++) {
      re += psi[2 * qp];
      im += psi[2 * qp + 1];
    }
    s.dsc[psi0_slot] = re;
    s.dsc[psi0_slot + 1] = im;
    (void)grnd(s.mt);  // sub.f90:72
  }
  __syncthreads();
}

// Sums NV values (a power of two, at most 32) over the warp together.  Each halving level trades half of
// the values with the partner lane, so the NV sums take NV - 1 + 5 - log2(NV) shuffles instead of 5 NV.
// Returns the warp total of value lane >> (5 - log2(NV)); v is overwritten.
template <int NV>
__device__ __forceinline__ double warp_transpose_sum(double (&v)[NV], int lane) {
  constexpr int L2 = NV >= 32 ? 5 : NV >= 16 ? 4 : NV >= 8 ? 3 : NV >= 4 ? 2 : NV >= 2 ? 1 : 0;
  static_assert((1 << L2) == NV && NV <= 32, "NV must be a power of two <= 32");
#pragma unroll
  for (int lev = 0; lev < L2; lev++) {
    const int h = NV >> (lev + 1), o = 16 >> lev;
    const bool hi = (lane & o) != 0;
#pragma unroll
    for (int i = 0; i < h; i++) {
      const double keep = hi ? v[h + i] : v[i];
      const double give = hi ? v[i] : v[h + i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, give, o);
    }
  }
  double r = v[0];
#pragma unroll
  for (int o = 16 >> L2; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  return r;
}

// Warp-level gather of the n x n block X(i, j) = XF(idx[i], idx[n + j]) into the tile T (leading dimension
// n + 1), lane <-> column.  Rows go in batches of B whose loads are all issued before any of their stores:
// the compiler cannot move a global load past a shared store it cannot prove disjoint, so a row-at-a-time
// loop would wait one L2 round trip per row.
template <int KPL, int NP, int B>
__device__ __forceinline__ void warp_gather_tile(double* T, const double* XFq, const int* idx, int n_rt, int N) {
  const int n = NP > 0 ? NP : n_rt, ld = n + 1;
  const int lane = threadIdx.x & 31;
  int col[KPL];
#pragma unroll
  for (int q = 0; q < KPL; q++) {
    const int j = lane + 32 * q;
    col[q] = idx[n + (j < n ? j : n - 1)];
  }
  for (int i0 = 0; i0 < n; i0 += B) {
    double v[B][KPL];
#pragma unroll
    for (int ii = 0; ii < B; ii++) {
      const int i = i0 + ii;
      const double* row = XFq + (size_t)idx[i < n ? i : n - 1] * N;
#pragma unroll
      for (int q = 0; q < KPL; q++) v[ii][q] = row[col[q]];
    }
#pragma unroll
    for (int ii = 0; ii < B; ii++) {
      const int i = i0 + ii;
#pragma unroll
      for (int q = 0; q < KPL; q++)
        if (i < n && lane + 32 * q < n) T[i * ld + lane + 32 * q] = v[ii][q];
    }
  }
  __syncwarp();
}

// Warp-level Gauss-Jordan inverse with partial pivoting (the role of dgetrf/dgetri, matrix.f90:155-177) of
// the n x n tile T with leading dimension n + 1 (n = NP when NP > 0, a compile-time size; otherwise n_rt).
// Returns det(X) (0 and singular = true on a zero pivot).  Column b of X^{-1} is column perm[b] of T
// afterwards.  The pivot search holds the pivot column in registers (rows lane + 32 p).  The elimination
// runs over batches of B rows, loading every row of a batch (and its multiplier) before storing any, so a
// step waits a shared-memory round trip per batch rather than per row.  Lanes past the last row or column load
// from a clamped, in-tile index (and discard the value): the compiler may issue a guarded shared load
// unconditionally, and a tile can end at the end of the block's shared memory.
template <int KPL, int NP, int B = 8>
__device__ __forceinline__ double warp_gj(double* T, int n_rt, int* perm, bool& singular) {
  static_assert(32 % B == 0, "row batches must tile a 32-row group");
  const int n = NP > 0 ? NP : n_rt, ld = n + 1;
  const int lane = threadIdx.x & 31;
  int jc[KPL];
#pragma unroll
  for (int q = 0; q < KPL; q++) {
    const int j = lane + 32 * q;
    jc[q] = j < n ? j : n - 1;
  }
  double det = 1.0;
  singular = false;
  for (int k = 0; k < n; k++) {
    double fc[KPL];
    double best = -1.0;
    int bi = k;
#pragma unroll
    for (int p = 0; p < KPL; p++) {
      const int i = lane + 32 * p;
      const double tv = T[(i < n ? i : n - 1) * ld + k];
      fc[p] = (i < n) ? tv : 0.0;
      if (i >= k && i < n) {
        const double v = fabs(fc[p]);
        if (v > best) {
          best = v;
          bi = i;
        }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (!(best > 0.0)) {
      singular = true;
      return 0.0;
    }
    // T(bi, k) and T(k, k) from their lanes
    double pv = 0.0, fkk = 0.0;
#pragma unroll
    for (int p = 0; p < KPL; p++) {
      if (p == (bi >> 5)) pv = fc[p];
      if (p == (k >> 5)) fkk = fc[p];
    }
    const double pivot = __shfl_sync(0xffffffffu, pv, bi & 31);
    fkk = __shfl_sync(0xffffffffu, fkk, k & 31);
    if (lane == 0) perm[k] = bi;
    double r[KPL];
#pragma unroll
    for (int q = 0; q < KPL; q++) {
      const int j = lane + 32 * q;
      const double a = T[k * ld + jc[q]], b = T[bi * ld + jc[q]];
      r[q] = 0.0;
      if (j < n) {
        if (bi != k) T[bi * ld + j] = a;
        r[q] = b / pivot;
      }
    }
    det = (bi != k ? -det : det) * pivot;
    __syncwarp();
    // rows i != k: T(i,j) -= f_i r_j for j != k, with f_i = T(i,k) after the interchange
    // The multiplier of row i is T(i, k) read back from the tile: a broadcast load, issued with the
    // batch's other loads.  After the interchange row bi holds the old row k, so T(bi, k) = fkk.
    auto batch = [&](const int p, const int l0) {
      double tv[B][KPL], fv[B];
#pragma unroll
      for (int ii = 0; ii < B; ii++) {
        const int i = 32 * p + l0 + ii, ic = i < n ? i : n - 1;
        fv[ii] = T[ic * ld + k];
#pragma unroll
        for (int q = 0; q < KPL; q++) tv[ii][q] = T[ic * ld + jc[q]];
      }
#pragma unroll
      for (int ii = 0; ii < B; ii++) {
        const int i = 32 * p + l0 + ii;
        if (i < n && i != k) {
#pragma unroll
          for (int q = 0; q < KPL; q++) {
            const int j = lane + 32 * q;
            if (j < n && j != k) T[i * ld + j] = tv[ii][q] - fv[ii] * r[q];
          }
        }
      }
    };
#pragma unroll
    for (int p = 0; p < KPL; p++) {
      if (32 * p >= n) break;
      if constexpr (NP > 0) {
#pragma unroll
        for (int l0 = 0; l0 < 32; l0 += B)
          if (32 * p + l0 < n) batch(p, l0);
      } else {
#pragma unroll 1
        for (int l0 = 0; l0 < 32 && 32 * p + l0 < n; l0 += B) batch(p, l0);
      }
    }
    __syncwarp();
#pragma unroll
    for (int p = 0; p < KPL; p++) {
      const int i = lane + 32 * p;
      if (i < n && i != k) T[i * ld + k] = -((i == bi) ? fkk : fc[p]) / pivot;
    }
#pragma unroll
    for (int q = 0; q < KPL; q++) {
      const int j = lane + 32 * q;
      if (j < n) T[k * ld + j] = (j == k) ? 1.0 / pivot : r[q];
    }
    __syncwarp();
  }
  // Source column of each column of the inverse: undo the interchanges in reverse, in place.  When step k
  // is undone, positions > k already hold source columns and positions < k are untouched (perm[k'] >= k').
  if (lane == 0)
    for (int k = n - 1; k >= 0; k--) {
      const int pk = perm[k];
      if (pk != k) {
        perm[k] = perm[pk];
        perm[pk] = k;
      } else {
        perm[k] = k;
      }
    }
  __syncwarp();
  return det;
}

// common.cuh -- device-side data layout and helpers shared by the sampler, estimator and SR kernels.
//
// Layout in HBM (all per-walker arrays are walker-major so one CTA streams one walker):
//   XF  [qp][p][q]  M entry for "up electron at site p, down electron at site q" (= -Slater_Elm(p, q+N))
//   XFT [qp][q][p]  its transpose (so both the new row and the new column of X are row gathers)
//   Y   [w][qp][j][k]  X^{-1} (rows: down electrons, cols: up electrons), row-major
//   th  [w][Mr], pf [w][n_qp], psi [w][n_qp] (complex), x/idx/cfg [w][N], mt [w][625]
//
// The Pfaffian matrix of the in-scope spin projection (beta in {0, pi}, spin_projection.f90:29-32) is
// block off-diagonal: M = [[A, X], [-X^T, D]] with A = D = 0 for beta = 0 and A, D of relative size
// cos(pi/2) = 6.1e-17 for beta = pi.  Pf(M) = (-1)^{Np(Np-1)/2} det(X), M^{-1} = [[0, -X^{-T}], [X^{-1}, 0]],
// so every quantity of pfupdate_two.f90 / matrix.f90 / slater.f90:68-170 is carried by the Np x Np
// block X and its inverse Y (Np = N/2).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

// Counts every kernel launch the library issues (process-wide); defined in capi.cu, read through
// rbmpp_query(ctx, 6, ...).
void rbmpp_note_launch();

#define RBMPP_MAX_N 512
#define RBMPP_MAX_KPL 8  // columns per lane in the warp streaming loops: Np <= 256

struct DevDims {
  int L, N, Np, n_mp, n_qp, alphar, Mr, n_slater, Nv, Nv_rbm;
  int alphac, Mc;     // complex RBM units (RBM.f90 thetac): Mc = 2 alphac n_mp complex angles, kept after the
                      //   Mr real ones in every theta array as (re, im) pairs
  int nw, ns, nupdate, nwarm;
  int orb_injective;  // Orbital_Idx is injective within each spin block for one projection
  int pf_sign;        // (-1)^{Np(Np-1)/2}
  int gj_global;      // the direct sampler's Gauss-Jordan tile lives in DevWalkers::gj (too large for SMEM)
  int trace_max;      // records per walker of DevWalkers::trace (0: no chain trace)
  int replay_max;     // checkpoint decisions per walker in DevWalkers::replay (0: none)
  int skip_load;      // verification hook: walker 0 of the streaming sampler never issues its load number
                      //   skip_load (1-based), so the wait on it runs out (0: off)
  int wait_polls;     // poll bound of the streaming sampler's pipeline waits (0: the default 2^22)
  int cplx;           // complex para_mp_trans: psi, H psi and O_k are complex; O keeps two rows per
                      //   configuration (real, imaginary parts: the Ovec_Store columns of calc_phys_quantity.f90:227-228)
  int skew;           // the same-spin blocks of Slater_Elm do not vanish (transverse spin projection): the
                      //   Pfaffian matrix is carried in its full N x N skew form (skew.cu), DevWalkers::Y holds
                      //   [w][qp][N][N] and DevParams::SE the Slater elements
  double J1, J2, shift;
  double sp_cc[2], sp_cs[2], sp_ss[2], para_sp[2];
};

struct DevTables {
  const int* wmap;        // [mp][N]  W_map(i, mp) 0-based  (MP_Trans_Idx)
  const int* winv;        // [mp][N]  inverse permutation of wmap
  const double* para_mp;  // [mp][2]  (re, im)
  const int* orb;         // [p][q]   Orbital_Idx(p, q) 0-based
  const unsigned char* subB;
  const int* bonds;       // [4N][2]  bond_map (i1, i2) for i0 = 1..4, i1 = 1..N
};

struct DevParams {
  const double* Wr;   // [f][N]   Wrirr(iw, f)
  const double* br;   // [f]
  const double* Wc;   // [f][N][2] Wcirr(iw, f) as (re, im)
  const double* bc;   // [f][2]
  const double* XF;   // [qp][N][N]
  const double* XFT;  // [qp][N][N]
  const double* SE;   // [qp][2N][2N] Slater_Elm(r, r') row-major (skew form only)
};

struct DevWalkers {
  int8_t* x;       // [w][N]
  int16_t* idx;    // [w][N]  Ele_Idx (0-based site of electron)
  int16_t* cfg;    // [w][N]  Ele_Cfg (0-based electron on site)
  double* th;      // [w][Mr]
  int8_t* sgn;     // [w][n_mp]
  double* pf;      // [w][n_qp]
  double* psi;     // [w][n_qp][2]
  double* Y;       // [w][qp][Np][Np]
  uint32_t* mt;    // [w][625]  624 words + mti
  int* nfastup;    // [w]
  int* naccept;    // [w]  accepted moves of the stored sweeps (i0 > 0)
  int* nacc_all;   // [w]  accepted moves of all sweeps
  int* status;     // [w]
  int8_t* xs;      // [w][s][N]
  double* pfs;     // [w][s][n_qp]
  double* psis;    // [w][s][n_qp+1][2]
  double* gj;      // [w][Np][Np+1] Gauss-Jordan scratch when DevDims::gj_global, else null
  int* events;     // [w][5] last make_sample: global flips tried, flips accepted, make_initial_x re-seeds,
                   //        Nfastup checkpoints (make_sample.f90:135-158, :61, :74-128), trace records
  double* trace;   // [w][trace_max][6] chain trace in draw order (null when trace_max = 0); records:
                   //   {0, i1, i2, ratio^2, u, accepted}   exchange proposal (make_sample.f90:160-220)
                   //   {1, i0, inverse drift, Pf drift, Nfastup before, after}   checkpoint (:74-128)
                   //   {2, 0, 0, ratio^2, u, accepted}     global spin flip (:135-158)
                   //   {3, 0, 0, 0, 0, 0}                  make_initial_x re-seed of a continued chain (:61)
  const int* replay;  // [w][replay_max][2] verification replay of checkpoint decisions {Nfastup after, extra
                      //   draw of :122}, used in place of the drift test for the first replay_max checkpoints
};

// One context of a batched launch (several lattices / couplings in one kernel)
struct BatchInst {
  DevDims d;
  DevTables t;
  DevParams p;
  DevWalkers W;
};

// ---- status codes (same numbering as include/rbmpp.h) ----
#define ST_CONFIG 2
#define ST_SIGN 3
#define ST_THETA 4
#define ST_CANDIDATE 5
#define ST_INITX 6
#define ST_SKEW 7
#define ST_SINGULAR 8

// ------------------------------------------------------------------------------------------------
// MT19937 with the reference's seeding and output mapping (mt.f:6-102).  The state lives in shared
// memory: mt[0..623] words, mt[624] = mti.  Only one thread draws.
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t mt_next(uint32_t* mt) {
  const uint32_t UMASK = 0x80000000u, LMASK = 0x7fffffffu, MATA = 0x9908b0dfu;
  uint32_t mti = mt[624];
  if (mti >= 624) {
    int kk;
    uint32_t y;
    for (kk = 0; kk < 624 - 397; kk++) {
      y = (mt[kk] & UMASK) | (mt[kk + 1] & LMASK);
      mt[kk] = mt[kk + 397] ^ (y >> 1) ^ ((y & 1u) ? MATA : 0u);
    }
    for (; kk < 623; kk++) {
      y = (mt[kk] & UMASK) | (mt[kk + 1] & LMASK);
      mt[kk] = mt[kk - 227] ^ (y >> 1) ^ ((y & 1u) ? MATA : 0u);
    }
    y = (mt[623] & UMASK) | (mt[0] & LMASK);
    mt[623] = mt[396] ^ (y >> 1) ^ ((y & 1u) ? MATA : 0u);
    mti = 0;
  }
  uint32_t y = mt[mti];
  mt[624] = mti + 1;
  y ^= (y >> 11);
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= (y >> 18);
  return y;
}

__device__ __forceinline__ double grnd(uint32_t* mt) { return __ddiv_rn((double)mt_next(mt), 4294967295.0); }

// nran(n) = mod(int(dble(n)*grnd()), n) + 1   (make_sample.f90:254,317)
__device__ __forceinline__ int nran(uint32_t* mt, int n) {
  return ((int)__dmul_rn((double)n, grnd(mt))) % n + 1;
}

// ------------------------------------------------------------------------------------------------
// warp / block reductions
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

struct cplx {
  double re, im;
};
__device__ __forceinline__ cplx cmul(cplx a, cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cplx cscale(cplx a, double s) { return {a.re * s, a.im * s}; }
__device__ __forceinline__ double cabs_(cplx a) { return hypot(a.re, a.im); }

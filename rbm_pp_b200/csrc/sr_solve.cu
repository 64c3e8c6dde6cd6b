// sr_solve.cu -- the solve of the SR step on the device: the blocked Cholesky factorisation and the two
// triangular solves that replace pdposv('U') (SR_pdposv.f90:200-249), the exact S applied matrix-free through
// the per-sample derivatives O (S_raw x = O^T (O x), calc_phys_quantity.f90:240), and the vector steps of the
// preconditioned conjugate-gradient refinement that uses both.  Matrices are column-major (Fortran layout).
//
// Cholesky (upper, A = U^T U, in place), panels of NB = 128 columns:
//   potrf_block_kernel   one CTA factors the NB x NB diagonal block in shared memory (32-column sub-panels:
//                        a warp factors each 32 x 32 diagonal piece in registers) and keeps 1 / U(i, i);
//   panel_kernel         U_kj = U_kk^{-T} A_kj by forward substitution, one warp per column j, U_kk in shared
//                        memory;
//   gemm_atb_upper<true> (linalg.cu) the trailing update A_22 -= U_12^T U_12.
//   invert_blocks_kernel all diagonal blocks inverted at once afterwards (one CTA per block).
// Triangular solves: one launch per block step; every CTA applies the inverted diagonal block to the block's
// right-hand side (redundantly, staged from L2) and then updates its share of the rest of the vector.
#include <cuda_runtime.h>
#include <stdint.h>

#include "tma.cuh"

void rbmpp_note_launch();  // capi.cu: counts kernel launches
cudaError_t rbmpp_gemm_atb_upper_acc(int n, int K, const double* A, long long sk, long long si, double alpha,
                                     double* C, long long ldc, int row0, cudaStream_t st);
cudaError_t rbmpp_gemv_ot(int, int, const double*, const double*, const double*, double*, double*, double*, int,
                          cudaStream_t);
cudaError_t rbmpp_gemv_o(int, int, const double*, const double*, double*, cudaStream_t);

namespace {

constexpr int NB = 128;
constexpr int NQ = NB / 32;  // rows of a block column held by one lane
// An inverted diagonal block is kept as two packed upper triangles (NB (NB + 1) / 2 doubles each, 16-byte
// multiples): by rows, V(q, q..NB-1) from off_rows(q), for the forward solve (y_p = sum_{q <= p} V(q, p) b_q
// reads consecutive p), and by columns, V(0..q, q) from off_cols(q), for the backward one
// (x_p = sum_{q >= p} V(p, q) y_q reads consecutive p).
constexpr int PK = NB * (NB + 1) / 2;
__host__ __device__ __forceinline__ int off_rows(int q) { return q * NB - q * (q - 1) / 2; }
__host__ __device__ __forceinline__ int off_cols(int q) { return q * (q + 1) / 2; }

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Copies the upper triangle (or all, FULL) of the nb x nb block at (k0, k0) of A into shared memory,
// dst[i * si + j * sj] = A(k0 + i, k0 + j), with eight loads in flight per thread before their stores (a
// store waits for its load, so a one-element loop would pay a full memory latency per element).
template <bool FULL>
__device__ __forceinline__ void load_block(int nb, const double* __restrict__ A, long long lda, int k0, double* dst,
                                           int si, int sj) {
  const int tot = nb * nb, step = blockDim.x;
  for (int e0 = threadIdx.x; e0 < tot; e0 += 8 * step) {
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int e = e0 + u * step, i = e % nb, j = e / nb;
      v[u] = (e < tot && (FULL || i <= j)) ? A[(long long)(k0 + i) + lda * (k0 + j)] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int e = e0 + u * step, i = e % nb, j = e / nb;
      if (e < tot && (FULL || i <= j)) dst[i * si + j * sj] = v[u];
    }
  }
}

// ---------------------------------------------------------------------------------------------------
// Diagonal block: Cholesky of the nb x nb block at (k0, k0) and the reciprocals of its diagonal.
// T (shared, column-major, ld NB + 1) holds the block; warp 0 factors each 32 x 32 diagonal piece with the
// piece's column c in lane c, then all warps solve the piece's row panel and update the trailing triangle.
// ---------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(512, 1)
    potrf_block_kernel(int n, double* __restrict__ A, long long lda, int k0, double* __restrict__ rdiag_out,
                       int* __restrict__ info) {
  extern __shared__ double T[];  // [NB][NB + 1] column-major: T[i + (NB + 1) j]
  __shared__ double rdiag[NB];   // 1 / U(i, i)
  constexpr int LD = NB + 1;
  const int nb = min(NB, n - k0);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nwarps = blockDim.x >> 5;
  for (int e = tid; e < NB * LD; e += blockDim.x) T[e] = 0.0;
  __syncthreads();
  load_block<false>(nb, A, lda, k0, T, 1, LD);
  __syncthreads();
  for (int p0 = 0; p0 < nb; p0 += 32) {
    const int pw = min(32, nb - p0);
    // (1) 32 x 32 piece in registers: col[r] = T(p0 + r, p0 + lane)
    if (warp == 0) {
      double col[32];
#pragma unroll
      for (int r = 0; r < 32; r++) col[r] = (r < pw && lane < pw) ? T[(p0 + r) + LD * (p0 + lane)] : 0.0;
#pragma unroll
      for (int k = 0; k < 32; k++) {
        if (k < pw) {
          double dkk = __shfl_sync(0xffffffffu, col[k], k);
          if (!(dkk > 0.0)) {
            if (lane == 0 && *info == 0) *info = k0 + p0 + k + 1;
            dkk = 1.0;
          }
          const double ukk = sqrt(dkk), rk = 1.0 / ukk;
          if (lane == 0) rdiag[p0 + k] = rk;
          // row k of U: U(k, c) = T(k, c) / U(k, k) for c > k (lane c), U(k, k) on lane k
          double ukc = col[k] * rk;
          if (lane == k) ukc = ukk;
          if (lane >= k) col[k] = ukc;
          // rows r > k of columns c >= r: T(r, c) -= U(k, r) U(k, c)
#pragma unroll
          for (int r = k + 1; r < 32; r++) {
            const double ukr = __shfl_sync(0xffffffffu, ukc, r);
            if (lane > k && lane >= r) col[r] -= ukr * ukc;
          }
        }
      }
#pragma unroll
      for (int r = 0; r < 32; r++)
        if (r < pw && lane < pw && r <= lane) T[(p0 + r) + LD * (p0 + lane)] = col[r];
    }
    __syncthreads();
    // (2) row panel: U(p0:p0+pw, c) = U_pp^{-T} T(p0:p0+pw, c) for c >= p0 + pw, one warp per column
    for (int c = p0 + pw + warp; c < nb; c += nwarps) {
      double x = (lane < pw) ? T[(p0 + lane) + LD * c] : 0.0;
      for (int r = 0; r < pw; r++) {
        const double xr = __shfl_sync(0xffffffffu, x, r) * rdiag[p0 + r];
        if (lane == r) x = xr;
        if (lane > r && lane < pw) x -= T[(p0 + r) + LD * (p0 + lane)] * xr;
      }
      if (lane < pw) T[(p0 + lane) + LD * c] = x;
    }
    __syncthreads();
    // (3) trailing triangle: T(i, j) -= sum_r U(p0 + r, i) U(p0 + r, j) for p0 + pw <= i <= j
    const int m = nb - (p0 + pw);
    for (int e = tid; e < m * m; e += blockDim.x) {
      const int i = p0 + pw + e % m, j = p0 + pw + e / m;
      if (i <= j) {
        double s = T[i + LD * j];
        for (int r = 0; r < pw; r++) s -= T[(p0 + r) + LD * i] * T[(p0 + r) + LD * j];
        T[i + LD * j] = s;
      }
    }
    __syncthreads();
  }
  for (int e = tid; e < nb * nb; e += blockDim.x) {
    const int i = e % nb, j = e / nb;
    if (i <= j) A[(long long)(k0 + i) + lda * (k0 + j)] = T[i + LD * j];
  }
  for (int i = tid; i < nb; i += blockDim.x) rdiag_out[k0 + i] = rdiag[i];
}

// U(k0:k0+nb, j) = U_kk^{-T} A(k0:k0+nb, j) for j >= k0 + nb by forward substitution: one warp per column,
// lane holding rows lane + 32 q; U_kk (upper) and its reciprocal diagonal in shared memory.
__global__ void __launch_bounds__(512) panel_kernel(int n, double* __restrict__ A, long long lda, int k0,
                                                    const double* __restrict__ rdiag) {
  extern __shared__ double U[];  // [NB][NB + 1] column-major
  __shared__ double rd[NB];
  constexpr int LD = NB + 1;
  const int nb = min(NB, n - k0);
  load_block<false>(nb, A, lda, k0, U, 1, LD);
  for (int i = threadIdx.x; i < nb; i += blockDim.x) rd[i] = rdiag[k0 + i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  for (int j = k0 + nb + blockIdx.x * nwarps + warp; j < n; j += gridDim.x * nwarps) {
    double* col = A + lda * j + k0;
    double x[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) x[q] = (lane + 32 * q < nb) ? col[lane + 32 * q] : 0.0;
    // x_r = (b_r - sum_{s < r} U(s, r) x_s) / U(r, r), applied column by column of U^T: after x_r,
    // x_p -= U(r, p) x_r for p > r
#pragma unroll
    for (int qr = 0; qr < NQ; qr++) {
      for (int rl = 0; rl < 32; rl++) {
        const int r = 32 * qr + rl;
        if (r >= nb) break;
        const double xr = __shfl_sync(0xffffffffu, x[qr], rl) * rd[r];
        if (lane == rl) x[qr] = xr;
#pragma unroll
        for (int q = qr; q < NQ; q++) {
          const int p = lane + 32 * q;
          if (p > r && p < nb) x[q] -= U[r + LD * p] * xr;
        }
      }
    }
#pragma unroll
    for (int q = 0; q < NQ; q++)
      if (lane + 32 * q < nb) col[lane + 32 * q] = x[q];
  }
}

// ---------------------------------------------------------------------------------------------------
// Inverses of all diagonal factor blocks at once (one CTA per block, after the factorisation): V_k = U_kk^{-1}
// (upper), column c by back substitution v_i = (delta_ic - sum_{i < j <= c} U(i, j) v_j) / U(i, i), one warp
// per column, U_kk in shared memory.  dinv: nblk triangles packed by rows, then nblk packed by columns.
// ---------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(512, 1) invert_blocks_kernel(int n, const double* __restrict__ A, long long lda,
                                                               const double* __restrict__ rdiag,
                                                               double* __restrict__ dinv) {
  extern __shared__ double U[];  // [NB][NB + 1] column-major
  constexpr int LD = NB + 1;
  const int k0 = blockIdx.x * NB, nb = min(NB, n - k0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  load_block<false>(nb, A, lda, k0, U, 1, LD);
  __syncthreads();
  double* VR = dinv + (size_t)blockIdx.x * PK;                          // packed by rows
  double* VC = dinv + (size_t)(gridDim.x + blockIdx.x) * PK;             // packed by columns
  for (int c = warp; c < NB; c += nwarps) {
    double v[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) v[q] = 0.0;
    if (c < nb) {
      for (int i = c; i >= 0; i--) {
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < NQ; q++) {
          const int j = lane + 32 * q;
          if (j > i && j <= c) s = fma(U[i + LD * j], v[q], s);
        }
        s = wsum(s);
        const double vi = ((i == c ? 1.0 : 0.0) - s) * rdiag[k0 + i];
#pragma unroll
        for (int q = 0; q < NQ; q++)
          if (lane + 32 * q == i) v[q] = vi;
      }
    }
#pragma unroll
    for (int q = 0; q < NQ; q++) {
      const int i = lane + 32 * q;  // V(i, c), i <= c
      if (i <= c) {
        const double vi = (c < nb && i < nb) ? v[q] : 0.0;
        VR[off_rows(i) + (c - i)] = vi;
        VC[off_cols(c) + i] = vi;
      }
    }
  }
}

// ---------------------------------------------------------------------------------------------------
// Triangular solves with the inverted diagonal blocks, one launch per block step.  Every CTA stages V_k in
// shared memory and forms the block's result itself: forward U^T y = b, y_k = V_k^T b_k, then
// b_j -= U(k-block, j) . y_k beyond the block (four columns per warp at a time); backward U x = y,
// x_k = V_k y_k, then y_i -= U(i, k-block) . x_k for i < k0.  The block's result goes to a separate vector, so
// no CTA reads what another one writes within the step.
// ---------------------------------------------------------------------------------------------------
// Vectors another CTA may have written since this CTA last read them are loaded past L1 (__ldcg) when the
// steps run inside one persistent launch.
template <bool COH>
__device__ __forceinline__ double ldv(const double* p) {
  return COH ? __ldcg(p) : *p;
}

// A packed triangle Vp (PK doubles) and the block's right-hand side rhs[0 .. nb) into shared memory
template <bool COH>
__device__ __forceinline__ void stage_v(int nb, const double* __restrict__ Vp, const double* rhs, double* Vs,
                                        double* sb) {
  const int step = blockDim.x;
  for (int e0 = threadIdx.x; e0 < PK; e0 += 8 * step) {
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) v[u] = (e0 + u * step < PK) ? Vp[e0 + u * step] : 0.0;
#pragma unroll
    for (int u = 0; u < 8; u++)
      if (e0 + u * step < PK) Vs[e0 + u * step] = v[u];
  }
  for (int p = threadIdx.x; p < nb; p += blockDim.x) sb[p] = ldv<COH>(rhs + p);
  __syncthreads();
}

struct StepSmem {
  double* Vs;  // a packed triangle (PK)
  double *sb, *sy, *hred, *red8;  // [NB], [NB], [2][NB], [8][32]
};

// One forward block step by CTA bid of nbk: y_k = V_k^T b_k into y (CTA 0 stores it), b_j -= U(k-block, j) . y_k
// V: the block's triangle packed by rows (staged here), or null when sm.Vs already holds it and only the
// right-hand side is to be staged
template <bool COH>
__device__ __forceinline__ void fwd_step(int n, const double* __restrict__ A, long long lda, int k0,
                                         const double* __restrict__ V, double* b, double* y, const StepSmem& sm,
                                         int bid, int nbk) {
  const int nb = min(NB, n - k0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  if (V) {
    stage_v<COH>(nb, V, b + k0, sm.Vs, sm.sb);
  } else {
    for (int p = threadIdx.x; p < nb; p += blockDim.x) sm.sb[p] = ldv<COH>(b + k0 + p);
    __syncthreads();
  }
  // sy[p] = sum_{q <= p} V(q, p) sb[q]: two threads per p (alternate q), consecutive p on consecutive lanes
  {
    const int p = threadIdx.x & (NB - 1), half = threadIdx.x / NB;
    double a0 = 0.0, a1 = 0.0;
    if (p < nb)
      for (int q = half; q <= p; q += 4) {
        a0 = fma(sm.Vs[off_rows(q) + p - q], sm.sb[q], a0);
        if (q + 2 <= p) a1 = fma(sm.Vs[off_rows(q + 2) + p - q - 2], sm.sb[q + 2], a1);
      }
    sm.hred[half * NB + p] = a0 + a1;
  }
  __syncthreads();
  for (int p = threadIdx.x; p < nb; p += blockDim.x) sm.sy[p] = sm.hred[p] + sm.hred[NB + p];
  __syncthreads();
  if (bid == 0)
    for (int p = threadIdx.x; p < nb; p += blockDim.x) y[k0 + p] = sm.sy[p];
  // b_j -= U(k-block, j) . y_k: four columns per warp at a time, all their loads issued before any sum
  double yl[NQ];
#pragma unroll
  for (int q = 0; q < NQ; q++) yl[q] = (lane + 32 * q < nb) ? sm.sy[lane + 32 * q] : 0.0;
  const int j0 = k0 + nb, ncol = n - j0, stride = nbk * nwarps;
  for (int c0 = (bid * nwarps + warp) * 4; c0 < ncol; c0 += stride * 4) {
    double v[4][NQ];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const double* col = A + lda * (j0 + c0 + u) + k0;
#pragma unroll
      for (int q = 0; q < NQ; q++) v[u][q] = (c0 + u < ncol && lane + 32 * q < nb) ? col[lane + 32 * q] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      double s = 0.0;
#pragma unroll
      for (int q = 0; q < NQ; q++) s = fma(v[u][q], yl[q], s);
      s = wsum(s);
      if (lane == 0 && c0 + u < ncol) b[j0 + c0 + u] = ldv<COH>(b + j0 + c0 + u) - s;
    }
  }
}

// One backward block step: x_k = V_k y_k into x (CTA 0 stores it), y_i -= U(i, k-block) . x_k for i < k0
// V: the block's triangle packed by columns (staged here), or null when sm.Vs already holds it
template <bool COH>
__device__ __forceinline__ void bwd_step(int n, const double* __restrict__ A, long long lda, int k0,
                                         const double* __restrict__ V, double* y, double* x, const StepSmem& sm,
                                         int bid, int nbk) {
  const int nb = min(NB, n - k0);
  const int lane = threadIdx.x & 31, wg = threadIdx.x >> 5;
  if (V) {
    stage_v<COH>(nb, V, y + k0, sm.Vs, sm.sb);
  } else {
    for (int p = threadIdx.x; p < nb; p += blockDim.x) sm.sb[p] = ldv<COH>(y + k0 + p);
    __syncthreads();
  }
  // sx[p] = sum_{q >= p} V(p, q) sb[q]: two threads per p (alternate q), consecutive p on consecutive lanes
  {
    const int p = threadIdx.x & (NB - 1), half = threadIdx.x / NB;
    double a0 = 0.0, a1 = 0.0;
    if (p < nb)
      for (int q = p + half; q < nb; q += 4) {
        a0 = fma(sm.Vs[off_cols(q) + p], sm.sb[q], a0);
        if (q + 2 < nb) a1 = fma(sm.Vs[off_cols(q + 2) + p], sm.sb[q + 2], a1);
      }
    sm.hred[half * NB + p] = a0 + a1;
  }
  __syncthreads();
  double* sx = sm.sy;
  for (int p = threadIdx.x; p < nb; p += blockDim.x) sx[p] = sm.hred[p] + sm.hred[NB + p];
  __syncthreads();
  if (bid == 0)
    for (int p = threadIdx.x; p < nb; p += blockDim.x) x[k0 + p] = sx[p];
  // y_i -= U(i, k-block) . x_k for i < k0: 32 rows per CTA pass, its 8 warps 16 columns each (each lane one
  // row, coalesced across the warp); the 8 partial sums of a row meet in shared memory
  for (int i0 = bid * 32; i0 < k0; i0 += nbk * 32) {
    const int i = i0 + lane;
    double a[16];
#pragma unroll
    for (int t = 0; t < 16; t++) {
      const int p = wg * 16 + t;
      a[t] = (i < k0 && p < nb) ? A[(long long)i + lda * (k0 + p)] : 0.0;
    }
    double s = 0.0;
#pragma unroll
    for (int t = 0; t < 16; t++) {
      const int p = wg * 16 + t;
      s = fma(a[t], p < nb ? sx[p] : 0.0, s);
    }
    sm.red8[wg * 32 + lane] = s;
    __syncthreads();
    if (wg == 0 && i < k0) {
      double t8 = 0.0;
      for (int g = 0; g < 8; g++) t8 += sm.red8[g * 32 + lane];
      y[i] = ldv<COH>(y + i) - t8;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) trsv_fwd_step(int n, const double* __restrict__ A, long long lda, int k0,
                                                     const double* __restrict__ V, double* b, double* y) {
  extern __shared__ double Vs[];
  __shared__ double sb[NB], sy[NB], hred[2 * NB], red8[8 * 32];
  fwd_step<false>(n, A, lda, k0, V, b, y, StepSmem{Vs, sb, sy, hred, red8}, blockIdx.x, gridDim.x);
}

__global__ void __launch_bounds__(256) trsv_bwd_step(int n, const double* __restrict__ A, long long lda, int k0,
                                                     const double* __restrict__ V, double* y, double* x) {
  extern __shared__ double Vs[];
  __shared__ double sb[NB], sy[NB], hred[2 * NB], red8[8 * 32];
  bwd_step<false>(n, A, lda, k0, V, y, x, StepSmem{Vs, sb, sy, hred, red8}, blockIdx.x, gridDim.x);
}

// Barrier of all CTAs of a cooperative launch: bar[0] arrival count, bar[1] generation, bar[2] set to 1 when a
// wait ran out (bounded: the CTA then goes on, and the host reports the error).
__device__ __forceinline__ void grid_sync(unsigned* bar, unsigned nblocks) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = bar + 1;
    const unsigned g = *gen;
    __threadfence();
    if (atomicAdd(bar, 1u) + 1u == nblocks) {
      bar[0] = 0u;
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      for (int it = 0; *gen == g; it++) {
        if (it > (1 << 24)) {
          atomicExch(bar + 2, 1u);
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

// Both triangular solves in one cooperative launch (all CTAs resident), a grid barrier between block steps:
// U^T y = b (y in tmp, b consumed), then U x = y (x in b).  Step s uses triangle s of the sequence (forward
// blocks 0..nblk-1 packed by rows, then backward blocks nblk-1..0 packed by columns); thread 0 copies the next
// step's triangle into the other shared-memory buffer (one bulk copy) while the current step computes.
__global__ void __launch_bounds__(256, 1) potrs_persistent_kernel(int n, const double* __restrict__ A,
                                                                  const double* __restrict__ dinv, double* b,
                                                                  double* tmp, unsigned* bar) {
  extern __shared__ __align__(128) double Vbuf[];  // [2][PK]
  __shared__ double sb[NB], sy[NB], hred[2 * NB], red8[8 * 32];
  __shared__ __align__(8) uint64_t full[2];
  const int nblk = (n + NB - 1) / NB, nsteps = 2 * nblk;
  auto tri = [&](int st) -> const double* {
    return st < nblk ? dinv + (size_t)st * PK : dinv + (size_t)(nblk + (2 * nblk - 1 - st)) * PK;
  };
  constexpr uint32_t kBytes = PK * sizeof(double);
  if (threadIdx.x == 0) {
    mbar_init(&full[0], 1);
    mbar_init(&full[1], 1);
    fence_mbar_init();
    mbar_arrive_expect_tx(&full[0], kBytes);
    bulk_load(Vbuf, tri(0), kBytes, &full[0]);
  }
  __syncthreads();
  for (int st = 0; st < nsteps; st++) {
    const int buf = st & 1;
    if (threadIdx.x == 0 && st + 1 < nsteps) {
      fence_proxy_async_smem();  // the other buffer's generic reads (step st - 1) come before its refill
      mbar_arrive_expect_tx(&full[buf ^ 1], kBytes);
      bulk_load(Vbuf + (buf ^ 1) * PK, tri(st + 1), kBytes, &full[buf ^ 1]);
    }
    if (!mbar_wait(&full[buf], (uint32_t)((st >> 1) & 1))) {
      atomicExch(bar + 2, 1u);
      // the copy may still land: wait for it (bounded) before its buffer is reused or the CTA exits
      (void)mbar_wait(&full[buf], (uint32_t)((st >> 1) & 1));
    }
    const StepSmem sm{Vbuf + buf * PK, sb, sy, hred, red8};
    if (st < nblk) {
      fwd_step<true>(n, A, n, st * NB, nullptr, b, tmp, sm, blockIdx.x, gridDim.x);
    } else {
      const int kb = 2 * nblk - 1 - st;
      bwd_step<true>(n, A, n, kb * NB, nullptr, tmp, b, sm, blockIdx.x, gridDim.x);
    }
    if (st + 1 < nsteps) grid_sync(bar, gridDim.x);
  }
}

// ---------------------------------------------------------------------------------------------------
// z = O^T (O y) in one pass over O (ns rows of nv FP64): each CTA keeps y and its partial z in shared memory
// and takes groups of kRows rows; the second read of a group's rows (z += t_r O_r) hits L2.  zpart[block][k];
// the partials are summed in block order afterwards, so the result does not depend on scheduling.
// ---------------------------------------------------------------------------------------------------
constexpr int kGramThreads = 512, kRows = 4;

template <bool VEC>
__global__ void __launch_bounds__(kGramThreads, 1)
    gram_apply_kernel(int ns, int nv, const double* __restrict__ O, const double* __restrict__ y,
                      double* __restrict__ zpart) {
  extern __shared__ double sh[];
  double* ys = sh;
  double* zs = sh + nv;
  double* red = zs + nv;  // [2][kRows][32]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int nwarps = kGramThreads / 32;
  for (int k = tid; k < nv; k += kGramThreads) {
    ys[k] = y[k];
    zs[k] = 0.0;
  }
  __syncthreads();
  const int ngroups = (ns + kRows - 1) / kRows;
  int buf = 0;
  for (int gi = blockIdx.x; gi < ngroups; gi += gridDim.x, buf ^= 1) {
    const int s0 = gi * kRows, nr = min(kRows, ns - s0);
    const double* Og = O + (size_t)s0 * nv;
    double d[kRows];
#pragma unroll
    for (int r = 0; r < kRows; r++) d[r] = 0.0;
    if (VEC) {
      const int nh = nv >> 1;
      for (int k2 = tid; k2 < nh; k2 += kGramThreads) {
        const double2 yk = reinterpret_cast<const double2*>(ys)[k2];
#pragma unroll
        for (int r = 0; r < kRows; r++)
          if (r < nr) {
            const double2 o = reinterpret_cast<const double2*>(Og + (size_t)r * nv)[k2];
            d[r] = fma(o.x, yk.x, d[r]);
            d[r] = fma(o.y, yk.y, d[r]);
          }
      }
    } else {
      for (int k = tid; k < nv; k += kGramThreads) {
        const double yk = ys[k];
#pragma unroll
        for (int r = 0; r < kRows; r++)
          if (r < nr) d[r] = fma(Og[(size_t)r * nv + k], yk, d[r]);
      }
    }
#pragma unroll
    for (int r = 0; r < kRows; r++) {
      const double v = wsum(d[r]);
      if (lane == 0) red[(buf * kRows + r) * 32 + warp] = v;
    }
    __syncthreads();
    double t[kRows];
#pragma unroll
    for (int r = 0; r < kRows; r++) {
      double a = 0.0;
      for (int w = 0; w < nwarps; w++) a += red[(buf * kRows + r) * 32 + w];
      t[r] = a;
    }
    if (VEC) {
      const int nh = nv >> 1;
      for (int k2 = tid; k2 < nh; k2 += kGramThreads) {
        double2 z = reinterpret_cast<double2*>(zs)[k2];
#pragma unroll
        for (int r = 0; r < kRows; r++)
          if (r < nr) {
            const double2 o = __ldcs(reinterpret_cast<const double2*>(Og + (size_t)r * nv) + k2);
            z.x = fma(t[r], o.x, z.x);
            z.y = fma(t[r], o.y, z.y);
          }
        reinterpret_cast<double2*>(zs)[k2] = z;
      }
    } else {
      for (int k = tid; k < nv; k += kGramThreads) {
        double z = zs[k];
#pragma unroll
        for (int r = 0; r < kRows; r++)
          if (r < nr) z = fma(t[r], Og[(size_t)r * nv + k], z);
        zs[k] = z;
      }
    }
  }
  __syncthreads();
  for (int k = tid; k < nv; k += kGramThreads) zpart[(size_t)blockIdx.x * nv + k] = zs[k];
}

__global__ void sum_blocks(int nv, int nparts, const double* __restrict__ part, double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nv) return;
  double a = 0.0;
  for (int c = 0; c < nparts; c++) a += part[(size_t)c * nv + k];
  out[k] = a;
}

// ---------------------------------------------------------------------------------------------------
// Vector steps of the refinement (one CTA of 1024 threads over the nv-vectors; sums in a fixed order).
// The conditioned matrix of SR_pdposv.f90:4-170 is A = D (S_raw / norm - m m^T) D + sigma I, with
// D = diag(1 on the RBM block, scal on the Pfaffian block) and m = Ovec / norm.
// ---------------------------------------------------------------------------------------------------
enum { SC_MX = 0, SC_RZ = 1, SC_RR = 2, SC_PAP = 3, SC_GG = 4, SC_ALPHA = 5 };

__device__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = wsum(v);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double a = 0.0;
  for (int w = 0; w < nw; w++) a += red[w];
  return a;
}

// xs = D x, sc[SC_MX] = m . xs
__global__ void __launch_bounds__(1024) sr_pre_kernel(int nv, int nrbm, const double* __restrict__ x, double scal,
                                                      const double* __restrict__ m, double* __restrict__ xs,
                                                      double* __restrict__ sc) {
  __shared__ double red[32];
  double a = 0.0;
  for (int k = threadIdx.x; k < nv; k += blockDim.x) {
    const double v = k < nrbm ? x[k] : x[k] * scal;
    xs[k] = v;
    a = fma(m[k], v, a);
  }
  a = block_sum(a, red);
  if (threadIdx.x == 0) sc[SC_MX] = a;
}

// y = D (z / norm - m sc[SC_MX]) + sigma x
__global__ void sr_post_kernel(int nv, int nrbm, const double* __restrict__ z, const double* __restrict__ m,
                               const double* __restrict__ sc, const double* __restrict__ x, double scal, double sigma,
                               double norm, double* __restrict__ y) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nv) return;
  const double v = z[k] / norm - m[k] * sc[SC_MX];
  y[k] = (k < nrbm ? v : v * scal) + sigma * x[k];
}

// r = g - Ax; sc[SC_GG] = g.g, sc[SC_RR] = r.r
__global__ void __launch_bounds__(1024) pcg_start_kernel(int nv, const double* __restrict__ g,
                                                         const double* __restrict__ ax, double* __restrict__ r,
                                                         double* __restrict__ sc) {
  __shared__ double red[32];
  double gg = 0.0, rr = 0.0;
  for (int k = threadIdx.x; k < nv; k += blockDim.x) {
    const double v = g[k] - ax[k];
    r[k] = v;
    gg = fma(g[k], g[k], gg);
    rr = fma(v, v, rr);
  }
  gg = block_sum(gg, red);
  rr = block_sum(rr, red);
  if (threadIdx.x == 0) {
    sc[SC_GG] = gg;
    sc[SC_RR] = rr;
  }
}

// mode 0: p = z, rz = r.z (first direction); mode 1: rz' = r.z, p = z + (rz' / rz) p
__global__ void __launch_bounds__(1024) pcg_dir_kernel(int nv, const double* __restrict__ r,
                                                       const double* __restrict__ z, double* __restrict__ p,
                                                       double* __restrict__ sc, int mode) {
  __shared__ double red[32];
  double a = 0.0;
  for (int k = threadIdx.x; k < nv; k += blockDim.x) a = fma(r[k], z[k], a);
  a = block_sum(a, red);
  const double beta = mode ? a / sc[SC_RZ] : 0.0;
  for (int k = threadIdx.x; k < nv; k += blockDim.x) p[k] = mode ? fma(beta, p[k], z[k]) : z[k];
  __syncthreads();
  if (threadIdx.x == 0) sc[SC_RZ] = a;
}

// alpha = rz / (p.Ap) (0 when p.Ap <= 0); x += alpha p; r -= alpha Ap; sc[SC_RR] = r.r; sc[SC_PAP] = p.Ap
__global__ void __launch_bounds__(1024) pcg_step_kernel(int nv, const double* __restrict__ p,
                                                        const double* __restrict__ ap, double* __restrict__ x,
                                                        double* __restrict__ r, double* __restrict__ sc) {
  __shared__ double red[32];
  double a = 0.0;
  for (int k = threadIdx.x; k < nv; k += blockDim.x) a = fma(p[k], ap[k], a);
  const double pap = block_sum(a, red);
  const double alpha = pap > 0.0 ? sc[SC_RZ] / pap : 0.0;
  double rr = 0.0;
  for (int k = threadIdx.x; k < nv; k += blockDim.x) {
    x[k] = fma(alpha, p[k], x[k]);
    const double v = fma(-alpha, ap[k], r[k]);
    r[k] = v;
    rr = fma(v, v, rr);
  }
  rr = block_sum(rr, red);
  if (threadIdx.x == 0) {
    sc[SC_PAP] = pap;
    sc[SC_ALPHA] = alpha;
    sc[SC_RR] = rr;
  }
}

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

}  // namespace

// ---------------------------------------------------------------------------------------------------
// host entry points
// ---------------------------------------------------------------------------------------------------
// Workspace of the factorisation: n reciprocal diagonal entries, then the inverted diagonal blocks.
size_t rbmpp_chol_work(int n) { return (size_t)2 * ((n + NB - 1) / NB) * PK + (size_t)n; }

// In-place Cholesky of the upper triangle of A (n x n, lda = n); work: rbmpp_chol_work(n) doubles, holding
// 1 / U(i, i) and the inverted diagonal blocks on return; *d_info = 0 or the first failing column (1-based).
cudaError_t rbmpp_potrf_upper(int n, double* A, double* work, int* d_info, cudaStream_t st) {
  double* rdiag = work + (size_t)2 * ((n + NB - 1) / NB) * PK;  // after the packed triangles (16-byte aligned)
  cudaError_t e = cudaMemsetAsync(d_info, 0, sizeof(int), st);
  if (e) return e;
  const size_t smem = (size_t)NB * (NB + 1) * sizeof(double);
  if ((e = cudaFuncSetAttribute(potrf_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem))) return e;
  if ((e = cudaFuncSetAttribute(panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem))) return e;
  const int nsm = sm_count();
  for (int k0 = 0; k0 < n; k0 += NB) {
    rbmpp_note_launch();
    potrf_block_kernel<<<1, 512, smem, st>>>(n, A, n, k0, rdiag, d_info);
    const int rest = n - (k0 + NB);
    if (rest > 0) {
      const int blocks = min(nsm, (rest + 15) / 16);
      rbmpp_note_launch();
      panel_kernel<<<blocks, 512, smem, st>>>(n, A, n, k0, rdiag);
      if ((e = rbmpp_gemm_atb_upper_acc(n, NB, A + k0, 1, n, -1.0, A, n, k0 + NB, st))) return e;
    }
  }
  if ((e = cudaFuncSetAttribute(invert_blocks_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)))
    return e;
  rbmpp_note_launch();
  invert_blocks_kernel<<<(n + NB - 1) / NB, 512, smem, st>>>(n, A, n, rdiag, work);
  return cudaGetLastError();
}

// b <- A^{-1} b with A = U^T U (upper factor in A, work as rbmpp_potrf_upper left it); tmp: n doubles.
// bar: 4 unsigned of device memory for the persistent form (one cooperative launch); bar[2] becomes 1 if one of
// its bounded barrier waits ran out.  Without bar, or where the cooperative launch is refused, one launch per
// block step.
cudaError_t rbmpp_potrs_upper(int n, const double* A, const double* work, double* b, double* tmp, unsigned* bar,
                              cudaStream_t st) {
  const double* dinv = work;
  const int nsm = sm_count();
  const int nblk = (n + NB - 1) / NB;
  const size_t smem = (size_t)PK * sizeof(double), psmem = 2 * smem;
  cudaError_t e;
  if (bar) {
    static int coop = -1;  // the device supports cooperative launches with this shape
    if (coop < 0) {
      int dev = 0, attr = 0, nb_sm = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&attr, cudaDevAttrCooperativeLaunch, dev);
      cudaFuncSetAttribute(potrs_persistent_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb_sm, potrs_persistent_kernel, 256, psmem);
      coop = (attr && nb_sm >= 1) ? 1 : 0;
      cudaGetLastError();
    }
    if (coop) {
      if ((e = cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), st))) return e;  // count, generation (bar[2] sticks)
      int nn = n;
      void* args[] = {&nn, (void*)&A, (void*)&dinv, &b, &tmp, &bar};
      rbmpp_note_launch();
      e = cudaLaunchCooperativeKernel((const void*)potrs_persistent_kernel, dim3(nsm), dim3(256), args, psmem, st);
      if (e == cudaSuccess) return cudaSuccess;
      cudaGetLastError();
      coop = 0;
    }
  }
  if ((e = cudaFuncSetAttribute(trsv_fwd_step, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem))) return e;
  if ((e = cudaFuncSetAttribute(trsv_bwd_step, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem))) return e;
  for (int kb = 0; kb < nblk; kb++) {  // U^T y = b: y in tmp, b consumed
    const int k0 = kb * NB, rest = n - (k0 + NB);
    const int blocks = rest > 0 ? min(nsm, (rest + 31) / 32) : 1;
    rbmpp_note_launch();
    trsv_fwd_step<<<blocks, 256, smem, st>>>(n, A, n, k0, dinv + (size_t)kb * PK, b, tmp);
  }
  for (int kb = nblk - 1; kb >= 0; kb--) {  // U x = y: x in b, tmp consumed
    const int k0 = kb * NB;
    const int blocks = k0 > 0 ? min(nsm, (k0 + 31) / 32) : 1;
    rbmpp_note_launch();
    trsv_bwd_step<<<blocks, 256, smem, st>>>(n, A, n, k0, dinv + (size_t)(nblk + kb) * PK, tmp, b);
  }
  return cudaGetLastError();
}

// Partial-sum buffer of rbmpp_gram_apply: rbmpp_gram_parts() * nv doubles.
int rbmpp_gram_parts() { return sm_count(); }

// Largest nv the one-pass kernel takes (its shared memory holds two nv-vectors).
int rbmpp_gram_max_nv() {
  int dev = 0, maxsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return (maxsm / (int)sizeof(double) - 2 * kRows * 32) / 2;
}

// z = O^T (O y): O is ns x nv (row per sample).  part: rbmpp_gram_parts() * nv doubles.  When two
// nv-vectors do not fit one block's shared memory, two passes: tmp_ns = O y, then O^T tmp_ns through
// part64 (64 * nv doubles).
cudaError_t rbmpp_gram_apply(int ns, int nv, const double* O, const double* y, double* z, double* part,
                             double* tmp_ns, double* part64, cudaStream_t st) {
  cudaError_t e;
  if (nv > rbmpp_gram_max_nv()) {
    if ((e = rbmpp_gemv_o(ns, nv, O, y, tmp_ns, st))) return e;
    return rbmpp_gemv_ot(ns, nv, O, tmp_ns, nullptr, z, nullptr, part64, 64, st);
  }
  const int nb = rbmpp_gram_parts();
  const size_t smem = (size_t)(2 * nv + 2 * kRows * 32) * sizeof(double);
  const bool vec = (nv % 2) == 0 && ((uintptr_t)O % 16) == 0;
  if (vec) {
    if ((e = cudaFuncSetAttribute(gram_apply_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)))
      return e;
    rbmpp_note_launch();
    gram_apply_kernel<true><<<nb, kGramThreads, smem, st>>>(ns, nv, O, y, part);
  } else {
    if ((e = cudaFuncSetAttribute(gram_apply_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)))
      return e;
    rbmpp_note_launch();
    gram_apply_kernel<false><<<nb, kGramThreads, smem, st>>>(ns, nv, O, y, part);
  }
  rbmpp_note_launch();
  sum_blocks<<<(nv + 255) / 256, 256, 0, st>>>(nv, nb, part, z);
  return cudaGetLastError();
}

// y = A x with A = D (S_raw / norm - m m^T) D + sigma I applied through O, in two halves so that a cross-rank
// sum of z = O^T (O D x) can come between them.  First half: ws = D x, sc[SC_MX] = m . ws, z = O^T (O ws);
// ws, z: nv doubles each; sc: device scalars.
cudaError_t rbmpp_sr_apply_gram(int ns, int nv, int nrbm, const double* O, const double* m, double scal,
                                const double* x, double* ws, double* z, double* part, double* tmp_ns, double* part64,
                                double* sc, cudaStream_t st) {
  rbmpp_note_launch();
  sr_pre_kernel<<<1, 1024, 0, st>>>(nv, nrbm, x, scal, m, ws, sc);
  return rbmpp_gram_apply(ns, nv, O, ws, z, part, tmp_ns, part64, st);
}

// Second half: y = D (z / norm - m sc[SC_MX]) + sigma x.
cudaError_t rbmpp_sr_apply_finish(int nv, int nrbm, const double* m, double norm, double scal, double sigma,
                                  const double* x, const double* z, const double* sc, double* y, cudaStream_t st) {
  rbmpp_note_launch();
  sr_post_kernel<<<(nv + 255) / 256, 256, 0, st>>>(nv, nrbm, z, m, sc, x, scal, sigma, norm, y);
  return cudaGetLastError();
}

cudaError_t rbmpp_pcg_start(int nv, const double* g, const double* ax, double* r, double* sc, cudaStream_t st) {
  rbmpp_note_launch();
  pcg_start_kernel<<<1, 1024, 0, st>>>(nv, g, ax, r, sc);
  return cudaGetLastError();
}

cudaError_t rbmpp_pcg_dir(int nv, const double* r, const double* z, double* p, double* sc, int mode, cudaStream_t st) {
  rbmpp_note_launch();
  pcg_dir_kernel<<<1, 1024, 0, st>>>(nv, r, z, p, sc, mode);
  return cudaGetLastError();
}

cudaError_t rbmpp_pcg_step(int nv, const double* p, const double* ap, double* x, double* r, double* sc,
                           cudaStream_t st) {
  rbmpp_note_launch();
  pcg_step_kernel<<<1, 1024, 0, st>>>(nv, p, ap, x, r, sc);
  return cudaGetLastError();
}

// linalg.cu -- FP64 dense kernels of the SR step: the S = O^T O build (the dgemm of
// calc_phys_quantity.f90:240) and the GEMM of the Cholesky's trailing update (sr_solve.cu holds the rest of
// the solve that replaces pdposv('U'), SR_pdposv.f90:232), GEMVs over the O matrix, and the element-wise SR
// conditioning (SR_pdposv.f90:1-170).  Matrices are column-major (Fortran layout), S is Nv x Nv.
#include <cuda_runtime.h>
#include <stdint.h>

void rbmpp_note_launch();  // capi.cu: counts kernel launches

namespace {

// C(i, j) = alpha * sum_k A(k, i) B(k, j) + beta * C(i, j) on upper-triangular 128 x 128 tiles.
// A(k, i) = A[k * sk + i * si] (same for B).  KCONTIG selects the coalesced load direction.
constexpr int BM = 128, BK = 8, TM = 8;

template <bool KCONTIG>
__global__ void __launch_bounds__(256) gemm_atb_upper(int n, int K, const double* __restrict__ A, long long sk,
                                                      long long si, double alpha, double beta, double* __restrict__ C,
                                                      long long ldc, int row0) {
  // upper-tile index -> (ti, tj) with ti <= tj
  const int nt = (n - row0 + BM - 1) / BM;
  int t = blockIdx.x, ti = 0;
  while (t >= nt - ti) {
    t -= nt - ti;
    ti++;
  }
  const int tj = ti + t;
  const int i0 = row0 + ti * BM, j0 = row0 + tj * BM;
  __shared__ double As[2][BK][BM];
  __shared__ double Bs[2][BK][BM];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  double acc[TM][TM];
#pragma unroll
  for (int a = 0; a < TM; a++)
#pragma unroll
    for (int b = 0; b < TM; b++) acc[a][b] = 0.0;

  auto load = [&](int buf, int k0) {
#pragma unroll
    for (int r = 0; r < (BK * BM) / 256; r++) {
      int e = tid + 256 * r;
      int kk, ii;
      if (KCONTIG) {
        kk = e % BK;
        ii = e / BK;
      } else {
        kk = e / BM;
        ii = e % BM;
      }
      int k = k0 + kk;
      int ia = i0 + ii, jb = j0 + ii;
      As[buf][kk][ii] = (k < K && ia < n) ? A[(long long)k * sk + (long long)ia * si] : 0.0;
      Bs[buf][kk][ii] = (k < K && jb < n) ? A[(long long)k * sk + (long long)jb * si] : 0.0;
    }
  };
  load(0, 0);
  __syncthreads();
  int buf = 0;
  for (int k0 = 0; k0 < K; k0 += BK) {
    if (k0 + BK < K) load(buf ^ 1, k0 + BK);
#pragma unroll
    for (int kk = 0; kk < BK; kk++) {
      double a[TM], b[TM];
#pragma unroll
      for (int m = 0; m < TM; m++) {
        a[m] = As[buf][kk][tx + 16 * m];
        b[m] = Bs[buf][kk][ty + 16 * m];
      }
#pragma unroll
      for (int p = 0; p < TM; p++)
#pragma unroll
        for (int q = 0; q < TM; q++) acc[p][q] = fma(a[p], b[q], acc[p][q]);
    }
    __syncthreads();
    buf ^= 1;
  }
#pragma unroll
  for (int q = 0; q < TM; q++) {
    int j = j0 + ty + 16 * q;
    if (j >= n) continue;
#pragma unroll
    for (int p = 0; p < TM; p++) {
      int i = i0 + tx + 16 * p;
      if (i >= n || i > j) continue;
      double* c = C + (long long)i + ldc * j;
      *c = (beta == 0.0) ? alpha * acc[p][q] : beta * (*c) + alpha * acc[p][q];
    }
  }
}

// mirror the upper triangle into the lower one
__global__ void symmetrize_kernel(int n, double* S) {
  __shared__ double tile[32][33];
  int bi = blockIdx.y, bj = blockIdx.x;
  if (bi > bj) return;
  int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int r = ty; r < 32; r += 8) {
    int i = bi * 32 + tx, j = bj * 32 + r;
    tile[r][tx] = (i < n && j < n) ? S[(long long)i + (long long)n * j] : 0.0;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    int i = bj * 32 + tx, j = bi * 32 + r;  // lower element (i, j) = upper (j, i)
    int ui = bi * 32 + r, uj = bj * 32 + tx;
    if (i < n && j < n && ui < uj) S[(long long)i + (long long)n * j] = tile[tx][r];
  }
}

// y = U x restricted: y(i) = sum_{j >= i} U(i, j) x(j)  (one warp per row)
__global__ void trmv_upper_kernel(int n, const double* A, long long lda, const double* x, double* y) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n) return;
  double s = 0.0;
  for (int j = warp + lane; j < n; j += 32) s += A[(long long)warp + lda * j] * x[j];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) y[warp] = s;
}

// out[c][k] = sum_{s in chunk c} coef[v][s] * O[s][k] for two coefficient vectors (v = 0, 1)
__global__ void gemv_ot_partial(int ns, int nv, const double* __restrict__ O, const double* __restrict__ c0,
                                const double* __restrict__ c1, int chunk, double* __restrict__ part0,
                                double* __restrict__ part1) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  int cb = blockIdx.y;
  if (k >= nv) return;
  int s0 = cb * chunk, s1 = min(ns, s0 + chunk);
  double a = 0.0, b = 0.0;
  for (int s = s0; s < s1; s++) {
    double o = O[(long long)s * nv + k];
    a += c0[s] * o;
    if (c1) b += c1[s] * o;
  }
  part0[(long long)cb * nv + k] = a;
  if (part1) part1[(long long)cb * nv + k] = b;
}

__global__ void sum_parts(int nv, int nparts, const double* part, double* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nv) return;
  double a = 0.0;
  for (int c = 0; c < nparts; c++) a += part[(long long)c * nv + k];
  out[k] = a;
}

// y[s] = sum_k O[s][k] x[k]   (warp per sample row)
__global__ void gemv_o_kernel(int ns, int nv, const double* __restrict__ O, const double* __restrict__ x,
                              double* __restrict__ y) {
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (row >= ns) return;
  const double* r = O + (long long)row * nv;
  double s = 0.0;
  for (int k = lane; k < nv; k += 32) s += r[k] * x[k];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) y[row] = s;
}

// S(i,j) = Sraw(i,j)/norm - Ovec(i) Ovec(j)   (SR_pdposv.f90:11-15), full matrix
__global__ void sr_form_kernel(int n, double* S, double norm, const double* ov) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // 2-D grid: no 64-bit division
  if (i >= n) return;
  for (int j = blockIdx.y; j < n; j += gridDim.y) {
    const long long e = (long long)j * n + i;
    S[e] = S[e] / norm - ov[i] * ov[j];
  }
}

// y = f x
__global__ void scale_copy_kernel(int n, const double* x, double f, double* y) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = x[i] * f;
}

// S(i, j) += f v_i v_j on the strict upper triangle (column-major)
__global__ void add_outer_offdiag_kernel(int n, double* S, const double* v, double f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  for (int j = blockIdx.y; j < n; j += gridDim.y)
    if (i < j) S[(long long)j * n + i] = fma(f * v[i], v[j], S[(long long)j * n + i]);
}

// PP-block scaling (SR_pdposv.f90:56-73): columns k2 > Nv_RBM, then rows k1 > Nv_RBM
__global__ void sr_scale_kernel(int n, int nrbm, double* S, double f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int j = blockIdx.y; j < n; j += gridDim.y) {
    const long long e = (long long)j * n + i;
    double v = S[e];
    if (j >= nrbm) v = v * f;
    if (i >= nrbm) v = v * f;
    S[e] = v;
  }
}

__global__ void get_diag_kernel(int n, const double* S, double* d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) d[i] = S[(long long)i + (long long)n * i];
}

__global__ void add_diag_kernel(int n, double* S, double v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) S[(long long)i + (long long)n * i] += v;
}

// max |S(k, :)|, |S(:, k)| for the listed indices (f_ii checks, SR_pdposv.f90:89-92)
__global__ void rowcol_absmax_kernel(int n, const double* S, const int* list, int nlist, double* out) {
  int li = blockIdx.x;
  if (li >= nlist) return;
  int k = list[li];
  double m = 0.0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    m = fmax(m, fabs(S[(long long)k + (long long)n * j]));
    m = fmax(m, fabs(S[(long long)j + (long long)n * k]));
  }
  __shared__ double r[256];
  r[threadIdx.x] = m;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) r[threadIdx.x] = fmax(r[threadIdx.x], r[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[li] = r[0];
}

// per-sample scalars of calc_phys_quantity.f90:102-109 and coefficient vectors of the gvec/Ovec GEMV:
// a_s = 2 Re(Eloc_s) (gvec, :229), b_s = w_s Re(psi_s) (Ovec, :230), with real O rows.
// Per-sample sums of calc_phys_quantity.f90:102-109 and the coefficients of gvec and Ovec per row of O:
// gvec += 2 Re(conj(E) O), Ovec += w Re(conj(psi) O).  With complex rows (cplx) sample s owns rows 2s (real part)
// and 2s + 1 (imaginary part) of O, so the coefficients are (2 Re E, 2 Im E) and (w Re psi, w Im psi).
__global__ void sample_scalars_kernel(int ns, const double* psi, int psi_stride, const double* eloc, double shift,
                                      double* a, double* b, double* acc4, int cplx) {
  __shared__ double r[4][256];
  double e1 = 0, e2 = 0, nn = 0, wf = 0;
  for (int s = threadIdx.x; s < ns; s += blockDim.x) {
    double pr = psi[(long long)s * psi_stride], pi = psi[(long long)s * psi_stride + 1];
    double ap = hypot(pr, pi);
    double w = 1.0 / (ap + shift);
    double er = eloc[2 * (long long)s], ei = eloc[2 * (long long)s + 1];
    e1 += w * (pr * er + pi * ei);
    e2 += er * er + ei * ei;
    nn += (ap * w) * (ap * w);
    wf += ap;
    if (cplx) {
      a[2 * s] = 2.0 * er;
      a[2 * s + 1] = 2.0 * ei;
      b[2 * s] = w * pr;
      b[2 * s + 1] = w * pi;
    } else {
      a[s] = 2.0 * er;
      b[s] = w * pr;
    }
  }
  r[0][threadIdx.x] = e1;
  r[1][threadIdx.x] = e2;
  r[2][threadIdx.x] = nn;
  r[3][threadIdx.x] = wf;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int q = 0; q < 4; q++) r[q][threadIdx.x] += r[q][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x < 4) acc4[threadIdx.x] = r[threadIdx.x][0];
}

}  // namespace

// ------------------------------------------------------------------------------------------------
// host wrappers
// ------------------------------------------------------------------------------------------------
cudaError_t rbmpp_syrk_ot_o(int nv, int ns, const double* O, double* S, cudaStream_t st) {
  int nt = (nv + BM - 1) / BM;
  int ntiles = nt * (nt + 1) / 2;
  rbmpp_note_launch();
  gemm_atb_upper<false><<<ntiles, 256, 0, st>>>(nv, ns, O, nv, 1, 1.0, 0.0, S, nv, 0);
  cudaError_t e = cudaGetLastError();
  if (e) return e;
  dim3 g((nv + 31) / 32, (nv + 31) / 32);
  rbmpp_note_launch();
  symmetrize_kernel<<<g, dim3(32, 8), 0, st>>>(nv, S);
  return cudaGetLastError();
}

// C(i, j) = sum_k A(k, i) A(k, j) for i <= j (upper triangle, column-major C), A(k, i) = A[k sk + i si]
cudaError_t rbmpp_gemm_atb_upper(int n, int K, const double* A, long long sk, long long si, double* C, long long ldc,
                                 cudaStream_t st) {
  int nt = (n + BM - 1) / BM;
  rbmpp_note_launch();
  gemm_atb_upper<false><<<nt * (nt + 1) / 2, 256, 0, st>>>(n, K, A, sk, si, 1.0, 0.0, C, ldc, 0);
  return cudaGetLastError();
}

cudaError_t rbmpp_symmetrize(int n, double* S, cudaStream_t st) {
  dim3 g((n + 31) / 32, (n + 31) / 32);
  rbmpp_note_launch();
  symmetrize_kernel<<<g, dim3(32, 8), 0, st>>>(n, S);
  return cudaGetLastError();
}

// C(i, j) += alpha * sum_k A(k, i) A(k, j) on the upper triangle of rows and columns >= row0 (the trailing
// update of the blocked Cholesky in sr_solve.cu; K = its panel width, A(k, i) contiguous in k)
cudaError_t rbmpp_gemm_atb_upper_acc(int n, int K, const double* A, long long sk, long long si, double alpha,
                                     double* C, long long ldc, int row0, cudaStream_t st) {
  const int rest = n - row0;
  if (rest <= 0) return cudaSuccess;
  const int nt = (rest + BM - 1) / BM;
  rbmpp_note_launch();
  gemm_atb_upper<true><<<nt * (nt + 1) / 2, 256, 0, st>>>(n, K, A, sk, si, alpha, 1.0, C, ldc, row0);
  return cudaGetLastError();
}

cudaError_t rbmpp_trmv_upper(int n, const double* A, const double* x, double* y, cudaStream_t st) {
  rbmpp_note_launch();
  trmv_upper_kernel<<<(n * 32 + 255) / 256, 256, 0, st>>>(n, A, n, x, y);
  return cudaGetLastError();
}

// out0 = O^T c0, out1 = O^T c1 (c1/out1 nullable); part: scratch of 2 * nparts * nv doubles
cudaError_t rbmpp_gemv_ot(int ns, int nv, const double* O, const double* c0, const double* c1, double* out0,
                          double* out1, double* part, int nparts, cudaStream_t st) {
  int chunk = (ns + nparts - 1) / nparts;
  dim3 g((nv + 127) / 128, nparts);
  rbmpp_note_launch();
  gemv_ot_partial<<<g, 128, 0, st>>>(ns, nv, O, c0, c1, chunk, part, c1 ? part + (long long)nparts * nv : nullptr);
  rbmpp_note_launch();
  sum_parts<<<(nv + 255) / 256, 256, 0, st>>>(nv, nparts, part, out0);
  if (c1) {
    rbmpp_note_launch();
    sum_parts<<<(nv + 255) / 256, 256, 0, st>>>(nv, nparts, part + (long long)nparts * nv, out1);
  }
  return cudaGetLastError();
}

cudaError_t rbmpp_gemv_o(int ns, int nv, const double* O, const double* x, double* y, cudaStream_t st) {
  rbmpp_note_launch();
  gemv_o_kernel<<<(ns * 32 + 255) / 256, 256, 0, st>>>(ns, nv, O, x, y);
  return cudaGetLastError();
}

cudaError_t rbmpp_sr_form(int n, double* S, double norm, const double* ov, cudaStream_t st) {
  rbmpp_note_launch();
  sr_form_kernel<<<dim3((n + 255) / 256, n < 65535 ? n : 65535), 256, 0, st>>>(n, S, norm, ov);
  return cudaGetLastError();
}

cudaError_t rbmpp_scale_copy(int n, const double* x, double f, double* y, cudaStream_t st) {
  rbmpp_note_launch();
  scale_copy_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, x, f, y);
  return cudaGetLastError();
}

cudaError_t rbmpp_add_outer_offdiag(int n, double* S, const double* v, double f, cudaStream_t st) {
  rbmpp_note_launch();
  add_outer_offdiag_kernel<<<dim3((n + 255) / 256, n < 65535 ? n : 65535), 256, 0, st>>>(n, S, v, f);
  return cudaGetLastError();
}

cudaError_t rbmpp_sr_scale(int n, int nrbm, double* S, double f, cudaStream_t st) {
  rbmpp_note_launch();
  sr_scale_kernel<<<dim3((n + 255) / 256, n < 65535 ? n : 65535), 256, 0, st>>>(n, nrbm, S, f);
  return cudaGetLastError();
}

cudaError_t rbmpp_get_diag(int n, const double* S, double* d, cudaStream_t st) {
  rbmpp_note_launch();
  get_diag_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, S, d);
  return cudaGetLastError();
}

cudaError_t rbmpp_add_diag(int n, double* S, double v, cudaStream_t st) {
  rbmpp_note_launch();
  add_diag_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, S, v);
  return cudaGetLastError();
}

cudaError_t rbmpp_rowcol_absmax(int n, const double* S, const int* list, int nlist, double* out, cudaStream_t st) {
  if (nlist <= 0) return cudaSuccess;
  rbmpp_note_launch();
  rowcol_absmax_kernel<<<nlist, 256, 0, st>>>(n, S, list, nlist, out);
  return cudaGetLastError();
}

cudaError_t rbmpp_sample_scalars(int ns, const double* psi, int psi_stride, const double* eloc, double shift,
                                 double* a, double* b, double* acc4, int cplx, cudaStream_t st) {
  rbmpp_note_launch();
  sample_scalars_kernel<<<1, 256, 0, st>>>(ns, psi, psi_stride, eloc, shift, a, b, acc4, cplx);
  return cudaGetLastError();
}

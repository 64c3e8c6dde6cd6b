// capi.cu -- the C ABI of include/rbmpp.h: context, device memory, tables, and the host logic of
// main.f90 / SR_pdposv.f90 around the device kernels (sampler.cu, estimator.cu, linalg.cu,
// gemm_bf16x3.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/rbmpp.h"
#include "common.cuh"

// launchers (sampler.cu, estimator.cu, linalg.cu, gemm_bf16x3.cu)
cudaError_t rbmpp_launch_sampler(const DevDims&, const DevTables&, const DevParams&, const DevWalkers&, int,
                                 cudaStream_t);
size_t rbmpp_sampler_smem(const DevDims&, int);
int rbmpp_stream_stages(const DevDims&, int);
cudaError_t rbmpp_launch_sampler_stream(const DevDims&, const DevTables&, const DevParams&, const DevWalkers&, int, int,
                                        cudaStream_t);
cudaError_t rbmpp_launch_estimator(const DevDims&, const DevTables&, const DevParams&, const int8_t*, int, double*,
                                   double*, double*, int*, int*, int, cudaStream_t);
size_t rbmpp_estimator_smem(const DevDims&, int);
size_t rbmpp_estimator_smem_any(const DevDims&, int);
cudaError_t rbmpp_launch_advance_rng(uint32_t*, const int*, int, int, int, cudaStream_t);
cudaError_t rbmpp_syrk_ot_o(int, int, const double*, double*, cudaStream_t);
cudaError_t rbmpp_symmetrize(int, double*, cudaStream_t);
cudaError_t rbmpp_potrf_upper(int, double*, double*, int*, cudaStream_t);
cudaError_t rbmpp_potrs_upper(int, const double*, const double*, double*, double*, unsigned*, cudaStream_t);
int rbmpp_gram_parts();
size_t rbmpp_chol_work(int);
cudaError_t rbmpp_sr_apply_gram(int, int, int, const double*, const double*, double, const double*, double*, double*,
                                double*, double*, double*, double*, cudaStream_t);
cudaError_t rbmpp_sr_apply_finish(int, int, const double*, double, double, double, const double*, const double*,
                                  const double*, double*, cudaStream_t);
cudaError_t rbmpp_pcg_start(int, const double*, const double*, double*, double*, cudaStream_t);
cudaError_t rbmpp_pcg_dir(int, const double*, const double*, double*, double*, int, cudaStream_t);
cudaError_t rbmpp_pcg_step(int, const double*, const double*, double*, double*, double*, cudaStream_t);
cudaError_t rbmpp_trmv_upper(int, const double*, const double*, double*, cudaStream_t);
cudaError_t rbmpp_gemv_ot(int, int, const double*, const double*, const double*, double*, double*, double*, int,
                          cudaStream_t);
cudaError_t rbmpp_gemv_o(int, int, const double*, const double*, double*, cudaStream_t);
cudaError_t rbmpp_sr_form(int, double*, double, const double*, cudaStream_t);
cudaError_t rbmpp_sr_scale(int, int, double*, double, cudaStream_t);
cudaError_t rbmpp_get_diag(int, const double*, double*, cudaStream_t);
cudaError_t rbmpp_add_diag(int, double*, double, cudaStream_t);
cudaError_t rbmpp_rowcol_absmax(int, const double*, const int*, int, double*, cudaStream_t);
cudaError_t rbmpp_sample_scalars(int, const double*, int, const double*, double, double*, double*, double*, int,
                                 cudaStream_t);
void rbmpp_bf16x3_pads(int, int, int*, int*);
int rbmpp_syrk_bf16x3(int, int, const double*, const double*, const double*, void*, void*, int*, double*, double*,
                      cudaStream_t);
cudaError_t rbmpp_scale_copy(int, const double*, double, double*, cudaStream_t);
cudaError_t rbmpp_add_outer_offdiag(int, double*, const double*, double, cudaStream_t);
int rbmpp_correlation_fits(const DevDims&, int);
int rbmpp_skew_max_n();
size_t rbmpp_skew_smem_shortfall(const DevDims&, int);
cudaError_t rbmpp_build_se(const DevDims&, const int*, const int*, const double*, double*, cudaStream_t);
cudaError_t rbmpp_launch_sampler_skew(const DevDims&, const DevTables&, const DevParams&, const DevWalkers&, int,
                                      cudaStream_t);
cudaError_t rbmpp_launch_estimator_skew(const DevDims&, const DevTables&, const DevParams&, const int8_t*, int,
                                        double*, double*, double*, int*, int*, int, cudaStream_t);
cudaError_t rbmpp_launch_correlation(const DevDims&, const DevTables&, const DevParams&, const int8_t*, int, double*,
                                     double*, double*, double*, int*, int*, cudaStream_t);
cudaError_t rbmpp_fill(double*, long long, double, cudaStream_t);
cudaError_t rbmpp_gemm_atb_upper(int, int, const double*, long long, long long, double*, long long, cudaStream_t);

static std::atomic<long long> g_launches{0};
void rbmpp_note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

namespace {

// update_slater_elements (slater.f90:7-64), block form: XF(p,q) = -Slater_Elm(p, q+N) for projection qp,
// with Slater_Elm(p, q+N) = -slt_ij*ss - slt_ji*cc, slt_ij = f(T q, T p), slt_ji = f(T p, T q).
__global__ void build_xf_kernel(int N, int n_mp, const int* wmap, const int* orb, const double* slater, double cc0,
                                double ss0, double cc1, double ss1, double* XF, double* XFT) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long tot = (long long)2 * n_mp * N * N;
  if (e >= tot) return;
  int q = (int)(e % N);
  long long r = e / N;
  int pp = (int)(r % N);
  int qp = (int)(r / N);
  int mp = qp >> 1, sp = qp & 1;
  double cc = sp ? cc1 : cc0, ss = sp ? ss1 : ss0;
  int tp = wmap[(long long)mp * N + pp], tq = wmap[(long long)mp * N + q];
  double slt_ij = slater[orb[(long long)tq * N + tp]];
  double slt_ji = slater[orb[(long long)tp * N + tq]];
  double se = __dsub_rn(__dmul_rn(-slt_ij, ss), __dmul_rn(slt_ji, cc));
  double xf = -se;
  XF[((long long)qp * N + pp) * N + q] = xf;
  XFT[((long long)qp * N + q) * N + pp] = xf;
}

__global__ void seed_kernel(uint32_t* mt, int nw, int iseed0, int ns, int w0) {
  int wl = blockIdx.x * blockDim.x + threadIdx.x;
  if (wl >= nw) return;
  const int w = w0 + wl;  // global rank
  uint32_t st[625];
  st[0] = (uint32_t)(iseed0 + w);
  for (int i = 1; i < 624; i++) st[i] = 69069u * st[i - 1];
  st[624] = 624;
  long long skip = (long long)ns * w + 1;  // main.f90:232-234
  for (long long i = 0; i < skip; i++) (void)mt_next(st);
  for (int k = 0; k < 625; k++) mt[(size_t)wl * 625 + k] = st[k];
}

__global__ void draw_kernel(uint32_t* mt, int n, double* out) {
  uint32_t st[625];
  for (int k = 0; k < 625; k++) st[k] = mt[k];
  for (int i = 0; i < n; i++) out[i] = grnd(st);
  for (int k = 0; k < 625; k++) mt[k] = st[k];
}

__global__ void int_to_i8_kernel(const int* in, int8_t* out, long long n) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) out[e] = (int8_t)in[e];
}
__global__ void i8_to_int_kernel(const int8_t* in, int* out, long long n) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) out[e] = (int)in[e];
}

}  // namespace

struct rbmpp_ctx {
  rbmpp_dims dims;
  DevDims d;
  cudaStream_t st = nullptr;
  std::string err;
  // host copies of the tables and parameters (Fortran layouts)
  std::vector<int> orb_host;     // Orbital_Idx 0-based [p][q] row-major (p*N+q)
  std::vector<double> Wr, br, slater;
  std::vector<double> Wc, bc;  // Wcirr(N, alphac), bcirr(alphac) as (re, im) pairs
  double shift = 0.0;
  bool tables_set = false, params_set = false, seeded = false, sampled = false, measured = false;
  // device tables / params
  int *d_wmap = nullptr, *d_winv = nullptr, *d_orb = nullptr, *d_bonds = nullptr;
  unsigned char* d_subB = nullptr;
  double *d_para = nullptr, *d_Wr = nullptr, *d_br = nullptr, *d_slater = nullptr, *d_XF = nullptr, *d_XFT = nullptr;
  double *d_Wc = nullptr, *d_bc = nullptr;
  DevWalkers W{};
  // measurement
  int ns_tot = 0;
  int nrows = 0;  // rows of O: ns_tot, or 2 ns_tot with complex projection weights
  double *d_O = nullptr, *d_psiS = nullptr, *d_eloc = nullptr, *d_a = nullptr, *d_b = nullptr, *d_acc4 = nullptr;
  int *d_nap = nullptr, *d_estat = nullptr;
  double *d_gvec = nullptr, *d_Ovec = nullptr, *d_S = nullptr, *d_part = nullptr, *d_vec = nullptr;
  double *d_tmp_ns = nullptr, *d_rv = nullptr;
  int *d_info = nullptr, *d_err = nullptr;
  double* d_Sb = nullptr;  // copy of the shifted split-precision S (preconditioner retries)
  double* d_dinv = nullptr;  // Cholesky workspace: 1 / U(i, i) and the inverted diagonal blocks
  double* d_pcg = nullptr;   // refinement vectors (10 x Nv)
  double* d_gpart = nullptr; // per-block partial sums of the one-pass O^T (O y)
  double* d_sc = nullptr;    // device scalars of the refinement
  unsigned* d_bar = nullptr; // grid barrier of the one-launch triangular solves
  double* h_sc = nullptr;    // pinned host copy of them
  // correlation measurement: per-sample rows (2 Nchi + 1), w SdotS rows (4N), ones, Chi_vbs blocks, sums
  double *d_crow = nullptr, *d_csd = nullptr, *d_cones = nullptr, *d_cvbs = nullptr, *d_cpart = nullptr,
         *d_csum = nullptr;
  void *d_hi = nullptr, *d_lo = nullptr;
  int ldk = 0;
  float* d_Sf = nullptr;
  double meas_scal[4] = {0, 0, 0, 0};
  long long naccept_total = 0;
  double n_samples_total = 0.0;  // samples behind meas_scal (all GPUs after a reduction)
  // main.f90 bookkeeping for rbmpp_iteration
  int iteration = 0;
  double s_factor0 = 0.0;
  bool s_factor_init = false;
  double wf_av_list[10] = {0};
  size_t bytes = 0;
  cudaEvent_t ev[12] = {};
  double stats[10] = {0};
  int stream_stages = 0;  // > 0: TMA-streamed sampler with this many stages
  bool est_fits = true;   // the estimator's workspace fits in shared memory (tiles there or in global scratch)
  bool est_smem_tiles = true;  // ... with its tiles in shared memory
  double* d_SE = nullptr;  // Slater_Elm [qp][2N][2N] of the skew form (transverse projection)
  // host-supplied cross-rank sum (rbmpp_set_allreduce) and its packed buffer: 6 scalars, gvec, Ovec
  rbmpp_allreduce_fn red_fn = nullptr;
  void* red_user = nullptr;
  double* d_xch = nullptr;
  // S of the current measurement: built lazily in the precision the SR step asks for
  bool S_valid = false, S_reduced = false;
  int S_prec = RBMPP_SR_FP64, meas_prec = RBMPP_SR_FP64;
};

namespace {

int fail(rbmpp_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CK(call)                                                                                  \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) return fail(c, RBMPP_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

template <class T>
int dalloc(rbmpp_ctx* c, T** p, size_t count) {
  cudaError_t e = cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(count, 1));
  if (e != cudaSuccess) return fail(c, RBMPP_E_CUDA, "cudaMalloc(%zu bytes): %s", sizeof(T) * count, cudaGetErrorString(e));
  c->bytes += sizeof(T) * count;
  return 0;
}

DevTables tables(const rbmpp_ctx* c) {
  DevTables t;
  t.wmap = c->d_wmap;
  t.winv = c->d_winv;
  t.para_mp = c->d_para;
  t.orb = c->d_orb;
  t.subB = c->d_subB;
  t.bonds = c->d_bonds;
  return t;
}

DevParams params(const rbmpp_ctx* c) {
  DevParams p;
  p.Wr = c->d_Wr;
  p.br = c->d_br;
  p.Wc = c->d_Wc;
  p.bc = c->d_bc;
  p.XF = c->d_XF;
  p.XFT = c->d_XFT;
  p.SE = c->d_SE;
  return p;
}

int upload_params(rbmpp_ctx* c) {
  const DevDims& d = c->d;
  std::vector<double> wr_dev((size_t)d.alphar * d.N);
  for (int f = 0; f < d.alphar; f++)
    for (int iw = 0; iw < d.N; iw++) wr_dev[(size_t)f * d.N + iw] = c->Wr[iw + (size_t)d.N * f];
  if (d.alphar > 0) {
    CK(cudaMemcpyAsync(c->d_Wr, wr_dev.data(), sizeof(double) * wr_dev.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->d_br, c->br.data(), sizeof(double) * d.alphar, cudaMemcpyHostToDevice, c->st));
  }
  CK(cudaMemcpyAsync(c->d_slater, c->slater.data(), sizeof(double) * d.n_slater, cudaMemcpyHostToDevice, c->st));
  if (d.alphac > 0) {  // Wcirr(iw, f) pairs in column-major order = the device's [f][N][2]
    CK(cudaMemcpyAsync(c->d_Wc, c->Wc.data(), sizeof(double) * c->Wc.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->d_bc, c->bc.data(), sizeof(double) * c->bc.size(), cudaMemcpyHostToDevice, c->st));
  }
  if (d.skew) {
    CK(rbmpp_build_se(d, c->d_wmap, c->d_orb, c->d_slater, c->d_SE, c->st));
  } else {
    long long tot = (long long)d.n_qp * d.N * d.N;
    rbmpp_note_launch();
    build_xf_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, c->st>>>(d.N, d.n_mp, c->d_wmap, c->d_orb, c->d_slater,
                                                                        d.sp_cc[0], d.sp_ss[0], d.sp_cc[1],
                                                                        d.sp_ss[1], c->d_XF, c->d_XFT);
    CK(cudaGetLastError());
  }
  c->d.shift = c->shift;
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int ensure_measure_buffers(rbmpp_ctx* c) {
  if (c->d_O) return 0;
  const DevDims& d = c->d;
  c->ns_tot = d.nw * d.ns;
  c->nrows = c->ns_tot * (d.cplx ? 2 : 1);
  int r;
  if ((r = dalloc(c, &c->d_O, (size_t)c->nrows * d.Nv))) return r;
  if ((r = dalloc(c, &c->d_psiS, (size_t)c->ns_tot * (d.n_qp + 1) * 2))) return r;
  if ((r = dalloc(c, &c->d_eloc, (size_t)c->ns_tot * 2))) return r;
  if ((r = dalloc(c, &c->d_a, (size_t)c->nrows))) return r;
  if ((r = dalloc(c, &c->d_b, (size_t)c->nrows))) return r;
  if ((r = dalloc(c, &c->d_tmp_ns, (size_t)c->nrows))) return r;
  if ((r = dalloc(c, &c->d_acc4, 4))) return r;
  if ((r = dalloc(c, &c->d_nap, (size_t)c->ns_tot))) return r;
  if ((r = dalloc(c, &c->d_estat, (size_t)c->ns_tot))) return r;
  if ((r = dalloc(c, &c->d_gvec, (size_t)d.Nv))) return r;
  if ((r = dalloc(c, &c->d_Ovec, (size_t)d.Nv))) return r;
  if ((r = dalloc(c, &c->d_vec, (size_t)4 * d.Nv))) return r;
  if ((r = dalloc(c, &c->d_S, (size_t)d.Nv * d.Nv))) return r;
  if ((r = dalloc(c, &c->d_part, (size_t)2 * 64 * d.Nv))) return r;
  if ((r = dalloc(c, &c->d_info, 4))) return r;
  if ((r = dalloc(c, &c->d_err, 4))) return r;
  if ((r = dalloc(c, &c->d_rv, (size_t)2 * d.Nv))) return r;
  if ((r = dalloc(c, &c->d_dinv, rbmpp_chol_work(d.Nv)))) return r;
  if ((r = dalloc(c, &c->d_pcg, (size_t)10 * d.Nv))) return r;
  if ((r = dalloc(c, &c->d_gpart, (size_t)rbmpp_gram_parts() * d.Nv))) return r;
  if ((r = dalloc(c, &c->d_sc, 8))) return r;
  if ((r = dalloc(c, &c->d_bar, 4))) return r;
  CK(cudaMallocHost(&c->h_sc, 8 * sizeof(double)));
  return 0;
}

// The host all-reduce of rbmpp_set_allreduce on n doubles at device address p, with the stream drained first.
int reduce_dev(rbmpp_ctx* c, double* p, long long n, const char* what) {
  CK(cudaStreamSynchronize(c->st));
  const int r = c->red_fn(c->red_user, p, n);
  if (r) return fail(c, RBMPP_E_COMM, "host all-reduce of %s returned %d", what, r);
  return 0;
}

// main.f90:348-369 across ranks: {Etot, Etot2, norm, wf_av, naccept_total, n_samples} and, when with_vectors,
// gvec and Ovec, summed in one call of the host all-reduce.
int reduce_measurement(rbmpp_ctx* c, bool with_vectors) {
  const size_t nv = c->d.Nv;
  int r;
  if (!c->d_xch && (r = dalloc(c, &c->d_xch, 6 + 2 * nv))) return r;
  double h6[6] = {c->meas_scal[0], c->meas_scal[1], c->meas_scal[2], c->meas_scal[3], (double)c->naccept_total,
                  c->n_samples_total};
  CK(cudaMemcpyAsync(c->d_xch, h6, sizeof(h6), cudaMemcpyHostToDevice, c->st));
  if (with_vectors) {
    CK(cudaMemcpyAsync(c->d_xch + 6, c->d_gvec, sizeof(double) * nv, cudaMemcpyDeviceToDevice, c->st));
    CK(cudaMemcpyAsync(c->d_xch + 6 + nv, c->d_Ovec, sizeof(double) * nv, cudaMemcpyDeviceToDevice, c->st));
  }
  if ((r = reduce_dev(c, c->d_xch, with_vectors ? 6 + 2 * (long long)nv : 6, "the measurement"))) return r;
  CK(cudaMemcpyAsync(h6, c->d_xch, sizeof(h6), cudaMemcpyDeviceToHost, c->st));
  if (with_vectors) {
    CK(cudaMemcpyAsync(c->d_gvec, c->d_xch + 6, sizeof(double) * nv, cudaMemcpyDeviceToDevice, c->st));
    CK(cudaMemcpyAsync(c->d_Ovec, c->d_xch + 6 + nv, sizeof(double) * nv, cudaMemcpyDeviceToDevice, c->st));
  }
  CK(cudaStreamSynchronize(c->st));
  for (int k = 0; k < 4; k++) c->meas_scal[k] = h6[k];
  c->naccept_total = (long long)h6[4];
  c->n_samples_total = h6[5];
  return 0;
}

// S_raw = sum over samples of O O^T (the dgemm of calc_phys_quantity.f90:240) for the current
// measurement, in FP64 or as split-BF16 products on the tensor cores (exact FP64 diagonal).
// The split-BF16 form multiplies the centred derivatives O' = O - b m^T (b: the per-sample weights of Ovec,
// m = Ovec / norm), whose products sum to S_raw - Ovec Ovec^T / norm, and adds Ovec Ovec^T / norm back in
// FP64: the BF16 pieces then carry the fluctuations only, not the mean that S = S_raw / norm - m m^T cancels,
// which would magnify their rounding.  The diagonal is the exact FP64 one of S_raw.
int build_S(rbmpp_ctx* c, int prec) {
  if (c->S_valid && c->S_prec == prec) return 0;
  if (c->S_reduced)
    return fail(c, RBMPP_E_STATE, "S was loaded by exchange_measurement in precision %d; cannot rebuild in %d",
                c->S_prec, prec);
  const DevDims& d = c->d;
  CK(cudaEventRecord(c->ev[5], c->st));
  const long long nS = (long long)d.Nv * d.Nv;
  if (prec == RBMPP_SR_FP64) {
    CK(rbmpp_syrk_ot_o(d.Nv, c->nrows, c->d_O, c->d_S, c->st));
    if (c->red_fn) {
      const int r = reduce_dev(c, c->d_S, nS, "S");
      if (r) return r;
    }
  } else if (prec == RBMPP_SR_SPLIT_BF16) {
    if (!c->d_hi) {
      int kp = 0, np = 0;
      rbmpp_bf16x3_pads(c->nrows, d.Nv, &kp, &np);
      const size_t bytes = (size_t)kp * np * 2;
      cudaError_t e = cudaMalloc(&c->d_hi, bytes);
      if (!e) e = cudaMalloc(&c->d_lo, bytes);
      if (e) return fail(c, RBMPP_E_CUDA, "cudaMalloc(split-BF16 operands, 2 x %zu bytes): %s", bytes,
                         cudaGetErrorString(e));
      c->bytes += 2 * bytes;
    }
    const double norm = c->meas_scal[2];
    double* d_m = c->d_rv;  // m = Ovec / norm
    CK(rbmpp_scale_copy(d.Nv, c->d_Ovec, 1.0 / norm, d_m, c->st));
    const int r = rbmpp_syrk_bf16x3(c->nrows, d.Nv, c->d_O, c->d_b, d_m, c->d_hi, c->d_lo, c->d_err, c->d_S,
                                    c->d_part, c->st);
    if (r == 1) return fail(c, RBMPP_E_CUDA, "cuTensorMapEncodeTiled unavailable from the driver");
    if (r) return fail(c, RBMPP_E_CUDA, "split-BF16 S build: %s", cudaGetErrorString((cudaError_t)(r - 100)));
    if (c->red_fn) {
      // every rank's centred product about the global mean, and its exact diagonal, summed over the ranks
      const int rr = reduce_dev(c, c->d_S, nS, "S");
      if (rr) return rr;
    }
    CK(rbmpp_add_outer_offdiag(d.Nv, c->d_S, c->d_Ovec, 1.0 / norm, c->st));  // upper triangle only
    CK(rbmpp_symmetrize(d.Nv, c->d_S, c->st));
  } else {
    return fail(c, RBMPP_E_ARG, "unknown S precision %d", prec);
  }
  CK(cudaEventRecord(c->ev[6], c->st));
  CK(cudaStreamSynchronize(c->st));
  if (prec == RBMPP_SR_SPLIT_BF16) {
    int err = 0;
    CK(cudaMemcpy(&err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return fail(c, RBMPP_E_TIMEOUT, "split-BF16 S build: a bounded device wait ran out");
  }
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, c->ev[5], c->ev[6]));
  c->stats[3] = ms;
  c->S_valid = true;
  c->S_prec = prec;
  return 0;
}

// y = A x with A = D (S_raw / norm - m m^T) D + sigma I, D = diag(1 on the RBM block, scal on the Pfaffian
// block), m = Ovec / norm in the refinement vector VM: the conditioned S of SR_pdposv.f90:4-170 applied
// exactly in FP64 through O (S_raw x = O^T (O x)) without forming S.  x, y: device vectors.
enum { VG = 0, VX, VR, VZ, VP, VAP, VWS, VZZ, VTMP, VM };
int apply_A(rbmpp_ctx* c, double norm, double scal, double sigma, const double* x, double* y) {
  const DevDims& d = c->d;
  double* v = c->d_pcg;
  const size_t Nv = d.Nv;
  CK(rbmpp_sr_apply_gram(c->nrows, d.Nv, d.Nv_rbm, c->d_O, v + VM * Nv, scal, x, v + VWS * Nv, v + VZZ * Nv,
                         c->d_gpart, c->d_tmp_ns, c->d_part, c->d_sc, c->st));
  if (c->red_fn) {
    const int r = reduce_dev(c, v + VZZ * Nv, d.Nv, "O^T O x");
    if (r) return r;
  }
  CK(rbmpp_sr_apply_finish(d.Nv, d.Nv_rbm, v + VM * Nv, norm, scal, sigma, x, v + VZZ * Nv, c->d_sc, y, c->st));
  return 0;
}

int check_walker_status(rbmpp_ctx* c, const int* d_status, int n, const char* what) {
  std::vector<int> st(n);
  CK(cudaMemcpy(st.data(), d_status, sizeof(int) * n, cudaMemcpyDeviceToHost));
  for (int i = 0; i < n; i++)
    if (st[i]) return fail(c, st[i], "%s failed on item %d (code %d)", what, i, st[i]);
  return 0;
}

}  // namespace

// ===================================================================================================
extern "C" {

int rbmpp_create(const rbmpp_dims* dims, rbmpp_ctx** out) {
  if (!dims || !out) return RBMPP_E_ARG;
  *out = nullptr;
  rbmpp_ctx* c = new rbmpp_ctx();
  c->dims = *dims;
  DevDims& d = c->d;
  std::memset(&d, 0, sizeof(d));
  if (dims->L < 2 || dims->L * dims->L > RBMPP_MAX_N || (dims->L * dims->L) % 2) {
    int r = fail(c, RBMPP_E_ARG, "unsupported L=%d (N must be even and <= %d)", dims->L, RBMPP_MAX_N);
    *out = c;
    return r;
  }
  if (dims->n_mp_trans < 1 || dims->alphar < 0 || dims->alphac < 0 || dims->n_slater < 1 || dims->nsample < 1 ||
      dims->n_walkers < 1) {
    *out = c;
    return fail(c, RBMPP_E_ARG, "bad dimensions");
  }
  d.L = dims->L;
  d.N = d.L * d.L;
  d.Np = d.N / 2;
  if ((d.Np + 31) / 32 > RBMPP_MAX_KPL) {
    *out = c;
    return fail(c, RBMPP_E_ARG, "N/2 = %d exceeds the supported Pfaffian block size", d.Np);
  }
  d.n_mp = dims->n_mp_trans;
  d.n_qp = 2 * d.n_mp;
  d.alphar = dims->alphar;
  d.Mr = dims->alphar * d.n_mp * 2;
  d.alphac = dims->alphac;
  d.Mc = dims->alphac * d.n_mp * 2;  // main.f90:134
  d.cplx = d.alphac > 0;             // complex units make psi complex
  d.n_slater = dims->n_slater;
  d.Nv = 2 * dims->alphac * (d.N + 1) + dims->alphar * (d.N + 1) + d.n_slater;  // main.f90:136
  d.Nv_rbm = d.Nv - d.n_slater;
  d.nw = dims->n_walkers;
  d.ns = dims->nsample;
  d.nupdate = d.N;                        // main.f90:139
  d.nwarm = std::max(30, d.ns / 100);     // make_sample.f90:66
  d.pf_sign = ((d.Np * (d.Np - 1) / 2) % 2) ? -1 : 1;
  d.J1 = dims->J1;
  d.J2 = dims->J2;
  // spin projection weights, spin_projection.f90:25-63 (beta = 0, pi)
  const double pi = std::acos(-1.0);
  double beta[2] = {0.0, pi};
  for (int s = 0; s < 2; s++) {
    double co = std::cos(0.5 * beta[s]), si = std::sin(0.5 * beta[s]);
    d.sp_cc[s] = co * co;
    d.sp_cs[s] = co * si;
    d.sp_ss[s] = si * si;
  }
  d.para_sp[0] = 1.0;
  d.para_sp[1] = dims->spin_parity == 1 ? 1.0 : -1.0;
  *out = c;
  cudaError_t e = cudaSetDevice(dims->device);
  if (e != cudaSuccess) return fail(c, RBMPP_E_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
  CK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
  for (auto& e : c->ev) CK(cudaEventCreate(&e));
  int maxsm = 0;
  CK(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dims->device));
  // large blocks (N/2 > ~120): the direct sampler's Gauss-Jordan tile moves to a per-walker global scratch
  if ((long long)rbmpp_sampler_smem(d, 256) > maxsm) d.gj_global = 1;
  if ((long long)rbmpp_sampler_smem(d, 256) > maxsm)
    return fail(c, RBMPP_E_ARG, "sampler workspace %zu B exceeds %d B of shared memory", rbmpp_sampler_smem(d, 256),
                maxsm);
  c->est_fits = (long long)rbmpp_estimator_smem_any(d, maxsm) <= maxsm;
  c->est_smem_tiles = (long long)rbmpp_estimator_smem(d, 256) <= maxsm;
  c->stream_stages = rbmpp_stream_stages(d, maxsm);
  if (getenv("RBMPP_SAMPLER") && std::string(getenv("RBMPP_SAMPLER")) == "direct") c->stream_stages = 0;
  if (d.alphac) c->stream_stages = 0;  // the streaming sampler carries real units only
  int r;
  const int N = d.N;
  if ((r = dalloc(c, &c->d_wmap, (size_t)d.n_mp * N))) return r;
  if ((r = dalloc(c, &c->d_winv, (size_t)d.n_mp * N))) return r;
  if ((r = dalloc(c, &c->d_orb, (size_t)N * N))) return r;
  if ((r = dalloc(c, &c->d_bonds, (size_t)8 * N))) return r;
  if ((r = dalloc(c, &c->d_subB, (size_t)N))) return r;
  if ((r = dalloc(c, &c->d_para, (size_t)2 * d.n_mp))) return r;
  if ((r = dalloc(c, &c->d_Wr, (size_t)std::max(1, d.alphar) * N))) return r;
  if ((r = dalloc(c, &c->d_br, (size_t)std::max(1, d.alphar)))) return r;
  if ((r = dalloc(c, &c->d_Wc, (size_t)2 * std::max(1, d.alphac) * N))) return r;
  if ((r = dalloc(c, &c->d_bc, (size_t)2 * std::max(1, d.alphac)))) return r;
  if ((r = dalloc(c, &c->d_slater, (size_t)d.n_slater))) return r;
  if ((r = dalloc(c, &c->d_XF, (size_t)d.n_qp * N * N))) return r;
  if ((r = dalloc(c, &c->d_XFT, (size_t)d.n_qp * N * N))) return r;
  DevWalkers& W = c->W;
  const size_t nw = d.nw, ns = d.ns;
  if ((r = dalloc(c, &W.x, nw * N))) return r;
  if ((r = dalloc(c, &W.idx, nw * N))) return r;
  if ((r = dalloc(c, &W.cfg, nw * N))) return r;
  if ((r = dalloc(c, &W.th, nw * std::max(1, d.Mr)))) return r;
  if ((r = dalloc(c, &W.sgn, nw * d.n_mp))) return r;
  if ((r = dalloc(c, &W.pf, nw * d.n_qp))) return r;
  if ((r = dalloc(c, &W.psi, nw * d.n_qp * 2))) return r;
  if ((r = dalloc(c, &W.Y, nw * d.n_qp * (size_t)d.Np * d.Np))) return r;
  if ((r = dalloc(c, &W.mt, nw * 625))) return r;
  if ((r = dalloc(c, &W.nfastup, nw))) return r;
  if ((r = dalloc(c, &W.naccept, nw))) return r;
  if ((r = dalloc(c, &W.nacc_all, nw))) return r;
  if ((r = dalloc(c, &W.status, nw))) return r;
  if ((r = dalloc(c, &W.events, nw * 5))) return r;
  CK(cudaMemset(W.events, 0, sizeof(int) * nw * 5));
  if ((r = dalloc(c, &W.xs, nw * ns * N))) return r;
  if ((r = dalloc(c, &W.pfs, nw * ns * d.n_qp))) return r;
  if ((r = dalloc(c, &W.psis, nw * ns * (d.n_qp + 1) * 2))) return r;
  if (d.gj_global && (r = dalloc(c, &W.gj, nw * (size_t)d.Np * (d.Np + 1)))) return r;
  std::vector<int> nf(nw, std::min(100, N * 2));  // main.f90:309
  CK(cudaMemcpy(W.nfastup, nf.data(), sizeof(int) * nw, cudaMemcpyHostToDevice));
  // sublattice and bonds: define_sublattice (interface_for_PP.f90:110-136), bond_map (:382-427)
  std::vector<unsigned char> subB(N);
  {
    int i = 0;
    for (int i2 = 0; i2 < d.L; i2++)
      for (int i1 = 0; i1 < d.L; i1++) subB[i++] = ((i1 + i2) % 2 == 1);
  }
  std::vector<int> bonds(8 * N);
  for (int i0 = 1; i0 <= 4; i0++)
    for (int i1 = 0; i1 < N; i1++) {
      int ix = i1 / d.L, iy = i1 % d.L;
      if (i0 == 1) ix = (ix + 1) % d.L;
      else if (i0 == 2) iy = (iy + 1) % d.L;
      else if (i0 == 3) {
        ix = (ix + 1) % d.L;
        iy = (iy + 1) % d.L;
      } else {
        ix = (ix + 1) % d.L;
        iy = (iy - 1 + d.L) % d.L;
      }
      int b = (i0 - 1) * N + i1;
      bonds[2 * b] = i1;
      bonds[2 * b + 1] = ix * d.L + iy;
    }
  CK(cudaMemcpy(c->d_subB, subB.data(), N, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_bonds, bonds.data(), sizeof(int) * 8 * N, cudaMemcpyHostToDevice));
  c->Wr.assign((size_t)N * d.alphar, 0.0);
  c->br.assign(d.alphar, 0.0);
  c->Wc.assign((size_t)2 * N * d.alphac, 0.0);
  c->bc.assign((size_t)2 * d.alphac, 0.0);
  c->slater.assign(d.n_slater, 0.0);
  return 0;
}

int rbmpp_destroy(rbmpp_ctx* c) {
  if (!c) return 0;
  void* ptrs[] = {c->d_wmap, c->d_winv, c->d_orb, c->d_bonds, c->d_subB, c->d_para, c->d_Wr, c->d_br, c->d_slater,
                  c->d_Wc, c->d_bc,
                  c->d_XF, c->d_XFT, c->W.x, c->W.idx, c->W.cfg, c->W.th, c->W.sgn, c->W.pf, c->W.psi, c->W.Y,
                  c->W.mt, c->W.nfastup, c->W.naccept, c->W.nacc_all, c->W.status, c->W.xs, c->W.pfs, c->W.psis, c->W.gj, c->W.events, c->W.trace, (void*)c->W.replay, c->d_O, c->d_psiS,
                  c->d_eloc, c->d_a, c->d_b, c->d_tmp_ns, c->d_acc4, c->d_nap, c->d_estat, c->d_gvec, c->d_Ovec,
                  c->d_vec, c->d_S, c->d_part, c->d_info, c->d_err, c->d_rv, c->d_hi, c->d_lo, c->d_Sf, c->d_Sb,
                  c->d_crow, c->d_csd, c->d_cones, c->d_cvbs, c->d_cpart, c->d_csum, c->d_dinv, c->d_pcg, c->d_gpart, c->d_sc, c->d_bar, c->d_xch, c->d_SE};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (c->h_sc) cudaFreeHost(c->h_sc);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  return 0;
}

const char* rbmpp_last_error(const rbmpp_ctx* c) { return c ? c->err.c_str() : "null context"; }

int rbmpp_query(const rbmpp_ctx* c, int what, long long* v) {
  if (!c || !v) return RBMPP_E_ARG;
  switch (what) {
    case 0: *v = c->d.Nv; break;
    case 1: *v = c->d.Nv_rbm; break;
    case 2: *v = c->d.Mr; break;
    case 3: *v = c->d.n_qp; break;
    case 4: *v = c->d.N; break;
    case 5: *v = (long long)c->bytes; break;
    case 6: *v = g_launches.load(std::memory_order_relaxed); break;
    default: return RBMPP_E_ARG;
  }
  return 0;
}

int rbmpp_set_tables(rbmpp_ctx* c, const int* W_map, const double* para, const int* orb_idx, const int* orb_sgn,
                     const int* subB, const double* sp_weights) {
  if (!c || !W_map || !para || !orb_idx) return fail(c, RBMPP_E_ARG, "null table");
  DevDims& d = c->d;
  const int N = d.N;
  if (sp_weights) {
    // InitSPWeight's products (spin_projection.f90:36-41).  When cos*sin vanishes at both points (beta in
    // {0, pi}) the same-spin blocks -(F - F^T) cos sin of slater.f90:36-44 vanish and the kernels carry the
    // Pfaffian as det X of the up-down block; otherwise (the transverse code's beta = -/+pi/2) they carry the
    // full N x N skew form.
    double cc[2], cs[2], ss[2];
    int skew = 0;
    for (int sp = 0; sp < 2; sp++) {
      const double co = sp_weights[3 * sp], si = sp_weights[3 * sp + 1], w = sp_weights[3 * sp + 2];
      if (!std::isfinite(co) || !std::isfinite(si) || !std::isfinite(w))
        return fail(c, RBMPP_E_ARG, "sp_weights: non-finite value at point %d", sp + 1);
      cc[sp] = co * co;
      cs[sp] = co * si;
      ss[sp] = si * si;
      if (!(std::fabs(cs[sp]) <= 1e-12 * std::max(cc[sp], ss[sp]))) skew = 1;
    }
    if (skew && d.N > rbmpp_skew_max_n())
      return fail(c, RBMPP_E_ARG, "sp_weights: the skew form (same-spin blocks present) supports N <= %d, not %d",
                  rbmpp_skew_max_n(), d.N);
    if (skew) {
      DevDims t = d;
      t.skew = 1;
      int maxsm = 0;
      CK(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->dims.device));
      const size_t need = rbmpp_skew_smem_shortfall(t, maxsm);
      if (need) return fail(c, RBMPP_E_ARG, "skew-form workspace %zu B exceeds %d B of shared memory", need, maxsm);
    }
    if (skew != d.skew) {
      // the per-walker inverses change shape: Np x Np blocks or N x N skew matrices
      const size_t nw = d.nw, np2 = (size_t)d.n_qp * (skew ? (size_t)d.N * d.N : (size_t)d.Np * d.Np);
      CK(cudaFree(c->W.Y));
      c->bytes -= sizeof(double) * nw * d.n_qp * (d.skew ? (size_t)d.N * d.N : (size_t)d.Np * d.Np);
      c->W.Y = nullptr;
      int r = dalloc(c, &c->W.Y, nw * np2);
      if (r) return r;
      if (skew && !c->d_SE && (r = dalloc(c, &c->d_SE, (size_t)d.n_qp * 4 * d.N * d.N))) return r;
      d.skew = skew;
      c->sampled = false;
    }
    for (int sp = 0; sp < 2; sp++) {
      d.sp_cc[sp] = cc[sp];
      d.sp_cs[sp] = cs[sp];
      d.sp_ss[sp] = ss[sp];
      d.para_sp[sp] = sp_weights[3 * sp + 2];
    }
  }
  if (subB) {
    std::vector<unsigned char> sb(N);
    for (int i = 0; i < N; i++) {
      if (subB[i] != 0 && subB[i] != 1) return fail(c, RBMPP_E_ARG, "subB(%d) = %d is neither 0 nor 1", i + 1, subB[i]);
      sb[i] = (unsigned char)subB[i];
    }
    CK(cudaMemcpy(c->d_subB, sb.data(), N, cudaMemcpyHostToDevice));
  }
  std::vector<int> wmap((size_t)d.n_mp * N), winv((size_t)d.n_mp * N);
  for (int mp = 0; mp < d.n_mp; mp++) {
    std::vector<char> seen(N, 0);
    for (int i = 0; i < N; i++) {
      int v = W_map[i + (size_t)N * mp];
      if (v < 1 || v > N) return fail(c, RBMPP_E_ARG, "W_map wrong 1 (sym_info.txt)");
      if (seen[v - 1]) return fail(c, RBMPP_E_ARG, "W_map wrong 2 (sym_info.txt)");
      seen[v - 1] = 1;
      wmap[(size_t)mp * N + i] = v - 1;
      winv[(size_t)mp * N + (v - 1)] = i;
    }
  }
  int cplx = d.alphac > 0;
  for (int mp = 0; mp < d.n_mp; mp++)
    if (para[2 * mp + 1] != 0.0) cplx = 1;
  if (cplx && d.skew)
    return fail(c, RBMPP_E_ARG, "complex para_mp_trans or complex RBM units with the transverse (skew-form) projection "
                                "are not supported");
  if (cplx != d.cplx && c->d_O)
    return fail(c, RBMPP_E_STATE, "complex para_mp_trans changed after measurement buffers were sized");
  d.cplx = cplx;
  c->orb_host.assign((size_t)N * N, 0);
  std::vector<int> cnt(d.n_slater, 0);
  for (int p = 0; p < N; p++)
    for (int q = 0; q < N; q++) {
      int v = orb_idx[p + (size_t)N * q];  // Orbital_Idx(p, q), column-major
      if (v < 1 || v > d.n_slater) return fail(c, RBMPP_E_ARG, "error4, orbitalidx");
      if (orb_sgn && orb_sgn[p + (size_t)N * q] != 1)
        return fail(c, RBMPP_E_ARG, "Orbital_Sgn /= 1 (anti-periodic boundary) is not supported");
      c->orb_host[(size_t)p * N + q] = v - 1;
      cnt[v - 1]++;
    }
  int inj = 1;
  for (int k = 0; k < d.n_slater; k++)
    if (cnt[k] > 1) inj = 0;
  c->d.orb_injective = inj;
  CK(cudaMemcpy(c->d_wmap, wmap.data(), sizeof(int) * wmap.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_winv, winv.data(), sizeof(int) * winv.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_para, para, sizeof(double) * 2 * d.n_mp, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_orb, c->orb_host.data(), sizeof(int) * c->orb_host.size(), cudaMemcpyHostToDevice));
  c->tables_set = true;
  return 0;
}

int rbmpp_set_params(rbmpp_ctx* c, const double* Wr, const double* br, const double* Wc, const double* bc,
                     const double* slater, double shift) {
  if (!c) return RBMPP_E_ARG;
  if ((Wc || bc) && c->d.alphac == 0) return fail(c, RBMPP_E_ARG, "complex RBM parameters given but alphac = 0");
  if (!c->tables_set) return fail(c, RBMPP_E_STATE, "rbmpp_set_tables must come first");
  if (Wc) std::memcpy(c->Wc.data(), Wc, sizeof(double) * c->Wc.size());
  if (bc) std::memcpy(c->bc.data(), bc, sizeof(double) * c->bc.size());
  if (Wr) std::memcpy(c->Wr.data(), Wr, sizeof(double) * c->Wr.size());
  if (br) std::memcpy(c->br.data(), br, sizeof(double) * c->br.size());
  if (slater) std::memcpy(c->slater.data(), slater, sizeof(double) * c->slater.size());
  c->shift = shift;
  c->params_set = true;
  return upload_params(c);
}

int rbmpp_get_params(rbmpp_ctx* c, double* Wr, double* br, double* slater, double* shift) {
  if (!c) return RBMPP_E_ARG;
  if (Wr) std::memcpy(Wr, c->Wr.data(), sizeof(double) * c->Wr.size());
  if (br) std::memcpy(br, c->br.data(), sizeof(double) * c->br.size());
  if (slater) std::memcpy(slater, c->slater.data(), sizeof(double) * c->slater.size());
  if (shift) *shift = c->shift;
  return 0;
}

int rbmpp_get_params_c(rbmpp_ctx* c, double* Wc, double* bc) {
  if (!c) return RBMPP_E_ARG;
  if (Wc) std::memcpy(Wc, c->Wc.data(), sizeof(double) * c->Wc.size());
  if (bc) std::memcpy(bc, c->bc.data(), sizeof(double) * c->bc.size());
  return 0;
}

int rbmpp_seed_walkers(rbmpp_ctx* c, int iseed0) {
  if (!c) return RBMPP_E_ARG;
  rbmpp_note_launch();
  seed_kernel<<<(c->d.nw + 63) / 64, 64, 0, c->st>>>(c->W.mt, c->d.nw, iseed0, c->d.ns, c->dims.walker_offset);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->st));
  c->seeded = true;
  return 0;
}

int rbmpp_rank0_grnd(rbmpp_ctx* c, int n, double* out) {
  if (!c || n < 0) return RBMPP_E_ARG;
  if (n == 0) return 0;
  double* d_out = nullptr;
  CK(cudaMalloc(&d_out, sizeof(double) * n));
  rbmpp_note_launch();
  draw_kernel<<<1, 1, 0, c->st>>>(c->W.mt, n, d_out);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
  cudaFree(d_out);
  if (e != cudaSuccess) return fail(c, RBMPP_E_CUDA, "rank0_grnd: %s", cudaGetErrorString(e));
  return 0;
}

int rbmpp_make_sample(rbmpp_ctx* c, int first, int* naccept, long long* naccept_total) {
  if (!c) return RBMPP_E_ARG;
  if (!c->params_set || !c->seeded) return fail(c, RBMPP_E_STATE, "set_params and seed_walkers must come first");
  if (!first && !c->sampled) return fail(c, RBMPP_E_STATE, "make_sample(first=0) before any sample exists");
  c->d.shift = c->shift;
  CK(cudaEventRecord(c->ev[0], c->st));
  if (c->d.skew)
    CK(rbmpp_launch_sampler_skew(c->d, tables(c), params(c), c->W, first ? 1 : 0, c->st));
  else if (c->stream_stages > 0)
    CK(rbmpp_launch_sampler_stream(c->d, tables(c), params(c), c->W, first ? 1 : 0, c->stream_stages, c->st));
  else
    CK(rbmpp_launch_sampler(c->d, tables(c), params(c), c->W, first ? 1 : 0, c->st));
  CK(cudaEventRecord(c->ev[1], c->st));
  CK(cudaStreamSynchronize(c->st));
  int r = check_walker_status(c, c->W.status, c->d.nw, "make_sample");
  if (r) return r;
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
  c->stats[0] = ms;
  std::vector<int> na(c->d.nw), naa(c->d.nw);
  CK(cudaMemcpy(na.data(), c->W.naccept, sizeof(int) * c->d.nw, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(naa.data(), c->W.nacc_all, sizeof(int) * c->d.nw, cudaMemcpyDeviceToHost));
  long long tot = 0, tot_all = 0;
  for (int v : na) tot += v;
  for (int v : naa) tot_all += v;
  c->stats[5] = (double)tot_all;
  c->stats[6] = (double)c->d.nw * (double)(c->d.nwarm + c->d.ns + 1) * (double)c->d.nupdate;
  if (naccept) std::memcpy(naccept, na.data(), sizeof(int) * c->d.nw);
  if (naccept_total) *naccept_total = tot;
  c->naccept_total = tot;
  c->sampled = true;
  c->measured = false;
  return 0;
}

int rbmpp_get_samples(rbmpp_ctx* c, int* x, double* psi, double* pf) {
  if (!c) return RBMPP_E_ARG;
  const DevDims& d = c->d;
  const long long nx = (long long)d.nw * d.ns * d.N;
  if (x) {
    int* dx = nullptr;
    CK(cudaMalloc(&dx, sizeof(int) * nx));
    rbmpp_note_launch();
    i8_to_int_kernel<<<(unsigned)((nx + 255) / 256), 256, 0, c->st>>>(c->W.xs, dx, nx);
    cudaError_t e = cudaMemcpyAsync(x, dx, sizeof(int) * nx, cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    cudaFree(dx);
    if (e != cudaSuccess) return fail(c, RBMPP_E_CUDA, "get_samples: %s", cudaGetErrorString(e));
  }
  if (psi) CK(cudaMemcpy(psi, c->W.psis, sizeof(double) * d.nw * d.ns * (d.n_qp + 1) * 2, cudaMemcpyDeviceToHost));
  if (pf) CK(cudaMemcpy(pf, c->W.pfs, sizeof(double) * d.nw * d.ns * d.n_qp, cudaMemcpyDeviceToHost));
  return 0;
}

int rbmpp_set_samples(rbmpp_ctx* c, const int* x) {
  if (!c || !x) return RBMPP_E_ARG;
  const DevDims& d = c->d;
  const long long nx = (long long)d.nw * d.ns * d.N;
  int* dx = nullptr;
  CK(cudaMalloc(&dx, sizeof(int) * nx));
  cudaError_t e = cudaMemcpyAsync(dx, x, sizeof(int) * nx, cudaMemcpyHostToDevice, c->st);
  if (e == cudaSuccess) {
    rbmpp_note_launch();
    int_to_i8_kernel<<<(unsigned)((nx + 255) / 256), 256, 0, c->st>>>(dx, c->W.xs, nx);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
  cudaFree(dx);
  if (e != cudaSuccess) return fail(c, RBMPP_E_CUDA, "set_samples: %s", cudaGetErrorString(e));
  c->sampled = true;
  return 0;
}

static int measure_common(rbmpp_ctx* c, bool with_o) {
  const DevDims& d = c->d;
  if (!c->est_fits && !d.skew)
    return fail(c, RBMPP_E_ARG, "the estimator's workspace for N/2 = %d exceeds the shared memory of one block", d.Np);
  int r = ensure_measure_buffers(c);
  if (r) return r;
  c->S_valid = false;
  c->S_reduced = false;
  c->d.shift = c->shift;
  CK(cudaEventRecord(c->ev[2], c->st));
  if (d.skew)
    CK(rbmpp_launch_estimator_skew(c->d, tables(c), params(c), c->W.xs, c->ns_tot, c->d_psiS, c->d_eloc,
                                   with_o ? c->d_O : nullptr, c->d_nap, c->d_estat, 1, c->st));
  else
    CK(rbmpp_launch_estimator(c->d, tables(c), params(c), c->W.xs, c->ns_tot, c->d_psiS, c->d_eloc,
                              with_o ? c->d_O : nullptr, c->d_nap, c->d_estat, 1, c->st));
  CK(cudaEventRecord(c->ev[3], c->st));
  CK(cudaStreamSynchronize(c->st));
  {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]));
    c->stats[1] = ms;
  }
  r = check_walker_status(c, c->d_estat, c->ns_tot, "calc_phys_quantity");
  if (r) return r;
  CK(rbmpp_sample_scalars(c->ns_tot, c->d_psiS, (d.n_qp + 1) * 2, c->d_eloc, c->shift, c->d_a, c->d_b, c->d_acc4,
                          d.cplx, c->st));
  CK(cudaMemcpyAsync(c->meas_scal, c->d_acc4, sizeof(double) * 4, cudaMemcpyDeviceToHost, c->st));
  c->n_samples_total = (double)d.nw * (double)d.ns;
  // the amplitude draws of the measurement advance each walker's stream
  CK(rbmpp_launch_advance_rng(c->W.mt, c->d_nap, d.ns, d.nw, 0, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int rbmpp_measure(rbmpp_ctx* c, double* scal, double* gvec, double* Ovec, double* Smat) {
  if (!c) return RBMPP_E_ARG;
  if (!c->sampled) return fail(c, RBMPP_E_STATE, "measure before make_sample");
  const DevDims& d = c->d;
  int r = measure_common(c, true);
  if (r) return r;
  CK(cudaEventRecord(c->ev[4], c->st));
  CK(rbmpp_gemv_ot(c->nrows, d.Nv, c->d_O, c->d_a, c->d_b, c->d_gvec, c->d_Ovec, c->d_part, 64, c->st));
  CK(cudaEventRecord(c->ev[11], c->st));
  CK(cudaStreamSynchronize(c->st));
  {
    float a1 = 0.f;
    CK(cudaEventElapsedTime(&a1, c->ev[4], c->ev[11]));
    c->stats[2] = a1;
  }
  if (c->red_fn && (r = reduce_measurement(c, true))) return r;
  // S itself is built when it is first needed (here if Smat is wanted, else by exchange or SR step)
  if (Smat && (r = build_S(c, c->meas_prec))) return r;
  if (scal) std::memcpy(scal, c->meas_scal, sizeof(double) * 4);
  if (gvec) CK(cudaMemcpy(gvec, c->d_gvec, sizeof(double) * d.Nv, cudaMemcpyDeviceToHost));
  if (Ovec) CK(cudaMemcpy(Ovec, c->d_Ovec, sizeof(double) * d.Nv, cudaMemcpyDeviceToHost));
  if (Smat) CK(cudaMemcpy(Smat, c->d_S, sizeof(double) * d.Nv * d.Nv, cudaMemcpyDeviceToHost));
  c->measured = true;
  return 0;
}

int rbmpp_measure_energy(rbmpp_ctx* c, double* scal) {
  if (!c) return RBMPP_E_ARG;
  if (!c->sampled) return fail(c, RBMPP_E_STATE, "measure before make_sample");
  int r = measure_common(c, false);
  if (r) return r;
  if (c->red_fn && (r = reduce_measurement(c, false))) return r;
  if (scal) std::memcpy(scal, c->meas_scal, sizeof(double) * 4);
  return 0;
}

// Calc_Correlation/calc_phys_quantity.f90:264-344 over the stored samples.  The per-sample rows are summed
// over samples by fixed partitions (rbmpp_gemv_ot with unit weights) and Chi_vbs(., t) = sum_s sdr sdr^T
// by the FP64 upper-triangle GEMM, so the sums do not depend on scheduling.
int rbmpp_measure_correlation(rbmpp_ctx* c, double* scal, double* chi_sp, double* chi_vbs) {
  if (!c) return RBMPP_E_ARG;
  if (!c->sampled) return fail(c, RBMPP_E_STATE, "measure before make_sample");
  if (c->d.skew)
    return fail(c, RBMPP_E_ARG, "correlation measurement: the Calc_Correlation program has no transverse projection");
  if (c->d.cplx)
    return fail(c, RBMPP_E_ARG, "correlation measurement with complex para_mp_trans is not supported");
  const DevDims& d = c->d;
  int dev = 0, maxsm = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (rbmpp_correlation_fits(d, maxsm) < 1)
    return fail(c, RBMPP_E_ARG, "the correlation workspace for N/2 = %d exceeds the shared memory of one block", d.Np);
  int r = ensure_measure_buffers(c);
  if (r) return r;
  const size_t nchi = (size_t)d.N * (d.N + 1) / 2, lr = 2 * nchi + 1;
  const int nparts = 64;
  if (!c->d_crow) {
    if ((r = dalloc(c, &c->d_crow, (size_t)c->ns_tot * lr))) return r;
    if ((r = dalloc(c, &c->d_csd, (size_t)c->ns_tot * 4 * d.N))) return r;
    if ((r = dalloc(c, &c->d_cones, (size_t)c->ns_tot))) return r;
    if ((r = dalloc(c, &c->d_cvbs, (size_t)4 * d.N * d.N))) return r;
    if ((r = dalloc(c, &c->d_cpart, (size_t)nparts * lr))) return r;
    if ((r = dalloc(c, &c->d_csum, lr))) return r;
    CK(rbmpp_fill(c->d_cones, c->ns_tot, 1.0, c->st));
  }
  c->S_valid = false;
  c->S_reduced = false;
  c->d.shift = c->shift;
  CK(cudaEventRecord(c->ev[2], c->st));
  CK(rbmpp_launch_correlation(c->d, tables(c), params(c), c->W.xs, c->ns_tot, c->d_psiS, c->d_eloc, c->d_crow,
                              c->d_csd, c->d_nap, c->d_estat, c->st));
  CK(cudaEventRecord(c->ev[3], c->st));
  CK(cudaStreamSynchronize(c->st));
  {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]));
    c->stats[1] = ms;
  }
  r = check_walker_status(c, c->d_estat, c->ns_tot, "calc_phys_quantity_after_opt (correlation)");
  if (r) return r;
  CK(rbmpp_sample_scalars(c->ns_tot, c->d_psiS, (d.n_qp + 1) * 2, c->d_eloc, c->shift, c->d_a, c->d_b, c->d_acc4,
                          0, c->st));
  CK(rbmpp_gemv_ot(c->ns_tot, (int)lr, c->d_crow, c->d_cones, nullptr, c->d_csum, nullptr, c->d_cpart, nparts, c->st));
  for (int t = 0; t < 4; t++)
    CK(rbmpp_gemm_atb_upper(d.N, c->ns_tot, c->d_csd + (size_t)t * d.N, 4LL * d.N, 1, c->d_cvbs + (size_t)t * d.N * d.N,
                            d.N, c->st));
  // one amplitude draw per sample, per antiparallel bond and per antiparallel site pair (N/2 x N/2 of them)
  CK(rbmpp_launch_advance_rng(c->W.mt, c->d_nap, d.ns, d.nw, d.ns * d.Np * d.Np, c->st));
  std::vector<double> sums(lr), vbs((size_t)4 * d.N * d.N);
  double s4[4];
  CK(cudaMemcpyAsync(s4, c->d_acc4, sizeof(double) * 4, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(sums.data(), c->d_csum, sizeof(double) * lr, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(vbs.data(), c->d_cvbs, sizeof(double) * vbs.size(), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  std::memcpy(c->meas_scal, s4, sizeof(s4));
  c->n_samples_total = (double)d.nw * (double)d.ns;
  if (scal) {
    std::memcpy(scal, s4, sizeof(s4));
    scal[4] = sums[2 * nchi];
  }
  if (chi_sp)
    for (size_t i0 = 0; i0 < nchi; i0++) {
      chi_sp[2 * i0] = sums[i0];
      chi_sp[2 * i0 + 1] = sums[nchi + i0];
    }
  if (chi_vbs)
    for (int t = 0; t < 4; t++) {
      const double* C = vbs.data() + (size_t)t * d.N * d.N;  // column-major, upper triangle
      size_t i0 = 0;
      for (int i2 = 0; i2 < d.N; i2++)
        for (int i1 = 0; i1 <= i2; i1++, i0++) chi_vbs[i0 + nchi * t] = C[i1 + (size_t)d.N * i2];
    }
  return 0;
}

int rbmpp_eval_configs(rbmpp_ctx* c, int n, const int* x, double* psi, double* hpsi, double* O) {
  if (!c || n < 0 || !x) return RBMPP_E_ARG;
  if (!c->params_set) return fail(c, RBMPP_E_STATE, "set_params must come first");
  if (n == 0) return 0;
  if (!c->est_fits && !c->d.skew)
    return fail(c, RBMPP_E_ARG, "the estimator's workspace for N/2 = %d exceeds the shared memory of one block",
                c->d.Np);
  const DevDims& d = c->d;
  int* dx = nullptr;
  int8_t* dx8 = nullptr;
  double *dpsi = nullptr, *dh = nullptr, *dO = nullptr;
  int* dst = nullptr;
  const long long nx = (long long)n * d.N;
  int rc = 0;
  cudaError_t e = cudaMalloc(&dx, sizeof(int) * nx);
  if (!e) e = cudaMalloc(&dx8, nx);
  if (!e) e = cudaMalloc(&dpsi, sizeof(double) * (size_t)n * (d.n_qp + 1) * 2);
  if (!e) e = cudaMalloc(&dh, sizeof(double) * 2 * (size_t)n);
  const size_t orows = (size_t)n * (d.cplx ? 2 : 1);  // complex weights: real and imaginary row per configuration
  if (!e && O) e = cudaMalloc(&dO, sizeof(double) * orows * d.Nv);
  if (!e) e = cudaMalloc(&dst, sizeof(int) * n);
  if (!e) e = cudaMemcpyAsync(dx, x, sizeof(int) * nx, cudaMemcpyHostToDevice, c->st);
  if (!e) {
    rbmpp_note_launch();
    int_to_i8_kernel<<<(unsigned)((nx + 255) / 256), 256, 0, c->st>>>(dx, dx8, nx);
    e = cudaGetLastError();
  }
  if (!e)
    e = d.skew ? rbmpp_launch_estimator_skew(c->d, tables(c), params(c), dx8, n, dpsi, dh, dO, nullptr, dst, 0, c->st)
               : rbmpp_launch_estimator(c->d, tables(c), params(c), dx8, n, dpsi, dh, dO, nullptr, dst, 0, c->st);
  if (!e) e = cudaStreamSynchronize(c->st);
  if (!e) rc = check_walker_status(c, dst, n, "eval_configs");
  if (!e && !rc && psi) e = cudaMemcpy(psi, dpsi, sizeof(double) * (size_t)n * (d.n_qp + 1) * 2, cudaMemcpyDeviceToHost);
  if (!e && !rc && hpsi) e = cudaMemcpy(hpsi, dh, sizeof(double) * 2 * (size_t)n, cudaMemcpyDeviceToHost);
  if (!e && !rc && O) e = cudaMemcpy(O, dO, sizeof(double) * orows * d.Nv, cudaMemcpyDeviceToHost);
  cudaFree(dx);
  cudaFree(dx8);
  cudaFree(dpsi);
  cudaFree(dh);
  if (dO) cudaFree(dO);
  cudaFree(dst);
  if (e) return fail(c, RBMPP_E_CUDA, "eval_configs: %s", cudaGetErrorString(e));
  return rc;
}

// ---------------------------------------------------------------------------------------------------
// SR step: SR_pdposv.f90:1-432 (Nsave = 1) with main.f90:351-369 normalisation.
// ---------------------------------------------------------------------------------------------------
int rbmpp_sr_step(rbmpp_ctx* c, const rbmpp_sr_in* in, rbmpp_sr_out* out, double* dx_out) {
  if (!c || !in || !out) return RBMPP_E_ARG;
  if (!c->measured) return fail(c, RBMPP_E_STATE, "sr_step before measure");
  if (in->precision != RBMPP_SR_FP64 && in->precision != RBMPP_SR_SPLIT_BF16)
    return fail(c, RBMPP_E_ARG, "unknown SR precision %d", in->precision);
  const DevDims& d = c->d;
  const int Nv = d.Nv, Nrbm = d.Nv_rbm, N = d.N;
  const bool refine = in->precision == RBMPP_SR_SPLIT_BF16 && in->refine_steps > 0;
  if (refine && c->n_samples_total != (double)c->ns_tot && !c->red_fn)
    return fail(c, RBMPP_E_ARG,
                "split-BF16 refinement applies S through this context's samples only; with a measurement reduced "
                "over several contexts use refine_steps = 0 or rbmpp_set_allreduce");
  std::memset(out, 0, sizeof(*out));
  const double norm = c->meas_scal[2];
  const double ntot = c->n_samples_total;
  out->norm = norm;
  out->Etot = c->meas_scal[0] / norm;
  out->Etot2 = c->meas_scal[1] / norm;
  out->wf_av = c->meas_scal[3] / ntot;
  out->accept_ratio = (double)c->naccept_total / ntot / (double)d.nupdate;
  const double Etot = out->Etot;
  std::vector<double> g(Nv), ov(Nv);
  CK(cudaMemcpy(g.data(), c->d_gvec, sizeof(double) * Nv, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(ov.data(), c->d_Ovec, sizeof(double) * Nv, cudaMemcpyDeviceToHost));
  for (int k = 0; k < Nv; k++) {
    g[k] = g[k] / norm;
    ov[k] = ov[k] / norm;
  }
  for (int k = 0; k < Nv; k++) g[k] = g[k] - 2.0 * Etot * ov[k];  // :4-6
  double* d_ov = c->d_vec;
  double* d_y = c->d_vec + 2 * Nv;
  double* d_diag = c->d_vec + 3 * Nv;
  CK(cudaMemcpyAsync(d_ov, ov.data(), sizeof(double) * Nv, cudaMemcpyHostToDevice, c->st));
  {
    int r = build_S(c, in->precision);  // S_raw of this measurement (the dgemm of calc_phys_quantity.f90:240)
    if (r) return r;
  }
  CK(rbmpp_sr_form(Nv, c->d_S, norm, d_ov, c->st));  // :11-15
  std::vector<double> dg(Nv);
  CK(rbmpp_get_diag(Nv, c->d_S, d_diag, c->st));
  CK(cudaMemcpyAsync(dg.data(), d_diag, sizeof(double) * Nv, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  double sr = 0, sp = 0;
  int i1 = 0, i2 = 0;
  for (int k = 0; k < Nv; k++)  // :18-31
    if (dg[k] > 0.0) {
      if (k < Nrbm) {
        i1++;
        sr += dg[k];
      } else {
        i2++;
        sp += dg[k];
      }
    }
  if (i1 != Nrbm) return fail(c, RBMPP_E_SDIAG, "i1/=Nv_RBM");
  if (i2 != d.n_slater - d.n_slater / N) return fail(c, RBMPP_E_SDIAG, "i2 /= N_Slater - N_Slater/N");
  sr = (Nrbm > 0) ? sr / (double)i1 : 1.0;
  sp = sp / (double)i2;
  const double scal = std::sqrt(sr / sp);  // :40
  for (int k = Nrbm; k < Nv; k++) g[k] = g[k] * scal;
  CK(rbmpp_sr_scale(Nv, Nrbm, c->d_S, scal, c->st));  // :54-74
  CK(rbmpp_get_diag(Nv, c->d_S, d_diag, c->st));
  CK(cudaMemcpyAsync(dg.data(), d_diag, sizeof(double) * Nv, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  // :78-100 f_ii checks
  std::vector<char> is_fii(Nv, 0);
  for (int i = 0; i < N; i++) is_fii[c->orb_host[(size_t)i * N + i] + Nv - d.n_slater] = 1;
  std::vector<int> zero_list;
  for (int k = 0; k < Nv; k++) {
    if (dg[k] < 0.0) return fail(c, RBMPP_E_SDIAG, "diagonal element of S matrix is not positive");
    if (dg[k] == 0.0) {
      if (!is_fii[k]) return fail(c, RBMPP_E_SDIAG, "diagonal element of S matrix is zero for other than f_ii parameters");
      if (std::fabs(ov[k]) > 1e-300 || std::fabs(g[k]) > 1e-300)
        return fail(c, RBMPP_E_SDIAG, "Ovec/gvec related with f_ii parameters is wrong");
      zero_list.push_back(k);
    } else if (is_fii[k]) {
      return fail(c, RBMPP_E_SDIAG, "diagonal element of S matrix is positive for f_ii parameters");
    }
  }
  if (!zero_list.empty()) {
    int* d_list = nullptr;
    double* d_m = nullptr;
    CK(cudaMalloc(&d_list, sizeof(int) * zero_list.size()));
    CK(cudaMalloc(&d_m, sizeof(double) * zero_list.size()));
    std::vector<double> mx(zero_list.size());
    cudaError_t e = cudaMemcpyAsync(d_list, zero_list.data(), sizeof(int) * zero_list.size(), cudaMemcpyHostToDevice, c->st);
    if (!e) e = rbmpp_rowcol_absmax(Nv, c->d_S, d_list, (int)zero_list.size(), d_m, c->st);
    if (!e) e = cudaMemcpyAsync(mx.data(), d_m, sizeof(double) * mx.size(), cudaMemcpyDeviceToHost, c->st);
    if (!e) e = cudaStreamSynchronize(c->st);
    cudaFree(d_list);
    cudaFree(d_m);
    if (e) return fail(c, RBMPP_E_CUDA, "f_ii check: %s", cudaGetErrorString(e));
    for (double m : mx)
      if (m > 1e-300) return fail(c, RBMPP_E_SDIAG, "Smat related with f_ii parameters is wrong");
  }
  double sdiag = 0, srb = 0, spp = 0;  // :104-140
  i1 = i2 = 0;
  for (int k = 0; k < Nv; k++)
    if (dg[k] > 0.0) {  // (the reference's Smax/Smin/kmaxS/kminS only feed its diagnostics output)
      sdiag += dg[k];
      if (k < Nrbm) {
        i1++;
        srb += dg[k];
      } else {
        i2++;
        spp += dg[k];
      }
    }
  sdiag = sdiag / (double)(i1 + i2);
  srb = (Nrbm > 0) ? srb / (double)i1 : 1.0;
  spp = spp / (double)i2;
  if (std::fabs(srb / spp - 1.0) > 1e-5) return fail(c, RBMPP_E_SDIAG, "Sdiag_av_RBM/=Sdiag_av_PP");
  const double rcut = sdiag * in->s_cut;
  int nS = 0;
  for (int k = 0; k < Nv; k++)
    if (dg[k] > rcut) nS++;
  const double s_factor = std::max(1e-4, in->s_factor0);  // :167-170
  CK(rbmpp_add_diag(Nv, c->d_S, sdiag * s_factor, c->st));
  // RNG: every rank draws at :172 (left-to-right .and.)
  CK(rbmpp_launch_advance_rng(c->W.mt, nullptr, 0, d.nw, 1, c->st));
  // pdposv('U') :232 -> Cholesky of the upper triangle + solve
  CK(cudaEventRecord(c->ev[7], c->st));
  const size_t s_bytes = (size_t)Nv * Nv * sizeof(double);
  if (in->precision == RBMPP_SR_SPLIT_BF16) {
    // the split-precision factor only preconditions the refinement on the exact S: if the split S plus the
    // reference's shift is not positive definite at working precision, factor it with a larger diagonal
    if (!c->d_Sb) {
      cudaError_t e = cudaMalloc(&c->d_Sb, s_bytes);
      if (e) return fail(c, RBMPP_E_CUDA, "cudaMalloc(S backup, %zu bytes): %s", s_bytes, cudaGetErrorString(e));
      c->bytes += s_bytes;
    }
    CK(cudaMemcpyAsync(c->d_Sb, c->d_S, s_bytes, cudaMemcpyDeviceToDevice, c->st));
  }
  int info = 0, attempts = 0;
  double tau = 0.0;
  for (int attempt = 0;; attempt++) {
    attempts = attempt + 1;
    CK(rbmpp_potrf_upper(Nv, c->d_S, c->d_dinv, c->d_info, c->st));
    CK(cudaMemcpyAsync(&info, c->d_info, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (info == 0 || in->precision != RBMPP_SR_SPLIT_BF16 || in->refine_steps <= 0 || attempt == 12) break;
    tau = tau == 0.0 ? sdiag * s_factor : 4.0 * tau;
    CK(cudaMemcpyAsync(c->d_S, c->d_Sb, s_bytes, cudaMemcpyDeviceToDevice, c->st));
    CK(rbmpp_add_diag(Nv, c->d_S, tau, c->st));
  }
  out->precond_shift = tau;
  double* v = c->d_pcg;
  const size_t nv = (size_t)Nv;
  double *d_g = v + VG * nv, *d_xv = v + VX * nv, *d_r = v + VR * nv, *d_z = v + VZ * nv, *d_p = v + VP * nv;
  double *d_ap = v + VAP * nv, *d_tmp = v + VTMP * nv, *d_m = v + VM * nv;
  CK(cudaMemcpyAsync(d_g, g.data(), sizeof(double) * Nv, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(d_xv, g.data(), sizeof(double) * Nv, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemsetAsync(c->d_bar, 0, 4 * sizeof(unsigned), c->st));
  CK(cudaStreamSynchronize(c->st));
  if (info != 0) return fail(c, RBMPP_E_CHOL, "info (pdposv): %d", info);
  CK(rbmpp_potrs_upper(Nv, c->d_S, c->d_dinv, d_xv, d_tmp, c->d_bar, c->st));
  CK(cudaEventRecord(c->ev[8], c->st));
  std::vector<double> x(Nv), ux(Nv), xr(Nv, 0.0), xp(Nv, 0.0);
  const double sigma = sdiag * s_factor;
  double lam2 = 0.0, lrr = 0.0, lpp = 0.0;
  float refine_ms = 0.f;
  if (refine) {
    // the split-precision solve refined against the exact FP64 S (applied through O in one pass per product):
    // conjugate gradients on A x = g preconditioned by the Cholesky factor of the split-precision S, started
    // from the split solve; stops at relative residual 1e-13 or after refine_steps iterations.  Every vector
    // stays on the device; the host reads the residual norm once per iteration.
    CK(cudaMemcpyAsync(d_m, ov.data(), sizeof(double) * Nv, cudaMemcpyHostToDevice, c->st));
    int r = apply_A(c, norm, scal, sigma, d_xv, d_ap);
    if (r) return r;
    CK(rbmpp_pcg_start(Nv, d_g, d_ap, d_r, c->d_sc, c->st));
    CK(cudaMemcpyAsync(d_z, d_r, sizeof(double) * Nv, cudaMemcpyDeviceToDevice, c->st));
    CK(rbmpp_potrs_upper(Nv, c->d_S, c->d_dinv, d_z, d_tmp, c->d_bar, c->st));
    CK(rbmpp_pcg_dir(Nv, d_r, d_z, d_p, c->d_sc, 0, c->st));
    CK(cudaMemcpyAsync(c->h_sc, c->d_sc, 8 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    const double gg = c->h_sc[4];
    double rr = c->h_sc[2];
    int it = 0;
    for (; it < in->refine_steps && gg > 0.0 && std::sqrt(rr) > 1e-13 * std::sqrt(gg); it++) {
      if ((r = apply_A(c, norm, scal, sigma, d_p, d_ap))) return r;
      CK(rbmpp_pcg_step(Nv, d_p, d_ap, d_xv, d_r, c->d_sc, c->st));
      CK(cudaMemcpyAsync(d_z, d_r, sizeof(double) * Nv, cudaMemcpyDeviceToDevice, c->st));
      CK(rbmpp_potrs_upper(Nv, c->d_S, c->d_dinv, d_z, d_tmp, c->d_bar, c->st));
      CK(rbmpp_pcg_dir(Nv, d_r, d_z, d_p, c->d_sc, 1, c->st));
      CK(cudaMemcpyAsync(c->h_sc, c->d_sc, 8 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
      CK(cudaStreamSynchronize(c->st));
      rr = c->h_sc[2];
      if (!(c->h_sc[3] > 0.0)) break;  // p.Ap <= 0: the step was not taken
    }
    out->refine_iterations = it;
    // lambda^2 = x^T A x and its block split (:251-277) with the exact A
    CK(cudaMemcpyAsync(x.data(), d_xv, sizeof(double) * Nv, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (int k = 0; k < Nv; k++) (k < Nrbm ? xr[k] : xp[k]) = x[k];
    std::vector<double> axr(Nv), axp(Nv);
    CK(cudaMemcpyAsync(d_p, xr.data(), sizeof(double) * Nv, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(d_z, xp.data(), sizeof(double) * Nv, cudaMemcpyHostToDevice, c->st));
    if ((r = apply_A(c, norm, scal, sigma, d_p, d_ap))) return r;
    if ((r = apply_A(c, norm, scal, sigma, d_z, d_r))) return r;
    CK(cudaEventRecord(c->ev[11], c->st));
    CK(cudaMemcpyAsync(axr.data(), d_ap, sizeof(double) * Nv, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(axp.data(), d_r, sizeof(double) * Nv, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    CK(cudaEventElapsedTime(&refine_ms, c->ev[8], c->ev[11]));
    for (int k = 0; k < Nv; k++) {
      lrr += xr[k] * axr[k];
      lpp += xp[k] * axp[k];
      lam2 += x[k] * (axr[k] + axp[k]);
    }
    // true residual of the final x
    double rn = 0.0, gn = 0.0;
    for (int k = 0; k < Nv; k++) {
      const double t = g[k] - (axr[k] + axp[k]);
      rn += t * t;
      gn += g[k] * g[k];
    }
    out->refine_residual = gn > 0.0 ? std::sqrt(rn / gn) : 0.0;
  } else {
    // lambda = sqrt(x^T S x) = ||U x|| and its block split (:251-277)
    CK(cudaMemcpyAsync(x.data(), d_xv, sizeof(double) * Nv, cudaMemcpyDeviceToHost, c->st));
    CK(rbmpp_trmv_upper(Nv, c->d_S, d_xv, d_y, c->st));
    CK(cudaMemcpyAsync(ux.data(), d_y, sizeof(double) * Nv, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (int k = 0; k < Nv; k++) lam2 += ux[k] * ux[k];
    for (int k = 0; k < Nv; k++) (k < Nrbm ? xr[k] : xp[k]) = x[k];
    CK(cudaMemcpyAsync(d_y, xr.data(), sizeof(double) * Nv, cudaMemcpyHostToDevice, c->st));
    CK(rbmpp_trmv_upper(Nv, c->d_S, d_y, d_diag, c->st));
    CK(cudaMemcpyAsync(ux.data(), d_diag, sizeof(double) * Nv, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (int k = 0; k < Nv; k++) lrr += ux[k] * ux[k];
    CK(cudaMemcpyAsync(d_y, xp.data(), sizeof(double) * Nv, cudaMemcpyHostToDevice, c->st));
    CK(rbmpp_trmv_upper(Nv, c->d_S, d_y, d_diag, c->st));
    CK(cudaMemcpyAsync(ux.data(), d_diag, sizeof(double) * Nv, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (int k = 0; k < Nv; k++) lpp += ux[k] * ux[k];
  }
  {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev[7], c->ev[8]));
    c->stats[4] = ms;
    c->stats[8] = refine_ms;
    c->stats[9] = attempts;
    unsigned bar[4];
    CK(cudaMemcpy(bar, c->d_bar, sizeof(bar), cudaMemcpyDeviceToHost));
    if (bar[2]) return fail(c, RBMPP_E_TIMEOUT, "triangular solve: a bounded grid-barrier wait ran out");
  }
  double lrp = lam2 - lrr - lpp;
  double lam = std::sqrt(lam2);
  // rank 0 draws at :281 and :313 (global walker 0 lives in the context with walker_offset 0)
  if (c->dims.walker_offset == 0) CK(rbmpp_launch_advance_rng(c->W.mt, nullptr, 0, 1, 2, c->st));
  lam = lam * 5.0 / (double)d.L;  // :309
  out->lambda = lam;
  out->lambda_rbm_rbm = lrr;
  out->lambda_pp_pp = lpp;
  out->lambda_rbm_pp = lrp;
  if (lam > 1.0)
    for (int k = 0; k < Nv; k++) x[k] = x[k] / lam;
  for (int k = Nrbm; k < Nv; k++) x[k] = x[k] * scal;  // :325-327
  double delW = 0.0;
  int kmax = -100, knz = 0;
  for (int k = 0; k < Nv; k++) {
    if (std::fabs(in->delta_tau * x[k]) > delW) {
      delW = std::fabs(in->delta_tau * x[k]);
      kmax = k + 1;
    }
    if (std::fabs(x[k]) > 1e-12) knz++;
  }
  // gamma: complex units as (re, im) pairs (bcirr, then Wcirr(iw, f)), real units, f_ij (SR_pdposv.f90:385-413)
  std::vector<double> gam(Nv);
  int k1 = 0;
  for (size_t q = 0; q < c->bc.size(); q++) gam[k1++] = c->bc[q];
  for (size_t q = 0; q < c->Wc.size(); q++) gam[k1++] = c->Wc[q];
  for (int f = 0; f < d.alphar; f++) gam[k1++] = c->br[f];
  for (int f = 0; f < d.alphar; f++)
    for (int iw = 0; iw < N; iw++) gam[k1++] = c->Wr[iw + (size_t)N * f];
  for (int o = 0; o < d.n_slater; o++) gam[k1++] = c->slater[o];
  const double max_change = 0.04;  // main.f90:50
  for (int k = 0; k < Nv; k++) {   // :347-354
    if (delW > max_change) gam[k] = gam[k] - in->delta_tau * x[k] * (max_change / delW);
    else gam[k] = gam[k] - in->delta_tau * x[k];
  }
  const int off = 2 * d.alphac * (N + 1) + d.alphar * (N + 1);  // :356-366
  double r1 = 0.0;
  for (int k = off; k < Nv; k++) r1 = r1 + std::fabs(gam[k]);
  r1 = r1 / (double)d.n_slater;
  for (int k = off; k < Nv; k++) gam[k] = gam[k] * 0.25 / r1;
  k1 = 0;  // :385-413
  for (size_t q = 0; q < c->bc.size(); q++) c->bc[q] = gam[k1++];
  for (size_t q = 0; q < c->Wc.size(); q++) c->Wc[q] = gam[k1++];
  for (int f = 0; f < d.alphar; f++) c->br[f] = gam[k1++];
  for (int f = 0; f < d.alphar; f++)
    for (int iw = 0; iw < N; iw++) c->Wr[iw + (size_t)N * f] = gam[k1++];
  r1 = 0.0;
  for (int o = 0; o < d.n_slater; o++) {
    c->slater[o] = gam[k1++];
    r1 += std::fabs(c->slater[o]);
  }
  r1 /= (double)d.n_slater;
  if (std::fabs(r1 - 0.25) > 1e-6) return fail(c, RBMPP_E_SLATER_NORM, "r1/=slater_abs_av");
  out->delW_max = delW;
  out->kmax = kmax;
  out->k_nonzero = knz;
  out->s_factor = s_factor;
  out->sdiag_av = sdiag;
  out->smat_scaling = scal;
  out->nSmat = nS;
  if (dx_out) std::memcpy(dx_out, x.data(), sizeof(double) * Nv);
  c->measured = false;  // S was factorised in place
  c->S_valid = false;
  return upload_params(c);
}

int rbmpp_exchange_measurement(rbmpp_ctx* c, int direction, double* d_S, double* d_g, double* d_ov, double* scal6) {
  if (!c || !scal6) return RBMPP_E_ARG;
  if (!c->measured) return fail(c, RBMPP_E_STATE, "exchange_measurement before measure");
  if (c->red_fn) return fail(c, RBMPP_E_STATE, "exchange_measurement with rbmpp_set_allreduce set: already reduced");
  const int Nv = c->d.Nv;
  const size_t nS = (size_t)Nv * Nv * sizeof(double), nV = (size_t)Nv * sizeof(double);
  if (direction == 0) {
    if (d_S) {
      int r = build_S(c, c->meas_prec);
      if (r) return r;
      CK(cudaMemcpyAsync(d_S, c->d_S, nS, cudaMemcpyDeviceToDevice, c->st));
    }
    if (d_g) CK(cudaMemcpyAsync(d_g, c->d_gvec, nV, cudaMemcpyDeviceToDevice, c->st));
    if (d_ov) CK(cudaMemcpyAsync(d_ov, c->d_Ovec, nV, cudaMemcpyDeviceToDevice, c->st));
    for (int k = 0; k < 4; k++) scal6[k] = c->meas_scal[k];
    scal6[4] = (double)c->naccept_total;
    scal6[5] = c->n_samples_total;
  } else {
    if (d_S) {
      CK(cudaMemcpyAsync(c->d_S, d_S, nS, cudaMemcpyDeviceToDevice, c->st));
      c->S_valid = true;
      c->S_reduced = true;
      c->S_prec = c->meas_prec;
    }
    if (d_g) CK(cudaMemcpyAsync(c->d_gvec, d_g, nV, cudaMemcpyDeviceToDevice, c->st));
    if (d_ov) CK(cudaMemcpyAsync(c->d_Ovec, d_ov, nV, cudaMemcpyDeviceToDevice, c->st));
    for (int k = 0; k < 4; k++) c->meas_scal[k] = scal6[k];
    c->naccept_total = (long long)scal6[4];
    c->n_samples_total = scal6[5];
  }
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int rbmpp_set_allreduce(rbmpp_ctx* c, rbmpp_allreduce_fn fn, void* user) {
  if (!c) return RBMPP_E_ARG;
  c->red_fn = fn;
  c->red_user = fn ? user : nullptr;
  return 0;
}

int rbmpp_set_s_precision(rbmpp_ctx* c, int precision) {
  if (!c) return RBMPP_E_ARG;
  if (precision != RBMPP_SR_FP64 && precision != RBMPP_SR_SPLIT_BF16)
    return fail(c, RBMPP_E_ARG, "unknown S precision %d", precision);
  c->meas_prec = precision;
  return 0;
}

int rbmpp_set_shift(rbmpp_ctx* c, double shift) {
  if (!c) return RBMPP_E_ARG;
  c->shift = shift;
  c->d.shift = shift;
  return 0;
}

int rbmpp_iteration(rbmpp_ctx* c, int precision, double delta_tau, double s_factor_scale, double s_cut,
                    double s_factor0_initial, rbmpp_sr_out* out) {
  if (!c || !out) return RBMPP_E_ARG;
  if (!c->s_factor_init) {
    c->s_factor0 = s_factor0_initial;
    c->s_factor_init = true;
  }
  if (precision != RBMPP_SR_FP64 && precision != RBMPP_SR_SPLIT_BF16)
    return fail(c, RBMPP_E_ARG, "unknown SR precision %d", precision);
  c->meas_prec = precision;
  c->iteration++;
  CK(cudaEventRecord(c->ev[9], c->st));
  int r = rbmpp_make_sample(c, c->iteration == 1 ? 1 : 0, nullptr, nullptr);
  if (r) return r;
  r = rbmpp_measure(c, nullptr, nullptr, nullptr, nullptr);
  if (r) return r;
  rbmpp_sr_in in;
  std::memset(&in, 0, sizeof(in));
  in.iteration = c->iteration;
  in.precision = precision;
  in.refine_steps = 50;
  in.delta_tau = delta_tau;
  in.s_factor0 = c->s_factor0;
  in.s_cut = s_cut;
  r = rbmpp_sr_step(c, &in, out, nullptr);
  if (r) return r;
  // main.f90:439-453
  c->s_factor0 = c->s_factor0 * s_factor_scale;
  for (int k = 1; k < 10; k++) c->wf_av_list[k - 1] = c->wf_av_list[k];
  c->wf_av_list[9] = out->wf_av;
  double wf = 0.0;
  for (int k = 0; k < 10; k++) wf = wf + c->wf_av_list[k];
  wf = wf / 10.0;
  // main.f90:451; transverse_code/main.f90:451 uses 0.003
  c->shift = wf * (c->d.skew ? 0.003 : 0.001) / (double)c->d.N / (double)c->d.N;
  c->d.shift = c->shift;
  CK(cudaEventRecord(c->ev[10], c->st));
  CK(cudaEventSynchronize(c->ev[10]));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, c->ev[9], c->ev[10]));
  c->stats[7] = ms;
  return 0;
}

int rbmpp_set_trace(rbmpp_ctx* c, int max_records) {
  if (!c || max_records < 0) return RBMPP_E_ARG;
  if (c->W.trace) {
    CK(cudaFree(c->W.trace));
    c->W.trace = nullptr;
  }
  c->d.trace_max = 0;
  if (max_records == 0) return 0;
  const size_t n = (size_t)c->d.nw * max_records * 6;
  int r = dalloc(c, &c->W.trace, n);
  if (r) return r;
  CK(cudaMemset(c->W.trace, 0, sizeof(double) * n));
  c->d.trace_max = max_records;
  return 0;
}

int rbmpp_set_replay(rbmpp_ctx* c, const int* decisions, int max_checkpoints) {
  if (!c || max_checkpoints < 0 || (max_checkpoints > 0 && !decisions)) return RBMPP_E_ARG;
  if (c->W.replay) {
    CK(cudaFree((void*)c->W.replay));
    c->W.replay = nullptr;
  }
  c->d.replay_max = 0;
  if (max_checkpoints == 0) return 0;
  const size_t n = (size_t)c->d.nw * max_checkpoints * 2;
  for (size_t k = 0; k < n; k += 2)
    if (decisions[k] < 1 || decisions[k] > 100 || (decisions[k + 1] != 0 && decisions[k + 1] != 1))
      return fail(c, RBMPP_E_ARG, "replay decision %zu out of range (Nfastup %d, extra draw %d)", k / 2,
                  decisions[k], decisions[k + 1]);
  int* p = nullptr;
  int r = dalloc(c, &p, n);
  if (r) return r;
  c->W.replay = p;
  CK(cudaMemcpy(p, decisions, sizeof(int) * n, cudaMemcpyHostToDevice));
  c->d.replay_max = max_checkpoints;
  return 0;
}

int rbmpp_debug_hook(rbmpp_ctx* c, int what, int value) {
  if (!c || value < 0) return RBMPP_E_ARG;
  switch (what) {
    case 1: c->d.skip_load = value; break;
    case 2: c->d.wait_polls = value; break;
    default: return fail(c, RBMPP_E_ARG, "unknown debug hook %d", what);
  }
  return 0;
}

int rbmpp_get_walker_events(const rbmpp_ctx* cc, int* events, double* trace) {
  rbmpp_ctx* c = const_cast<rbmpp_ctx*>(cc);
  if (!c) return RBMPP_E_ARG;
  if (events) CK(cudaMemcpy(events, c->W.events, sizeof(int) * 5 * c->d.nw, cudaMemcpyDeviceToHost));
  if (trace && c->W.trace)
    CK(cudaMemcpy(trace, c->W.trace, sizeof(double) * 6 * c->d.trace_max * c->d.nw, cudaMemcpyDeviceToHost));
  return 0;
}

int rbmpp_copy_state(rbmpp_ctx* dst, const rbmpp_ctx* src) {
  if (!dst || !src || dst == src) return RBMPP_E_ARG;
  rbmpp_ctx* c = dst;  // errors are reported on the destination context
  const DevDims &a = dst->d, &b = src->d;
  if (a.L != b.L || a.n_mp != b.n_mp || a.alphar != b.alphar || a.n_slater != b.n_slater || a.nw != b.nw ||
      a.ns != b.ns || a.skew != b.skew || a.alphac != b.alphac || dst->dims.device != src->dims.device)
    return fail(dst, RBMPP_E_ARG, "copy_state: the two contexts differ in shape or device");
  if (!src->tables_set || !dst->tables_set) return fail(dst, RBMPP_E_STATE, "copy_state: tables must be set on both");
  const size_t nw = a.nw, ns = a.ns, N = a.N;
  const DevWalkers &S = src->W, &D = dst->W;
  CK(cudaStreamSynchronize(src->st));
  auto cp = [&](void* d, const void* s, size_t bytes) -> cudaError_t {
    return cudaMemcpyAsync(d, s, bytes, cudaMemcpyDeviceToDevice, dst->st);
  };
  CK(cp(D.x, S.x, nw * N));
  CK(cp(D.idx, S.idx, 2 * nw * N));
  CK(cp(D.cfg, S.cfg, 2 * nw * N));
  CK(cp(D.th, S.th, 8 * nw * std::max(1, a.Mr)));
  CK(cp(D.sgn, S.sgn, nw * a.n_mp));
  CK(cp(D.pf, S.pf, 8 * nw * a.n_qp));
  CK(cp(D.psi, S.psi, 16 * nw * a.n_qp));
  CK(cp(D.Y, S.Y, 8 * nw * a.n_qp * (a.skew ? (size_t)N * N : (size_t)a.Np * a.Np)));
  CK(cp(D.mt, S.mt, 4 * nw * 625));
  CK(cp(D.nfastup, S.nfastup, 4 * nw));
  CK(cp(D.naccept, S.naccept, 4 * nw));
  CK(cp(D.nacc_all, S.nacc_all, 4 * nw));
  CK(cp(D.xs, S.xs, nw * ns * N));
  CK(cp(D.pfs, S.pfs, 8 * nw * ns * a.n_qp));
  CK(cp(D.psis, S.psis, 16 * nw * ns * (a.n_qp + 1)));
  CK(cp(D.events, S.events, 4 * 5 * nw));
  CK(cudaStreamSynchronize(dst->st));
  dst->Wr = src->Wr;
  dst->br = src->br;
  dst->Wc = src->Wc;
  dst->bc = src->bc;
  dst->slater = src->slater;
  dst->shift = src->shift;
  dst->params_set = src->params_set;
  dst->seeded = src->seeded;
  dst->sampled = src->sampled;
  dst->measured = false;
  dst->S_valid = false;
  dst->naccept_total = src->naccept_total;
  dst->iteration = src->iteration;
  dst->s_factor0 = src->s_factor0;
  dst->s_factor_init = src->s_factor_init;
  std::memcpy(dst->wf_av_list, src->wf_av_list, sizeof(dst->wf_av_list));
  return src->params_set ? upload_params(dst) : 0;
}

int rbmpp_get_walker_state(const rbmpp_ctx* cc, int* nfastup, int* nacc_all) {
  rbmpp_ctx* c = const_cast<rbmpp_ctx*>(cc);
  if (!c) return RBMPP_E_ARG;
  if (nfastup) CK(cudaMemcpy(nfastup, c->W.nfastup, sizeof(int) * c->d.nw, cudaMemcpyDeviceToHost));
  if (nacc_all) CK(cudaMemcpy(nacc_all, c->W.nacc_all, sizeof(int) * c->d.nw, cudaMemcpyDeviceToHost));
  return 0;
}

int rbmpp_get_stats(const rbmpp_ctx* c, double* out, int n) {
  if (!c || !out || n < 0) return RBMPP_E_ARG;
  for (int k = 0; k < n && k < 10; k++) out[k] = c->stats[k];
  return 0;
}

}  // extern "C"

// ===================================================================================================
// Batched make_sample: several contexts (lattice sizes, couplings, parameter sets) on one device sampled
// by one persistent launch of the direct sampler, with the launch shape and the walker order chosen by a
// measuring autotuner.
// ===================================================================================================
cudaError_t rbmpp_launch_sampler_batch(const BatchInst*, const int2*, int, int, int, int, size_t, long long*,
                                       cudaStream_t);
int rbmpp_batch_occupancy(int, int, size_t);

struct rbmpp_batch {
  std::vector<rbmpp_ctx*> ctx;
  std::vector<int> off;  // first block of each context in context-major order
  int total = 0, kpl = 1, threads = 256, order = 0, nsm = 0;
  size_t smem[3] = {0, 0, 0};  // dynamic shared memory for 128, 256, 512 threads
  std::vector<double> cost;    // per-walker cost of each context (model, then measured)
  BatchInst* d_inst = nullptr;
  int2* d_sched = nullptr;
  long long* d_cycles = nullptr;
  cudaEvent_t ev[2] = {};
  std::string err;
};

namespace {

int bfail(rbmpp_batch* b, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (b) b->err = buf;
  return code;
}

#define BCK(call)                                                                                  \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) return bfail(b, RBMPP_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

int thr_index(int threads) { return threads == 128 ? 0 : threads == 256 ? 1 : 2; }

// Block order of the whole batch.  0: context after context; 1: round robin over contexts;
// 2: longest walkers first (by the per-walker cost), the list-scheduling order that bounds the makespan.
std::vector<int2> make_schedule(const rbmpp_batch* b, int order) {
  std::vector<int2> s;
  s.reserve(b->total);
  const int n = (int)b->ctx.size();
  if (order == 0) {
    for (int k = 0; k < n; k++)
      for (int w = 0; w < b->ctx[k]->d.nw; w++) s.push_back(make_int2(k, w));
  } else if (order == 1) {
    int wmax = 0;
    for (auto* c : b->ctx) wmax = std::max(wmax, c->d.nw);
    for (int w = 0; w < wmax; w++)
      for (int k = 0; k < n; k++)
        if (w < b->ctx[k]->d.nw) s.push_back(make_int2(k, w));
  } else {
    std::vector<int> ks(n);
    for (int k = 0; k < n; k++) ks[k] = k;
    std::stable_sort(ks.begin(), ks.end(), [&](int a, int c2) { return b->cost[a] > b->cost[c2]; });
    int wmax = 0;
    for (auto* c : b->ctx) wmax = std::max(wmax, c->d.nw);
    // contexts of (nearly) equal cost interleave, which spreads each context's walkers over the SMs
    for (int w = 0; w < wmax; w++)
      for (int k : ks)
        if (w < b->ctx[k]->d.nw) s.push_back(make_int2(k, w));
    std::stable_sort(s.begin(), s.end(), [&](const int2& a, const int2& c2) { return b->cost[a.x] > b->cost[c2.x]; });
  }
  return s;
}

// Makespan of a block order under greedy list scheduling on `slots` identical block slots.
double makespan(const std::vector<int2>& sched, const std::vector<double>& cost, int slots) {
  std::vector<double> load(std::max(1, slots), 0.0);
  for (const int2& j : sched) {
    auto it = std::min_element(load.begin(), load.end());
    *it += cost[j.x];
  }
  return *std::max_element(load.begin(), load.end());
}

int upload_insts(rbmpp_batch* b, const std::vector<DevDims>* dims_override) {
  std::vector<BatchInst> h(b->ctx.size());
  for (size_t k = 0; k < b->ctx.size(); k++) {
    rbmpp_ctx* c = b->ctx[k];
    c->d.shift = c->shift;
    h[k].d = dims_override ? (*dims_override)[k] : c->d;
    h[k].t = tables(c);
    h[k].p = params(c);
    h[k].W = c->W;
  }
  BCK(cudaMemcpy(b->d_inst, h.data(), sizeof(BatchInst) * h.size(), cudaMemcpyHostToDevice));
  return 0;
}

}  // namespace

extern "C" {

int rbmpp_batch_create(rbmpp_ctx* const* ctxs, int n, rbmpp_batch** out) {
  if (!ctxs || n < 1 || !out) return RBMPP_E_ARG;
  rbmpp_batch* b = new rbmpp_batch();
  *out = b;
  int dev = -1;
  for (int k = 0; k < n; k++) {
    rbmpp_ctx* c = ctxs[k];
    if (!c) return bfail(b, RBMPP_E_ARG, "context %d is null", k);
    if (!c->tables_set || !c->params_set) return bfail(b, RBMPP_E_STATE, "context %d: tables and params first", k);
    if (c->d.skew) return bfail(b, RBMPP_E_ARG, "context %d: the batched sampler carries the block form only", k);
    if (c->d.alphac) return bfail(b, RBMPP_E_ARG, "context %d: the batched sampler carries real RBM units only", k);
    if (dev < 0) dev = c->dims.device;
    if (c->dims.device != dev) return bfail(b, RBMPP_E_ARG, "contexts on different devices");
    b->ctx.push_back(c);
    b->off.push_back(b->total);
    b->total += c->d.nw;
    b->kpl = std::max(b->kpl, (c->d.Np + 31) / 32);
    // cost model until measured: proposals x (Y bytes read per proposal + the per-proposal fixed work)
    const double sweeps = (double)(c->d.nwarm + c->d.ns + 1);
    b->cost.push_back(sweeps * c->d.N * ((double)c->d.n_qp * c->d.Np * c->d.Np + 64.0 * c->d.N));
  }
  BCK(cudaSetDevice(dev));
  int maxsm = 0;
  BCK(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  BCK(cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, dev));
  const int opts[3] = {128, 256, 512};
  for (int i = 0; i < 3; i++) {
    size_t m = 0;
    for (auto* c : b->ctx) m = std::max(m, rbmpp_sampler_smem(c->d, opts[i]));
    b->smem[i] = (long long)m <= maxsm ? m : 0;
  }
  if (!b->smem[1] && !b->smem[0]) return bfail(b, RBMPP_E_ARG, "sampler workspace exceeds shared memory");
  b->threads = b->smem[1] ? 256 : 128;
  BCK(cudaMalloc(&b->d_inst, sizeof(BatchInst) * n));
  BCK(cudaMalloc(&b->d_sched, sizeof(int2) * b->total));
  BCK(cudaMalloc(&b->d_cycles, sizeof(long long) * b->total));
  for (auto& e : b->ev) BCK(cudaEventCreate(&e));
  b->order = 2;
  std::vector<int2> sched = make_schedule(b, b->order);
  BCK(cudaMemcpy(b->d_sched, sched.data(), sizeof(int2) * sched.size(), cudaMemcpyHostToDevice));
  return 0;
}

int rbmpp_batch_destroy(rbmpp_batch* b) {
  if (!b) return 0;
  if (b->d_inst) cudaFree(b->d_inst);
  if (b->d_sched) cudaFree(b->d_sched);
  if (b->d_cycles) cudaFree(b->d_cycles);
  for (auto& e : b->ev)
    if (e) cudaEventDestroy(e);
  delete b;
  return 0;
}

const char* rbmpp_batch_last_error(const rbmpp_batch* b) { return b ? b->err.c_str() : "null batch"; }

int rbmpp_batch_tune(rbmpp_batch* b, int* threads_out, int* order_out, double* probe_ms) {
  if (!b) return RBMPP_E_ARG;
  const int n = (int)b->ctx.size();
  for (auto* c : b->ctx) {
    if (!c->seeded) return bfail(b, RBMPP_E_STATE, "seed every context before tuning");
    if (c->sampled) return bfail(b, RBMPP_E_STATE, "tune before the first batched make_sample");
  }
  // probe: up to 8 walkers of each context, 2 sweeps from a fresh configuration (first_iteration)
  std::vector<int2> probe;
  std::vector<DevDims> pd(n);
  for (int k = 0; k < n; k++) {
    pd[k] = b->ctx[k]->d;
    pd[k].nwarm = 1;
    pd[k].ns = 0;
    for (int w = 0; w < std::min(8, b->ctx[k]->d.nw); w++) probe.push_back(make_int2(k, w));
  }
  // the probed walkers' random streams and Nfastup are saved and restored
  std::vector<std::vector<uint32_t>> mt(n);
  std::vector<std::vector<int>> nf(n);
  for (int k = 0; k < n; k++) {
    rbmpp_ctx* c = b->ctx[k];
    const int m = std::min(8, c->d.nw);
    mt[k].resize((size_t)m * 625);
    nf[k].resize(m);
    BCK(cudaMemcpy(mt[k].data(), c->W.mt, sizeof(uint32_t) * mt[k].size(), cudaMemcpyDeviceToHost));
    BCK(cudaMemcpy(nf[k].data(), c->W.nfastup, sizeof(int) * m, cudaMemcpyDeviceToHost));
  }
  int r = upload_insts(b, &pd);
  if (r) return r;
  cudaStream_t st = b->ctx[0]->st;
  BCK(cudaMemcpy(b->d_sched, probe.data(), sizeof(int2) * probe.size(), cudaMemcpyHostToDevice));
  const int opts[3] = {128, 256, 512};
  double best_est = 1e300, best_ms = 0.0;
  int best_thr = b->threads, best_order = b->order;
  std::vector<double> best_cost = b->cost;
  for (int i = 0; i < 3; i++) {
    if (!b->smem[i]) continue;
    const int occ = rbmpp_batch_occupancy(b->kpl, opts[i], b->smem[i]);
    if (occ < 1) continue;
    BCK(cudaEventRecord(b->ev[0], st));
    BCK(rbmpp_launch_sampler_batch(b->d_inst, b->d_sched, (int)probe.size(), 1, b->kpl, opts[i], b->smem[i],
                                   b->d_cycles, st));
    BCK(cudaEventRecord(b->ev[1], st));
    BCK(cudaStreamSynchronize(st));
    float ms = 0.f;
    BCK(cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]));
    std::vector<long long> cyc(probe.size());
    BCK(cudaMemcpy(cyc.data(), b->d_cycles, sizeof(long long) * cyc.size(), cudaMemcpyDeviceToHost));
    // per-walker cost of a full make_sample: probe cycles per sweep x sweeps of the real call
    std::vector<double> cost(n, 0.0);
    std::vector<int> cnt(n, 0);
    for (size_t j = 0; j < probe.size(); j++) {
      cost[probe[j].x] += (double)cyc[j];
      cnt[probe[j].x]++;
    }
    for (int k = 0; k < n; k++)
      cost[k] = cnt[k] ? cost[k] / cnt[k] / 2.0 * (double)(b->ctx[k]->d.nwarm + b->ctx[k]->d.ns + 1) : 0.0;
    const std::vector<double> keep = b->cost;
    b->cost = cost;
    for (int order = 0; order < 3; order++) {
      const double est = makespan(make_schedule(b, order), cost, b->nsm * occ);
      if (est < best_est) {
        best_est = est;
        best_thr = opts[i];
        best_order = order;
        best_ms = ms;
        best_cost = cost;
      }
    }
    b->cost = keep;
  }
  for (int k = 0; k < n; k++) {
    rbmpp_ctx* c = b->ctx[k];
    BCK(cudaMemcpy(c->W.mt, mt[k].data(), sizeof(uint32_t) * mt[k].size(), cudaMemcpyHostToDevice));
    BCK(cudaMemcpy(c->W.nfastup, nf[k].data(), sizeof(int) * nf[k].size(), cudaMemcpyHostToDevice));
  }
  b->threads = best_thr;
  b->order = best_order;
  b->cost = best_cost;
  std::vector<int2> sched = make_schedule(b, b->order);
  BCK(cudaMemcpy(b->d_sched, sched.data(), sizeof(int2) * sched.size(), cudaMemcpyHostToDevice));
  if (threads_out) *threads_out = b->threads;
  if (order_out) *order_out = b->order;
  if (probe_ms) *probe_ms = best_ms;
  return 0;
}

int rbmpp_batch_make_sample(rbmpp_batch* b, int first, long long* naccept_total) {
  if (!b) return RBMPP_E_ARG;
  for (size_t k = 0; k < b->ctx.size(); k++) {
    rbmpp_ctx* c = b->ctx[k];
    if (!c->params_set || !c->seeded) return bfail(b, RBMPP_E_STATE, "context %zu: set_params and seed first", k);
    if (!first && !c->sampled) return bfail(b, RBMPP_E_STATE, "context %zu: make_sample(first=0) before any sample", k);
    BCK(cudaStreamSynchronize(c->st));
  }
  int r = upload_insts(b, nullptr);
  if (r) return r;
  cudaStream_t st = b->ctx[0]->st;
  const int ti = thr_index(b->threads);
  BCK(cudaEventRecord(b->ev[0], st));
  BCK(rbmpp_launch_sampler_batch(b->d_inst, b->d_sched, b->total, first ? 1 : 0, b->kpl, b->threads, b->smem[ti],
                                 nullptr, st));
  BCK(cudaEventRecord(b->ev[1], st));
  BCK(cudaStreamSynchronize(st));
  float ms = 0.f;
  BCK(cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]));
  for (size_t k = 0; k < b->ctx.size(); k++) {
    rbmpp_ctx* c = b->ctx[k];
    const int nw = c->d.nw;
    std::vector<int> stv(nw), na(nw), naa(nw);
    BCK(cudaMemcpy(stv.data(), c->W.status, sizeof(int) * nw, cudaMemcpyDeviceToHost));
    for (int w = 0; w < nw; w++)
      if (stv[w]) return bfail(b, stv[w], "context %zu walker %d: make_sample failed (code %d)", k, w, stv[w]);
    BCK(cudaMemcpy(na.data(), c->W.naccept, sizeof(int) * nw, cudaMemcpyDeviceToHost));
    BCK(cudaMemcpy(naa.data(), c->W.nacc_all, sizeof(int) * nw, cudaMemcpyDeviceToHost));
    long long tot = 0, tot_all = 0;
    for (int v : na) tot += v;
    for (int v : naa) tot_all += v;
    c->stats[0] = ms;
    c->stats[5] = (double)tot_all;
    c->stats[6] = (double)nw * (double)(c->d.nwarm + c->d.ns + 1) * (double)c->d.nupdate;
    c->naccept_total = tot;
    c->sampled = true;
    c->measured = false;
    if (naccept_total) naccept_total[k] = tot;
  }
  return 0;
}

}  // extern "C"

// ===================================================================================================
// rbmpp_eval_configs_noalloc: rbmpp_eval_configs for callers that must not allocate device memory.
//
// rbmpp_eval_configs allocates and frees device buffers on every call.  Some callers can't allow that:
// a host code whose own pool allocator has reserved the GPU's memory up front (a cudaMalloc from the
// library would then fail, or fragment the pool), or a loop that must not stall other streams (cudaFree
// waits for all work on the device).  This entry point takes the configurations and the results in
// device memory that the caller owns.  Its only scratch, the int8 copy of the configurations and one
// status word per configuration, lives in the fixed array below, which is part of the library's device
// image: every GPU that loads the library holds it until the process exits.
//
// Every call shares that array, and it keeps what the last call wrote.  The status words are written
// for every configuration of the call and the error word is cleared at the start of each call, so no
// stale value is read; but two calls whose work overlaps on the GPU (two contexts on one device driven
// from two host threads, say) race on the array.
// ===================================================================================================
namespace {

constexpr int kNoAllocMaxConfigs = 4096;                                        // configurations per call
constexpr size_t kNoAllocX8 = (size_t)kNoAllocMaxConfigs * RBMPP_MAX_N;         // int8 spins: 2 MiB
constexpr size_t kNoAllocStatus = kNoAllocX8;                                   // offset of the status words
constexpr size_t kNoAllocBad = kNoAllocStatus + 4 * (size_t)kNoAllocMaxConfigs;  // offset of the error word
constexpr size_t kNoAllocBytes = kNoAllocBad + 256;

static __device__ __align__(256) unsigned char g_eval_scratch[kNoAllocBytes];

// Records n - i for the first configuration i whose status is non-zero (atomicMax keeps the smallest i).
__global__ void first_bad_kernel(const int* status, int n, int* bad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && status[i] != 0) atomicMax(bad, n - i);
}

int noalloc_run(rbmpp_ctx* c, int n, const int* d_x, double* d_psi, double* d_hpsi, double* d_O) {
  // the array's device address on the current device, looked up on every call (a cheap runtime query that
  // stays right if the host code resets the device between calls)
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_eval_scratch);
  if (e != cudaSuccess || !p)
    return fail(c, RBMPP_E_CUDA, "cudaGetSymbolAddress(g_eval_scratch) on device %d: %s", c->dims.device,
                cudaGetErrorString(e));
  unsigned char* base = (unsigned char*)p;
  int8_t* x8 = (int8_t*)base;
  int* status = (int*)(base + kNoAllocStatus);
  int* bad = (int*)(base + kNoAllocBad);
  const long long nx = (long long)n * c->d.N;
  CK(cudaMemsetAsync(bad, 0, sizeof(int), c->st));
  rbmpp_note_launch();
  int_to_i8_kernel<<<(unsigned)((nx + 255) / 256), 256, 0, c->st>>>(d_x, x8, nx);
  CK(cudaGetLastError());
  CK(rbmpp_launch_estimator(c->d, tables(c), params(c), x8, n, d_psi, d_hpsi, d_O, nullptr, status, 0, c->st));
  rbmpp_note_launch();
  first_bad_kernel<<<(n + 255) / 256, 256, 0, c->st>>>(status, n, bad);
  CK(cudaGetLastError());
  int hbad = 0;
  CK(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (hbad) {
    const int i = n - hbad;
    int code = 0;
    CK(cudaMemcpy(&code, status + i, sizeof(int), cudaMemcpyDeviceToHost));
    return fail(c, code, "eval_configs_noalloc failed on configuration %d (code %d)", i, code);
  }
  return 0;
}

}  // namespace

extern "C" int rbmpp_eval_configs_noalloc(rbmpp_ctx* c, int n, const int* d_x, double* d_psi, double* d_hpsi,
                                          double* d_O) {
  if (!c || n < 0 || (n > 0 && !d_x)) return fail(c, RBMPP_E_ARG, "eval_configs_noalloc: bad arguments");
  if (n > kNoAllocMaxConfigs)
    return fail(c, RBMPP_E_ARG, "eval_configs_noalloc: n = %d configurations exceeds the fixed scratch limit of %d",
                n, kNoAllocMaxConfigs);
  if (c->dims.device < 0 || c->dims.device >= 64)
    return fail(c, RBMPP_E_ARG, "eval_configs_noalloc: device ordinal %d outside 0..63", c->dims.device);
  if (!c->params_set) return fail(c, RBMPP_E_STATE, "set_params must come first");
  if (c->d.skew || c->d.cplx)
    return fail(c, RBMPP_E_ARG, "eval_configs_noalloc takes real projection weights and the block form only; use "
                                "eval_configs");
  if (!c->est_smem_tiles)  // larger blocks need a global scratch buffer, which this entry point may not allocate
    return fail(c, RBMPP_E_ARG, "the estimator's workspace for N/2 = %d exceeds the shared memory of one block",
                c->d.Np);
  if (n == 0) return 0;
  // the scratch address and every launch belong to the context's device: make it current for the call
  int prev = -1;
  CK(cudaGetDevice(&prev));
  if (prev != c->dims.device) CK(cudaSetDevice(c->dims.device));
  const int r = noalloc_run(c, n, d_x, d_psi, d_hpsi, d_O);
  if (prev != c->dims.device) cudaSetDevice(prev);
  return r;
}

// estimator.cu -- per-configuration estimators (calc_phys_quantity.f90:20-246, 250-302, 306-427) and
// the adjoint O_k kernel: one CTA per configuration.
//
// For each projection qp the CTA inverts X from scratch in shared memory (the role of calculate_MAll,
// calc_phys_quantity.f90:85), then
//   * evaluates the exchange ratio of every antiparallel J1/J2 bond against that inverse
//     (calc_local_energy_correlation, calc_phys_quantity.f90:338-374), one warp per bond;
//   * scatters d Pf / d f_k (calculate_derivative_Pfaffian, slater.f90:94-170) times psi_wo_pf into
//     the configuration's O row (plain read-add-write: for one projection Orbital_Idx maps distinct
//     electron pairs to distinct parameters when it is injective; atomics otherwise).
// The RBM part of O_k (calc_phys_quantity.f90:165-201) is a gather over the inverse translation
// tables.  Outputs are the raw psi, H psi and d psi/d theta_k, optionally reweighted by
// 1/(|psi| + shift) as calc_phys_quantity.f90:102-109,221 do.
#include "walker_ops.cuh"

namespace {

struct EstShared {
  int* ap;        // [4N][2] antiparallel bonds (i1, i2)
  double* apc;    // [4N]    2 J sgn
  double* psib;   // [4N][2] psi(x') accumulators
  int* nap;       // [1]
  double* diag;   // [1]     sum J x x
  double* P;      // [Np][Np+1]  P(e, j) = XF(d_e, d_j)   (down-down gathers)
  double* Q;      // [Np][Np+1]  Q(i, a) = XF(u_i, u_a)   (up-up gathers)
  double* YQ;     // [Np][Np+1]  Y Q
};

__host__ __device__ __forceinline__ size_t est_layout(const DevDims& d, int nwarps, char* base, WS* w, EstShared* e) {
  size_t off = ws_layout(d, nwarps, base, w);
  auto take = [&](size_t bytes) -> char* {
    char* p = base ? base + off : nullptr;
    off = align16(off + bytes);
    return p;
  };
  EstShared t;
  t.ap = (int*)take((size_t)4 * d.N * 2 * 4);
  t.apc = (double*)take((size_t)4 * d.N * 8);
  t.psib = (double*)take((size_t)4 * d.N * 16);
  t.nap = (int*)take(16);
  t.diag = (double*)take(16);
  const size_t tb = (size_t)d.Np * (d.Np + 1) * 8;
  t.P = (double*)take(tb);
  t.Q = (double*)take(tb);
  t.YQ = (double*)take(tb);
  if (e) *e = t;
  return off;
}

// C = A B for n x n row-major shared-memory matrices with leading dimension ld (rows of 2, interleaved
// columns so that a warp reads consecutive columns of B)
__device__ __forceinline__ void cta_gemm(int n, int ld, const double* A, const double* B, double* C) {
  const int nr = (n + 1) / 2, nc = (n + 3) / 4;
  for (int blk = threadIdx.x; blk < nr * nc; blk += blockDim.x) {
    const int bi = blk / nc, bj = blk - bi * nc;
    const int i0 = 2 * bi;
    double acc[2][4];
#pragma unroll
    for (int r = 0; r < 2; r++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[r][q] = 0.0;
    const bool r1ok = i0 + 1 < n;
#pragma unroll 2
    for (int k = 0; k < n; k++) {
      const double a0 = A[i0 * ld + k], a1 = r1ok ? A[(i0 + 1) * ld + k] : 0.0;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int j = bj + q * nc;
        const double b = (j < n) ? B[k * ld + j] : 0.0;
        acc[0][q] = fma(a0, b, acc[0][q]);
        acc[1][q] = fma(a1, b, acc[1][q]);
      }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int j = bj + q * nc;
      if (j < n) {
        C[i0 * ld + j] = acc[0][q];
        if (r1ok) C[(i0 + 1) * ld + j] = acc[1][q];
      }
    }
  }
}

template <int KPL>
__global__ void __launch_bounds__(512, 1)
    estimator_kernel(const __grid_constant__ DevDims d, const __grid_constant__ DevTables t,
                     const __grid_constant__ DevParams p, const int8_t* xs, int n, double* out_psi, double* out_hpsi,
                     double* O, int* out_nap, int* out_status, int reweight) {
  extern __shared__ __align__(16) char smem[];
  __shared__ WS s;
  __shared__ EstShared e;
  if (threadIdx.x == 0) est_layout(d, blockDim.x >> 5, smem, &s, &e);
  __syncthreads();
  const int tid = threadIdx.x;
  const int N = d.N, Np = d.Np, ld = Np + 1;
  const int cfgi = blockIdx.x;
  if (cfgi >= n) return;
  double* Orow = O ? O + (size_t)cfgi * d.Nv : nullptr;

  for (int i = tid; i < N; i += blockDim.x) s.x[i] = (int)xs[(size_t)cfgi * N + i];
  if (Orow)
    for (int k = tid; k < d.Nv; k += blockDim.x) Orow[k] = 0.0;
  if (tid == 0) s.iflag[F_STATUS] = 0;
  __syncthreads();
  if (tid == 0) {
    int st = x_to_ele(d, s.x, s.idx, s.cfg);
    if (st) s.iflag[F_STATUS] = st;
    // bond list (bond_map, calc_phys_quantity.f90:382-427) and the diagonal part
    int na = 0;
    double dg = 0.0;
    for (int b = 0; b < 4 * N; b++) {
      int i1 = t.bonds[2 * b], i2 = t.bonds[2 * b + 1];
      double J = (b < 2 * N) ? d.J1 : d.J2, sg = (b < 2 * N) ? -1.0 : 1.0;
      dg = dg + J * (double)s.x[i1] * (double)s.x[i2];
      if (s.x[i1] != s.x[i2]) {
        e.ap[2 * na] = i1;
        e.ap[2 * na + 1] = i2;
        e.apc[na] = 2.0 * J * sg;
        na++;
      }
    }
    e.nap[0] = na;
    e.diag[0] = dg;
  }
  __syncthreads();
  if (s.iflag[F_STATUS]) {
    if (tid == 0 && out_status) out_status[cfgi] = s.iflag[F_STATUS];
    return;
  }
  const int nap = e.nap[0];
  for (int b = tid; b < nap; b += blockDim.x) {
    e.psib[2 * b] = 0.0;
    e.psib[2 * b + 1] = 0.0;
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
  const int off_pp = d.alphar * (N + 1);
  for (int qp = 0; qp < d.n_qp; qp++) {
    const int mp = qp >> 1, sp = qp & 1;
    cta_build_x(d, p, qp, s.idx, s.tile);
    {
      const double* XFq = p.XF + (size_t)qp * N * N;
      for (int i = tid >> 5; i < Np; i += blockDim.x >> 5) {
        const double* rowP = XFq + (size_t)s.idx[Np + i] * N;
        const double* rowQ = XFq + (size_t)s.idx[i] * N;
        for (int j = tid & 31; j < Np; j += 32) {
          e.P[i * ld + j] = rowP[s.idx[Np + j]];
          e.Q[i * ld + j] = rowQ[s.idx[j]];
        }
      }
    }
    __syncthreads();
    cta_gauss_jordan(d, s);
    if (s.iflag[F_SINGULAR]) {
      if (tid == 0 && out_status) out_status[cfgi] = ST_SINGULAR;
      return;
    }
    // Y with the column interchanges applied (into the YQ buffer, which then swaps roles with the tile)
    for (int a = tid >> 5; a < Np; a += blockDim.x >> 5)
      for (int b = tid & 31; b < Np; b += 32) e.YQ[a * ld + b] = s.tile[a * ld + s.perm[b]];
    __syncthreads();
    double* const Yt = e.YQ;
    double* const YQb = s.tile;
    const double pfq = (double)d.pf_sign * s.dsc[D_DET];
    const cplx cw = psi_wo_pf(d, t, s.rbm[qp], s.sgn[mp], qp);
    if (tid == 0) {
      s.pf[qp] = pfq;
      s.psi[2 * qp] = cw.re * pfq;
      s.psi[2 * qp + 1] = cw.im * pfq;
    }
    // local energy: exchange ratios of the antiparallel bonds (calc_phys_quantity.f90:347-373) for all
    // bonds at once.  With u_b = P(db,:) + du e_db, v_b = Q(:,ua) + dv e_ua (du = c - P(db,db),
    // dv = c - Q(ua,ua), c = XF(d_db, u_ua)), the entries of u^T Y, Y v and u^T Y v that the ratio
    // needs are (PY)(db,ua), (YQ)(db,ua), (P YQ)(db,ua) and Y(db,ua).
    cta_gemm(Np, ld, Yt, e.Q, YQb);
    __syncthreads();
    for (int b = tid; b < nap; b += blockDim.x) {
      const int i1 = e.ap[2 * b], i2 = e.ap[2 * b + 1];
      const int i3 = s.cfg[i1], i4 = s.cfg[i2];
      int ua, db, s_up, s_dn;
      if (s.x[i1] == 1) {
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
      const double c = p.XF[((size_t)qp * N + s_dn) * N + s_up];
      const double du = c - e.P[db * ld + db], dv = c - e.Q[ua * ld + ua];
      double py = 0.0, pyq = 0.0;
      for (int j = 0; j < Np; j++) {
        const double pj = e.P[db * ld + j];
        py = fma(pj, Yt[j * ld + ua], py);
        pyq = fma(pj, YQb[j * ld + ua], pyq);
      }
      const double y = Yt[db * ld + ua], yq = YQb[db * ld + ua];
      const double ra = py + du * y, sb = yq + dv * y;
      const double wv = pyq + du * yq + dv * py + du * dv * y;
      const double R = ra * sb - y * (wv - c);
      // theta' for this projection (update_theta on the qp's alphar slots) and the cosh product
      const int s_sign = sp == 0 ? 1 : -1;
      const int iw1 = t.wmap[(size_t)mp * N + i1], iw2 = t.wmap[(size_t)mp * N + i2];
      double r = 1.0;
      for (int f = 0; f < d.alphar; f++) {
        double th = s.th[qp * d.alphar + f];
        th = th - 2.0 * p.Wr[(size_t)f * N + iw1] * (double)s.x[i1] * (double)s_sign;
        th = th - 2.0 * p.Wr[(size_t)f * N + iw2] * (double)s.x[i2] * (double)s_sign;
        r = r * cosh(th);
      }
      const int sg = -s.sgn[mp] * (t.subB[i1] ? -1 : 1) * (t.subB[i2] ? -1 : 1);
      const cplx cb = psi_wo_pf(d, t, r, sg, qp);
      const double pn = R * pfq;
      e.psib[2 * b] += cb.re * pn;
      e.psib[2 * b + 1] += cb.im * pn;
    }
    // d Pf / d f_k scatter (slater.f90:140-167, block form)
    if (Orow) {
      const int* wm = t.wmap + (size_t)mp * N;
      const double cc = pfq * d.sp_cc[sp] * cw.re, ss = pfq * d.sp_ss[sp] * cw.re;
      for (int pr = tid; pr < Np * Np; pr += blockDim.x) {
        const int i = pr / Np, j = pr - i * Np;  // i: up electron, j: down electron
        const double y = Yt[j * ld + i];        // Y(j, i) = (M^-1)(Np+j, i)
        const int tu = wm[s.idx[i]], td = wm[s.idx[Np + j]];
        double* o1 = Orow + off_pp + t.orb[(size_t)tu * N + td];
        double* o2 = Orow + off_pp + t.orb[(size_t)td * N + tu];
        if (d.orb_injective) {
          if (cc != 0.0) *o1 = *o1 + y * cc;
          if (ss != 0.0) *o2 = *o2 + y * ss;
        } else {
          if (cc != 0.0) atomicAdd(o1, y * cc);
          if (ss != 0.0) atomicAdd(o2, y * ss);
        }
      }
    }
    __syncthreads();
  }
  // psi(0), H psi
  if (tid == 0) {
    double re = 0.0, im = 0.0;
    for (int qp = 0; qp < d.n_qp; qp++) {
      re += s.psi[2 * qp];
      im += s.psi[2 * qp + 1];
    }
    s.dsc[D_PSI0R] = re;
    s.dsc[D_PSI0I] = im;
    double hr = e.diag[0] * re, hi = e.diag[0] * im;
    for (int b = 0; b < nap; b++) {
      hr += e.apc[b] * e.psib[2 * b];
      hi += e.apc[b] * e.psib[2 * b + 1];
    }
    s.dsc[D_PSIPR] = hr;
    s.dsc[D_PSIPI] = hi;
    if (out_nap) out_nap[cfgi] = nap;
    if (out_status) out_status[cfgi] = 0;
  }
  __syncthreads();
  const double w = reweight ? 1.0 / (hypot(s.dsc[D_PSI0R], s.dsc[D_PSI0I]) + d.shift) : 1.0;
  if (Orow) {
    // RBM part, real branch (calc_phys_quantity.f90:165-201); psi_qp real for real para_mp_trans
    for (int k = tid; k < d.alphar * (N + 1); k += blockDim.x) {
      double acc = 0.0;
      if (k < d.alphar) {
        const int f = k;
        for (int qp = 0; qp < d.n_qp; qp++) acc = acc + tanh(s.th[qp * d.alphar + f]) * s.psi[2 * qp];
      } else {
        const int f = (k - d.alphar) / N, iw = (k - d.alphar) - f * N;
        for (int mp = 0; mp < d.n_mp; mp++) {
          const double xi = (double)s.x[t.winv[(size_t)mp * N + iw]];
          const int q0 = 2 * mp, q1 = 2 * mp + 1;
          acc = acc + tanh(s.th[q0 * d.alphar + f]) * s.psi[2 * q0] * xi;
          acc = acc - tanh(s.th[q1 * d.alphar + f]) * s.psi[2 * q1] * xi;
        }
      }
      Orow[k] = acc * w;
    }
    for (int k = off_pp + tid; k < d.Nv; k += blockDim.x) Orow[k] = Orow[k] * w;
  }
  if (tid == 0) {
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
      out_hpsi[2 * (size_t)cfgi] = s.dsc[D_PSIPR] * w;
      out_hpsi[2 * (size_t)cfgi + 1] = s.dsc[D_PSIPI] * w;
    }
  }
}

// Advances every walker's MT19937 by its measurement draws: one per amplitude call, i.e.
// 1 + n_antiparallel per stored sample (sub.f90:72 called from calc_phys_quantity.f90:95,369).
__global__ void advance_rng_kernel(uint32_t* mt, const int* nap, int ns, int nw, int extra) {
  int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nw) return;
  uint32_t st[625];
  for (int k = 0; k < 625; k++) st[k] = mt[(size_t)w * 625 + k];
  long long draws = extra;
  if (nap)
    for (int s = 0; s < ns; s++) draws += 1 + nap[(size_t)w * ns + s];
  for (long long i = 0; i < draws; i++) (void)mt_next(st);
  for (int k = 0; k < 625; k++) mt[(size_t)w * 625 + k] = st[k];
}

}  // namespace

size_t rbmpp_estimator_smem(const DevDims& d, int threads) { return est_layout(d, threads / 32, nullptr, nullptr, nullptr); }
static const int kEstThreads = 512;

cudaError_t rbmpp_launch_estimator(const DevDims& d, const DevTables& t, const DevParams& p, const int8_t* xs, int n,
                                   double* out_psi, double* out_hpsi, double* O, int* out_nap, int* out_status,
                                   int reweight, cudaStream_t st) {
  const int threads = kEstThreads;
  size_t smem = rbmpp_estimator_smem(d, threads);
  int kpl = (d.Np + 31) / 32;
#define LAUNCH(K)                                                                                          \
  do {                                                                                                     \
    cudaError_t e = cudaFuncSetAttribute(estimator_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                         (int)smem);                                                       \
    if (e != cudaSuccess) return e;                                                                        \
    estimator_kernel<K><<<n, threads, smem, st>>>(d, t, p, xs, n, out_psi, out_hpsi, O, out_nap, out_status, \
                                                  reweight);                                               \
    return cudaGetLastError();                                                                             \
  } while (0)
  if (n <= 0) return cudaSuccess;
  if (kpl <= 1) LAUNCH(1);
  if (kpl <= 2) LAUNCH(2);
  if (kpl <= 4) LAUNCH(4);
  if (kpl <= 8) LAUNCH(8);
#undef LAUNCH
  return cudaErrorInvalidValue;
}

cudaError_t rbmpp_launch_advance_rng(uint32_t* mt, const int* nap, int ns, int nw, int extra, cudaStream_t st) {
  advance_rng_kernel<<<(nw + 63) / 64, 64, 0, st>>>(mt, nap, ns, nw, extra);
  return cudaGetLastError();
}

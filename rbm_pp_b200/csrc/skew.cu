// skew.cu -- the Pfaffian matrix in its full N x N skew form, for spin projections whose same-spin blocks of
// Slater_Elm do not vanish: the transverse code's beta = -pi/2, pi/2 with sqrt(2)-scaled weights
// (transverse_code/spin_projection.f90:30-38), where cos sin = -/+1 and every block of
//     B(i, j) = -Slater_Elm(rho_i, rho_j),   rho = site of the electron (+ N for a down electron)
// (matrix.f90:70-77; electrons 0..Np-1 up, Np..N-1 down) is non-zero.  Per walker and projection the device
// keeps G = B^{-1} (N x N, skew, row-major) in DevWalkers::Y.
//
// Exchange of electron a (moving to rho'_a) and electron b (to rho'_b): columns and rows a and b of B change.
// With x = B'(:, a), y = B'(:, b), and x^, y^ the same vectors with entries a and b set to zero, the Schur
// complement of the index pair {a, b} gives (the role of calculate_new_PfM_two, pfupdate_two.f90:27-88)
//     Pf(B') / Pf(B) = -G_ab (y_a + x^ . G y^) + (G x^)_a (G y^)_b - (G x^)_b (G y^)_a,
// one pass over G per projection.  An accepted exchange is B' = B + U J U^T with U = [dx, e_a, dy, e_b]
// (dx = x - B(:, a); dy = y - B(:, b) with entry a zeroed) and J = diag(j2, j2), j2 = [[0, 1], [-1, 0]], so
// Woodbury gives G' = G + V K^{-1} V^T, V = G U, K = U^T G U - J, a 4 x 4 skew matrix inverted in closed form
// (its Pfaffian is the ratio again); the role of calculate_new_InvM_two, pfupdate_two.f90:113-224.
// From scratch (calculate_MAll, matrix.f90:55-108): the Pfaffian by Parlett-Reid elimination with pivoting
// (a skew L T L^T; restated from M. Wimmer, ACM TOMS 38(4) 2012, the role of dskpfa('U', 'P')), the inverse by
// warp Gauss-Jordan, skew-symmetrised as matrix.f90:96-105 does, with its skew check.
//
// Kernels: the direct Metropolis sampler (one CTA per walker, one warp per projection at a time, G streamed
// from HBM), the estimator (one CTA per configuration; local energy over the antiparallel J1/J2 bonds,
// dPf/df_k over the four spin blocks of slater.f90:140-167) and the Slater-element table.
#include "sampler_common.cuh"

namespace {

constexpr int kSkThreads = 256;
constexpr int kSkWarps = kSkThreads / 32;

__device__ __forceinline__ int rho_of(const int* idx, int e, int Np, int N) { return idx[e] + (e >= Np ? N : 0); }

// row r of Slater_Elm for projection qp: SE(r, .)
__device__ __forceinline__ const double* se_row(const DevDims& d, const DevParams& p, int qp, int r) {
  return p.SE + ((size_t)qp * 2 * d.N + r) * 2 * (size_t)d.N;
}

// update_slater_elements, slater.f90:7-64, all four blocks: row site rj, column site ri,
// slt_ij = f(orb(T ri, T rj)), slt_ji = f(orb(T rj, T ri)).  Products and sums rounded one at a time.
__global__ void build_se_kernel(int N, int n_mp, const int* wmap, const int* orb, const double* slater, double cs0,
                                double cs1, double cc0, double cc1, double ss0, double ss1, double* SE) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long tot = (long long)2 * n_mp * N * N;
  if (e >= tot) return;
  const int ri = (int)(e % N);
  const long long r = e / N;
  const int rj = (int)(r % N);
  const int qp = (int)(r / N), mp = qp >> 1, sp = qp & 1;
  const double cs = sp ? cs1 : cs0, cc = sp ? cc1 : cc0, ss = sp ? ss1 : ss0;
  const int tri = wmap[(long long)mp * N + ri], trj = wmap[(long long)mp * N + rj];
  const double sij = slater[orb[(long long)tri * N + trj]];
  const double sji = slater[orb[(long long)trj * N + tri]];
  const long long N2 = 2LL * N;
  double* S = SE + (long long)qp * N2 * N2;
  const double dsl = __dsub_rn(sij, sji);
  S[(long long)rj * N2 + ri] = __dmul_rn(-dsl, cs);                                         // up - up
  S[(long long)(rj + N) * N2 + ri] = __dadd_rn(__dmul_rn(sij, cc), __dmul_rn(sji, ss));     // down row, up column
  S[(long long)rj * N2 + ri + N] = __dsub_rn(__dmul_rn(-sij, ss), __dmul_rn(sji, cc));      // up row, down column
  S[(long long)(rj + N) * N2 + ri + N] = __dmul_rn(dsl, cs);                                // down - down
}

// B(i, j) = -SE(rho_i, rho_j) into a warp tile (ld = N + 1)
__device__ __forceinline__ void warp_gather_skew(double* T, const DevDims& d, const DevParams& p, int qp,
                                                 const int* idx) {
  const int N = d.N, Np = d.Np, ld = N + 1, lane = threadIdx.x & 31;
  for (int i = 0; i < N; i++) {
    const double* row = se_row(d, p, qp, rho_of(idx, i, Np, N));
    for (int j = lane; j < N; j += 32) T[i * ld + j] = -row[rho_of(idx, j, Np, N)];
  }
  __syncwarp();
}

// Pf(T) by Parlett-Reid elimination with row/column pivoting; T (n x n, ld = n + 1) is destroyed.
template <int KPL>
__device__ double warp_pfaffian(double* T, int n, bool& singular) {
  const int ld = n + 1, lane = threadIdx.x & 31;
  double pf = 1.0;
  singular = false;
  for (int k = 0; k + 1 < n; k += 2) {
    double best = -1.0;
    int bi = k + 1;
    for (int i = k + 1 + lane; i < n; i += 32) {
      const double v = fabs(T[i * ld + k]);
      if (v > best) {
        best = v;
        bi = i;
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
    if (bi != k + 1) {  // interchange rows, then columns, k + 1 and bi of the trailing matrix
      for (int j = k + lane; j < n; j += 32) {
        const double t0 = T[(k + 1) * ld + j];
        T[(k + 1) * ld + j] = T[bi * ld + j];
        T[bi * ld + j] = t0;
      }
      __syncwarp();
      for (int i = k + lane; i < n; i += 32) {
        const double t0 = T[i * ld + k + 1];
        T[i * ld + k + 1] = T[i * ld + bi];
        T[i * ld + bi] = t0;
      }
      __syncwarp();
      pf = -pf;
    }
    const double piv = T[(k + 1) * ld + k];
    pf *= T[k * ld + k + 1];
    if (k + 2 < n) {
      // rows and columns i, j >= k + 2: T(i, j) += -tau_i T(k+1, j) + T(k+1, i) tau_j, tau = T(., k) / T(k+1, k)
      double tau[KPL], rr[KPL];
#pragma unroll
      for (int m = 0; m < KPL; m++) {
        const int j = lane + 32 * m;
        const bool in = j >= k + 2 && j < n;
        tau[m] = in ? T[j * ld + k] / piv : 0.0;
        rr[m] = in ? T[(k + 1) * ld + j] : 0.0;
      }
      __syncwarp();
      for (int i = k + 2; i < n; i++) {
        const double ti = T[i * ld + k] / piv, ri = T[(k + 1) * ld + i];
#pragma unroll
        for (int m = 0; m < KPL; m++) {
          const int j = lane + 32 * m;
          if (j >= k + 2 && j < n) T[i * ld + j] = fma(ri, tau[m], fma(-ti, rr[m], T[i * ld + j]));
        }
      }
      __syncwarp();
    }
  }
  return pf;
}

// G = (B^-1 - B^-T) / 2 in place (matrix.f90:96-105) from warp_gj's inverse, whose column j sits at perm[j].
// The symmetric part of the computed inverse is rounding noise, which the exchange-ratio formula would amplify
// by the conditioning of B; the skew part alone gives ratios to about 1e-13.
template <int KPL>
__device__ void warp_unpermute_skew(double* T, int n, const int* perm) {
  const int ld = n + 1, lane = threadIdx.x & 31;
  for (int i = 0; i < n; i++) {
    double v[KPL];
#pragma unroll
    for (int m = 0; m < KPL; m++) {
      const int j = lane + 32 * m;
      v[m] = j < n ? T[i * ld + perm[j]] : 0.0;
    }
    __syncwarp();
#pragma unroll
    for (int m = 0; m < KPL; m++) {
      const int j = lane + 32 * m;
      if (j < n) T[i * ld + j] = v[m];
    }
    __syncwarp();
  }
  for (int i = 0; i < n; i++) {
    for (int j = i + 1 + lane; j < n; j += 32) {
      const double g = 0.5 * (T[i * ld + j] - T[j * ld + i]);
      T[i * ld + j] = g;
      T[j * ld + i] = -g;
    }
    if (lane == 0) T[i * ld + i] = 0.0;
    __syncwarp();
  }
}

// calculate_MAll for the skew form (policy of the walker routines of sampler_common.cuh): one warp per
// projection on its own shared-memory tile; writes G (when write_y) and pf_out; with diff, the drift measure
// of make_sample.f90:106-113 against the stored G.
template <int KPL>
struct SkewScratch {
  static __device__ void run(const SCtx& c, const int* idx, double* pf_out, bool write_y, bool diff) {
    const DevDims& d = c.d;
    const WS& s = c.s;
    const int N = d.N, ld = N + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double wratio = -1.0;
    int bad = 0;  // 1: singular, 2: inverse not skew (matrix.f90:103)
    if (warp < c.par_ntile) {
      double* T = c.par_tiles + (size_t)warp * N * ld;
      int* perm = (int*)(s.wS + (size_t)warp * d.Np);
      for (int qp = warp; qp < d.n_qp && !bad; qp += c.par_ntile) {
        warp_gather_skew(T, d, c.p, qp, idx);
        bool sing;
        const double pfq = warp_pfaffian<KPL>(T, N, sing);
        if (!sing) {
          warp_gather_skew(T, d, c.p, qp, idx);
          (void)warp_gj<KPL, 0, 4>(T, N, perm, sing);
        }
        if (sing) {
          bad = 1;
          break;
        }
        double* Gq = c.Yw + (size_t)qp * N * N;
        double mx = 0.0, md = 0.0, mraw = 0.0, msym = 0.0;
        for (int i = 0; i < N; i++)
          for (int j = lane; j < N; j += 32) {
            const double a = T[i * ld + perm[j]], b = T[j * ld + perm[i]];
            const double g = 0.5 * (a - b);
            mraw = fmax(mraw, fabs(a));
            msym = fmax(msym, fabs(0.5 * (a + b)));
            mx = fmax(mx, fabs(g));
            if (diff) md = fmax(md, fabs(Gq[(size_t)i * N + j] - g));
            if (write_y) Gq[(size_t)i * N + j] = g;
          }
        mx = warp_max(mx);
        md = warp_max(md);
        mraw = warp_max(mraw);
        msym = warp_max(msym);
        if (msym > 2.0e-3 * mraw) bad = 2;
        if (diff) wratio = fmax(wratio, md / mx);
        if (lane == 0) pf_out[qp] = pfq;
        __syncwarp();
      }
    }
    if (lane == 0) {
      s.red[warp] = wratio;
      s.red[32 + warp] = (double)bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double di = -1.0;
      int b = 0;
      for (int w = 0; w < c.par_ntile; w++) {
        di = fmax(di, s.red[w]);
        if (s.red[32 + w] != 0.0 && !b) b = (int)s.red[32 + w];
      }
      if (b) status(c) = b == 1 ? ST_SINGULAR : ST_SKEW;
      s.dsc[D_DIFFINV] = di;
    }
    __syncthreads();
  }
};

// x^_i = B'(i, a) = SE(rho'_a, rho_i) and y^_i = SE(rho'_b, rho_i) (skew Slater_Elm), zero at i = a, b
__device__ __forceinline__ void warp_gather_xy(const DevDims& d, const double* SEa, const double* SEb, const int* idx,
                                               int a, int b, double* xh, double* yh) {
  const int N = d.N, Np = d.Np, lane = threadIdx.x & 31;
  for (int i = lane; i < N; i += 32) {
    const int ri = rho_of(idx, i, Np, N);
    const bool ab = i == a || i == b;
    xh[i] = ab ? 0.0 : SEa[ri];
    yh[i] = ab ? 0.0 : SEb[ri];
  }
  __syncwarp();
}

// (G x^)_j and (G y^)_j for this lane's columns j = lane + 32 m (G skew: (G v)_j = -sum_i v_i G(i, j))
template <int KPL>
__device__ __forceinline__ void warp_gxy(const double* Gq, int N, const double* xh, const double* yh, double (&gx)[KPL],
                                         double (&gy)[KPL]) {
  const int lane = threadIdx.x & 31;
  double ax[KPL], ay[KPL];
#pragma unroll
  for (int m = 0; m < KPL; m++) ax[m] = ay[m] = 0.0;
  int i = 0;
  for (; i + 2 <= N; i += 2) {
    const double x0 = xh[i], y0 = yh[i], x1 = xh[i + 1], y1 = yh[i + 1];
    double g0[KPL], g1[KPL];
#pragma unroll
    for (int m = 0; m < KPL; m++) {
      const int j = lane + 32 * m;
      g0[m] = j < N ? Gq[(size_t)i * N + j] : 0.0;
      g1[m] = j < N ? Gq[(size_t)(i + 1) * N + j] : 0.0;
    }
#pragma unroll
    for (int m = 0; m < KPL; m++) {
      ax[m] = fma(x1, g1[m], fma(x0, g0[m], ax[m]));
      ay[m] = fma(y1, g1[m], fma(y0, g0[m], ay[m]));
    }
  }
  for (; i < N; i++) {
    const double x0 = xh[i], y0 = yh[i];
#pragma unroll
    for (int m = 0; m < KPL; m++) {
      const int j = lane + 32 * m;
      if (j < N) {
        const double g = Gq[(size_t)i * N + j];
        ax[m] = fma(x0, g, ax[m]);
        ay[m] = fma(y0, g, ay[m]);
      }
    }
  }
#pragma unroll
  for (int m = 0; m < KPL; m++) {
    gx[m] = -ax[m];
    gy[m] = -ay[m];
  }
}

// Pf(B') / Pf(B) for the exchange of electrons a -> rho'_a, b -> rho'_b (valid on all lanes)
template <int KPL>
__device__ double warp_skew_ratio(const DevDims& d, const DevParams& p, const double* Gq, int qp, const int* idx,
                                  int a, int b, int ra_new, int rb_new, double* xh, double* yh) {
  const int lane = threadIdx.x & 31, N = d.N;
  const double* SEa = se_row(d, p, qp, ra_new);
  const double* SEb = se_row(d, p, qp, rb_new);
  warp_gather_xy(d, SEa, SEb, idx, a, b, xh, yh);
  const double ya = -SEa[rb_new];  // B'(a, b)
  double gx[KPL], gy[KPL];
  warp_gxy<KPL>(Gq, N, xh, yh, gx, gy);
  double xgy = 0.0, gxa = 0.0, gxb = 0.0, gya = 0.0, gyb = 0.0;
#pragma unroll
  for (int m = 0; m < KPL; m++) {
    const int j = lane + 32 * m;
    if (j < N) {
      xgy = fma(xh[j], gy[m], xgy);
      if (j == a) {
        gxa = gx[m];
        gya = gy[m];
      }
      if (j == b) {
        gxb = gx[m];
        gyb = gy[m];
      }
    }
  }
  xgy = warp_sum(xgy);
  gxa = warp_sum(gxa);
  gxb = warp_sum(gxb);
  gya = warp_sum(gya);
  gyb = warp_sum(gyb);
  const double gab = Gq[(size_t)a * N + b];
  __syncwarp();
  return -gab * (ya + xgy) + gxa * gyb - gxb * gya;
}

// G' = G + V K^{-1} V^T after the accepted exchange; v: [4][N] per-warp scratch for the columns of V
template <int KPL>
__device__ void warp_skew_update(const DevDims& d, const DevParams& p, double* Gq, int qp, const int* idx, int a,
                                 int b, int ra_old, int rb_old, int ra_new, int rb_new, double* xh, double* yh,
                                 double* v) {
  const int lane = threadIdx.x & 31, N = d.N;
  const double* SEa = se_row(d, p, qp, ra_new);
  const double* SEb = se_row(d, p, qp, rb_new);
  warp_gather_xy(d, SEa, SEb, idx, a, b, xh, yh);
  const double xb = SEa[rb_new];                           // B'(b, a)
  const double bab = -se_row(d, p, qp, ra_old)[rb_old];    // B(a, b) before the move
  double gx[KPL], gy[KPL];
  warp_gxy<KPL>(Gq, N, xh, yh, gx, gy);
  // V = [G dx, G e_a, G dy, G e_b]: G dx = G x^ + x_b G(:, b) - e_a, G dy = G y^ - e_b + B(a, b) G(:, a)
  double V[KPL][4];
  double v0a = 0.0, v0b = 0.0, v2a = 0.0, v2b = 0.0, xv2 = 0.0;
#pragma unroll
  for (int m = 0; m < KPL; m++) {
    const int j = lane + 32 * m;
    V[m][0] = V[m][1] = V[m][2] = V[m][3] = 0.0;
    if (j < N) {
      const double ga = -Gq[(size_t)a * N + j], gb = -Gq[(size_t)b * N + j];  // G(j, a), G(j, b)
      V[m][0] = gx[m] + xb * gb - (j == a ? 1.0 : 0.0);
      V[m][1] = ga;
      V[m][2] = gy[m] - (j == b ? 1.0 : 0.0) + bab * ga;
      V[m][3] = gb;
#pragma unroll
      for (int q = 0; q < 4; q++) v[q * N + j] = V[m][q];
      xv2 = fma(xh[j] + (j == b ? xb : 0.0), V[m][2], xv2);
      if (j == a) {
        v0a = V[m][0];
        v2a = V[m][2];
      }
      if (j == b) {
        v0b = V[m][0];
        v2b = V[m][2];
      }
    }
  }
  xv2 = warp_sum(xv2);
  v0a = warp_sum(v0a);
  v0b = warp_sum(v0b);
  v2a = warp_sum(v2a);
  v2b = warp_sum(v2b);
  const double gab = Gq[(size_t)a * N + b];
  __syncwarp();
  // K = U^T G U - J (skew): upper entries
  const double k01 = -v0a - 1.0, k02 = xv2, k03 = -v0b, k12 = v2a, k13 = gab, k23 = -v2b - 1.0;
  const double pk = k01 * k23 - k02 * k13 + k03 * k12;
  const double ip = 1.0 / pk;
  // K^{-1} = [[0, -k23, k13, -k12], [k23, 0, -k03, k02], [-k13, k03, 0, -k01], [k12, -k02, k01, 0]] / Pf(K)
  const double Ki[4][4] = {{0.0, -k23 * ip, k13 * ip, -k12 * ip},
                           {k23 * ip, 0.0, -k03 * ip, k02 * ip},
                           {-k13 * ip, k03 * ip, 0.0, -k01 * ip},
                           {k12 * ip, -k02 * ip, k01 * ip, 0.0}};
  for (int i = 0; i < N; i++) {
    double z[4];
    const double vi[4] = {v[i], v[N + i], v[2 * N + i], v[3 * N + i]};
#pragma unroll
    for (int q = 0; q < 4; q++) z[q] = vi[0] * Ki[0][q] + vi[1] * Ki[1][q] + vi[2] * Ki[2][q] + vi[3] * Ki[3][q];
    double* Gr = Gq + (size_t)i * N;
#pragma unroll
    for (int m = 0; m < KPL; m++) {
      const int j = lane + 32 * m;
      if (j < N) {
        double g = Gr[j];
#pragma unroll
        for (int q = 0; q < 4; q++) g = fma(z[q], V[m][q], g);
        Gr[j] = g;
      }
    }
  }
  __syncwarp();
}

// Shared memory of the skew sampler: the walker workspace, 6 N doubles per warp (x^, y^, the columns of V),
// and ntile from-scratch tiles of N x (N + 1) doubles.
__host__ __device__ size_t skew_sampler_smem(const DevDims& d, int ntile, size_t* vec_off, size_t* tile_off) {
  size_t off = ws_layout(d, kSkWarps, nullptr, nullptr, false);
  if (vec_off) *vec_off = off;
  off = align16(off + (size_t)kSkWarps * 6 * d.N * 8);
  if (tile_off) *tile_off = off;
  return off + (size_t)ntile * d.N * (d.N + 1) * 8;
}

template <int KPL>
__global__ void __launch_bounds__(kSkThreads, 1)
    sampler_skew_kernel(const __grid_constant__ DevDims d, const __grid_constant__ DevTables t,
                        const __grid_constant__ DevParams p, const __grid_constant__ DevWalkers W, int first,
                        int ntile) {
  extern __shared__ __align__(16) char smem[];
  __shared__ WS ws;
  const int w = blockIdx.x;
  if (w >= d.nw) return;
  size_t vec_off = 0, tile_off = 0;
  skew_sampler_smem(d, ntile, &vec_off, &tile_off);
  if (threadIdx.x == 0) ws_layout(d, kSkWarps, smem, &ws, false);
  __syncthreads();
  const int N = d.N, Np = d.Np;
  const SCtx c{d, t, p, W, w, ws, W.Y + (size_t)w * d.n_qp * N * N, (double*)(smem + tile_off), ntile};
  const WS& s = ws;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nwarps = blockDim.x >> 5;
  double* xh = (double*)(smem + vec_off) + (size_t)warp * 6 * N;
  double* yh = xh + N;
  double* vv = xh + 2 * N;
  using F = SkewScratch<KPL>;

  for (int k = tid; k < 625; k += blockDim.x) s.mt[k] = W.mt[(size_t)w * 625 + k];
  if (tid == 0) {
    status(c) = 0;
    events_reset(s);
  }
  __syncthreads();
  int nfastup = W.nfastup[w];
  if (first) {
    make_initial_x<0, 0, F>(c);
  } else {
    for (int i = tid; i < N; i += blockDim.x) s.x[i] = W.xs[((size_t)w * d.ns + (d.ns - 1)) * N + i];
    __syncthreads();
    full_state<0, 0, F>(c);
    if (!status(c)) {
      if (tid == 0) {
        s.iflag[F_AUX] = grnd(s.mt) < 0.05;  // make_sample.f90:61
        s.iflag[F_EV_RESEED] += s.iflag[F_AUX];
        if (s.iflag[F_AUX] && W.trace) trace_rec(c, 3, 0.0, 0.0, 0.0, 0.0, 0.0);
      }
      __syncthreads();
      if (s.iflag[F_AUX]) make_initial_x<0, 0, F>(c);
    }
  }

  int naccept = 0, nacc_tmp = 0, nacc_all = 0;
  for (int i0 = -d.nwarm; i0 <= d.ns && !status(c); i0++) {
    if (nacc_tmp > nfastup) {
      checkpoint<0, 0, F>(c, nfastup, i0);
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
        global_flip<0, 0, F>(c);
        if (status(c)) break;
      }
      if (tid == 0) candidate_search(c);
      __syncthreads();
      if (status(c)) break;
      const int i1 = s.iflag[F_I1], i2 = s.iflag[F_I2];
      const int i3 = s.cfg[i1], i4 = s.cfg[i2];  // electron a = i3 moves to i2, electron b = i4 to i1
      const int ra_old = i1 + (i3 >= Np ? N : 0), rb_old = i2 + (i4 >= Np ? N : 0);
      const int ra_new = i2 + (i3 >= Np ? N : 0), rb_new = i1 + (i4 >= Np ? N : 0);
      cta_update_theta(d, t, p, s.x, i1, i2, s.th, s.thp);
      const int flipsign = (t.subB[i1] ? -1 : 1) * (t.subB[i2] ? -1 : 1);
      for (int mp = tid; mp < d.n_mp; mp += blockDim.x) s.sgnp[mp] = -s.sgn[mp] * flipsign;
      __syncthreads();
      cta_rbm_factors(d, s.thp, s.rbm);
      __syncthreads();
      double pre = 0.0, pim = 0.0;
      for (int qp = warp; qp < d.n_qp; qp += nwarps) {
        const double R = warp_skew_ratio<KPL>(d, p, c.Yw + (size_t)qp * N * N, qp, s.idx, i3, i4, ra_new, rb_new,
                                              xh, yh);
        if (lane == 0) {
          const double pfn = R * s.pf[qp];
          s.pfp[qp] = pfn;
          const cplx cw = psi_wo_pf(d, t, s.rbm[qp], s.sgnp[qp >> 1], qp);
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
        const double r1 = (hypot(re, im) + d.shift) / (hypot(s.dsc[D_PSI0R], s.dsc[D_PSI0I]) + d.shift);
        const double u = grnd(s.mt);
        s.iflag[F_ACCEPT] = u < r1 * r1;  // make_sample.f90:203-204
        if (W.trace) trace_rec(c, 0, (double)i1, (double)i2, r1 * r1, u, (double)s.iflag[F_ACCEPT]);
      }
      __syncthreads();
      if (s.iflag[F_ACCEPT]) {  // make_sample.f90:205-219
        for (int qp = warp; qp < d.n_qp; qp += nwarps)
          warp_skew_update<KPL>(d, p, c.Yw + (size_t)qp * N * N, qp, s.idx, i3, i4, ra_old, rb_old, ra_new, rb_new,
                                xh, yh, vv);
        for (int j = tid; j < d.Mr; j += blockDim.x) s.th[j] = s.thp[j];
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
      const size_t sidx = (size_t)w * d.ns + (i0 - 1);
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

// ---- estimator ----
struct SkEst {
  int* ap;       // [4N][2] antiparallel bonds (i1, i2) in bond_map order
  double* apc;   // [4N]    2 J sgn
  double* Rb;    // [kSkWarps][4N] exchange ratios of the warp's current projection
  double* vec;   // [kSkWarps][3N] x^, y^, G y^
  double* tiles; // [nqw][N (N + 1)]
  int* perm;     // [nqw][N]
  double* pfw;   // [n_qp]
  int* nap;
  double* diag;
  int nqw;
};

__host__ __device__ __forceinline__ size_t skest_layout(const DevDims& d, int nqw, char* base, WS* w, SkEst* e) {
  size_t off = 0;
  auto take = [&](size_t bytes) -> char* {
    char* p = base ? base + off : nullptr;
    off = align16(off + bytes);
    return p;
  };
  const int N = d.N, NB = 4 * N;
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
  t.pf = t.pfp = nullptr;
  t.psi = (double*)take((size_t)d.n_qp * 16);
  t.psip = nullptr;
  t.rbm = (double*)take((size_t)d.n_qp * 8);
  t.tile = t.colbuf = t.rowbuf = nullptr;
  t.perm = nullptr;
  t.wu = (double*)take((size_t)kSkWarps * N * 4);  // per-warp N-int buffers of cta_sign_pp
  t.wv = t.wA = t.wS = nullptr;
  t.red = (double*)take(64 * 8);
  t.iflag = (int*)take(32 * 4);
  t.dsc = (double*)take(32 * 8);
  SkEst x;
  x.ap = (int*)take((size_t)NB * 2 * 4);
  x.apc = (double*)take((size_t)NB * 8);
  x.Rb = (double*)take((size_t)kSkWarps * NB * 8);
  x.vec = (double*)take((size_t)kSkWarps * 3 * N * 8);
  x.perm = (int*)take((size_t)kSkWarps * N * 4);
  x.pfw = (double*)take((size_t)d.n_qp * 8);
  x.nap = (int*)take(16);
  x.diag = (double*)take(16);
  x.tiles = (double*)take((size_t)nqw * N * (N + 1) * 8);
  x.nqw = nqw;
  if (w) *w = t;
  if (e) *e = x;
  return off;
}

// d Pf / d f_k coefficients of B(i, j), i < j, by the spins of i (row) and j (column): B(i, j) = c1 f(k1) + c2 f(k2)
// + ..., k1 = orb(T site_j, T site_i), k2 = orb(T site_i, T site_j) (slater.f90:36-44 with B = -Slater_Elm)
__device__ __forceinline__ void skew_coef(const DevDims& d, int sp, bool dn_i, bool dn_j, double& c1, double& c2) {
  const double cs = d.sp_cs[sp], cc = d.sp_cc[sp], ss = d.sp_ss[sp];
  if (!dn_i && !dn_j) {
    c1 = cs;
    c2 = -cs;
  } else if (dn_i && !dn_j) {
    c1 = -cc;
    c2 = -ss;
  } else if (!dn_i && dn_j) {
    c1 = ss;
    c2 = cc;
  } else {
    c1 = -cs;
    c2 = cs;
  }
}

template <int KPL>
__global__ void __launch_bounds__(kSkThreads, 1)
    estimator_skew_kernel(const __grid_constant__ DevDims d, const __grid_constant__ DevTables t,
                          const __grid_constant__ DevParams p, const int8_t* xs, int n, double* out_psi,
                          double* out_hpsi, double* O, int* out_nap, int* out_status, int reweight, int nqw) {
  extern __shared__ __align__(16) char smem[];
  __shared__ WS s;
  __shared__ SkEst e;
  if (threadIdx.x == 0) skest_layout(d, nqw, smem, &s, &e);
  __syncthreads();
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int N = d.N, Np = d.Np, ld = N + 1, NB = 4 * N;
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
    for (int b = 0; b < NB && !st; b++) {
      const int i1 = t.bonds[2 * b], i2 = t.bonds[2 * b + 1];
      const double J = (b < 2 * N) ? d.J1 : d.J2, sg = (b < 2 * N) ? -1.0 : 1.0;
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
  double* Rw = e.Rb + (size_t)warp * NB;
  double* xh = e.vec + (size_t)warp * 3 * N;
  double* yh = xh + N;
  double* gy = yh + N;
  int bad = 0;
  double hacc = 0.0;
  for (int q0 = 0; q0 < d.n_qp; q0 += e.nqw) {
    const int qp = q0 + warp;
    if (warp < e.nqw && qp < d.n_qp) {
      const int mp = qp >> 1, sp = qp & 1;
      double* T = e.tiles + (size_t)warp * N * ld;
      int* src = e.perm + (size_t)warp * N;
      warp_gather_skew(T, d, p, qp, s.idx);
      bool sing;
      const double pfq = warp_pfaffian<KPL>(T, N, sing);
      if (!sing) {
        warp_gather_skew(T, d, p, qp, s.idx);
        (void)warp_gj<KPL, 0, 4>(T, N, src, sing);
        if (!sing) warp_unpermute_skew<KPL>(T, N, src);
      }
      if (sing) bad = 1;
      const cplx cw = psi_wo_pf(d, t, s.rbm[qp], s.sgn[mp], qp);
      if (lane == 0) {
        e.pfw[qp] = sing ? 0.0 : pfq;
        s.psi[2 * qp] = cw.re * pfq;
        s.psi[2 * qp + 1] = cw.im * pfq;
      }
      // exchange ratio of every antiparallel bond against G = B^{-1} (the tile, skew-symmetrised)
      for (int b = 0; b < nap && !sing; b++) {
        const int i1 = e.ap[2 * b], i2 = e.ap[2 * b + 1];
        const int ea = s.cfg[i1], eb = s.cfg[i2];  // electron ea moves to i2, eb to i1
        const int ra = i2 + (ea >= Np ? N : 0), rb = i1 + (eb >= Np ? N : 0);
        const double* SEa = se_row(d, p, qp, ra);
        const double* SEb = se_row(d, p, qp, rb);
        warp_gather_xy(d, SEa, SEb, s.idx, ea, eb, xh, yh);
        const double ya = -SEa[rb];
        // (G y^)_i for this lane's rows
        double xgy = 0.0;
        for (int i = lane; i < N; i += 32) {
          const double* Tr = T + i * ld;
          double acc = 0.0;
          for (int j = 0; j < N; j++) acc = fma(Tr[j], yh[j], acc);
          gy[i] = acc;
          xgy = fma(xh[i], acc, xgy);
        }
        double gxa = 0.0, gxb = 0.0;
        for (int j = lane; j < N; j += 32) {
          gxa = fma(T[ea * ld + j], xh[j], gxa);
          gxb = fma(T[eb * ld + j], xh[j], gxb);
        }
        xgy = warp_sum(xgy);
        gxa = warp_sum(gxa);
        gxb = warp_sum(gxb);
        __syncwarp();
        const double gab = T[ea * ld + eb];
        if (lane == 0) Rw[b] = -gab * (ya + xgy) + gxa * gy[eb] - gxb * gy[ea];
        __syncwarp();
      }
      __syncwarp();
      // weigh every bond: cosh product of theta' for this projection (update_theta on the qp's alphar slots)
      if (!sing) {
        const int* wm = t.wmap + (size_t)mp * N;
        const double s_sign = sp == 0 ? 1.0 : -1.0;
        for (int b = lane; b < nap; b += 32) {
          const int i1 = e.ap[2 * b], i2 = e.ap[2 * b + 1];
          const int iw1 = wm[i1], iw2 = wm[i2];
          const double x1 = (double)s.x[i1], x2 = (double)s.x[i2];
          double ch = 1.0;
          for (int f = 0; f < d.alphar; f++) {
            double th = s.th[qp * d.alphar + f];
            th = th - 2.0 * p.Wr[(size_t)f * N + iw1] * x1 * s_sign;
            th = th - 2.0 * p.Wr[(size_t)f * N + iw2] * x2 * s_sign;
            ch = ch * cosh(th);
          }
          const int sg = -s.sgn[mp] * (t.subB[i1] ? -1 : 1) * (t.subB[i2] ? -1 : 1);
          const cplx cbw = psi_wo_pf(d, t, ch, sg, qp);
          hacc = hacc + e.apc[b] * (cbw.re * (Rw[b] * pfq));
        }
      }
      __syncwarp();
    }
    __syncthreads();
    // d Pf / d f_k of this round's projections, in projection order: Pf sum_{i<j} G(j, i) dB(i, j)/df_k
    if (Orow) {
      for (int w = 0; w < e.nqw && q0 + w < d.n_qp; w++) {
        const int qp = q0 + w, mp = qp >> 1, sp = qp & 1;
        const double* Tw = e.tiles + (size_t)w * N * ld;
        const int* wm = t.wmap + (size_t)mp * N;
        const cplx cw = psi_wo_pf(d, t, s.rbm[qp], s.sgn[mp], qp);
        const double pw = e.pfw[qp] * cw.re;
        const int npr = N * (N - 1) / 2;
        for (int pr = tid; pr < npr; pr += blockDim.x) {
          // pair (i, j), i < j, from the triangular index pr = j (j - 1) / 2 + i
          int j = (int)((1.0 + sqrt(1.0 + 8.0 * (double)pr)) * 0.5);
          while (j * (j - 1) / 2 > pr) j--;
          while ((j + 1) * j / 2 <= pr) j++;
          const int i = pr - j * (j - 1) / 2;
          const double gji = Tw[j * ld + i];
          const int ti = wm[s.idx[i]], tj = wm[s.idx[j]];
          double c1, c2;
          skew_coef(d, sp, i >= Np, j >= Np, c1, c2);
          const int k1 = off_pp + t.orb[(size_t)tj * N + ti], k2 = off_pp + t.orb[(size_t)ti * N + tj];
          if (d.orb_injective) {
            if (c1 != 0.0) Orow[k1] += gji * c1 * pw;
            if (c2 != 0.0) Orow[k2] += gji * c2 * pw;
          } else {
            if (c1 != 0.0) atomicAdd(Orow + k1, gji * c1 * pw);
            if (c2 != 0.0) atomicAdd(Orow + k2, gji * c2 * pw);
          }
        }
        __syncthreads();
      }
    }
    __syncthreads();
  }
  if (lane == 0 && bad) s.iflag[F_STATUS] = ST_SINGULAR;
  hacc = warp_sum(hacc);
  if (lane == 0) s.red[warp] = hacc;
  __syncthreads();
  if (s.iflag[F_STATUS]) {
    if (tid == 0 && out_status) out_status[cfgi] = s.iflag[F_STATUS];
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
    double hr = e.diag[0] * re, hi = e.diag[0] * im;
    for (int w = 0; w < kSkWarps; w++) hr += s.red[w];
    s.dsc[D_PSIPR] = hr;
    s.dsc[D_PSIPI] = hi;
    if (out_nap) out_nap[cfgi] = nap;
    if (out_status) out_status[cfgi] = 0;
  }
  __syncthreads();
  const double wgt = reweight ? 1.0 / (hypot(s.dsc[D_PSI0R], s.dsc[D_PSI0I]) + d.shift) : 1.0;
  if (Orow) {
    // RBM part, real branch (calc_phys_quantity.f90:165-201)
    for (int k = tid; k < d.alphar * (N + 1); k += blockDim.x) {
      double acc = 0.0;
      if (k < d.alphar) {
        const int f = k;
        for (int qp = 0; qp < d.n_qp; qp++) acc = acc + tanh(s.th[qp * d.alphar + f]) * s.psi[2 * qp];
      } else {
        const int f = (k - d.alphar) / N, iw = (k - d.alphar) - f * N;
        for (int mp = 0; mp < d.n_mp; mp++) {
          const double xi = (double)s.x[t.winv[(size_t)mp * N + iw]];
          const int qa = 2 * mp, qb = 2 * mp + 1;
          acc = acc + tanh(s.th[qa * d.alphar + f]) * s.psi[2 * qa] * xi;
          acc = acc - tanh(s.th[qb * d.alphar + f]) * s.psi[2 * qb] * xi;
        }
      }
      Orow[k] = acc * wgt;
    }
    for (int k = off_pp + tid; k < d.Nv; k += blockDim.x) Orow[k] = Orow[k] * wgt;
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
      out_hpsi[2 * (size_t)cfgi] = s.dsc[D_PSIPR] * wgt;
      out_hpsi[2 * (size_t)cfgi + 1] = s.dsc[D_PSIPI] * wgt;
    }
  }
}

int max_smem_optin() {
  int dev = 0, maxsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return maxsm;
}

int skew_sampler_tiles(const DevDims& d, int maxsm) {
  for (int q = kSkWarps; q >= 1; q--)
    if ((long long)skew_sampler_smem(d, q, nullptr, nullptr) <= maxsm) return q;
  return 0;
}

int skew_est_tiles(const DevDims& d, int maxsm) {
  for (int q = kSkWarps; q >= 1; q--)
    if ((long long)skest_layout(d, q, nullptr, nullptr, nullptr) <= maxsm) return q;
  return 0;
}

}  // namespace

// Largest N the skew kernels take (lanes hold N / 32 columns each).
int rbmpp_skew_max_n() { return 128; }

// 0 when the skew sampler and estimator fit one block's shared memory at this shape, else the bytes one of them
// needs at its smallest.
size_t rbmpp_skew_smem_shortfall(const DevDims& d, int maxsm) {
  if (skew_sampler_tiles(d, maxsm) < 1) return skew_sampler_smem(d, 1, nullptr, nullptr);
  if (skew_est_tiles(d, maxsm) < 1) return skest_layout(d, 1, nullptr, nullptr, nullptr);
  return 0;
}

cudaError_t rbmpp_build_se(const DevDims& d, const int* wmap, const int* orb, const double* slater, double* SE,
                           cudaStream_t st) {
  const long long tot = (long long)d.n_qp * d.N * d.N;
  rbmpp_note_launch();
  build_se_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(d.N, d.n_mp, wmap, orb, slater, d.sp_cs[0],
                                                                   d.sp_cs[1], d.sp_cc[0], d.sp_cc[1], d.sp_ss[0],
                                                                   d.sp_ss[1], SE);
  return cudaGetLastError();
}

cudaError_t rbmpp_launch_sampler_skew(const DevDims& d, const DevTables& t, const DevParams& p, const DevWalkers& W,
                                      int first, cudaStream_t st) {
  const int ntile = skew_sampler_tiles(d, max_smem_optin());
  if (ntile < 1 || d.N > rbmpp_skew_max_n()) return cudaErrorInvalidValue;
  const size_t smem = skew_sampler_smem(d, ntile, nullptr, nullptr);
#define LAUNCH_SK(K)                                                                                            \
  do {                                                                                                          \
    cudaError_t e = cudaFuncSetAttribute(sampler_skew_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,   \
                                         (int)smem);                                                            \
    if (e != cudaSuccess) return e;                                                                             \
    rbmpp_note_launch();                                                                                        \
    sampler_skew_kernel<K><<<d.nw, kSkThreads, smem, st>>>(d, t, p, W, first, ntile);                           \
    return cudaGetLastError();                                                                                  \
  } while (0)
  const int kpl = (d.N + 31) / 32;
  if (kpl <= 1) LAUNCH_SK(1);
  if (kpl <= 2) LAUNCH_SK(2);
  if (kpl <= 3) LAUNCH_SK(3);
  LAUNCH_SK(4);
#undef LAUNCH_SK
}

cudaError_t rbmpp_launch_estimator_skew(const DevDims& d, const DevTables& t, const DevParams& p, const int8_t* xs,
                                        int n, double* out_psi, double* out_hpsi, double* O, int* out_nap,
                                        int* out_status, int reweight, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int nqw = skew_est_tiles(d, max_smem_optin());
  if (nqw < 1 || d.N > rbmpp_skew_max_n()) return cudaErrorInvalidValue;
  const size_t smem = skest_layout(d, nqw, nullptr, nullptr, nullptr);
#define LAUNCH_SE(K)                                                                                             \
  do {                                                                                                           \
    cudaError_t e = cudaFuncSetAttribute(estimator_skew_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,  \
                                         (int)smem);                                                             \
    if (e != cudaSuccess) return e;                                                                              \
    rbmpp_note_launch();                                                                                         \
    estimator_skew_kernel<K><<<n, kSkThreads, smem, st>>>(d, t, p, xs, n, out_psi, out_hpsi, O, out_nap,         \
                                                          out_status, reweight, nqw);                            \
    return cudaGetLastError();                                                                                   \
  } while (0)
  const int kpl = (d.N + 31) / 32;
  if (kpl <= 1) LAUNCH_SE(1);
  if (kpl <= 2) LAUNCH_SE(2);
  if (kpl <= 3) LAUNCH_SE(3);
  LAUNCH_SE(4);
#undef LAUNCH_SE
}

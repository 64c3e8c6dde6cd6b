// rbmpp_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU FP64 restatement of the RBM_PP variational-Monte-Carlo hot path (sampling, local energy,
// O_k, stochastic reconfiguration).  It is the checker for the CUDA path: only tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm may load it.  The product
// (rbm_pp_b200/) never links, imports or executes anything from this directory.
//
// Every routine cites the reference file:line it restates (paths relative to
// code/normal_code/ of yusukenomura/RBM_PP).  Emulated MPI ranks are independent walkers, each
// with its own MT19937 stream, exactly as one rank of the reference.
//
// Parity status: the reference (Fortran + MKL + a binary-only PFAPACK) cannot be compiled here, so
// no reference outputs exist to pin against ("parity unpinned" with respect to reference-run
// outputs).  The oracle is pinned instead against independent known answers: numpy's MT19937
// core, brute-force Pfaffians, LAPACK (scipy) inverses and Cholesky, exact diagonalisation of the
// 4x4 J1-J2 model, and central finite differences of ln psi.
//
// Conventions that the Fortran source leaves open and this restatement fixes:
//  * `.and.` is evaluated left to right with short circuit (make_sample.f90:122,
//    SR_pdposv.f90:172,281,313), which fixes how many RNG draws those lines consume.
//  * PFAPACK dskpfa('U','P') is restated as Parlett-Reid skew LTL^T elimination with pivoting
//    (M. Wimmer, ACM TOMS 38(4), 2012); MKL dgetrf/dgetri as LU with partial pivoting.
//
// Build: oracle/Makefile (g++ -O2 -ffp-contract=off -fopenmp, shared library for ctypes).

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cplx;

// ------------------------------------------------------------------------------------------------
// MT19937 with Knuth-69069 seeding: mt.f:6-29 (sgrnd), mt.f:32-102 (grnd).
// grnd() returns y/(2^32-1) in [0,1] inclusive (mt.f:95-99).
// ------------------------------------------------------------------------------------------------
struct MT {
  uint32_t mt[624];
  int mti;
};

static void mt_seed(MT& s, int32_t seed) {  // mt.f:23-26
  s.mt[0] = (uint32_t)seed;
  for (int i = 1; i < 624; i++) s.mt[i] = 69069u * s.mt[i - 1];
  s.mti = 624;
}

static uint32_t mt_next_u32(MT& s) {  // mt.f:67-93
  const uint32_t UMASK = 0x80000000u, LMASK = 0x7fffffffu, MATA = 0x9908b0dfu;
  if (s.mti >= 624) {
    int kk;
    uint32_t y;
    for (kk = 0; kk < 624 - 397; kk++) {
      y = (s.mt[kk] & UMASK) | (s.mt[kk + 1] & LMASK);
      s.mt[kk] = s.mt[kk + 397] ^ (y >> 1) ^ ((y & 1u) ? MATA : 0u);
    }
    for (; kk < 623; kk++) {
      y = (s.mt[kk] & UMASK) | (s.mt[kk + 1] & LMASK);
      s.mt[kk] = s.mt[kk + (397 - 624)] ^ (y >> 1) ^ ((y & 1u) ? MATA : 0u);
    }
    y = (s.mt[623] & UMASK) | (s.mt[0] & LMASK);
    s.mt[623] = s.mt[396] ^ (y >> 1) ^ ((y & 1u) ? MATA : 0u);
    s.mti = 0;
  }
  uint32_t y = s.mt[s.mti++];
  y ^= (y >> 11);
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= (y >> 18);
  return y;
}

static double grnd(MT& s) { return (double)mt_next_u32(s) / 4294967295.0; }  // mt.f:95-99

// nran(n) = mod(int(dble(n)*grnd()),n) + 1   (make_sample.f90:254,317), 1-based result
static int nran(MT& s, int n) { return ((int)((double)n * grnd(s))) % n + 1; }

// ------------------------------------------------------------------------------------------------
// Context: module globals of module.f90 plus one record per emulated rank.
// ------------------------------------------------------------------------------------------------
enum {
  ORC_OK = 0,
  ORC_E_ARG = 1,
  ORC_E_CONFIG = 2,       // x / Ele_Idx bookkeeping (interface_for_PP.f90:26-30,37-65)
  ORC_E_SIGN = 3,         // sign_PP consistency (interface_for_PP.f90:101-103, make_sample.f90:90-92)
  ORC_E_THETA = 4,        // theta drift (make_sample.f90:84-89)
  ORC_E_CANDIDATE = 5,    // make_spin_flip_candidate fails (make_sample.f90:290-291)
  ORC_E_INITX = 6,        // make_initial_x fails (make_sample.f90:337,359)
  ORC_E_SKEW = 7,         // InvM not skew-symmetric (matrix.f90:103)
  ORC_E_SINGULAR = 8,     // LU/Pfaffian breakdown (matrix.f90:145-148,171-174)
  ORC_E_SDIAG = 9,        // S-matrix diagonal checks (SR_pdposv.f90:32-33,78-100,132,140)
  ORC_E_CHOL = 10,        // pdposv info /= 0 (SR_pdposv.f90:233-236)
  ORC_E_SLATER_NORM = 11, // f renormalisation (SR_pdposv.f90:414)
  ORC_E_LAMBDA = 12,      // lambda split (SR_pdposv.f90:308)
};

struct Rank {
  MT rng;
  int nfastup;
  int naccept;
  // diagnostics of the last make_sample: global flips tried / accepted, make_initial_x re-seeds,
  // checkpoints, trace records; and the chain trace (6 doubles per record, the library's record layout)
  int ev[5] = {0, 0, 0, 0, 0};
  std::vector<double> trace;
  void rec(int max, int type, double a, double b, double x, double u, double e) {
    if (ev[4] < max) {
      double* q = &trace[(size_t)ev[4] * 6];
      q[0] = type;
      q[1] = a;
      q[2] = b;
      q[3] = x;
      q[4] = u;
      q[5] = e;
    }
    ev[4]++;
  }
  std::vector<int> x_sample;      // x_sample(N, Nsample)            module.f90:39
  std::vector<cplx> psi_sample;   // psi_x_sample(0:N_QP, Nsample)   module.f90:40
  std::vector<double> pf_sample;  // PfM_sample(N_QP, Nsample)       module.f90:41
  int err;
};

struct Ctx {
  int L, N, Npair, n_mp, alphac, alphar, n_slater, n_qp, Mr, Mc, Nv, Nv_rbm, nsample, nranks, nupdate;
  int spin_parity;
  double J1, J2;
  std::vector<int> W_map;  // W_map(N, n_mp), 0-based values          module.f90:34
  std::vector<cplx> para_mp;
  std::vector<int> orb_idx, orb_sgn;  // Orbital_Idx(N,N) 0-based, Orbital_Sgn
  std::vector<char> subB;
  double sp_cos[2], sp_sin[2], sp_cc[2], sp_cs[2], sp_ss[2], para_sp[2];
  std::vector<double> Wr, br, slater;  // Wrirr(N,alphar), brirr(alphar), Slater(N_Slater)
  std::vector<cplx> Wc, bc;            // Wcirr(N,alphac), bcirr(alphac)
  double shift;
  std::vector<double> SE;  // Slater_Elm(2N, 2N, N_QP)                module.f90:55
  std::vector<Rank> ranks;
  int rank0 = 0;  // global MPI rank of local rank 0 (a shard of the ranks)
  int trace_max = 0;  // chain-trace records kept per rank
  int err;
  char msg[256];
};

static int set_err(Ctx& c, int code, const char* m) {
  if (!c.err) {
    c.err = code;
    snprintf(c.msg, sizeof(c.msg), "%s", m);
  }
  return code;
}

// ------------------------------------------------------------------------------------------------
// Spin-projection weights: spin_projection.f90:5-79 (N_SP_Gauss_Leg = 2, beta = {0, pi}).
// ------------------------------------------------------------------------------------------------
static void init_sp_weight(Ctx& c) {
  const double pi = std::acos(-1.0);
  double beta[2] = {0.0, pi};  // spin_projection.f90:29-32
  for (int s = 0; s < 2; s++) {
    c.sp_cos[s] = std::cos(0.5 * beta[s]);
    c.sp_sin[s] = std::sin(0.5 * beta[s]);
    c.sp_cc[s] = c.sp_cos[s] * c.sp_cos[s];
    c.sp_cs[s] = c.sp_cos[s] * c.sp_sin[s];
    c.sp_ss[s] = c.sp_sin[s] * c.sp_sin[s];
  }
  c.para_sp[0] = 1.0;  // spin_projection.f90:55-62
  c.para_sp[1] = (c.spin_parity == 1) ? 1.0 : -1.0;
}

// define_sublattice: interface_for_PP.f90:110-136 (site i = i2*L + i1 + 1, B if i1+i2 odd)
static void define_sublattice(Ctx& c) {
  c.subB.assign(c.N, 0);
  int i = 0;
  for (int i2 = 0; i2 < c.L; i2++)
    for (int i1 = 0; i1 < c.L; i1++) c.subB[i++] = ((i1 + i2) % 2 == 1);
}

// ------------------------------------------------------------------------------------------------
// update_slater_elements: slater.f90:7-64.  SE(r, r', qp) column-major, 2N x 2N per qp.
// ------------------------------------------------------------------------------------------------
static int update_slater_elements(Ctx& c) {
  const int N = c.N, N2 = 2 * N;
  c.SE.assign((size_t)N2 * N2 * c.n_qp, 0.0);
  int qp = 0;
  for (int mp = 0; mp < c.n_mp; mp++) {
    for (int sp = 0; sp < 2; sp++, qp++) {
      double cs = c.sp_cs[sp], cc = c.sp_cc[sp], ss = c.sp_ss[sp];
      double* S = &c.SE[(size_t)N2 * N2 * qp];
      for (int ri = 0; ri < N; ri++) {
        int tri = c.W_map[ri + N * mp];  // MP_Trans_Idx = W_map(:,1,mp), parameter.f90:105-109
        for (int rj = 0; rj < N; rj++) {
          int trj = c.W_map[rj + N * mp];
          int i1 = c.orb_idx[tri + N * trj], i2 = c.orb_idx[trj + N * tri];
          double slt_ij = c.slater[i1] * (double)(c.orb_sgn[tri + N * trj]);
          double slt_ji = c.slater[i2] * (double)(c.orb_sgn[trj + N * tri]);
          S[rj + N2 * ri] = -(slt_ij - slt_ji) * cs;             // up - up
          S[(rj + N) + N2 * ri] = slt_ij * cc + slt_ji * ss;     // up - down
          S[rj + N2 * (ri + N)] = -slt_ij * ss - slt_ji * cc;    // down - up
          S[(rj + N) + N2 * (ri + N)] = (slt_ij - slt_ji) * cs;  // down - down
        }
      }
      for (int i2 = 0; i2 < N2; i2++)  // slater.f90:51-56
        for (int i1 = 0; i1 < N2; i1++)
          if (std::fabs(S[i1 + N2 * i2] + S[i2 + N2 * i1]) > 1e-10)
            return set_err(c, ORC_E_SKEW, "Slater_Elm is not skew-symmetric");
    }
  }
  return 0;
}

// ------------------------------------------------------------------------------------------------
// RBM theta: calc_theta RBM.f90:31-91, update_theta RBM.f90:95-148.
// th holds thetar (Mr reals, index j = mp*2*alphar + (s==+1 ? 0 : alphar) + f) followed by thetac
// (Mc complex as (re, im) pairs, the same index pattern with alphac).
// ------------------------------------------------------------------------------------------------
static int n_theta(const Ctx& c) { return c.Mr + 2 * c.Mc; }
static cplx thc(const Ctx& c, const double* th, int j) { return cplx(th[c.Mr + 2 * j], th[c.Mr + 2 * j + 1]); }

static void calc_theta(const Ctx& c, const int* x, double* th) {
  const int N = c.N;
  for (int mp = 0; mp < c.n_mp; mp++) {
    int j = mp * 2 * c.alphac;
    for (int s = 1; s >= -1; s -= 2)
      for (int f = 0; f < c.alphac; f++) {
        cplx t = c.bc[f];
        for (int i = 0; i < N; i++) {
          int iw = c.W_map[i + N * mp];
          t = t + c.Wc[iw + N * f] * (double)x[i] * (double)s;
        }
        th[c.Mr + 2 * j] = t.real();
        th[c.Mr + 2 * j + 1] = t.imag();
        j++;
      }
  }
  for (int mp = 0; mp < c.n_mp; mp++) {
    int j = mp * 2 * c.alphar;
    for (int s = 1; s >= -1; s -= 2)
      for (int f = 0; f < c.alphar; f++) {
        double t = c.br[f];
        for (int i = 0; i < N; i++) {
          int iw = c.W_map[i + N * mp];
          t = t + c.Wr[iw + N * f] * (double)x[i] * (double)s;
        }
        th[j++] = t;
      }
  }
}

static void update_theta(const Ctx& c, const int* x, int i1, int i2, double* th) {
  const int N = c.N;
  for (int mp = 0; mp < c.n_mp; mp++) {
    int j = mp * 2 * c.alphac;
    int iw1 = c.W_map[i1 + N * mp], iw2 = c.W_map[i2 + N * mp];
    for (int s = 1; s >= -1; s -= 2)
      for (int f = 0; f < c.alphac; f++) {
        cplx t = thc(c, th, j);
        t = t - 2.0 * c.Wc[iw1 + N * f] * (double)x[i1] * (double)s;
        t = t - 2.0 * c.Wc[iw2 + N * f] * (double)x[i2] * (double)s;
        th[c.Mr + 2 * j] = t.real();
        th[c.Mr + 2 * j + 1] = t.imag();
        j++;
      }
  }
  for (int mp = 0; mp < c.n_mp; mp++) {
    int j = mp * 2 * c.alphar;
    int iw1 = c.W_map[i1 + N * mp], iw2 = c.W_map[i2 + N * mp];
    for (int s = 1; s >= -1; s -= 2)
      for (int f = 0; f < c.alphar; f++) {
        th[j] = th[j] - 2.0 * c.Wr[iw1 + N * f] * (double)x[i1] * (double)s;
        th[j] = th[j] - 2.0 * c.Wr[iw2 + N * f] * (double)x[i2] * (double)s;
        j++;
      }
  }
}

// ------------------------------------------------------------------------------------------------
// Electron bookkeeping: x_to_Ele_Idx_Ele_Cfg interface_for_PP.f90:5-33 (0-based sites/labels)
// ------------------------------------------------------------------------------------------------
static int x_to_ele(const Ctx& c, const int* x, int* idx, int* cfg) {
  int i1 = 0, i2 = c.Npair;
  for (int i = 0; i < c.N; i++) {
    if (x[i] == 1) {
      if (i1 >= c.Npair) return ORC_E_CONFIG;
      idx[i1] = i;
      cfg[i] = i1++;
    } else if (x[i] == -1) {
      if (i2 >= c.N) return ORC_E_CONFIG;
      idx[i2] = i;
      cfg[i] = i2++;
    } else
      return ORC_E_CONFIG;
  }
  if (i1 != c.Npair || i2 != c.N) return ORC_E_CONFIG;
  return 0;
}

// check_Ele_Idx_Ele_Cfg interface_for_PP.f90:37-65
static int check_ele(const Ctx& c, const int* x, const int* idx, const int* cfg) {
  std::vector<char> chk(c.N, 0);
  for (int i = 0; i < c.N; i++) {
    if (cfg[idx[i]] != i) return ORC_E_CONFIG;
    if (x[idx[i]] != (i < c.Npair ? 1 : -1)) return ORC_E_CONFIG;
    chk[idx[i]] = 1;
  }
  for (int i = 0; i < c.N; i++)
    if (!chk[i]) return ORC_E_CONFIG;
  return 0;
}

// sign_PP interface_for_PP.f90:71-106
static int sign_pp(const Ctx& c, const int* idx, int* sgn) {
  const int N = c.N;
  std::vector<int> t(N);
  int st0 = 0;
  for (int mp = 0; mp < c.n_mp; mp++) {
    for (int i1 = 0; i1 < N; i1++) t[i1] = c.W_map[idx[i1] + N * mp];
    int s = 1, st = 1;
    for (int i1 = 1; i1 < N; i1++) {
      if (i1 >= c.Npair && c.subB[t[i1]]) {
        s = -s;
        st = -st;
      }
      for (int i2 = 0; i2 < i1; i2++)
        if (t[i2] > t[i1]) s = -s;
    }
    sgn[mp] = s;
    if (mp == 0) st0 = st;
    else if (st != st0) return ORC_E_SIGN;
  }
  return 0;
}

// ------------------------------------------------------------------------------------------------
// Amplitude: calc_amplitude_RBM_PP sub.f90:4-89 (Ncopy = 1). qp = 2*mp + sp.
// Consumes exactly one grnd() per call (sub.f90:72); the self-check it guards only prints.
// psi has n_qp+1 entries: psi[0] = total, psi[1+qp] = per projection.
// ------------------------------------------------------------------------------------------------
static void amplitude(const Ctx& c, const double* th, const double* pf, const int* sgn, cplx* psi_wo_pf,
                      cplx* psi, MT& rng) {
  for (int qp = 0; qp < c.n_qp; qp++) {
    int mp = qp / 2, sp = qp % 2;
    cplx c1 = std::pow(0.5, c.alphac);  // sub.f90:37-41
    for (int f = 0; f < c.alphac; f++) {
      const cplx t = thc(c, th, qp * c.alphac + f);
      c1 = c1 * cplx(std::cosh(t.real()) * std::cos(t.imag()), std::sinh(t.real()) * std::sin(t.imag()));
    }
    double r1 = 1.0;
    for (int f = 0; f < c.alphar; f++) r1 = r1 * std::cosh(th[qp * c.alphar + f]);
    c1 = c1 * r1;
    c1 = c1 * (double)sgn[mp];
    c1 = c1 * c.para_mp[mp];
    c1 = c1 * c.para_sp[sp];
    psi_wo_pf[qp] = c1;
    psi[1 + qp] = c1 * pf[qp];
  }
  cplx s = 0.0;
  for (int qp = 0; qp < c.n_qp; qp++) s = s + psi[1 + qp];
  psi[0] = s;
  (void)grnd(rng);
}

// ------------------------------------------------------------------------------------------------
// Dense FP64 kernels used by calculate_MAll (matrix.f90:55-177).
// ------------------------------------------------------------------------------------------------
// Pfaffian of a real skew matrix by Parlett-Reid elimination with pivoting (restated from
// M. Wimmer, "Algorithm 923", ACM TOMS 38(4) 2012).  A is n x n column-major, destroyed.
static double pfaffian_pr(int n, double* A) {
  if (n % 2) return 0.0;
  double pf = 1.0;
  for (int k = 0; k < n - 1; k += 2) {
    int kp = k + 1;
    double amax = std::fabs(A[(k + 1) + (size_t)n * k]);
    for (int i = k + 2; i < n; i++) {
      double v = std::fabs(A[i + (size_t)n * k]);
      if (v > amax) {
        amax = v;
        kp = i;
      }
    }
    if (kp != k + 1) {
      for (int j = 0; j < n; j++) std::swap(A[(k + 1) + (size_t)n * j], A[kp + (size_t)n * j]);
      for (int i = 0; i < n; i++) std::swap(A[i + (size_t)n * (k + 1)], A[i + (size_t)n * kp]);
      pf = -pf;
    }
    if (A[(k + 1) + (size_t)n * k] == 0.0) return 0.0;
    double akk1 = A[k + (size_t)n * (k + 1)];
    pf = pf * akk1;
    if (k + 2 < n) {
      // tau(i) = A(k,i)/A(k,k+1);  A(i,j) += tau(i)*A(j,k+1) - A(i,k+1)*tau(j),  i,j >= k+2
      std::vector<double> tau(n), col(n);
      for (int i = k + 2; i < n; i++) {
        tau[i] = A[k + (size_t)n * i] / akk1;
        col[i] = A[i + (size_t)n * (k + 1)];
      }
      for (int j = k + 2; j < n; j++)
        for (int i = k + 2; i < n; i++)
          A[i + (size_t)n * j] = A[i + (size_t)n * j] + tau[i] * col[j] - col[i] * tau[j];
    }
  }
  return pf;
}

// In-place inverse by LU with partial pivoting (the role of dgetrf + dgetri, matrix.f90:155-177).
static int inverse_lu(int n, double* A) {
  std::vector<int> piv(n);
  for (int k = 0; k < n; k++) {
    int p = k;
    double amax = std::fabs(A[k + (size_t)n * k]);
    for (int i = k + 1; i < n; i++) {
      double v = std::fabs(A[i + (size_t)n * k]);
      if (v > amax) {
        amax = v;
        p = i;
      }
    }
    piv[k] = p;
    if (amax == 0.0) return ORC_E_SINGULAR;
    if (p != k)
      for (int j = 0; j < n; j++) std::swap(A[k + (size_t)n * j], A[p + (size_t)n * j]);
    double d = A[k + (size_t)n * k];
    for (int i = k + 1; i < n; i++) A[i + (size_t)n * k] /= d;
    for (int j = k + 1; j < n; j++) {
      double akj = A[k + (size_t)n * j];
      if (akj != 0.0)
        for (int i = k + 1; i < n; i++) A[i + (size_t)n * j] -= A[i + (size_t)n * k] * akj;
    }
  }
  // solve A * X = P^T ... column by column: inv(A) = inv(U) inv(L) P
  std::vector<double> X((size_t)n * n, 0.0), b(n);
  for (int col = 0; col < n; col++) {
    for (int i = 0; i < n; i++) b[i] = (i == col) ? 1.0 : 0.0;
    for (int k = 0; k < n; k++)
      if (piv[k] != k) std::swap(b[k], b[piv[k]]);
    for (int i = 0; i < n; i++) {  // L y = b (unit lower)
      double s = b[i];
      for (int k = 0; k < i; k++) s -= A[i + (size_t)n * k] * b[k];
      b[i] = s;
    }
    for (int i = n - 1; i >= 0; i--) {  // U x = y
      double s = b[i];
      for (int k = i + 1; k < n; k++) s -= A[i + (size_t)n * k] * b[k];
      b[i] = s / A[i + (size_t)n * i];
    }
    for (int i = 0; i < n; i++) X[i + (size_t)n * col] = b[i];
  }
  std::memcpy(A, X.data(), sizeof(double) * (size_t)n * n);
  return 0;
}

// calculate_MAll_child matrix.f90:55-110.  invM is the transposed inverse (matrix.f90:96-107).
static int calc_mall_qp(const Ctx& c, int qp, const int* idx, double* pf, double* invM, bool calc_inv,
                        std::vector<double>& b1, std::vector<double>& b2) {
  const int N = c.N, N2 = 2 * N, Np = c.Npair;
  const double* S = &c.SE[(size_t)N2 * N2 * qp];
  b1.resize((size_t)N * N);
  b2.resize((size_t)N * N);
  for (int msj = 0; msj < N; msj++) {
    int rsj = idx[msj] + (msj / Np) * N;
    for (int msi = 0; msi < N; msi++) {
      int rsi = idx[msi] + (msi / Np) * N;
      b1[msi + (size_t)N * msj] = -S[rsi + (size_t)N2 * rsj];
    }
  }
  b2 = b1;
  *pf = pfaffian_pr(N, b2.data());
  if (!calc_inv) return 0;
  if (inverse_lu(N, b1.data())) return ORC_E_SINGULAR;
  double r1 = 0.0;
  for (size_t k = 0; k < (size_t)N * N; k++) r1 = std::max(r1, std::fabs(b1[k]));
  for (int msj = 0; msj < N; msj++)
    for (int msi = 0; msi < N; msi++) {
      double a = b1[msj + (size_t)N * msi], b = b1[msi + (size_t)N * msj];
      double r2 = 0.5 * (a - b), r3 = 0.5 * (a + b);
      if (std::fabs(r3 / r1) > 2.0e-3) return ORC_E_SKEW;
      invM[msi + (size_t)N * msj] = r2;
    }
  return 0;
}

static int calc_mall(const Ctx& c, const int* idx, double* pf, double* invM, bool calc_inv) {
  std::vector<double> b1, b2;
  for (int qp = 0; qp < c.n_qp; qp++) {
    int e = calc_mall_qp(c, qp, idx, &pf[qp], invM ? invM + (size_t)c.N * c.N * qp : nullptr, calc_inv, b1, b2);
    if (e) return e;
  }
  return 0;
}

// ------------------------------------------------------------------------------------------------
// Fast updates: calculate_new_PfM_two_child pfupdate_two.f90:27-88 and
// calculate_new_InvM_two_child pfupdate_two.f90:113-224 (0-based msa, msb).
// ------------------------------------------------------------------------------------------------
static double new_pf_two_qp(const Ctx& c, int qp, int msa, int msb, const int* tidx, const double* InvM,
                            double pf_old, double* va, double* vb) {
  const int N = c.N, N2 = 2 * N, Np = c.Npair;
  const double* S = &c.SE[(size_t)N2 * N2 * qp];
  int rsa = tidx[msa] + (msa / Np) * N, rsb = tidx[msb] + (msb / Np) * N;
  for (int msi = 0; msi < N; msi++) {
    int rsi = tidx[msi] + (msi / Np) * N;
    va[msi] = S[rsi + (size_t)N2 * rsa];
    vb[msi] = S[rsi + (size_t)N2 * rsb];
  }
  double vec_ba = vb[msa];
  double InvM_ab = InvM[msb + (size_t)N * msa];
  double p_a = 0, p_b = 0, q_a = 0, q_b = 0, bMa = 0;
  for (int msi = 0; msi < N; msi++) {
    p_a = p_a + InvM[msi + (size_t)N * msa] * va[msi];
    p_b = p_b + InvM[msi + (size_t)N * msb] * va[msi];
    q_a = q_a + InvM[msi + (size_t)N * msa] * vb[msi];
    q_b = q_b + InvM[msi + (size_t)N * msb] * vb[msi];
  }
  for (int msi = 0; msi < N; msi++) {
    double rtmp = 0.0;
    for (int msj = 0; msj < N; msj++) rtmp = rtmp + InvM[msj + (size_t)N * msi] * va[msj];
    bMa = bMa + vb[msi] * rtmp;
  }
  double ratio = InvM_ab * vec_ba + InvM_ab * bMa + p_a * q_b - p_b * q_a;
  return ratio * pf_old;
}

static void new_invm_two_qp(const Ctx& c, int qp, int msa, int msb, const int* tidx, double* InvM) {
  const int N = c.N, N2 = 2 * N, Np = c.Npair;
  const double* S = &c.SE[(size_t)N2 * N2 * qp];
  std::vector<double> P(N), Q(N), Sv(N), T(N);
  int rsa = tidx[msa] + (msa / Np) * N, rsb = tidx[msb] + (msb / Np) * N;
  for (int msi = 0; msi < N; msi++) {
    int rsi = tidx[msi] + (msi / Np) * N;
    Sv[msi] = S[rsi + (size_t)N2 * rsa];
    T[msi] = S[rsi + (size_t)N2 * rsb];
  }
  for (int msi = 0; msi < N; msi++) {
    double p = 0.0, q = 0.0;
    for (int msj = 0; msj < N; msj++) {
      p = p + InvM[msj + (size_t)N * msi] * Sv[msj];
      q = q + InvM[msj + (size_t)N * msi] * T[msj];
    }
    P[msi] = p;
    Q[msi] = q;
  }
  double bMa = 0.0;
  for (int msi = 0; msi < N; msi++) bMa = bMa + T[msi] * P[msi];
  double a = -P[msa], b = P[msb], cc = Q[msa], d = -Q[msb], e = -bMa - T[msa];
  double f = InvM[msb + (size_t)N * msa];
  double Det = a * d - b * cc - e * f;
  double InvDet = 1.0 / Det;
  for (int msi = 0; msi < N; msi++) {
    Sv[msi] = InvDet * InvM[msi + (size_t)N * msa];
    T[msi] = InvDet * InvM[msi + (size_t)N * msb];
  }
  for (int msi = 0; msi < N; msi++) {
    double p_i = P[msi], q_i = Q[msi], s_i = Sv[msi], t_i = T[msi];
    for (int msj = 0; msj < N; msj++) {
      double p_j = P[msj], q_j = Q[msj], s_j = Sv[msj], t_j = T[msj];
      double& m = InvM[msj + (size_t)N * msi];
      m = m + a * (q_i * t_j - q_j * t_i) + b * (q_i * s_j - q_j * s_i) + cc * (p_i * t_j - p_j * t_i) +
          d * (p_i * s_j - p_j * s_i) + e * Det * (s_i * t_j - s_j * t_i) + f * InvDet * (p_i * q_j - q_i * p_j);
    }
    double& ma = InvM[msa + (size_t)N * msi];
    ma = ma - cc * t_i - d * s_i - f * InvDet * q_i;
    double& mb = InvM[msb + (size_t)N * msi];
    mb = mb - a * t_i - b * s_i + f * InvDet * p_i;
  }
  for (int msi = 0; msi < N; msi++) {
    double p_i = P[msi], q_i = Q[msi], s_i = Sv[msi], t_i = T[msi];
    double& ma = InvM[msi + (size_t)N * msa];
    ma = ma + cc * t_i + d * s_i + f * InvDet * q_i;
    double& mb = InvM[msi + (size_t)N * msb];
    mb = mb + a * t_i + b * s_i - f * InvDet * p_i;
  }
  InvM[msa + (size_t)N * msb] = InvM[msa + (size_t)N * msb] - f * InvDet;
  InvM[msb + (size_t)N * msa] = InvM[msb + (size_t)N * msa] + f * InvDet;
}

// ------------------------------------------------------------------------------------------------
// Per-walker state (make_sample.f90:14-33)
// ------------------------------------------------------------------------------------------------
struct WState {
  std::vector<int> x, idx, cfg, sgn;
  std::vector<double> th, pf, inv;
  std::vector<cplx> psi, psi_wo;
  void init(const Ctx& c) {
    x.assign(c.N, 0);
    idx.assign(c.N, 0);
    cfg.assign(c.N, 0);
    sgn.assign(c.n_mp, 1);
    th.assign(n_theta(c), 0.0);
    pf.assign(c.n_qp, 0.0);
    inv.assign((size_t)c.N * c.N * c.n_qp, 0.0);
    psi.assign(c.n_qp + 1, 0.0);
    psi_wo.assign(c.n_qp, 0.0);
  }
};

// make_spin_flip_candidate make_sample.f90:244-294 (returns 0-based sites)
static int spin_flip_candidate(const Ctx& c, const int* x, MT& rng, int* o1, int* o2) {
  const int L = c.L, N = c.N;
  int dist_max = nran(rng, L - 1) + 1;
  if (dist_max <= 1) return ORC_E_CANDIDATE;
  for (int it = 0; it < 1000000; it++) {
    int i1 = nran(rng, N);
    int ix = (i1 - 1) / L, iy = (i1 - 1) - ix * L;
    ix = ix + nran(rng, dist_max) - 1;
    iy = iy + nran(rng, dist_max) - 1;
    if (ix >= L) ix -= L;
    if (iy >= L) iy -= L;
    int i2 = ix * L + iy + 1;
    if (x[i1 - 1] != x[i2 - 1]) {
      *o1 = i1 - 1;
      *o2 = i2 - 1;
      return 0;
    }
  }
  return ORC_E_CANDIDATE;
}

// Full recompute of a walker's state from x (the calc_theta / x_to_Ele_Idx / calculate_MAll /
// sign_PP / calc_amplitude sequence of make_sample.f90:54-60 and :345-350).
static int full_state(const Ctx& c, WState& w, MT& rng) {
  calc_theta(c, w.x.data(), w.th.data());
  if (x_to_ele(c, w.x.data(), w.idx.data(), w.cfg.data())) return ORC_E_CONFIG;
  if (check_ele(c, w.x.data(), w.idx.data(), w.cfg.data())) return ORC_E_CONFIG;
  int e = calc_mall(c, w.idx.data(), w.pf.data(), w.inv.data(), true);
  if (e) return e;
  if (sign_pp(c, w.idx.data(), w.sgn.data())) return ORC_E_SIGN;
  amplitude(c, w.th.data(), w.pf.data(), w.sgn.data(), w.psi_wo.data(), w.psi.data(), rng);
  return 0;
}

// make_initial_x make_sample.f90:298-362
static int make_initial_x(const Ctx& c, WState& w, MT& rng) {
  for (int it1 = 0; it1 < 1000000; it1++) {
    std::fill(w.x.begin(), w.x.end(), -1);
    int i3 = 0;
    bool ok2 = false;
    for (int it2 = 0; it2 < 1000000; it2++) {
      int i = nran(rng, c.N) - 1;
      if (w.x[i] == -1) {
        i3++;
        w.x[i] = 1;
      }
      if (i3 == c.N / 2) {
        ok2 = true;
        break;
      }
    }
    if (!ok2) return ORC_E_INITX;
    int e = full_state(c, w, rng);
    if (e) return e;
    if (std::abs(w.psi[0]) > 1e-300) return 0;
  }
  return ORC_E_INITX;
}

static inline double lround_pos(double v) { return std::floor(v + 0.5); }  // idnint for v >= 0

// make_sample make_sample.f90:4-240 for one emulated rank.
static int make_sample_rank(const Ctx& c, Rank& R, bool first) {
  const int N = c.N;
  MT& rng = R.rng;
  WState w, t;
  w.init(c);
  t.init(c);
  std::vector<double> va(N), vb(N);
  std::vector<int> tidx(N);
  int e;
  for (int k = 0; k < 5; k++) R.ev[k] = 0;
  R.trace.assign((size_t)c.trace_max * 6, 0.0);
  if (first) {
    if ((e = make_initial_x(c, w, rng))) return e;
  } else {
    for (int i = 0; i < N; i++) w.x[i] = R.x_sample[(size_t)N * (c.nsample - 1) + i];
    if ((e = full_state(c, w, rng))) return e;
    if (grnd(rng) < 0.05) {
      R.ev[2]++;
      R.rec(c.trace_max, 3, 0, 0, 0, 0, 0);
      if ((e = make_initial_x(c, w, rng))) return e;
    }
  }
  const int nwarm = std::max(30, c.nsample / 100);
  int naccept = 0, nacc_tmp = 0;
  for (int i0 = -nwarm; i0 <= c.nsample; i0++) {
    if (nacc_tmp > R.nfastup) {  // make_sample.f90:74-128
      std::vector<double> th_old = w.th;
      std::vector<int> sgn_old = w.sgn;
      calc_theta(c, w.x.data(), w.th.data());
      if (check_ele(c, w.x.data(), w.idx.data(), w.cfg.data())) return ORC_E_CONFIG;
      if (sign_pp(c, w.idx.data(), w.sgn.data())) return ORC_E_SIGN;
      for (int j = 0; j < c.Mc; j++)  // make_sample.f90:84-86
        if (std::abs(thc(c, w.th.data(), j) - thc(c, th_old.data(), j)) > 1.0e-5) return ORC_E_THETA;
      for (int j = 0; j < c.Mr; j++)
        if (std::fabs(w.th[j] - th_old[j]) > 1.0e-5) return ORC_E_THETA;
      for (int mp = 0; mp < c.n_mp; mp++)
        if (sgn_old[mp] != w.sgn[mp]) return ORC_E_SIGN;
      std::vector<double> inv_old = w.inv, pf_old = w.pf;
      if ((e = calc_mall(c, w.idx.data(), w.pf.data(), w.inv.data(), true))) return e;
      amplitude(c, w.th.data(), w.pf.data(), w.sgn.data(), w.psi_wo.data(), w.psi.data(), rng);
      double r2 = 0.0;
      for (int qp = 0; qp < c.n_qp; qp++) r2 = r2 + std::fabs(w.pf[qp]);
      r2 = r2 / (double)c.n_qp;
      double diff_pf = -1.0, diff_inv = -1.0;
      for (int qp = 0; qp < c.n_qp; qp++) diff_pf = std::max(diff_pf, std::fabs(pf_old[qp] - w.pf[qp]) / r2);
      for (int qp = 0; qp < c.n_qp; qp++) {
        const double* Mn = &w.inv[(size_t)N * N * qp];
        const double* Mo = &inv_old[(size_t)N * N * qp];
        double r3 = 0.0;
        for (size_t k = 0; k < (size_t)N * N; k++) r3 = std::max(r3, std::fabs(Mn[k]));
        for (size_t k = 0; k < (size_t)N * N; k++) diff_inv = std::max(diff_inv, std::fabs(Mo[k] - Mn[k]) / r3);
      }
      nacc_tmp = 0;
      const int nf0 = R.nfastup;
      (void)grnd(rng);  // make_sample.f90:116 (diagnostic print only)
      if (diff_inv > 1.0e-5 || diff_pf > 1.0e-5) {
        R.nfastup = std::max(1, (int)lround_pos((double)R.nfastup / 1.2));
        if (diff_inv > 10.0 && diff_pf > 10.0) (void)grnd(rng);  // make_sample.f90:122
      } else {
        R.nfastup = std::min(100, (int)lround_pos((double)R.nfastup * 1.1));
      }
      R.ev[3]++;
      R.rec(c.trace_max, 1, i0, diff_inv, diff_pf, nf0, R.nfastup);
    }
    for (int iu = 0; iu < c.nupdate; iu++) {
      if (grnd(rng) < 3.0e-4) {  // global spin flip, make_sample.f90:135-158
        R.ev[0]++;
        for (int i = 0; i < N; i++) t.x[i] = -w.x[i];
        calc_theta(c, t.x.data(), t.th.data());
        if (x_to_ele(c, t.x.data(), t.idx.data(), t.cfg.data())) return ORC_E_CONFIG;
        if (check_ele(c, t.x.data(), t.idx.data(), t.cfg.data())) return ORC_E_CONFIG;
        if ((e = calc_mall(c, t.idx.data(), t.pf.data(), t.inv.data(), true))) return e;
        if (sign_pp(c, t.idx.data(), t.sgn.data())) return ORC_E_SIGN;
        amplitude(c, t.th.data(), t.pf.data(), t.sgn.data(), t.psi_wo.data(), t.psi.data(), rng);
        double r1 = (std::abs(t.psi[0]) + c.shift) / (std::abs(w.psi[0]) + c.shift);
        const double u = grnd(rng);
        R.rec(c.trace_max, 2, 0, 0, r1 * r1, u, u < r1 * r1);
        if (u < r1 * r1) {
          R.ev[1]++;
          (void)grnd(rng);  // make_sample.f90:146
          w.x = t.x;
          w.th = t.th;
          w.idx = t.idx;
          w.cfg = t.cfg;
          w.pf = t.pf;
          w.inv = t.inv;
          w.sgn = t.sgn;
          w.psi = t.psi;
        }
      }
      int i1, i2;
      if ((e = spin_flip_candidate(c, w.x.data(), rng, &i1, &i2))) return e;
      t.th = w.th;
      update_theta(c, w.x.data(), i1, i2, t.th.data());
      int i3 = w.cfg[i1], i4 = w.cfg[i2];
      if (w.idx[i3] != i1 || w.idx[i4] != i2) return ORC_E_CONFIG;
      for (int i = 0; i < N; i++) tidx[i] = w.idx[i];
      tidx[i3] = i2;
      tidx[i4] = i1;
      for (int qp = 0; qp < c.n_qp; qp++)
        t.pf[qp] = new_pf_two_qp(c, qp, i3, i4, tidx.data(), &w.inv[(size_t)N * N * qp], w.pf[qp], va.data(), vb.data());
      for (int mp = 0; mp < c.n_mp; mp++) {
        int s = -w.sgn[mp];
        if (c.subB[i1]) s = -s;
        if (c.subB[i2]) s = -s;
        t.sgn[mp] = s;
      }
      amplitude(c, t.th.data(), t.pf.data(), t.sgn.data(), t.psi_wo.data(), t.psi.data(), rng);
      double r1 = (std::abs(t.psi[0]) + c.shift) / (std::abs(w.psi[0]) + c.shift);
      const double u = grnd(rng);
      R.rec(c.trace_max, 0, i1, i2, r1 * r1, u, u < r1 * r1);
      if (u < r1 * r1) {  // make_sample.f90:203-220
        if (i0 > 0) naccept++;
        nacc_tmp++;
        w.x[i1] = -w.x[i1];
        w.x[i2] = -w.x[i2];
        w.th = t.th;
        w.cfg[i1] = i4;
        w.cfg[i2] = i3;
        w.idx[i3] = i2;
        w.idx[i4] = i1;
        w.pf = t.pf;
        for (int qp = 0; qp < c.n_qp; qp++) new_invm_two_qp(c, qp, i3, i4, w.idx.data(), &w.inv[(size_t)N * N * qp]);
        w.sgn = t.sgn;
        w.psi = t.psi;
      }
    }
    if (i0 > 0) {  // make_sample.f90:228-232
      int s = i0 - 1;
      for (int i = 0; i < N; i++) R.x_sample[(size_t)N * s + i] = w.x[i];
      for (int qp = 0; qp < c.n_qp; qp++) R.pf_sample[(size_t)c.n_qp * s + qp] = w.pf[qp];
      for (int k = 0; k <= c.n_qp; k++) R.psi_sample[(size_t)(c.n_qp + 1) * s + k] = w.psi[k];
    }
  }
  R.naccept = naccept;
  return 0;
}

// ------------------------------------------------------------------------------------------------
// Estimators: bond_map calc_phys_quantity.f90:382-427; calc_local_energy_correlation :306-378;
// calculate_derivative_Pfaffian slater.f90:68-170; calc_phys_quantity_opt :20-246.
// ------------------------------------------------------------------------------------------------
static int bond_map(const Ctx& c, int i0, int i1) {  // i0 in 1..4, i1 0-based -> 0-based
  const int L = c.L;
  int ix = i1 / L, iy = i1 - ix * L;
  if (i0 == 1) {
    ix++;
    if (ix >= L) ix -= L;
  } else if (i0 == 2) {
    iy++;
    if (iy >= L) iy -= L;
  } else if (i0 == 3) {
    ix++;
    if (ix >= L) ix -= L;
    iy++;
    if (iy >= L) iy -= L;
  } else {
    ix++;
    if (ix >= L) ix -= L;
    iy--;
    if (iy < 0) iy += L;
  }
  return ix * L + iy;
}

static cplx local_energy(const Ctx& c, const int* x, cplx psi0, const double* th, const int* idx, const int* cfg,
                         const int* sgn, const double* pf, const double* inv, MT& rng) {
  const int N = c.N;
  std::vector<double> thp(n_theta(c)), tpf(c.n_qp), va(N), vb(N);
  std::vector<int> tidx(N), tsgn(c.n_mp);
  std::vector<cplx> psip(c.n_qp + 1), psipw(c.n_qp);
  cplx E = 0.0;
  for (int i0 = 1; i0 <= 4; i0++) {
    double J = (i0 <= 2) ? c.J1 : c.J2, sg = (i0 <= 2) ? -1.0 : 1.0;
    for (int i1 = 0; i1 < N; i1++) {
      int i2 = bond_map(c, i0, i1);
      E = E + J * (double)x[i1] * (double)x[i2] * psi0;
      if (x[i1] != x[i2]) {
        for (int j = 0; j < n_theta(c); j++) thp[j] = th[j];
        update_theta(c, x, i1, i2, thp.data());
        int i3 = cfg[i1], i4 = cfg[i2];
        for (int i = 0; i < N; i++) tidx[i] = idx[i];
        tidx[i3] = i2;
        tidx[i4] = i1;
        for (int qp = 0; qp < c.n_qp; qp++)
          tpf[qp] = new_pf_two_qp(c, qp, i3, i4, tidx.data(), &inv[(size_t)N * N * qp], pf[qp], va.data(), vb.data());
        for (int mp = 0; mp < c.n_mp; mp++) {
          int s = -sgn[mp];
          if (c.subB[i1]) s = -s;
          if (c.subB[i2]) s = -s;
          tsgn[mp] = s;
        }
        amplitude(c, thp.data(), tpf.data(), tsgn.data(), psipw.data(), psip.data(), rng);
        E = E + 2.0 * J * sg * psip[0];
      }
    }
  }
  return E;
}

// deriv(orbidx, qp) scatter of slater.f90:94-170
static void deriv_pfaffian(const Ctx& c, const int* idx, const double* pf, const double* inv, double* deriv) {
  const int N = c.N, Np = c.Npair;
  std::fill(deriv, deriv + (size_t)c.n_slater * c.n_qp, 0.0);
  std::vector<int> toi((size_t)N * N), tos((size_t)N * N);
  for (int mp = 0; mp < c.n_mp; mp++) {
    for (int msj = 0; msj < N; msj++) {
      int trj = c.W_map[idx[msj] + N * mp];
      for (int msi = 0; msi < N; msi++) {
        int tri = c.W_map[idx[msi] + N * mp];
        toi[msi + (size_t)N * msj] = c.orb_idx[tri + N * trj];
        tos[msi + (size_t)N * msj] = c.orb_sgn[tri + N * trj];
      }
    }
    for (int sp = 0; sp < 2; sp++) {
      int qp = 2 * mp + sp;
      double* d = deriv + (size_t)c.n_slater * qp;
      const double* M = inv + (size_t)N * N * qp;
      double cs = pf[qp] * c.sp_cs[sp], cc = pf[qp] * c.sp_cc[sp], ss = pf[qp] * c.sp_ss[sp];
      for (int msj = 0; msj < Np; msj++)
        for (int msi = 0; msi < Np; msi++) {
          size_t k;
          k = msi + (size_t)N * msj;
          d[toi[k]] = d[toi[k]] - M[k] * cs * tos[k];
          k = msi + (size_t)N * (msj + Np);
          d[toi[k]] = d[toi[k]] + M[k] * cc * tos[k];
          k = (msi + Np) + (size_t)N * msj;
          d[toi[k]] = d[toi[k]] - M[k] * ss * tos[k];
          k = (msi + Np) + (size_t)N * (msj + Np);
          d[toi[k]] = d[toi[k]] + M[k] * cs * tos[k];
        }
    }
  }
}

// Raw per-configuration quantities: psi(0..N_QP), Hpsi (= Eloc_x before reweighting) and the raw
// derivative d psi / d theta_k (Ovec_loc_x before reweighting), calc_phys_quantity.f90:74-220.
static int eval_config(const Ctx& c, const int* x, MT& rng, cplx* psi_out, cplx* hpsi, cplx* Oraw,
                       std::vector<double>* pf_out = nullptr) {
  const int N = c.N;
  std::vector<double> th(n_theta(c)), pf(c.n_qp), inv((size_t)N * N * c.n_qp), deriv((size_t)c.n_slater * c.n_qp);
  std::vector<int> idx(N), cfg(N), sgn(c.n_mp);
  std::vector<cplx> psi(c.n_qp + 1), psiw(c.n_qp);
  calc_theta(c, x, th.data());
  if (x_to_ele(c, x, idx.data(), cfg.data())) return ORC_E_CONFIG;
  int e = calc_mall(c, idx.data(), pf.data(), inv.data(), true);
  if (e) return e;
  if (sign_pp(c, idx.data(), sgn.data())) return ORC_E_SIGN;
  amplitude(c, th.data(), pf.data(), sgn.data(), psiw.data(), psi.data(), rng);
  if (psi_out)
    for (int k = 0; k <= c.n_qp; k++) psi_out[k] = psi[k];
  if (pf_out) *pf_out = pf;
  if (hpsi) *hpsi = local_energy(c, x, psi[0], th.data(), idx.data(), cfg.data(), sgn.data(), pf.data(), inv.data(), rng);
  if (Oraw) {
    for (int k = 0; k < c.Nv; k++) Oraw[k] = 0.0;
    // complex RBM branch, calc_phys_quantity.f90:115-160: (re, im) parameter pairs, the imaginary partner
    // derivative being i times the real one; tanh(t) of a complex t as (tanh a + i tan b) / (1 + i tanh a tan b)
    auto ctanh = [](cplx t) {
      return cplx(std::tanh(t.real()), std::tan(t.imag())) / cplx(1.0, std::tanh(t.real()) * std::tan(t.imag()));
    };
    const cplx ci(0.0, 1.0);
    for (int f = 0; f < c.alphac; f++) {
      int k1 = 2 * f, itmp = 0;
      for (int mp = 0; mp < c.n_mp; mp++)
        for (int s = 1; s >= -1; s -= 2) {
          int j = itmp * c.alphac + f;
          itmp++;
          Oraw[k1] = Oraw[k1] + ctanh(thc(c, th.data(), j)) * psi[itmp];
        }
      Oraw[k1 + 1] = Oraw[k1] * ci;
    }
    for (int f = 0; f < c.alphac; f++) {
      int off = 2 * c.alphac + f * N * 2, itmp = 0;
      for (int mp = 0; mp < c.n_mp; mp++)
        for (int s = 1; s >= -1; s -= 2) {
          int j = itmp * c.alphac + f;
          itmp++;
          cplx c1 = ctanh(thc(c, th.data(), j)) * psi[itmp];
          for (int i = 0; i < N; i++) {
            int k1 = off + 2 * c.W_map[i + N * mp];
            Oraw[k1] = Oraw[k1] + c1 * (double)x[i] * (double)s;
            if (mp == c.n_mp - 1) Oraw[k1 + 1] = Oraw[k1] * ci;
          }
        }
    }
    // real RBM branch, calc_phys_quantity.f90:165-201
    const int offr = 2 * c.alphac * (N + 1);
    for (int f = 0; f < c.alphar; f++) {
      int k1 = offr + f, itmp = 0;
      for (int mp = 0; mp < c.n_mp; mp++)
        for (int s = 1; s >= -1; s -= 2) {
          int j = itmp * c.alphar + f;
          itmp++;
          Oraw[k1] = Oraw[k1] + std::tanh(th[j]) * psi[itmp];
        }
    }
    for (int f = 0; f < c.alphar; f++) {
      int off = offr + c.alphar + f * N, itmp = 0;
      for (int mp = 0; mp < c.n_mp; mp++)
        for (int s = 1; s >= -1; s -= 2) {
          int j = itmp * c.alphar + f;
          itmp++;
          cplx c1 = std::tanh(th[j]) * psi[itmp];
          for (int i = 0; i < N; i++) {
            int iw = c.W_map[i + N * mp];
            Oraw[off + iw] = Oraw[off + iw] + c1 * (double)x[i] * (double)s;
          }
        }
    }
    deriv_pfaffian(c, idx.data(), pf.data(), inv.data(), deriv.data());
    int off = offr + c.alphar * (N + 1);
    for (int o = 0; o < c.n_slater; o++) {
      cplx acc = Oraw[off + o];
      for (int qp = 0; qp < c.n_qp; qp++) acc = acc + deriv[o + (size_t)c.n_slater * qp] * psiw[qp];
      Oraw[off + o] = acc;
    }
  }
  return 0;
}

// ------------------------------------------------------------------------------------------------
// Dense Cholesky solve (upper, the role of pdposv('U') / dposv('U'), SR_pdposv.f90:232, SR.f90:123)
// ------------------------------------------------------------------------------------------------
static int chol_solve_upper(int n, std::vector<double>& A, std::vector<double>& b) {
  // A = U^T U using the upper triangle of A (column-major); b overwritten by the solution.
  for (int j = 0; j < n; j++) {
    for (int i = 0; i <= j; i++) {
      double s = A[i + (size_t)n * j];
      for (int k = 0; k < i; k++) s -= A[k + (size_t)n * i] * A[k + (size_t)n * j];
      if (i == j) {
        if (!(s > 0.0)) return ORC_E_CHOL;
        A[j + (size_t)n * j] = std::sqrt(s);
      } else {
        A[i + (size_t)n * j] = s / A[i + (size_t)n * i];
      }
    }
  }
  for (int i = 0; i < n; i++) {  // U^T y = b
    double s = b[i];
    for (int k = 0; k < i; k++) s -= A[k + (size_t)n * i] * b[k];
    b[i] = s / A[i + (size_t)n * i];
  }
  for (int i = n - 1; i >= 0; i--) {  // U x = y
    double s = b[i];
    for (int k = i + 1; k < n; k++) s -= A[i + (size_t)n * k] * b[k];
    b[i] = s / A[i + (size_t)n * i];
  }
  return 0;
}

// ================================================================================================
// C API (ctypes)
// ================================================================================================
extern "C" {

struct orc_sr_in {
  int iteration;
  double delta_tau, s_factor0, s_cut;
  double Etot, Etot2;  // already divided by norm (main.f90:357-361)
};
struct orc_sr_out {
  double lambda, lambda_rbm_rbm, lambda_pp_pp, lambda_rbm_pp;
  double delW_max, s_factor, sdiag_av, smat_scaling;
  int kmax, k_nonzero, nSmat;
};

void* orc_create(int L, int n_mp, int alphac, int alphar, int n_slater, int nsample_per_rank, int nranks,
                 int spin_parity, double J1, double J2) {
  if (L < 2 || n_mp < 1 || alphac < 0 || alphar < 0 || n_slater < 1 || nsample_per_rank < 1 || nranks < 1)
    return nullptr;
  Ctx* c = new Ctx();
  c->L = L;
  c->N = L * L;
  if (c->N % 2) {
    delete c;
    return nullptr;
  }
  c->Npair = c->N / 2;
  c->n_mp = n_mp;
  c->alphac = alphac;
  c->alphar = alphar;
  c->n_slater = n_slater;
  c->n_qp = 2 * n_mp;
  c->Mr = alphar * n_mp * 2;                                   // main.f90:135
  c->Mc = alphac * n_mp * 2;                                   // main.f90:134
  c->Nv = alphac * 2 * (c->N + 1) + alphar * (c->N + 1) + n_slater;  // main.f90:136
  c->Nv_rbm = c->Nv - n_slater;
  c->nsample = nsample_per_rank;
  c->nranks = nranks;
  c->nupdate = c->N;  // main.f90:139
  c->spin_parity = spin_parity;
  c->J1 = J1;
  c->J2 = J2;
  c->shift = 0.0;
  c->err = 0;
  c->msg[0] = 0;
  init_sp_weight(*c);
  define_sublattice(*c);
  c->ranks.resize(nranks);
  for (auto& r : c->ranks) {
    r.nfastup = std::min(100, c->N * 2);  // main.f90:309
    r.naccept = 0;
    r.err = 0;
    r.x_sample.assign((size_t)c->N * c->nsample, 0);
    r.psi_sample.assign((size_t)(c->n_qp + 1) * c->nsample, 0.0);
    r.pf_sample.assign((size_t)c->n_qp * c->nsample, 0.0);
    mt_seed(r.rng, 4357);
  }
  c->Wr.assign((size_t)c->N * alphar, 0.0);
  c->br.assign(alphar, 0.0);
  c->Wc.assign((size_t)c->N * alphac, 0.0);
  c->bc.assign(alphac, 0.0);
  c->slater.assign(n_slater, 0.0);
  return c;
}

void orc_destroy(void* h) { delete (Ctx*)h; }
const char* orc_errmsg(void* h) { return ((Ctx*)h)->msg; }
int orc_nv(void* h) { return ((Ctx*)h)->Nv; }

// W_map(N, n_mp) with 1-based values (sym_info.txt), para_mp (re,im) pairs, Orbital_Idx(N,N) 1-based,
// Orbital_Sgn(N,N) or NULL (all +1; l_AP = .false. in parameter.f90:80).
int orc_set_tables(void* h, const int* W_map, const double* para_mp, const int* orb_idx, const int* orb_sgn) {
  Ctx& c = *(Ctx*)h;
  const int N = c.N;
  c.W_map.resize((size_t)N * c.n_mp);
  for (size_t k = 0; k < c.W_map.size(); k++) {
    if (W_map[k] < 1 || W_map[k] > N) return set_err(c, ORC_E_ARG, "W_map out of range");
    c.W_map[k] = W_map[k] - 1;
  }
  c.para_mp.resize(c.n_mp);
  for (int mp = 0; mp < c.n_mp; mp++) c.para_mp[mp] = cplx(para_mp[2 * mp], para_mp[2 * mp + 1]);
  c.orb_idx.resize((size_t)N * N);
  c.orb_sgn.assign((size_t)N * N, 1);
  for (size_t k = 0; k < c.orb_idx.size(); k++) {
    if (orb_idx[k] < 1 || orb_idx[k] > c.n_slater) return set_err(c, ORC_E_ARG, "Orbital_Idx out of range");
    c.orb_idx[k] = orb_idx[k] - 1;
    if (orb_sgn) c.orb_sgn[k] = orb_sgn[k];
  }
  return 0;
}

int orc_set_params(void* h, const double* Wr, const double* br, const double* slater, double shift) {
  Ctx& c = *(Ctx*)h;
  if (Wr) std::memcpy(c.Wr.data(), Wr, sizeof(double) * c.Wr.size());
  if (br) std::memcpy(c.br.data(), br, sizeof(double) * c.br.size());
  if (slater) std::memcpy(c.slater.data(), slater, sizeof(double) * c.slater.size());
  c.shift = shift;
  if (c.W_map.empty()) return set_err(c, ORC_E_ARG, "tables not set");
  return update_slater_elements(c);
}

// InitSPWeight with given weights w(3, 2) = {SP_GL_Cos, SP_GL_Sin, para_spin_proj} of the two points, as the
// transverse code's spin_projection.f90:30-38 sets them (beta = -pi/2, pi/2, sqrt(2)-scaled); the
// CosCos/CosSin/SinSin products follow spin_projection.f90:39-41.  Rebuilds Slater_Elm when parameters are set.
int orc_set_sp_weights(void* h, const double* w) {
  Ctx& c = *(Ctx*)h;
  for (int s = 0; s < 2; s++) {
    c.sp_cos[s] = w[3 * s];
    c.sp_sin[s] = w[3 * s + 1];
    c.para_sp[s] = w[3 * s + 2];
    c.sp_cc[s] = c.sp_cos[s] * c.sp_cos[s];
    c.sp_cs[s] = c.sp_cos[s] * c.sp_sin[s];
    c.sp_ss[s] = c.sp_sin[s] * c.sp_sin[s];
  }
  if (!c.slater.empty() && !c.W_map.empty()) return update_slater_elements(c);
  return 0;
}

// Complex RBM parameters Wcirr(N, alphac), bcirr(alphac) as (re, im) pairs (module.f90 mod_RBM).
int orc_set_params_c(void* h, const double* Wc, const double* bc) {
  Ctx& c = *(Ctx*)h;
  for (size_t k = 0; k < c.Wc.size(); k++) c.Wc[k] = cplx(Wc[2 * k], Wc[2 * k + 1]);
  for (size_t k = 0; k < c.bc.size(); k++) c.bc[k] = cplx(bc[2 * k], bc[2 * k + 1]);
  return 0;
}

int orc_get_params_c(void* h, double* Wc, double* bc) {
  Ctx& c = *(Ctx*)h;
  for (size_t k = 0; k < c.Wc.size(); k++) {
    Wc[2 * k] = c.Wc[k].real();
    Wc[2 * k + 1] = c.Wc[k].imag();
  }
  for (size_t k = 0; k < c.bc.size(); k++) {
    bc[2 * k] = c.bc[k].real();
    bc[2 * k + 1] = c.bc[k].imag();
  }
  return 0;
}

int orc_get_params(void* h, double* Wr, double* br, double* slater, double* shift) {
  Ctx& c = *(Ctx*)h;
  if (Wr) std::memcpy(Wr, c.Wr.data(), sizeof(double) * c.Wr.size());
  if (br) std::memcpy(br, c.br.data(), sizeof(double) * c.br.size());
  if (slater) std::memcpy(slater, c.slater.data(), sizeof(double) * c.slater.size());
  if (shift) *shift = c.shift;
  return 0;
}

int orc_get_slater_elements(void* h, double* out) {
  Ctx& c = *(Ctx*)h;
  std::memcpy(out, c.SE.data(), sizeof(double) * c.SE.size());
  return 0;
}

// main.f90:224-234: every rank seeds sgrnd(iseed0 + rank) and skips Nsample_rank*rank + 1 draws.
// Local rank r is global rank offset + r (the context holds one shard of the ranks).
int orc_seed_offset(void* h, int iseed0, int offset) {
  Ctx& c = *(Ctx*)h;
  c.rank0 = offset;
  for (int r = 0; r < c.nranks; r++) {
    const int g = offset + r;
    mt_seed(c.ranks[r].rng, (int32_t)(iseed0 + g));
    long long skip = (long long)c.nsample * g + 1;
    for (long long i = 0; i < skip; i++) (void)grnd(c.ranks[r].rng);
  }
  return 0;
}

int orc_seed(void* h, int iseed0) { return orc_seed_offset(h, iseed0, 0); }

int orc_rank_grnd(void* h, int rank, int n, double* out) {
  Ctx& c = *(Ctx*)h;
  if (rank < 0 || rank >= c.nranks) return ORC_E_ARG;
  for (int i = 0; i < n; i++) {
    double u = grnd(c.ranks[rank].rng);
    if (out) out[i] = u;
  }
  return 0;
}

int orc_get_rng_state(void* h, int rank, uint32_t* mt, int* mti) {
  Ctx& c = *(Ctx*)h;
  std::memcpy(mt, c.ranks[rank].rng.mt, sizeof(uint32_t) * 624);
  *mti = c.ranks[rank].rng.mti;
  return 0;
}

int orc_get_nfastup(void* h, int* out) {
  Ctx& c = *(Ctx*)h;
  for (int r = 0; r < c.nranks; r++) out[r] = c.ranks[r].nfastup;
  return 0;
}

int orc_make_sample(void* h, int first, int* naccept, int nthreads) {
  Ctx& c = *(Ctx*)h;
  std::vector<int> errs(c.nranks, 0);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
  for (int r = 0; r < c.nranks; r++) errs[r] = make_sample_rank(c, c.ranks[r], first != 0);
  for (int r = 0; r < c.nranks; r++) {
    if (errs[r]) {
      char m[128];
      snprintf(m, sizeof(m), "make_sample failed on rank %d (code %d)", r, errs[r]);
      return set_err(c, errs[r], m);
    }
    if (naccept) naccept[r] = c.ranks[r].naccept;
  }
  return 0;
}

// x (N, Nsample, nranks) int; psi ((N_QP+1) complex, Nsample, nranks) as (re,im); pf (N_QP, Nsample, nranks)
int orc_set_trace(void* h, int max_records) {
  ((Ctx*)h)->trace_max = max_records < 0 ? 0 : max_records;
  return 0;
}

// events (5, nranks) and, when a trace is kept, the trace (6, trace_max, nranks) of the last make_sample
int orc_get_events(void* h, int* events, double* trace) {
  Ctx& c = *(Ctx*)h;
  for (int r = 0; r < c.nranks; r++) {
    const Rank& R = c.ranks[r];
    if (events)
      for (int k = 0; k < 5; k++) events[5 * r + k] = R.ev[k];
    if (trace && c.trace_max > 0)
      for (size_t k = 0; k < (size_t)c.trace_max * 6; k++)
        trace[(size_t)r * c.trace_max * 6 + k] = k < R.trace.size() ? R.trace[k] : 0.0;
  }
  return 0;
}

int orc_get_samples(void* h, int* x, double* psi, double* pf) {
  Ctx& c = *(Ctx*)h;
  for (int r = 0; r < c.nranks; r++) {
    Rank& R = c.ranks[r];
    if (x) std::memcpy(x + (size_t)c.N * c.nsample * r, R.x_sample.data(), sizeof(int) * R.x_sample.size());
    if (pf) std::memcpy(pf + (size_t)c.n_qp * c.nsample * r, R.pf_sample.data(), sizeof(double) * R.pf_sample.size());
    if (psi)
      std::memcpy(psi + (size_t)2 * (c.n_qp + 1) * c.nsample * r, R.psi_sample.data(), sizeof(cplx) * R.psi_sample.size());
  }
  return 0;
}

int orc_set_samples(void* h, const int* x) {
  Ctx& c = *(Ctx*)h;
  for (int r = 0; r < c.nranks; r++)
    std::memcpy(c.ranks[r].x_sample.data(), x + (size_t)c.N * c.nsample * r, sizeof(int) * c.ranks[r].x_sample.size());
  return 0;
}

// calc_phys_quantity_opt (calc_phys_quantity.f90:20-246) over all ranks, summed in rank order like
// the MPI reductions of main.f90:348-369 (before the division by norm).
//   scal[0..3] = Etot, Etot2, norm, wf_av (sums);  gvec, Ovec (Nv sums);  Smat (Nv*Nv, optional)
//   Ostore (optional): Nv x (2*Nsample*nranks) column-major, the Ovec_Store columns of every rank.
//   eloc_out (optional): complex reweighted Eloc_x per stored sample (rank-major order).
int orc_measure(void* h, double* scal, double* gvec, double* Ovec, double* Smat, double* Ostore, double* eloc_out,
                int nthreads) {
  Ctx& c = *(Ctx*)h;
  const int Nv = c.Nv, Ns = c.nsample;
  const size_t ncols = (size_t)2 * Ns * c.nranks;
  std::vector<double> O;
  bool keepO = (Smat != nullptr) || (Ostore != nullptr);
  if (keepO) O.assign((size_t)Nv * ncols, 0.0);
  std::vector<double> rE(c.nranks, 0), rE2(c.nranks, 0), rN(c.nranks, 0), rW(c.nranks, 0);
  std::vector<double> rg((size_t)Nv * c.nranks, 0), rO((size_t)Nv * c.nranks, 0);
  std::vector<int> errs(c.nranks, 0);
  std::vector<cplx> elocs((size_t)Ns * c.nranks);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
  for (int r = 0; r < c.nranks; r++) {
    Rank& R = c.ranks[r];
    std::vector<cplx> psi(c.n_qp + 1), Oloc(Nv);
    double Etot = 0, Etot2 = 0, norm = 0, wf = 0;
    double* g = &rg[(size_t)Nv * r];
    double* ov = &rO[(size_t)Nv * r];
    for (int s = 0; s < Ns && !errs[r]; s++) {
      const int* x = &R.x_sample[(size_t)c.N * s];
      cplx E;
      int e = eval_config(c, x, R.rng, psi.data(), &E, Oloc.data());
      if (e) {
        errs[r] = e;
        break;
      }
      double w = 1.0 / (std::abs(psi[0]) + c.shift);
      E = E * w;
      elocs[(size_t)Ns * r + s] = E;
      Etot = Etot + w * std::real(std::conj(psi[0]) * E);
      Etot2 = Etot2 + std::real(std::conj(E) * E);
      norm = norm + (std::abs(psi[0]) * w) * (std::abs(psi[0]) * w);
      wf = wf + std::abs(psi[0]);
      for (int k = 0; k < Nv; k++) {
        cplx o = Oloc[k] * w;
        g[k] = std::real(g[k] + 2.0 * std::conj(E) * o);
        ov[k] = ov[k] + w * std::real(std::conj(psi[0]) * o);
        if (keepO) {
          size_t col = (size_t)2 * Ns * r + 2 * s;
          O[k + (size_t)Nv * col] = std::real(o);
          O[k + (size_t)Nv * (col + 1)] = std::imag(o);
        }
      }
    }
    rE[r] = Etot;
    rE2[r] = Etot2;
    rN[r] = norm;
    rW[r] = wf;
  }
  for (int r = 0; r < c.nranks; r++)
    if (errs[r]) return set_err(c, errs[r], "calc_phys_quantity_opt failed");
  double E = 0, E2 = 0, nn = 0, wf = 0;
  for (int r = 0; r < c.nranks; r++) {
    E += rE[r];
    E2 += rE2[r];
    nn += rN[r];
    wf += rW[r];
  }
  scal[0] = E;
  scal[1] = E2;
  scal[2] = nn;
  scal[3] = wf;
  for (int k = 0; k < Nv; k++) {
    double a = 0, b = 0;
    for (int r = 0; r < c.nranks; r++) {
      a += rg[(size_t)Nv * r + k];
      b += rO[(size_t)Nv * r + k];
    }
    if (gvec) gvec[k] = a;
    if (Ovec) Ovec[k] = b;
  }
  if (eloc_out)
    for (size_t i = 0; i < elocs.size(); i++) {
      eloc_out[2 * i] = elocs[i].real();
      eloc_out[2 * i + 1] = elocs[i].imag();
    }
  if (Ostore) std::memcpy(Ostore, O.data(), sizeof(double) * O.size());
  if (Smat) {  // dgemm('N','T',Nv,Nv,2*Nsample) summed over ranks: calc_phys_quantity.f90:240
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads > 0 ? nthreads : 1)
    for (int k2 = 0; k2 < Nv; k2++)
      for (int k1 = 0; k1 <= k2; k1++) {
        double s = 0.0;
        for (size_t col = 0; col < ncols; col++) s += O[k1 + (size_t)Nv * col] * O[k2 + (size_t)Nv * col];
        Smat[k1 + (size_t)Nv * k2] = s;
        Smat[k2 + (size_t)Nv * k1] = s;
      }
  }
  return 0;
}

// calc_phys_quantity_after_opt (calc_phys_quantity.f90:250-302): scal = Etot, Etot2, norm, wf_av sums
int orc_measure_energy(void* h, double* scal, int nthreads) {
  Ctx& c = *(Ctx*)h;
  std::vector<double> rE(c.nranks, 0), rE2(c.nranks, 0), rN(c.nranks, 0), rW(c.nranks, 0);
  std::vector<int> errs(c.nranks, 0);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
  for (int r = 0; r < c.nranks; r++) {
    std::vector<cplx> psi(c.n_qp + 1);
    for (int s = 0; s < c.nsample; s++) {
      cplx E;
      int e = eval_config(c, &c.ranks[r].x_sample[(size_t)c.N * s], c.ranks[r].rng, psi.data(), &E, nullptr);
      if (e) {
        errs[r] = e;
        break;
      }
      double w = 1.0 / (std::abs(psi[0]) + c.shift);
      E = E * w;
      rE[r] += w * std::real(std::conj(psi[0]) * E);
      rE2[r] += std::real(std::conj(E) * E);
      rN[r] += (std::abs(psi[0]) * w) * (std::abs(psi[0]) * w);
      rW[r] += std::abs(psi[0]);
    }
  }
  for (int r = 0; r < c.nranks; r++)
    if (errs[r]) return set_err(c, errs[r], "calc_phys_quantity_after_opt failed");
  scal[0] = scal[1] = scal[2] = scal[3] = 0;
  for (int r = 0; r < c.nranks; r++) {
    scal[0] += rE[r];
    scal[1] += rE2[r];
    scal[2] += rN[r];
    scal[3] += rW[r];
  }
  return 0;
}

// ------------------------------------------------------------------------------------------------
// Correlation measurement of the Calc_Correlation program (Calc_Correlation/calc_phys_quantity.f90):
// calc_local_energy_correlation :348-424 (local energy and SdotS per bond), calc_local_correlation
// :477-550 (SzSz and exchange parts for every site pair i1 <= i2) and their accumulation in
// calc_phys_quantity_after_opt :264-344.  Pair index i0 = i2 (i2 - 1) / 2 + i1 (1-based, i1 <= i2).
// Every exchanged amplitude consumes one draw (sub.f90:72), in the reference's loop order.
// ------------------------------------------------------------------------------------------------
struct ExchangeBuf {
  std::vector<double> thp, tpf, va, vb;
  std::vector<int> tidx, tsgn;
  std::vector<cplx> psip, psipw;
  explicit ExchangeBuf(const Ctx& c)
      : thp(n_theta(c)), tpf(c.n_qp), va(c.N), vb(c.N), tidx(c.N), tsgn(c.n_mp), psip(c.n_qp + 1), psipw(c.n_qp) {}
};

// psi(x') for the exchange of the antiparallel spins on sites i1, i2 (0-based), as in
// calc_local_correlation :507-533.
static cplx exchange_psi(const Ctx& c, const int* x, const double* th, const int* idx, const int* cfg,
                         const int* sgn, const double* pf, const double* inv, MT& rng, int i1, int i2, ExchangeBuf& b) {
  const int N = c.N;
  for (int j = 0; j < n_theta(c); j++) b.thp[j] = th[j];
  update_theta(c, x, i1, i2, b.thp.data());
  const int i3 = cfg[i1], i4 = cfg[i2];
  for (int i = 0; i < N; i++) b.tidx[i] = idx[i];
  b.tidx[i3] = i2;
  b.tidx[i4] = i1;
  for (int qp = 0; qp < c.n_qp; qp++)
    b.tpf[qp] = new_pf_two_qp(c, qp, i3, i4, b.tidx.data(), &inv[(size_t)N * N * qp], pf[qp], b.va.data(), b.vb.data());
  for (int mp = 0; mp < c.n_mp; mp++) {
    int s = -sgn[mp];
    if (c.subB[i1]) s = -s;
    if (c.subB[i2]) s = -s;
    b.tsgn[mp] = s;
  }
  amplitude(c, b.thp.data(), b.tpf.data(), b.tsgn.data(), b.psipw.data(), b.psip.data(), rng);
  return b.psip[0];
}

// One stored sample: psi(0), Eloc_x (before reweighting), SdotS(N, 4) (before reweighting) and
// Chi_loc_x(2, Nchi).
static int corr_sample(const Ctx& c, const int* x, MT& rng, cplx& psi0, cplx& eloc, cplx* sdots, cplx* chi) {
  const int N = c.N;
  std::vector<double> th(n_theta(c)), pf(c.n_qp), inv((size_t)N * N * c.n_qp);
  std::vector<int> idx(N), cfg(N), sgn(c.n_mp);
  std::vector<cplx> psi(c.n_qp + 1), psiw(c.n_qp);
  ExchangeBuf b(c);
  calc_theta(c, x, th.data());
  if (x_to_ele(c, x, idx.data(), cfg.data())) return ORC_E_CONFIG;
  int e = calc_mall(c, idx.data(), pf.data(), inv.data(), true);
  if (e) return e;
  if (sign_pp(c, idx.data(), sgn.data())) return ORC_E_SIGN;
  amplitude(c, th.data(), pf.data(), sgn.data(), psiw.data(), psi.data(), rng);
  psi0 = psi[0];
  // calc_local_energy_correlation :364-421
  eloc = 0.0;
  for (int k = 0; k < 4 * N; k++) sdots[k] = 0.0;
  for (int i0 = 1; i0 <= 4; i0++) {
    const double J = (i0 <= 2) ? c.J1 : c.J2, sg = (i0 <= 2) ? -1.0 : 1.0;
    for (int i1 = 0; i1 < N; i1++) {
      const int i2 = bond_map(c, i0, i1);
      cplx& sd = sdots[i1 + (size_t)N * (i0 - 1)];
      eloc = eloc + J * (double)x[i1] * (double)x[i2] * psi0;
      sd = sd + (double)x[i1] * (double)x[i2] * psi0;
      if (x[i1] != x[i2]) {
        const cplx pp = exchange_psi(c, x, th.data(), idx.data(), cfg.data(), sgn.data(), pf.data(), inv.data(), rng,
                                     i1, i2, b);
        eloc = eloc + 2.0 * J * sg * pp;
        sd = sd + 2.0 * sg * pp;
      }
    }
  }
  // calc_local_correlation :495-547
  size_t i0 = 0;
  for (int i2 = 0; i2 < N; i2++)
    for (int i1 = 0; i1 <= i2; i1++, i0++) {
      chi[2 * i0] = (double)x[i1] * (double)x[i2] * psi0;
      chi[2 * i0 + 1] = (i1 == i2) ? psi0 : cplx(0.0);
      if (x[i1] != x[i2]) {
        const cplx pp = exchange_psi(c, x, th.data(), idx.data(), cfg.data(), sgn.data(), pf.data(), inv.data(), rng,
                                     i1, i2, b);
        double sgs = 1.0;
        if (c.subB[i1]) sgs = -sgs;
        if (c.subB[i2]) sgs = -sgs;
        chi[2 * i0 + 1] = sgs * pp;
      }
    }
  return 0;
}

// calc_phys_quantity_after_opt of the Calc_Correlation program (:264-344) over all ranks, summed in rank
// order like the MPI_REDUCE calls of Calc_Correlation/main.f90:553-581 (before the division by norm):
// scal = Etot, Etot2, norm, wf_av, Re wf_sgn; chi_sp = Chi_sp(2, Nchi); chi_vbs = Chi_vbs(Nchi, 4)
// (Fortran column-major).
int orc_measure_correlation(void* h, double* scal, double* chi_sp, double* chi_vbs, int nthreads) {
  Ctx& c = *(Ctx*)h;
  const int N = c.N;
  const size_t nchi = (size_t)N * (N + 1) / 2;
  std::vector<double> rs((size_t)c.nranks * 5, 0.0), rsp((size_t)c.nranks * 2 * nchi, 0.0),
      rvb((size_t)c.nranks * 4 * nchi, 0.0);
  std::vector<int> errs(c.nranks, 0);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
  for (int r = 0; r < c.nranks; r++) {
    std::vector<cplx> sd((size_t)4 * N), chi(2 * nchi);
    double* S = &rs[(size_t)5 * r];
    double* sp = &rsp[(size_t)2 * nchi * r];
    double* vb = &rvb[(size_t)4 * nchi * r];
    for (int s = 0; s < c.nsample; s++) {
      cplx psi0, E;
      int e = corr_sample(c, &c.ranks[r].x_sample[(size_t)N * s], c.ranks[r].rng, psi0, E, sd.data(), chi.data());
      if (e) {
        errs[r] = e;
        break;
      }
      const double w = 1.0 / (std::abs(psi0) + c.shift);
      E = E * w;
      S[0] += w * std::real(std::conj(psi0) * E);
      S[1] += std::real(std::conj(E) * E);
      S[2] += (std::abs(psi0) * w) * (std::abs(psi0) * w);
      S[3] += std::abs(psi0);
      S[4] += std::real(psi0 / std::abs(psi0));
      for (auto& v : sd) v = v * w;
      for (int i3 = 0; i3 < 4; i3++) {
        size_t i0 = 0;
        for (int i2 = 0; i2 < N; i2++)
          for (int i1 = 0; i1 <= i2; i1++, i0++)
            vb[i0 + nchi * i3] += std::real(std::conj(sd[i1 + (size_t)N * i3]) * sd[i2 + (size_t)N * i3]);
      }
      for (size_t k = 0; k < 2 * nchi; k++) sp[k] += w * w * std::real(std::conj(psi0) * chi[k]);
    }
  }
  for (int r = 0; r < c.nranks; r++)
    if (errs[r]) return set_err(c, errs[r], "calc_phys_quantity_after_opt (correlation) failed");
  for (int k = 0; k < 5; k++) scal[k] = 0.0;
  for (size_t k = 0; k < 2 * nchi; k++) chi_sp[k] = 0.0;
  for (size_t k = 0; k < 4 * nchi; k++) chi_vbs[k] = 0.0;
  for (int r = 0; r < c.nranks; r++) {
    for (int k = 0; k < 5; k++) scal[k] += rs[(size_t)5 * r + k];
    for (size_t k = 0; k < 2 * nchi; k++) chi_sp[k] += rsp[(size_t)2 * nchi * r + k];
    for (size_t k = 0; k < 4 * nchi; k++) chi_vbs[k] += rvb[(size_t)4 * nchi * r + k];
  }
  return 0;
}

// Per-configuration evaluation for tests: psi (N_QP+1 complex), raw H psi (complex), raw dpsi/dtheta
// (Nv complex).  Uses a private RNG (the amplitude draws do not affect values).
int orc_eval_configs(void* h, int n, const int* x, double* psi, double* hpsi, double* Oraw, double* pf) {
  Ctx& c = *(Ctx*)h;
  MT rng;
  mt_seed(rng, 1);
  std::vector<cplx> ps(c.n_qp + 1), O(c.Nv);
  std::vector<double> pfv;
  for (int s = 0; s < n; s++) {
    cplx E;
    int e = eval_config(c, x + (size_t)c.N * s, rng, ps.data(), hpsi ? &E : nullptr, Oraw ? O.data() : nullptr, &pfv);
    if (e) return set_err(c, e, "eval_config failed");
    if (psi) std::memcpy(psi + (size_t)2 * (c.n_qp + 1) * s, ps.data(), sizeof(cplx) * (c.n_qp + 1));
    if (hpsi) {
      hpsi[2 * s] = E.real();
      hpsi[2 * s + 1] = E.imag();
    }
    if (Oraw) std::memcpy(Oraw + (size_t)2 * c.Nv * s, O.data(), sizeof(cplx) * c.Nv);
    if (pf) std::memcpy(pf + (size_t)c.n_qp * s, pfv.data(), sizeof(double) * c.n_qp);
  }
  return 0;
}

// Fast-update ratio for one proposal on a configuration (for kernel-level parity tests):
// returns Pf_new(qp) for exchanging the electrons on sites i1, i2 (0-based, x(i1) /= x(i2)).
int orc_proposal_pf(void* h, const int* x, int i1, int i2, double* pf_old, double* pf_new) {
  Ctx& c = *(Ctx*)h;
  const int N = c.N;
  std::vector<int> idx(N), cfg(N), tidx(N);
  std::vector<double> inv((size_t)N * N * c.n_qp), va(N), vb(N);
  if (x_to_ele(c, x, idx.data(), cfg.data())) return ORC_E_CONFIG;
  int e = calc_mall(c, idx.data(), pf_old, inv.data(), true);
  if (e) return e;
  int i3 = cfg[i1], i4 = cfg[i2];
  tidx = idx;
  tidx[i3] = i2;
  tidx[i4] = i1;
  for (int qp = 0; qp < c.n_qp; qp++)
    pf_new[qp] = new_pf_two_qp(c, qp, i3, i4, tidx.data(), &inv[(size_t)N * N * qp], pf_old[qp], va.data(), vb.data());
  return 0;
}

// SR block: SR_pdposv.f90:1-432 with the normalisation of main.f90:357-369 already applied to
// Etot/Etot2/gvec/Ovec; mat_tmp = S_raw summed over ranks (not normalised), norm = summed norm.
// Updates the parameters in place (rank 0's gamma_save, Nsave = 1) and consumes the RNG draws of
// SR_pdposv.f90:172 (every rank) and :281, :313 (rank 0).
int orc_sr_step(void* h, const orc_sr_in* in, const double* mat_tmp, double norm, double* gvec, const double* Ovec,
                orc_sr_out* out, double* dx_out) {
  Ctx& c = *(Ctx*)h;
  const int Nv = c.Nv, Nrbm = c.Nv_rbm, N = c.N;
  std::vector<double> S((size_t)Nv * Nv), g(gvec, gvec + Nv);
  for (int k = 0; k < Nv; k++) g[k] = g[k] - 2.0 * in->Etot * Ovec[k];  // :4-6
  for (int k2 = 0; k2 < Nv; k2++)                                          // :11-15
    for (int k1 = 0; k1 < Nv; k1++) S[k1 + (size_t)Nv * k2] = mat_tmp[k1 + (size_t)Nv * k2] / norm - Ovec[k1] * Ovec[k2];
  double sr = 0, sp = 0;
  int i1 = 0, i2 = 0;
  for (int k = 0; k < Nv; k++)  // :18-31
    if (S[k + (size_t)Nv * k] > 0.0) {
      if (k < Nrbm) {
        i1++;
        sr += S[k + (size_t)Nv * k];
      } else {
        i2++;
        sp += S[k + (size_t)Nv * k];
      }
    }
  if (i1 != Nrbm) return set_err(c, ORC_E_SDIAG, "i1/=Nv_RBM");
  if (i2 != c.n_slater - c.n_slater / N) return set_err(c, ORC_E_SDIAG, "i2 /= N_Slater - N_Slater/N");
  sr = (Nrbm > 0) ? sr / (double)i1 : 1.0;
  sp = sp / (double)i2;
  double scal = std::sqrt(sr / sp);  // :40
  for (int k = Nrbm; k < Nv; k++) g[k] = g[k] * scal;  // :56-58
  for (int k2 = Nrbm; k2 < Nv; k2++)
    for (int k1 = 0; k1 < Nv; k1++) S[k1 + (size_t)Nv * k2] *= scal;
  for (int k1 = Nrbm; k1 < Nv; k1++)
    for (int k2 = 0; k2 < Nv; k2++) S[k1 + (size_t)Nv * k2] *= scal;
  for (int k1 = 0; k1 < Nv; k1++) {  // :78-100
    double d = S[k1 + (size_t)Nv * k1];
    int cnt = 0;
    for (int i = 0; i < N; i++)
      if (k1 == c.orb_idx[i + N * i] + Nv - c.n_slater) cnt++;
    if (d < 0.0) return set_err(c, ORC_E_SDIAG, "diagonal element of S matrix is not positive");
    if (d == 0.0) {
      if (cnt == 0) return set_err(c, ORC_E_SDIAG, "diagonal element of S matrix is zero for other than f_ii parameters");
      if (std::fabs(Ovec[k1]) > 1e-300 || std::fabs(g[k1]) > 1e-300)
        return set_err(c, ORC_E_SDIAG, "Ovec/gvec related with f_ii parameters is wrong");
      for (int k2 = 0; k2 < Nv; k2++)
        if (std::fabs(S[k2 + (size_t)Nv * k1]) > 1e-300 || std::fabs(S[k1 + (size_t)Nv * k2]) > 1e-300)
          return set_err(c, ORC_E_SDIAG, "Smat related with f_ii parameters is wrong");
    } else if (cnt != 0)
      return set_err(c, ORC_E_SDIAG, "diagonal element of S matrix is positive for f_ii parameters");
  }
  double sdiag = 0, srb = 0, spp = 0;  // :104-140
  i1 = i2 = 0;
  for (int k = 0; k < Nv; k++) {
    double d = S[k + (size_t)Nv * k];
    if (d > 0.0) {
      sdiag += d;
      if (k < Nrbm) {
        i1++;
        srb += d;
      } else {
        i2++;
        spp += d;
      }
    }
  }
  sdiag = sdiag / (double)(i1 + i2);
  srb = (Nrbm > 0) ? srb / (double)i1 : 1.0;
  spp = spp / (double)i2;
  if (std::fabs(srb / spp - 1.0) > 1e-5) return set_err(c, ORC_E_SDIAG, "Sdiag_av_RBM/=Sdiag_av_PP");
  double rcut = sdiag * in->s_cut;
  int nS = 0;
  for (int k = 0; k < Nv; k++)
    if (S[k + (size_t)Nv * k] > rcut) nS++;
  double s_factor = std::max(1e-4, in->s_factor0);  // :167-170
  for (int k = 0; k < Nv; k++) S[k + (size_t)Nv * k] += sdiag * s_factor;
  for (int r = 0; r < c.nranks; r++) (void)grnd(c.ranks[r].rng);  // :172, every rank
  std::vector<double> Ssave = S;
  std::vector<double> x = g;
  if (chol_solve_upper(Nv, S, x)) return set_err(c, ORC_E_CHOL, "pdposv info /= 0");
  double lam = 0, lrr = 0, lpp = 0, lrp = 0;  // :251-267
  for (int k2 = 0; k2 < Nv; k2++)
    for (int k1 = 0; k1 < Nv; k1++) {
      double r1 = x[k1] * Ssave[k1 + (size_t)Nv * k2] * x[k2];
      lam += r1;
      if (k2 < Nrbm && k1 < Nrbm) lrr += r1;
      else if (k2 >= Nrbm && k1 >= Nrbm) lpp += r1;
      else lrp += r1;
    }
  lam = std::sqrt(lam);
  if (c.rank0 == 0) (void)grnd(c.ranks[0].rng);  // :281 (rank 0)
  if (std::fabs(lam * lam - lrr - lpp - lrp) > 1e-5) return set_err(c, ORC_E_LAMBDA, "lambda division is wrong");
  lam = lam * 5.0 / (double)c.L;  // :309
  out->lambda = lam;
  out->lambda_rbm_rbm = lrr;
  out->lambda_pp_pp = lpp;
  out->lambda_rbm_pp = lrp;
  if (lam > 1.0)
    for (int k = 0; k < Nv; k++) x[k] = x[k] / lam;
  if (c.rank0 == 0) (void)grnd(c.ranks[0].rng);  // :313 (rank 0; left-to-right .and.)
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
  // gamma_save(:,Nsave) = current parameters (main.f90:263-294 ordering: complex b and W(iw,f) as (re, im)
  // pairs, then real b, W(iw,f), then f_ij)
  std::vector<double> gam(Nv);
  int k1 = 0;
  for (int f = 0; f < c.alphac; f++) {
    gam[k1++] = c.bc[f].real();
    gam[k1++] = c.bc[f].imag();
  }
  for (int f = 0; f < c.alphac; f++)
    for (int iw = 0; iw < N; iw++) {
      gam[k1++] = c.Wc[iw + (size_t)N * f].real();
      gam[k1++] = c.Wc[iw + (size_t)N * f].imag();
    }
  for (int f = 0; f < c.alphar; f++) gam[k1++] = c.br[f];
  for (int f = 0; f < c.alphar; f++)
    for (int iw = 0; iw < N; iw++) gam[k1++] = c.Wr[iw + (size_t)N * f];
  for (int o = 0; o < c.n_slater; o++) gam[k1++] = c.slater[o];
  const double max_change = 0.04;
  for (int k = 0; k < Nv; k++) {  // :347-354
    if (delW > max_change) gam[k] = gam[k] - in->delta_tau * x[k] * (max_change / delW);
    else gam[k] = gam[k] - in->delta_tau * x[k];
  }
  int off = 2 * c.alphac * (N + 1) + c.alphar * (N + 1);  // :356-366
  double r1 = 0.0;
  for (int k = off; k < Nv; k++) r1 = r1 + std::fabs(gam[k]);
  r1 = r1 / (double)c.n_slater;
  for (int k = off; k < Nv; k++) gam[k] = gam[k] * 0.25 / r1;
  k1 = 0;  // :385-413 (parameter averaging is a no-op for Nsave = 1)
  for (int f = 0; f < c.alphac; f++, k1 += 2) c.bc[f] = cplx(gam[k1], gam[k1 + 1]);
  for (int f = 0; f < c.alphac; f++)
    for (int iw = 0; iw < N; iw++, k1 += 2) c.Wc[iw + (size_t)N * f] = cplx(gam[k1], gam[k1 + 1]);
  for (int f = 0; f < c.alphar; f++) c.br[f] = gam[k1++];
  for (int f = 0; f < c.alphar; f++)
    for (int iw = 0; iw < N; iw++) c.Wr[iw + (size_t)N * f] = gam[k1++];
  r1 = 0.0;
  for (int o = 0; o < c.n_slater; o++) {
    c.slater[o] = gam[k1++];
    r1 += std::fabs(c.slater[o]);
  }
  r1 /= (double)c.n_slater;
  if (std::fabs(r1 - 0.25) > 1e-6) return set_err(c, ORC_E_SLATER_NORM, "r1/=slater_abs_av");
  out->delW_max = delW;
  out->kmax = kmax;
  out->k_nonzero = knz;
  out->s_factor = s_factor;
  out->sdiag_av = sdiag;
  out->smat_scaling = scal;
  out->nSmat = nS;
  if (dx_out) std::memcpy(dx_out, x.data(), sizeof(double) * Nv);
  for (int k = 0; k < Nv; k++) gvec[k] = g[k];
  return update_slater_elements(c);
}

// ---- small standalone kernels for tests ----
double orc_pfaffian(int n, const double* A) {
  std::vector<double> B(A, A + (size_t)n * n);
  return pfaffian_pr(n, B.data());
}

int orc_inverse(int n, double* A) { return inverse_lu(n, A); }

int orc_mt_u32(int seed, int skip, int n, uint32_t* out) {
  MT s;
  mt_seed(s, seed);
  for (int i = 0; i < skip; i++) (void)mt_next_u32(s);
  for (int i = 0; i < n; i++) out[i] = mt_next_u32(s);
  return 0;
}

int orc_mt_state(int seed, uint32_t* mt) {
  MT s;
  mt_seed(s, seed);
  std::memcpy(mt, s.mt, sizeof(s.mt));
  return 0;
}

int orc_grnd(int seed, int skip, int n, double* out) {
  MT s;
  mt_seed(s, seed);
  for (int i = 0; i < skip; i++) (void)grnd(s);
  for (int i = 0; i < n; i++) out[i] = grnd(s);
  return 0;
}

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"

// estimator.cu -- per-configuration estimators (calc_phys_quantity.f90:20-246, 250-302, 306-427) and
// the adjoint O_k kernel: one CTA per configuration, one warp per Pfaffian projection.
//
// Each warp owns a padded shared-memory tile and, for its projections qp, inverts X from scratch with
// warp-level Gauss-Jordan (the role of calculate_MAll, calc_phys_quantity.f90:85), then evaluates the
// exchange ratio of every antiparallel J1/J2 bond (calc_local_energy_correlation,
// calc_phys_quantity.f90:338-374) against that inverse.  Bonds are grouped by their up electron ua:
// with v_ua(i) = XF(u_i, u_ua) and W = Y v_ua (one mat-vec per ua), a bond (ua, db) needs only
//     r_a = u.Y(:,ua),  s_b = W(db) + dv Y(db,ua),  u^T Y v = u.W + dv r_a,  dv = c - XF(u_ua, u_ua),
// so the Np^2 work is per up electron, not per bond.  The up to eight bonds of one up electron gather
// their rows u together and reduce their 16 dot products in one transposed butterfly; lane t then
// finishes bond t.  W and the needed column of Y stay in registers (lane <-> row) and reach other lanes
// by shuffles.  A warp first stores every bond's ratio,
// then weighs the bonds lane-parallel (cosh products of the moved spins, calc_phys_quantity.f90:338-374)
// into per-lane sums of sum_b 2 J sgn psi(x'_b).  After each round of projections the CTA scatters
// d Pf / d f_k (calculate_derivative_Pfaffian, slater.f90:94-170) in projection order.
// The RBM part of O_k (calc_phys_quantity.f90:165-201) is a gather over the inverse translation
// tables.  Outputs are the raw psi, H psi and d psi/d theta_k, optionally reweighted by
// 1/(|psi| + shift) as calc_phys_quantity.f90:102-109,221 do.
#include "walker_ops.cuh"

namespace {

constexpr int kEstThreads = 256;
constexpr int kEstWarps = kEstThreads / 32;

struct Est {
  int* ap;       // [4N][2] antiparallel bonds (i1, i2) in bond_map order
  double* apc;   // [4N]    2 J sgn
  int* bua;      // [4N]    up electron of the bond
  int* bdb;      // [4N]    down electron (local index) of the bond
  int* order;    // [4N]    bonds sorted by ua
  int* ustart;   // [Np+1]  CSR offsets into order
  double* Rb;    // [kEstWarps][4N] per-warp exchange ratios of the current projection
  double* tiles; // [nqw][Np*(Np+1)]
  int* perm;     // [kEstWarps][Np] column map of each warp's inverse
  double* vp;    // [kEstWarps][Np]  v_ua stored at the tile's column positions
  double* pfw;   // [n_qp] Pf per projection
  int* nap;
  double* diag;
  int nqw;
};

// Shared-memory layout of one estimator block.  With gtiles the nqw Gauss-Jordan tiles live in global memory (a
// per-block slice of a scratch buffer, for block sizes whose tiles do not fit one block's shared memory).
__host__ __device__ __forceinline__ size_t est_layout(const DevDims& d, int nqw, char* base, WS* w, Est* e,
                                                      bool gtiles = false) {
  size_t off = 0;
  auto take = [&](size_t bytes) -> char* {
    char* p = base ? base + off : nullptr;
    off = align16(off + bytes);
    return p;
  };
  const int N = d.N, Np = d.Np, NB = 4 * N;
  WS t;
  t.mt = nullptr;
  t.x = (int*)take(N * 4);
  t.idx = (int*)take(N * 4);
  t.cfg = (int*)take(N * 4);
  t.x2 = t.idx2 = t.cfg2 = nullptr;
  t.th = (double*)take((size_t)(d.Mr + 2 * d.Mc) * 8);
  t.thp = nullptr;
  t.sgn = (int*)take(d.n_mp * 4);
  t.sgnp = nullptr;
  t.pb = (int*)take(d.n_mp * 4);
  t.pf = nullptr;
  t.pfp = nullptr;
  t.psi = (double*)take((size_t)d.n_qp * 16);
  t.psip = nullptr;
  t.rbm = (double*)take((size_t)d.n_qp * 8);
  t.rbmc = d.alphac ? (double*)take((size_t)d.n_qp * 16) : nullptr;
  t.colbuf = t.rowbuf = nullptr;
  t.perm = nullptr;
  t.wA = t.wS = nullptr;
  t.red = (double*)take(64 * 8);
  t.iflag = (int*)take(32 * 4);
  t.dsc = (double*)take(32 * 8);
  Est x;
  x.ap = (int*)take((size_t)NB * 2 * 4);
  x.apc = (double*)take((size_t)NB * 8);
  x.bua = (int*)take((size_t)NB * 4);
  x.bdb = (int*)take((size_t)NB * 4);
  x.order = (int*)take((size_t)NB * 4);
  x.ustart = (int*)take((size_t)(Np + 1) * 4);
  x.Rb = (double*)take((size_t)kEstWarps * NB * 8);
  x.perm = (int*)take((size_t)kEstWarps * Np * 4);
  x.vp = (double*)take((size_t)kEstWarps * Np * 8);
  x.pfw = (double*)take((size_t)d.n_qp * 8);
  x.nap = (int*)take(16);
  x.diag = (double*)take(16);
  const size_t tile = (size_t)Np * (Np + 1) * 8;
  const size_t signbuf = (size_t)kEstWarps * N * 4;
  if (gtiles) {
    x.tiles = nullptr;  // set per block from the scratch buffer
    t.wu = (double*)take(signbuf);  // per-warp N-int buffers of cta_sign_pp
  } else {
    size_t tiles_bytes = (size_t)nqw * tile;
    if (tiles_bytes < signbuf) tiles_bytes = signbuf;  // sign_PP scratch reuses the tile area
    x.tiles = (double*)take(tiles_bytes);
    t.wu = x.tiles;  // per-warp N-int buffers of cta_sign_pp (used before the projection loop)
  }
  x.nqw = nqw;
  t.tile = x.tiles;
  t.wv = nullptr;
  if (w) *w = t;
  if (e) *e = x;
  return off;
}

template <int KPL, int NP>
__device__ __forceinline__ void estimator_config(const DevDims& d, const DevTables& t, const DevParams& p,
                                                 const int8_t* xs, int n, double* out_psi, double* out_hpsi,
                                                 double* O, int* out_nap, int* out_status, int reweight, const WS& s,
                                                 const Est& e, int cfgi) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int N = d.N, Np = NP > 0 ? NP : d.Np, ld = Np + 1, NB = 4 * N;
  // complex projection weights: a real row and an imaginary row per configuration
  double* Orow = O ? O + (size_t)cfgi * d.Nv * (d.cplx ? 2 : 1) : nullptr;
  double* OrowI = (Orow && d.cplx) ? Orow + d.Nv : nullptr;

  for (int i = tid; i < N; i += blockDim.x) s.x[i] = (int)xs[(size_t)cfgi * N + i];
  if (Orow)
    for (int k = tid; k < d.Nv * (d.cplx ? 2 : 1); k += blockDim.x) Orow[k] = 0.0;
  if (tid == 0) s.iflag[F_STATUS] = 0;
  __syncthreads();
  if (tid == 0) {
    int st = x_to_ele(d, s.x, s.idx, s.cfg);
    if (st) s.iflag[F_STATUS] = st;
    // bond list (bond_map, calc_phys_quantity.f90:382-427), diagonal part, CSR by up electron
    int na = 0;
    double dg = 0.0;
    for (int a = 0; a <= Np; a++) e.ustart[a] = 0;
    for (int b = 0; b < NB && !st; b++) {
      const int i1 = t.bonds[2 * b], i2 = t.bonds[2 * b + 1];
      const double J = (b < 2 * N) ? d.J1 : d.J2, sg = (b < 2 * N) ? -1.0 : 1.0;
      dg = dg + J * (double)s.x[i1] * (double)s.x[i2];
      if (s.x[i1] != s.x[i2]) {
        const int i3 = s.cfg[i1], i4 = s.cfg[i2];
        const int ua = (s.x[i1] == 1) ? i3 : i4, db = ((s.x[i1] == 1) ? i4 : i3) - Np;
        e.ap[2 * na] = i1;
        e.ap[2 * na + 1] = i2;
        e.apc[na] = 2.0 * J * sg;
        e.bua[na] = ua;
        e.bdb[na] = db;
        e.ustart[ua + 1]++;
        na++;
      }
    }
    for (int a = 0; a < Np; a++) e.ustart[a + 1] += e.ustart[a];
    int fill[RBMPP_MAX_N / 2];
    for (int a = 0; a < Np; a++) fill[a] = e.ustart[a];
    for (int b = 0; b < na; b++) e.order[fill[e.bua[b]]++] = b;
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
  cta_rbm_factors(d, s.th, s.rbm, s.rbmc);
  __syncthreads();
  if (s.iflag[F_STATUS]) {
    if (tid == 0 && out_status) out_status[cfgi] = s.iflag[F_STATUS];
    return;
  }
  const int off_r = 2 * d.alphac * (N + 1), off_pp = off_r + d.alphar * (N + 1);  // calc_phys_quantity.f90:205
  double* Rw = e.Rb + (size_t)warp * NB;
  int* src = e.perm + (size_t)warp * Np;
  double* vp = e.vp + (size_t)warp * Np;
  int jc[KPL];
#pragma unroll
  for (int q = 0; q < KPL; q++) {
    const int j = lane + 32 * q;
    jc[q] = j < Np ? j : Np - 1;  // in-tile index for every lane
  }
  bool bad = false;
  double hacc = 0.0, hacci = 0.0;  // this lane's share of sum_b 2 J sgn psi(x'_b) (real, imaginary part)
  // rounds of nqw projections: warp w < nqw handles qp = round*nqw + w
  for (int q0 = 0; q0 < d.n_qp; q0 += e.nqw) {
    const int qp = q0 + warp;
    double* T = e.tiles + (size_t)warp * Np * ld;
    if (warp < e.nqw && qp < d.n_qp) {
      const int mp = qp >> 1, sp = qp & 1;
      const double* XFq = p.XF + (size_t)qp * N * N;
      const double* XFTq = p.XFT + (size_t)qp * N * N;
      warp_gather_tile<KPL, NP, 8>(T, XFq, s.idx, Np, N);
      bool sing;
      const double det = warp_gj<KPL, NP, (KPL <= 2 ? 16 : (KPL <= 4 ? 8 : 4))>(T, Np, src, sing);
      if (sing) bad = true;
      const double pfq = (double)d.pf_sign * det;
      const cplx cw = psi_wo_pf_s(d, t, s, s.sgn[mp], qp);
      if (lane == 0) {
        e.pfw[qp] = pfq;
        s.psi[2 * qp] = cw.re * pfq;
        s.psi[2 * qp + 1] = cw.im * pfq;
      }
      // down-electron sites of this lane's rows (the columns of every u row)
      int dsite[KPL];
#pragma unroll
      for (int q = 0; q < KPL; q++) dsite[q] = s.idx[Np + jc[q]];
      // exchange ratios, grouped by up electron
      for (int ua = 0; ua < Np && !sing; ua++) {
        const int b0 = e.ustart[ua], b1 = e.ustart[ua + 1];
        if (b0 == b1) continue;
        const int s_up = s.idx[ua];
        const int cu = src[ua];
        double vv[KPL];
#pragma unroll
        for (int q = 0; q < KPL; q++) vv[q] = XFTq[(size_t)s_up * N + s.idx[jc[q]]];
        const double xfuu = XFq[(size_t)s_up * N + s_up];
        constexpr int MB = KPL <= 2 ? 8 : (KPL <= 4 ? 4 : 2);  // a site lies on 4 J1 and 4 J2 bonds
        constexpr int NV = 2 * MB, SH = MB == 8 ? 1 : (MB == 4 ? 2 : 3);  // value v ends in lane v << SH
        for (int c0 = b0; c0 < b1; c0 += MB) {
          const int m = b1 - c0 < MB ? b1 - c0 : MB;
          // bond t of the chunk in lane t: its index, down electron, down site and X'(ua, db) = XF(s_dn, s_up)
          int b_l = 0, db_l = 0, sdn_l = 0;
          double c_l = 0.0;
          if (lane < m) {
            b_l = e.order[c0 + lane];
            db_l = e.bdb[b_l];
            sdn_l = s.idx[Np + db_l];
            c_l = XFq[(size_t)sdn_l * N + s_up];
          }
          // rows u of the m bonds: u_j = XF(s_dn, down site j), gathered before any use
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
              dbv[t2] = __shfl_sync(0xffffffffu, db_l, t2);
              const double* urow = XFq + (size_t)sdn * N;
#pragma unroll
              for (int q = 0; q < KPL; q++) uu[t2][q] = urow[dsite[q]];
            }
          }
#pragma unroll
          for (int t2 = 0; t2 < MB; t2++)
            if (t2 < m) cb[t2] = __shfl_sync(0xffffffffu, c_l, t2);
          if (c0 == b0) {
            // v_ua(i) = XF(u_i, s_up) at the tile's column positions, W = Y v_ua (lane <-> row)
#pragma unroll
            for (int q = 0; q < KPL; q++)
              if (lane + 32 * q < Np) vp[src[lane + 32 * q]] = vv[q];
            __syncwarp();
          }
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
          // partial sums: val[t] = u_t . Y(:, ua), val[MB + t] = u_t . W
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
          // lane t < m finishes bond t
          const double ra = __shfl_sync(0xffffffffu, tot, (lane << SH) & 31);
          const double uw = __shfl_sync(0xffffffffu, tot, ((MB + lane) << SH) & 31);
          double y = 0.0, wdb = 0.0;
#pragma unroll
          for (int q = 0; q < KPL; q++) {
            const double a = __shfl_sync(0xffffffffu, tj[q], db_l & 31);   // Y(db, ua)
            const double w = __shfl_sync(0xffffffffu, wv[q], db_l & 31);   // W(db)
            if (q == (db_l >> 5)) {
              y = a;
              wdb = w;
            }
          }
          if (lane < m) {
            const double dv = c_l - xfuu;
            const double sb = wdb + dv * y;
            const double wvv = uw + dv * ra;
            Rw[b_l] = ra * sb - y * (wvv - c_l);
          }
        }
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
          cplx cbw = psi_wo_pf(d, t, ch, sg, qp);
          if (d.alphac) {  // complex units: 0.5^alphac prod cosh(thetac') of the exchanged configuration
            cplx cf = {1.0, 0.0};
            for (int f = 0; f < d.alphac; f++) {
              const int j = d.Mr + 2 * (qp * d.alphac + f);
              const double* Wf = p.Wc + (size_t)f * N * 2;
              const double ar = s.th[j] - 2.0 * Wf[2 * iw1] * x1 * s_sign - 2.0 * Wf[2 * iw2] * x2 * s_sign;
              const double ai = s.th[j + 1] - 2.0 * Wf[2 * iw1 + 1] * x1 * s_sign - 2.0 * Wf[2 * iw2 + 1] * x2 * s_sign;
              cf = cscale(cmul(cf, ccosh_(ar, ai)), 0.5);
            }
            cbw = cmul(cbw, cf);
          }
          hacc = hacc + e.apc[b] * (cbw.re * (Rw[b] * pfq));
          hacci = hacci + e.apc[b] * (cbw.im * (Rw[b] * pfq));
        }
      }
      __syncwarp();
    }
    __syncthreads();
    // d Pf / d f_k scatter of this round's projections, in projection order (slater.f90:140-167); with complex
    // weights the imaginary row takes the same scatter with the imaginary part of psi_x_wo_pf
    if (OrowI) {
      for (int w = 0; w < e.nqw && q0 + w < d.n_qp; w++) {
        const int qp = q0 + w, mp = qp >> 1, sp = qp & 1;
        const double* Tw = e.tiles + (size_t)w * Np * ld;
        const int* srcw = e.perm + (size_t)w * Np;
        const int* wm = t.wmap + (size_t)mp * N;
        const double pfq = e.pfw[qp];
        const cplx cw = psi_wo_pf_s(d, t, s, s.sgn[mp], qp);
        const double cc = pfq * d.sp_cc[sp] * cw.im, ss = pfq * d.sp_ss[sp] * cw.im;
        for (int pr = tid; pr < Np * Np; pr += blockDim.x) {
          const int j = pr / Np, i = pr - j * Np;
          const double y = Tw[j * ld + srcw[i]];
          const int tu = wm[s.idx[i]], td = wm[s.idx[Np + j]];
          if (d.orb_injective) {
            if (cc != 0.0) OrowI[off_pp + t.orb[(size_t)tu * N + td]] += y * cc;
            if (ss != 0.0) OrowI[off_pp + t.orb[(size_t)td * N + tu]] += y * ss;
          } else {
            if (cc != 0.0) atomicAdd(OrowI + off_pp + t.orb[(size_t)tu * N + td], y * cc);
            if (ss != 0.0) atomicAdd(OrowI + off_pp + t.orb[(size_t)td * N + tu], y * ss);
          }
        }
        __syncthreads();
      }
    }
    if (Orow) {
      for (int w = 0; w < e.nqw && q0 + w < d.n_qp; w++) {
        const int qp = q0 + w, mp = qp >> 1, sp = qp & 1;
        const double* Tw = e.tiles + (size_t)w * Np * ld;
        const int* srcw = e.perm + (size_t)w * Np;
        const int* wm = t.wmap + (size_t)mp * N;
        const double pfq = e.pfw[qp];
        const cplx cw = psi_wo_pf_s(d, t, s, s.sgn[mp], qp);
        const double cc = pfq * d.sp_cc[sp] * cw.re, ss = pfq * d.sp_ss[sp] * cw.re;
        const int npr = Np * Np;
        // Each thread loads the values and targets of SB pairs before it adds any, and adds with fire-and-forget
        // reductions in L2 (the thread never waits for the old value).  With an injective orbital map every
        // (up, down) pair of one projection has its own two targets, and projections follow one another
        // (barrier below), so every target receives its terms in projection order: the sums are
        // deterministic.  A non-injective map can hit a target twice within one projection.
        constexpr int SB = 8;
        for (int pr0 = tid; pr0 < npr; pr0 += SB * kEstThreads) {
          double y[SB];
          int a1[SB], a2[SB];
#pragma unroll
          for (int u = 0; u < SB; u++) {
            const int pr = pr0 + u * kEstThreads, prc = pr < npr ? pr : npr - 1;
            const int j = prc / Np, i = prc - j * Np;  // j: down electron, i: up electron
            y[u] = Tw[j * ld + srcw[i]];               // Y(j, i) = (M^-1)(Np+j, i)
            const int tu = wm[s.idx[i]], td = wm[s.idx[Np + j]];
            a1[u] = off_pp + t.orb[(size_t)tu * N + td];
            a2[u] = off_pp + t.orb[(size_t)td * N + tu];
          }
#pragma unroll
          for (int u = 0; u < SB; u++)
            if (pr0 + u * kEstThreads < npr) {
              if (cc != 0.0) atomicAdd(Orow + a1[u], y[u] * cc);
              if (ss != 0.0) atomicAdd(Orow + a2[u], y[u] * ss);
            }
        }
        __syncthreads();
      }
    }
    __syncthreads();
  }
  if (lane == 0 && bad) s.iflag[F_STATUS] = ST_SINGULAR;
  hacc = warp_sum(hacc);
  hacci = warp_sum(hacci);
  if (lane == 0) {
    s.red[warp] = hacc;
    s.red[32 + warp] = hacci;
  }
  __syncthreads();
  if (s.iflag[F_STATUS]) {
    if (tid == 0 && out_status) out_status[cfgi] = s.iflag[F_STATUS];
    return;
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
    for (int w = 0; w < kEstWarps; w++) {
      hr += s.red[w];
      hi += s.red[32 + w];
    }
    s.dsc[D_PSIPR] = hr;
    s.dsc[D_PSIPI] = hi;
    if (out_nap) out_nap[cfgi] = nap;
    if (out_status) out_status[cfgi] = 0;
  }
  __syncthreads();
  const double w = reweight ? 1.0 / (hypot(s.dsc[D_PSI0R], s.dsc[D_PSI0I]) + d.shift) : 1.0;
  if (Orow) {
    // RBM part, real branch (calc_phys_quantity.f90:165-201): tanh(theta) psi_qp, whose imaginary part comes from
    // complex para_mp_trans
    for (int k = tid; k < d.alphar * (N + 1); k += blockDim.x) {
      double acc = 0.0, acci = 0.0;
      if (k < d.alphar) {
        const int f = k;
        for (int qp = 0; qp < d.n_qp; qp++) {
          const double th = tanh(s.th[qp * d.alphar + f]);
          acc = acc + th * s.psi[2 * qp];
          acci = acci + th * s.psi[2 * qp + 1];
        }
      } else {
        const int f = (k - d.alphar) / N, iw = (k - d.alphar) - f * N;
        for (int mp = 0; mp < d.n_mp; mp++) {
          const double xi = (double)s.x[t.winv[(size_t)mp * N + iw]];
          const int q0 = 2 * mp, q1 = 2 * mp + 1;
          const double t0 = tanh(s.th[q0 * d.alphar + f]), t1 = tanh(s.th[q1 * d.alphar + f]);
          acc = acc + t0 * s.psi[2 * q0] * xi;
          acc = acc - t1 * s.psi[2 * q1] * xi;
          acci = acci + t0 * s.psi[2 * q0 + 1] * xi;
          acci = acci - t1 * s.psi[2 * q1 + 1] * xi;
        }
      }
      Orow[off_r + k] = acc * w;
      if (OrowI) OrowI[off_r + k] = acci * w;
    }
    // complex RBM part (calc_phys_quantity.f90:115-160): parameter pairs (re, im) with d psi / d Im = i d psi / d Re;
    // tanh of a complex angle as (tanh a + i tan b) / (1 + i tanh a tan b)
    for (int k = tid; k < d.alphac * (N + 1); k += blockDim.x) {
      cplx v = {0.0, 0.0};
      auto ctanh = [&](int qp, int f) {
        const int j = d.Mr + 2 * (qp * d.alphac + f);
        const double ta = tanh(s.th[j]), tb = tan(s.th[j + 1]);
        const cplx num = {ta, tb}, den = {1.0, ta * tb};
        const double dd = den.re * den.re + den.im * den.im;
        return cplx{(num.re * den.re + num.im * den.im) / dd, (num.im * den.re - num.re * den.im) / dd};
      };
      int pos;
      if (k < d.alphac) {
        const int f = k;
        for (int qp = 0; qp < d.n_qp; qp++) v = cadd(v, cmul(ctanh(qp, f), cplx{s.psi[2 * qp], s.psi[2 * qp + 1]}));
        pos = 2 * f;
      } else {
        const int f = (k - d.alphac) / N, iw = (k - d.alphac) - f * N;
        for (int mp = 0; mp < d.n_mp; mp++) {
          const double xi = (double)s.x[t.winv[(size_t)mp * N + iw]];
          const int qa = 2 * mp, qb = 2 * mp + 1;
          v = cadd(v, cscale(cmul(ctanh(qa, f), cplx{s.psi[2 * qa], s.psi[2 * qa + 1]}), xi));
          v = cadd(v, cscale(cmul(ctanh(qb, f), cplx{s.psi[2 * qb], s.psi[2 * qb + 1]}), -xi));
        }
        pos = 2 * d.alphac + f * 2 * N + 2 * iw;
      }
      Orow[pos] = v.re * w;        // d psi / d Re
      OrowI[pos] = v.im * w;
      Orow[pos + 1] = -v.im * w;   // d psi / d Im = i d psi / d Re
      OrowI[pos + 1] = v.re * w;
    }
    for (int k = off_pp + tid; k < d.Nv; k += blockDim.x) {
      Orow[k] = Orow[k] * w;
      if (OrowI) OrowI[k] = OrowI[k] * w;
    }
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

template <int KPL, int NP>
__global__ void __launch_bounds__(kEstThreads, 1)
    estimator_kernel(const __grid_constant__ DevDims d, const __grid_constant__ DevTables t,
                     const __grid_constant__ DevParams p, const int8_t* xs, int n, double* out_psi, double* out_hpsi,
                     double* O, int* out_nap, int* out_status, int reweight, int nqw, double* gtiles) {
  extern __shared__ __align__(16) char smem[];
  __shared__ WS s;
  __shared__ Est e;
  const int Np = NP > 0 ? NP : d.Np, ld = Np + 1;
  if (threadIdx.x == 0) {
    est_layout(d, nqw, smem, &s, &e, gtiles != nullptr);
    if (gtiles) {
      e.tiles = gtiles + (size_t)blockIdx.x * nqw * Np * ld;
      s.tile = e.tiles;
    }
  }
  __syncthreads();
  // one configuration per block, or (global tiles) the configurations blockIdx.x, blockIdx.x + gridDim.x, ...
  for (int cfgi = blockIdx.x; cfgi < n; cfgi += gridDim.x) {
    __syncthreads();
    estimator_config<KPL, NP>(d, t, p, xs, n, out_psi, out_hpsi, O, out_nap, out_status, reweight, s, e, cfgi);
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

int est_tile_warps(const DevDims& d, int max_smem) {
  for (int q = kEstWarps; q >= 1; q--)
    if ((long long)est_layout(d, q, nullptr, nullptr, nullptr) <= max_smem) return q;
  return 0;
}

}  // namespace

// Shared memory of the estimator with its tiles in shared memory (one tile at least); larger than the opt-in
// limit for N/2 beyond about 120, where the tiles move to a global scratch buffer.
size_t rbmpp_estimator_smem(const DevDims& d, int threads) {
  (void)threads;
  return est_layout(d, 1, nullptr, nullptr, nullptr);
}

// Shared memory of the estimator in the mode its launch will use (global tiles when the shared ones do not fit).
size_t rbmpp_estimator_smem_any(const DevDims& d, int max_smem) {
  if (est_tile_warps(d, max_smem) >= 1) return est_layout(d, 1, nullptr, nullptr, nullptr);
  return est_layout(d, kEstWarps, nullptr, nullptr, nullptr, true);
}

cudaError_t rbmpp_launch_estimator(const DevDims& d, const DevTables& t, const DevParams& p, const int8_t* xs, int n,
                                   double* out_psi, double* out_hpsi, double* O, int* out_nap, int* out_status,
                                   int reweight, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  int dev = 0, maxsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  int nqw = est_tile_warps(d, maxsm);
  size_t smem = 0;
  double* gtiles = nullptr;
  int grid = n;
  if (nqw >= 1) {
    smem = est_layout(d, nqw, nullptr, nullptr, nullptr);
  } else {
    // tiles beyond one block's shared memory (N/2 beyond about 120): one block per SM loops over the
    // configurations with its tiles in a stream-ordered scratch slice of global memory
    nqw = kEstWarps;
    smem = est_layout(d, nqw, nullptr, nullptr, nullptr, true);
    if ((long long)smem > maxsm) return cudaErrorInvalidValue;
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    grid = n < nsm ? n : nsm;
    const size_t bytes = (size_t)grid * nqw * d.Np * (d.Np + 1) * sizeof(double);
    cudaError_t e = cudaMallocAsync((void**)&gtiles, bytes, st);
    if (e != cudaSuccess) return e;
  }
  int kpl = (d.Np + 31) / 32;
  cudaError_t rc = cudaErrorInvalidValue;
#define LAUNCH(K, NPC)                                                                                     \
  do {                                                                                                     \
    rc = cudaFuncSetAttribute(estimator_kernel<K, NPC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
    if (rc == cudaSuccess) {                                                                               \
      rbmpp_note_launch();                                                                                 \
      estimator_kernel<K, NPC><<<grid, kEstThreads, smem, st>>>(d, t, p, xs, n, out_psi, out_hpsi, O, out_nap, \
                                                                out_status, reweight, nqw, gtiles);         \
      rc = cudaGetLastError();                                                                             \
    }                                                                                                      \
    if (gtiles) cudaFreeAsync(gtiles, st);                                                                 \
    return rc;                                                                                             \
  } while (0)
  switch (d.Np) {  // block sizes of the even-L lattices with a compile-time specialisation
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
  if (gtiles) cudaFreeAsync(gtiles, st);
  return rc;
}

cudaError_t rbmpp_launch_advance_rng(uint32_t* mt, const int* nap, int ns, int nw, int extra, cudaStream_t st) {
  rbmpp_note_launch();
  advance_rng_kernel<<<(nw + 63) / 64, 64, 0, st>>>(mt, nap, ns, nw, extra);
  return cudaGetLastError();
}

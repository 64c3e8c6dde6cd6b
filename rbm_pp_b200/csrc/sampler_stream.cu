// sampler_stream.cu -- Metropolis sampler that streams each walker's projections through shared memory
// with TMA bulk copies (make_sample.f90:4-240, same RNG order as sampler.cu).
//
// One CTA per walker.  Warp 0 is the control warp: its lane 0 draws every random number, and the warp
// evaluates theta', the cosh products and the amplitude weights of the proposal.  Warp 1 is the producer
// (its lane 0 issues the bulk loads).  Warps 2..15 are seven pairs of consumers.  A tile is one projection's
// Y = X^{-1} (Np x Np FP64, row major); pair g takes tiles g, g + 7, ..., each warp of the pair half of the
// rows.  Every proposal is one pass over the n_qp tiles through an ST-stage ring, ST >= 7 where shared
// memory allows, so that loads are in flight while every pair computes:
//   producer:  cp.async.bulk global->shared (mbarrier complete_tx) into stage T mod ST as soon as tile
//              T - ST has released it, after posting the stage's ticket T;
//   pair:      waits for the ticket and the load, applies the deferred rank-2 update of the previously
//              accepted exchange (if any) to the tile in place, evaluates the determinant ratio of the
//              current proposal on it, writes an updated tile back with cp.async.bulk shared->global, and
//              releases the stage.
// The halves combine only vectors and scalars (partial column sums, row db, the ratio's terms) through
// shared memory at two pair barriers per tile.  A proposal costs one read of Y and an accepted move one
// write: the algorithmic minimum (pfupdate_two.f90 reads InvM once per ratio and rewrites it per accepted
// move).  The producer starts a pass at once; the control warp publishes the candidate as soon as it is
// drawn and computes theta' and the weights while the pairs work, and the amplitude of the proposal is
// summed after the pass.
#include "sampler_common.cuh"

namespace {

constexpr int kPairs = 7;
constexpr int kWarps = 2 + 2 * kPairs;  // warp 0: control (RNG, candidate, theta'); 1: producer; 2..15: pairs
constexpr int kMaxStages = 16;
#define ST_TIMEOUT 22

struct Stream {
  double* stage;  // [ST][Np*Np]; also the Gauss-Jordan tile outside passes
  uint64_t* full;
  uint64_t* empty;
  int* ticket;    // [ST] tile index last issued into the stage (the producer posts it before the load)
  double* pAS;    // [kPairs][Np][2] (A_j, S_j) = (Y(j, ua), (Y v)_j) of the deferred exchange (each half its rows)
  double* pscal;  // [kPairs][2 slots][2 halves][4] ratio terms of each half
  int ST;
  uint32_t tile_bytes;
};

// Per-warp vectors come from the walker workspace: wu = u of the proposal, wA = u and wv = v of the
// deferred exchange, wS = this warp's partial column sums.
__host__ __device__ __forceinline__ size_t stream_layout(const DevDims& d, int ST, char* base, WS* w, Stream* st) {
  size_t off = ws_layout(d, kWarps, base, w, false);
  auto take = [&](size_t bytes, size_t align) -> char* {
    off = (off + align - 1) / align * align;
    char* p = base ? base + off : nullptr;
    off += bytes;
    return p;
  };
  Stream t;
  t.ST = ST;
  t.tile_bytes = 8u * (uint32_t)d.Np * (uint32_t)d.Np;
  size_t stage_bytes = (size_t)ST * t.tile_bytes, gj = (size_t)d.Np * (d.Np + 1) * 8;
  t.stage = (double*)take(stage_bytes > gj ? stage_bytes : gj, 128);
  t.full = (uint64_t*)take(8 * (size_t)ST, 8);
  t.empty = (uint64_t*)take(8 * (size_t)ST, 8);
  t.ticket = (int*)take(4 * (size_t)ST, 4);
  t.pAS = (double*)take((size_t)kPairs * d.Np * 16, 16);
  t.pscal = (double*)take((size_t)kPairs * 16 * 8, 16);
  if (w) w->tile = t.stage;
  if (st) *st = t;
  return off;
}

struct Move {
  int ua, db, s_up, s_dn;  // up electron, down electron (local index), their sites before the move
};

// Tile math.  NP is the block size Np, a compile-time constant: the even-L square lattices 4x4 .. 10x10 have
// Np = 8, 18, 32, 50, the shapes this sampler takes.  Lane l of a consumer warp owns the column pair
// (2l, 2l+1) of every tile row, so a row is read and written with one 16-byte shared access per lane (rows
// start on 16-byte boundaries because Np is even).  Lanes with 2l >= NP hold nothing.
__device__ __forceinline__ double2 ld2(const double* p) { return *reinterpret_cast<const double2*>(p); }
__device__ __forceinline__ void st2(double* p, double2 v) { *reinterpret_cast<double2*>(p) = v; }

// Lane-held gathers of one exchange for one projection at the lane's column pair: u = new row ua of X,
// v = new column db of X, c = their shared corner, which u holds at column db and v at column ua (the
// gathers of pfupdate_two.f90:48-52 in block form).
struct UV {
  double2 u, v;
  double c;
};

template <int NP>
__device__ __forceinline__ void gather_regs(const DevDims& d, const DevParams& p, int qp, const int* idx,
                                            const Move& m, UV& g) {
  const int k = 2 * (threadIdx.x & 31), N = d.N;
  const double* xr = p.XF + (size_t)qp * N * N + (size_t)m.s_dn * N;
  const double* xc = p.XFT + (size_t)qp * N * N + (size_t)m.s_up * N;
  g.c = __ldg(xr + m.s_up);
  g.u = make_double2(0.0, 0.0);
  g.v = make_double2(0.0, 0.0);
  if (k < NP) {
    const int2 iu = *reinterpret_cast<const int2*>(idx + NP + k);
    const int2 iv = *reinterpret_cast<const int2*>(idx + k);
    g.u.x = (k == m.db) ? g.c : __ldg(xr + iu.x);
    g.u.y = (k + 1 == m.db) ? g.c : __ldg(xr + iu.y);
    g.v.x = (k == m.ua) ? g.c : __ldg(xc + iv.x);
    g.v.y = (k + 1 == m.ua) ? g.c : __ldg(xc + iv.y);
  }
}

// u (and v) of the lane's columns into the warp's shared vectors
template <int NP>
__device__ __forceinline__ void store_u(const UV& g, double* u) {
  const int k = 2 * (threadIdx.x & 31);
  if (k < NP) st2(u + k, g.u);
}
template <int NP>
__device__ __forceinline__ void store_uv(const UV& g, double* u, double* v) {
  const int k = 2 * (threadIdx.x & 31);
  if (k < NP) {
    st2(u + k, g.u);
    st2(v + k, g.v);
  }
}

// Barrier of the two warps of pair g (named barrier 1 + g, 64 threads) that also returns, on every thread,
// whether any thread of the pair passed a non-zero flag: both warps take the same branch afterwards.
// The warp is reconverged first and the barrier is the non-aligned form, which counts threads one by one,
// so lanes that arrive from a divergent branch (lane 0's bookkeeping) are counted exactly once.
__device__ __forceinline__ bool pair_sync_or(int g, bool flag) {
  __syncwarp();
  uint32_t out;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 q, %1, 0;\n barrier.red.or.pred p, %2, 64, q;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(out)
      : "r"((uint32_t)flag), "r"(1 + g)
      : "memory");
  return out != 0;
}

// (u^T Y)_k at the lane's column pair over the NR rows r0 .. r0+NR-1 (one half of a tile), as two
// interleaved FMA chains per column (even and odd rows).
template <int NP, int NR>
__device__ __forceinline__ double2 col_sums(const double* Y, const double* u, int r0) {
  const int k = 2 * (threadIdx.x & 31);
  double2 a = make_double2(0.0, 0.0), b = make_double2(0.0, 0.0);
  if (k < NP) {
    const double* y = Y + r0 * NP + k;
    const double* uu = u + r0;
#pragma unroll
    for (int jj = 0; jj + 1 < NR; jj += 2) {
      const double2 y0 = ld2(y + jj * NP), y1 = ld2(y + (jj + 1) * NP);
      const double u0 = uu[jj], u1 = uu[jj + 1];
      a.x = fma(u0, y0.x, a.x);
      a.y = fma(u0, y0.y, a.y);
      b.x = fma(u1, y1.x, b.x);
      b.y = fma(u1, y1.y, b.y);
    }
    if (NR & 1) {
      const double2 y0 = ld2(y + (NR - 1) * NP);
      const double u0 = uu[NR - 1];
      a.x = fma(u0, y0.x, a.x);
      a.y = fma(u0, y0.y, a.y);
    }
  }
  return make_double2(a.x + b.x, a.y + b.y);
}

// value of a lane-pair vector at column col, taken from the lane that owns it (valid on all lanes)
__device__ __forceinline__ double pick(double2 a, int col) {
  return __shfl_sync(0xffffffffu, (col & 1) ? a.y : a.x, col >> 1);
}

// (Y v)_j for row j (one row per lane).  The column pairs are visited in the order c ^ sig(j): rows are NP/2
// 16-byte words apart, so when gcd(NP/2, 8) = G > 1 the rows of a quarter-warp fall G to a bank group, and
// sig(j) in [0, G) moves those G rows onto distinct groups (G = 1 for NP = 18, 50: sig = 0 at compile time).
template <int NP>
__device__ __forceinline__ double row_dot(const double* Y, const double* v, int j) {
  constexpr int M2 = NP / 2;
  constexpr int G = (M2 & -M2) < 8 ? (M2 & -M2) : 8;
  const int sig = (j / (8 / G)) & (G - 1);
  const double* yr = Y + j * NP;
  double a0 = 0.0, a1 = 0.0;
#pragma unroll
  for (int cc = 0; cc < M2; cc++) {
    const int c2 = 2 * (cc ^ sig);
    const double2 y = ld2(yr + c2), w = ld2(v + c2);
    a0 = fma(y.x, w.x, a0);
    a1 = fma(y.y, w.y, a1);
  }
  return a0 + a1;
}

// Half h (rows h*NP/2 .. ) of the deferred rank-2 update of a tile for an accepted exchange (the algebra of
// pfupdate_two.f90:113-224 in block form): Y' = Y - A B^T / R1 - s1 t1^T / R2, with A = Y e_ua,
// B = u^T Y - e_ua^T, s1 = Y v - A (u^T Y v - c)/R1 - e_db, t1 = e_db^T Y - Y(db,ua) B^T / R1, R2 = R / R1.
// With S = Y v, bk = B / R1, tk = t1 / R2 and wc = (u^T Y v - c) / R1 this is
//   Y'_jk = Y_jk - A_j (bk_k - wc tk_k) - S_j tk_k + [j = db] tk_k,
// one pass over the rows with (A_j, S_j) read as one 16-byte word.  Each half forms its rows' part of u^T Y
// and its rows' A and S, the pair exchanges them at one barrier, and each half rewrites its own rows.
// bad enters as this warp's failure flag and leaves as the pair's (uniform).
template <int NP>
__device__ __forceinline__ bool update_half(double* Y, const Move& m, double c, const double* u, const double* v,
                                            int g, int h, double* my_acc, const double* other_acc, double* pAS,
                                            bool bad) {
  constexpr int NR = NP / 2;
  const int lane = threadIdx.x & 31, k = 2 * lane, r0 = h * NR;
  double2 accp = make_double2(0.0, 0.0), rho = make_double2(0.0, 0.0);
  double ydbua = 0.0;
  if (!bad) {
    accp = col_sums<NP, NR>(Y, u, r0);
    if (lane < NR) {
      const int j = r0 + lane;
      st2(pAS + 2 * j, make_double2(Y[j * NP + m.ua], row_dot<NP>(Y, v, j)));
    }
    if (k < NP) {
      rho = ld2(Y + m.db * NP + k);  // row db, read before either half rewrites it
      st2(my_acc + k, accp);
    }
    ydbua = Y[m.db * NP + m.ua];
  }
  if (pair_sync_or(g, bad)) return true;
  double2 acc = make_double2(0.0, 0.0);
  double wv = 0.0;
  if (k < NP) {
    const double2 o = ld2(other_acc + k), vk = ld2(v + k);
    acc = make_double2(accp.x + o.x, accp.y + o.y);  // both halves form the same sums (addition commutes)
    wv = fma(acc.y, vk.y, acc.x * vk.x);
  }
  const double ra = pick(acc, m.ua);
  wv = warp_sum(wv);
  const double R1 = ra, R = ra * pAS[2 * m.db + 1] - ydbua * (wv - c);
  const double inv_r1 = 1.0 / R1, r1_over_r = R1 / R, wc = (wv - c) * inv_r1;
  const double bx = (acc.x - (k == m.ua ? 1.0 : 0.0)) * inv_r1, by = (acc.y - (k + 1 == m.ua ? 1.0 : 0.0)) * inv_r1;
  const double tx = (rho.x - ydbua * bx) * r1_over_r, ty = (rho.y - ydbua * by) * r1_over_r;
  const double cx = bx - wc * tx, cy = by - wc * ty;
  if (k < NP) {
    double* y = Y + r0 * NP + k;
    const double* as = pAS + 2 * r0;
#pragma unroll 5
    for (int jj = 0; jj < NR; jj++) {
      const double2 a = ld2(as + 2 * jj);
      double2 yv = ld2(y + jj * NP);
      yv.x = yv.x - a.x * cx - a.y * tx;
      yv.y = yv.y - a.x * cy - a.y * ty;
      st2(y + jj * NP, yv);
    }
    if (m.db >= r0 && m.db < r0 + NR) {
      double2 yv = ld2(Y + m.db * NP + k);
      yv.x += tx;
      yv.y += ty;
      st2(Y + m.db * NP + k, yv);
    }
  }
  __syncwarp();
  return false;
}

// Half h's terms of the ratio R = (u^T Y)_ua (Y v)_db - Y(db,ua) (u^T Y v - c): its rows' part of u^T Y v
// and of (u^T Y)_ua, and, from the half that holds row db, (Y v)_db and Y(db,ua).  v comes from the
// lane's registers.  The two warp sums share one shuffle tree; lanes 0 and 16 write scal[0..3].
template <int NP>
__device__ __forceinline__ void ratio_half(const double* Y, const Move& m, const double* u, const UV& g, int h,
                                           double* scal) {
  constexpr int NR = NP / 2;
  const int lane = threadIdx.x & 31, k = 2 * lane, r0 = h * NR;
  const double2 acc = col_sums<NP, NR>(Y, u, r0);
  const bool owner = m.db >= r0 && m.db < r0 + NR;
  double t[2] = {0.0, 0.0};  // u^T Y v, (Y v)_db
  if (k < NP) {
    t[0] = fma(acc.y, g.v.y, acc.x * g.v.x);
    if (owner) {
      const double2 yd = ld2(Y + m.db * NP + k);
      t[1] = fma(yd.y, g.v.y, yd.x * g.v.x);
    }
  }
  const double ra = pick(acc, m.ua);
  const double s = warp_transpose_sum<2>(t, lane);  // lanes 0-15: sum of t[0]; lanes 16-31: sum of t[1]
  if (lane == 0) {
    scal[0] = s;
    scal[1] = ra;
    if (owner) scal[3] = Y[m.db * NP + m.ua];
  }
  if (lane == 16 && owner) scal[2] = s;
}

struct Pipe {
  uint32_t T0;                  // tiles issued before this pass (same value in every thread)
  int last_issued[kMaxStages];  // per stage: last tile index loaded (producer thread only), -1 if none
};

// Thread of warp 1 that issues the bulk loads; its Pipe::last_issued is the one that counts.
constexpr int kProducerThread = 32;

// Verification hook: walker 0 never issues load number skip_load (1-based over the launch), so the consumer's
// bounded wait on it runs out and the CTA takes its timeout path.  The load is not recorded as issued.
__device__ __forceinline__ bool skipped_load(const SCtx& c, uint32_t T) {
  return c.d.skip_load > 0 && c.w == 0 && T + 1 == (uint32_t)c.d.skip_load;
}
__device__ __forceinline__ int wait_polls(const SCtx& c) { return c.d.wait_polls > 0 ? c.d.wait_polls : (1 << 22); }

// Load of tile t (global index T) into its stage: the ticket first, so that a consumer waiting on the stage
// knows that the stage's previous load was consumed and the full barrier's next phase is this load's.
__device__ __forceinline__ void issue_tile(const SCtx& c, const Stream& sm, Pipe& pp, int t, uint32_t T) {
  const size_t NN = (size_t)c.d.Np * c.d.Np;
  const int s = (int)(T % sm.ST);
  if (skipped_load(c, T)) return;
  *(volatile int*)&sm.ticket[s] = (int)T;
  __threadfence_block();
  mbar_arrive_expect_tx(&sm.full[s], sm.tile_bytes);
  bulk_load(sm.stage + (size_t)s * NN, c.Yw + (size_t)t * NN, sm.tile_bytes, &sm.full[s]);
  pp.last_issued[s] = (int)T;
}

// Producer (one thread): the first min(ST, n_qp) loads of a pass at once (every stage was released in the
// previous pass and every store of that pass has completed: the consumer that issued it waited for it before
// the pass-ending barrier), then each further load as soon as the stage's previous tile is released.  The
// waits on a release give up after wait_polls polls, or when a consumer has aborted the pass.
__device__ __forceinline__ bool pass_produce(const SCtx& c, const Stream& sm, Pipe& pp, volatile int* abort_flag) {
  const int n = c.d.n_qp, ST = sm.ST, n0 = n < ST ? n : ST;
  fence_proxy_async_global();
  for (int t = 0; t < n0; t++) issue_tile(c, sm, pp, t, pp.T0 + t);
  const int polls = wait_polls(c);
  for (int t = ST; t < n; t++) {
    const uint32_t T = pp.T0 + t, Tp = T - ST;
    const int s = (int)(T % ST);
    bool released = false;
    for (int it = 0; it < polls && !released; it++) {
      released = mbar_try_wait(&sm.empty[s], (Tp / ST) & 1u);
      if (!released && *abort_flag) return false;
    }
    if (!released || *abort_flag) return false;
    issue_tile(c, sm, pp, t, T);
  }
  return true;
}

// Consumer side of a stage's ticket: true once the producer has posted tile T on it (bounded; gives up when
// the pass is aborted).
__device__ __forceinline__ bool wait_ticket(const Stream& sm, int st, uint32_t T, int polls, volatile int* abort_flag) {
  for (int it = 0; it < polls; it++) {
    if (*(volatile int*)&sm.ticket[st] == (int)T) {
      __threadfence_block();
      return true;
    }
    if (*abort_flag) return false;
    __nanosleep(32);
  }
  return false;
}

// Control warp, proposal pass: the candidate (thread 0), published to the pairs at once; then, while the
// pairs work, theta', sgn' and the cosh products on the warp, and the weight psi_wo_pf of every projection
// into psip (the pass's end multiplies it by the new Pfaffian).  A failed candidate search is published too:
// the pairs read the status.
__device__ __forceinline__ void control_propose(const SCtx& c, volatile int* cand_flag, int pass_id, int* mv) {
  const DevDims& d = c.d;
  const WS& s = c.s;
  const int lane = threadIdx.x & 31;
  if (lane == 0) {
    candidate_search(c);
    if (!status(c)) {
      const int i1 = s.iflag[F_I1], i2 = s.iflag[F_I2];
      const int i3 = s.cfg[i1], i4 = s.cfg[i2];
      if (s.x[i1] == 1) {
        mv[0] = i3;
        mv[1] = i4 - d.Np;
        mv[2] = i1;
        mv[3] = i2;
      } else {
        mv[0] = i4;
        mv[1] = i3 - d.Np;
        mv[2] = i2;
        mv[3] = i1;
      }
    }
    __threadfence_block();
    *cand_flag = pass_id;
  }
  __syncwarp();
  if (status(c)) return;
  const int i1 = s.iflag[F_I1], i2 = s.iflag[F_I2];
  // update_theta RBM.f90:95-148 and the new signs (make_sample.f90:195-197) on the warp
  const int A2 = 2 * d.alphar;
  const double x1 = (double)s.x[i1], x2 = (double)s.x[i2];
  for (int j = lane; j < d.Mr; j += 32) {
    int mp = j / A2, rem = j - mp * A2;
    double sg = rem < d.alphar ? 1.0 : -1.0;
    int f = rem < d.alphar ? rem : rem - d.alphar;
    const double* Wf = c.p.Wr + (size_t)f * d.N;
    int iw1 = c.t.wmap[(size_t)mp * d.N + i1], iw2 = c.t.wmap[(size_t)mp * d.N + i2];
    double v = s.th[j];
    v = v - 2.0 * Wf[iw1] * x1 * sg;
    v = v - 2.0 * Wf[iw2] * x2 * sg;
    s.thp[j] = v;
  }
  const int flipsign = (c.t.subB[i1] ? -1 : 1) * (c.t.subB[i2] ? -1 : 1);
  for (int mp = lane; mp < d.n_mp; mp += 32) s.sgnp[mp] = -s.sgn[mp] * flipsign;
  __syncwarp();
  for (int qp = lane; qp < d.n_qp; qp += 32) {
    double r = 1.0;
    for (int f = 0; f < d.alphar; f++) r = r * cosh(s.thp[qp * d.alphar + f]);
    s.rbm[qp] = r;
    const cplx cw = psi_wo_pf(d, c.t, r, s.sgnp[qp >> 1], qp);
    s.psip[2 * qp] = cw.re;
    s.psip[2 * qp + 1] = cw.im;
  }
}

// Pairs: deferred update (pend) and/or proposal ratio (prop) per tile.  Pair g takes tiles g, g + kPairs, ...
// Every warp of a pair reaches the same pair barriers in the same order, and a failure (a bounded wait that
// ran out, an abort) is agreed at those barriers, so both warps leave together.
template <int KPL, int NP>
__device__ __forceinline__ bool pass_consume(const SCtx& c, const Stream& sm, const Pipe& pp, bool pend,
                                             const Move& mk, bool prop, volatile int* cand_flag, int pass_id,
                                             const int* mv, volatile int* abort_flag) {
  const DevDims& d = c.d;
  const WS& s = c.s;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, Np = NP, n = d.n_qp;
  const int cw = warp - 2, g = cw >> 1, h = cw & 1, partner = 2 + 2 * g + (1 - h);
  const int polls = wait_polls(c);
  const size_t NN = (size_t)Np * Np;
  double* u = s.wu + (size_t)warp * Np;
  double* U0 = s.wA + (size_t)warp * Np;
  double* V0 = s.wv + (size_t)warp * Np;
  double* my_acc = s.wS + (size_t)warp * Np;
  const double* other_acc = s.wS + (size_t)partner * Np;
  double* pAS = sm.pAS + (size_t)g * 2 * Np;
  double* pscal = sm.pscal + (size_t)g * 16;
  UV gk, gn;
  Move mn{0, 0, 0, 0};
  bool have_move = false, stored = false;
  int slot = 0;
  int t = g;
  if (pend && t < n) gather_regs<NP>(d, c.p, t, s.idx, mk, gk);
  for (; t < n; t += kPairs) {
    const uint32_t T = pp.T0 + t;
    const int st = (int)(T % sm.ST);
    const int tn = t + kPairs;
    double ck = 0.0;
    if (pend) {
      store_uv<NP>(gk, U0, V0);
      ck = gk.c;
      if (tn < n) gather_regs<NP>(d, c.p, tn, s.idx, mk, gk);
    }
    __syncwarp();
    bool bad = (*abort_flag != 0) || !wait_ticket(sm, st, T, polls, abort_flag) ||
               !mbar_wait(&sm.full[st], (T / sm.ST) & 1u, polls);
    double* Y = sm.stage + (size_t)st * NN;
    if (pend) {
      if (update_half<NP>(Y, mk, ck, U0, V0, g, h, my_acc, other_acc, pAS, bad)) return false;
      fence_proxy_async_smem();
    }
    double* sc = pscal + slot * 8 + h * 4;
    double cn = 0.0;
    if (prop && !bad) {
      if (!have_move) {
        bool ok = false;
        for (int it = 0; it < (1 << 24); it++) {
          if (*cand_flag == pass_id) {
            ok = true;
            break;
          }
          if (*abort_flag) break;
          __nanosleep(64);
        }
        __syncwarp();
        __threadfence_block();
        if (!ok || status(c)) bad = true;
        if (!bad) {
          mn = Move{mv[0], mv[1], mv[2], mv[3]};
          have_move = true;
          gather_regs<NP>(d, c.p, t, s.idx, mn, gn);
        }
      }
      if (!bad) {
        store_u<NP>(gn, u);
        cn = gn.c;
        __syncwarp();
        ratio_half<NP>(Y, mn, u, gn, h, sc);
        if (tn < n) gather_regs<NP>(d, c.p, tn, s.idx, mn, gn);
      }
    }
    if (pair_sync_or(g, bad)) return false;
    if (h == 0 && lane == 0) {
      if (prop) {
        const double* s0 = pscal + slot * 8;
        const double* s1 = s0 + 4;
        const double* so = (mn.db < NP / 2) ? s0 : s1;
        const double wv = s0[0] + s1[0], ra = s0[1] + s1[1];
        const double R = ra * so[2] - so[3] * (wv - cn);
        s.pfp[t] = R * s.pf[t];
      }
      if (pend) {  // write the updated tile back; the stage is released once the copy has read it
        bulk_store(c.Yw + (size_t)t * NN, Y, sm.tile_bytes);
        bulk_commit();
        bulk_wait_read_all();
        stored = true;
      }
      mbar_arrive(&sm.empty[st]);
    }
    slot ^= 1;
  }
  if (lane == 0 && stored) {  // the next pass reloads these tiles: their stores must have landed
    bulk_wait_all();
    fence_proxy_async_global();
  }
  __syncwarp();
  return true;
}

// One pass over all projections (all threads).  prop: evaluate a new proposal (control warp draws
// it); pend: apply the deferred update of the previously accepted exchange mk.
template <int KPL, int NP>
__device__ __forceinline__ void run_pass(const SCtx& c, const Stream& sm, Pipe& pp, bool pend, const Move& mk,
                                         bool prop, volatile int* cand_flag, int pass_id, int* mv,
                                         volatile int* abort_flag) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const WS& s = c.s;
  bool ok = true;
  if (warp == 0) {
    if (prop) control_propose(c, cand_flag, pass_id, mv);
  } else if (warp == 1) {
    if (lane == 0) ok = pass_produce(c, sm, pp, abort_flag);
  } else {
    ok = pass_consume<KPL, NP>(c, sm, pp, pend, mk, prop, cand_flag, pass_id, mv, abort_flag);
  }
  if (!ok) {
    *abort_flag = 1;
    if (!status(c)) status(c) = ST_TIMEOUT;
    bulk_wait_all();  // this thread's stores in flight, if any
  }
  __syncthreads();
  // psi' = sum over projections of weight x new Pfaffian (sub.f90:47-70), each lane over every 32nd projection
  if (prop && warp == 0 && !status(c)) {
    double re = 0.0, im = 0.0;
    for (int t = lane; t < c.d.n_qp; t += 32) {
      const double pf = s.pfp[t];
      const double a = s.psip[2 * t] * pf, b = s.psip[2 * t + 1] * pf;
      s.psip[2 * t] = a;
      s.psip[2 * t + 1] = b;
      re += a;
      im += b;
    }
    re = warp_sum(re);
    im = warp_sum(im);
    if (lane == 0) {
      s.dsc[D_PSIPR] = re;
      s.dsc[D_PSIPI] = im;
    }
  }
  if (prop) __syncthreads();
  pp.T0 += (uint32_t)c.d.n_qp;
}

// all stores of this CTA performed and visible to generic accesses of Y
__device__ __forceinline__ void drain(const SCtx& c) {
  if (threadIdx.x == 0) {
    bulk_wait_all();
    fence_proxy_async_global();
  }
  __syncthreads();
}

template <int KPL, int NP>
__global__ void __launch_bounds__(kWarps * 32, 1)
    sampler_stream_kernel(const __grid_constant__ DevDims d, const __grid_constant__ DevTables t,
                          const __grid_constant__ DevParams p, const __grid_constant__ DevWalkers W, int first,
                          int ST) {
  extern __shared__ __align__(128) char smem[];
  __shared__ WS ws;
  __shared__ Stream sm;
  __shared__ int pend_s[5];
  __shared__ int mv[4];
  __shared__ int abort_flag, cand_flag;
  const int tid = threadIdx.x;
  if (tid == 0) {
    stream_layout(d, ST, smem, &ws, &sm);
    for (int k = 0; k < ST; k++) {
      mbar_init(&sm.full[k], 1);
      mbar_init(&sm.empty[k], 1);
      sm.ticket[k] = -1;
    }
    fence_mbar_init();
    pend_s[0] = 0;
    abort_flag = 0;
    cand_flag = -1;
  }
  __syncthreads();
  // from-scratch recomputes invert up to kWarps - 1 projections in parallel, one per tile of the stage area
  const size_t gj_tile = (size_t)d.Np * (d.Np + 1) * 8;
  const size_t area = (size_t)sm.ST * sm.tile_bytes > gj_tile ? (size_t)sm.ST * sm.tile_bytes : gj_tile;
  int ntile = (int)(area / gj_tile);
  ntile = ntile < kWarps - 1 ? ntile : kWarps - 1;
  const SCtx c{d, t, p, W, (int)blockIdx.x, ws, W.Y + (size_t)blockIdx.x * d.n_qp * d.Np * d.Np, sm.stage,
               ntile >= 2 ? ntile : 0};
  const WS& s = ws;
  const int w = c.w, N = d.N;
  Pipe pp;
  pp.T0 = 0;
  for (int k = 0; k < kMaxStages; k++) pp.last_issued[k] = -1;
  int pass_id = 0;

  for (int k = tid; k < 625; k += blockDim.x) s.mt[k] = W.mt[(size_t)w * 625 + k];
  if (tid == 0) {
    status(c) = 0;
    events_reset(s);
  }
  __syncthreads();
  int nfastup = W.nfastup[w];

  if (first) {
    make_initial_x<KPL, NP>(c);
  } else {
    for (int i = tid; i < N; i += blockDim.x) s.x[i] = W.xs[((size_t)w * d.ns + (d.ns - 1)) * N + i];
    __syncthreads();
    full_state<KPL, NP>(c);
    if (!status(c)) {
      if (tid == 0) {
        s.iflag[F_AUX] = grnd(s.mt) < 0.05;  // make_sample.f90:61
        s.iflag[F_EV_RESEED] += s.iflag[F_AUX];
        if (s.iflag[F_AUX] && W.trace) trace_rec(c, 3, 0.0, 0.0, 0.0, 0.0, 0.0);
      }
      __syncthreads();
      if (s.iflag[F_AUX]) make_initial_x<KPL, NP>(c);
    }
  }
  int naccept = 0, nacc_tmp = 0, nacc_all = 0;
  for (int i0 = -d.nwarm; i0 <= d.ns && !status(c); i0++) {
    if (nacc_tmp > nfastup) {
      if (pend_s[0]) {  // apply the deferred update before the drift check
        const Move mk{pend_s[1], pend_s[2], pend_s[3], pend_s[4]};
        run_pass<KPL, NP>(c, sm, pp, true, mk, false, &cand_flag, ++pass_id, mv, &abort_flag);
        if (tid == 0) pend_s[0] = 0;
      }
      drain(c);
      if (status(c)) break;
      checkpoint<KPL, NP>(c, nfastup, i0);
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
        drain(c);
        global_flip<KPL, NP>(c);
        if (status(c)) break;
        if (tid == 0 && s.iflag[F_ACCEPT]) pend_s[0] = 0;  // Y recomputed for the flipped state
        __syncthreads();
      }
      const bool pend = pend_s[0] != 0;
      const Move mk{pend_s[1], pend_s[2], pend_s[3], pend_s[4]};
      run_pass<KPL, NP>(c, sm, pp, pend, mk, true, &cand_flag, ++pass_id, mv, &abort_flag);
      if (status(c)) break;
      const int i1 = s.iflag[F_I1], i2 = s.iflag[F_I2];
      const int i3 = s.cfg[i1], i4 = s.cfg[i2];
      if (tid == 0) {
        const double re = s.dsc[D_PSIPR], im = s.dsc[D_PSIPI];
        (void)grnd(s.mt);  // sub.f90:72
        double r1 = (hypot(re, im) + d.shift) / (hypot(s.dsc[D_PSI0R], s.dsc[D_PSI0I]) + d.shift);
        const double u = grnd(s.mt);
        s.iflag[F_ACCEPT] = u < r1 * r1;  // make_sample.f90:203-204
        if (W.trace) trace_rec(c, 0, (double)i1, (double)i2, r1 * r1, u, (double)s.iflag[F_ACCEPT]);
      }
      __syncthreads();
      if (s.iflag[F_ACCEPT]) {  // make_sample.f90:205-219; the Y update is deferred to the next pass
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
          pend_s[0] = 1;
          pend_s[1] = mv[0];
          pend_s[2] = mv[1];
          pend_s[3] = mv[2];
          pend_s[4] = mv[3];
        }
        if (i0 > 0) naccept++;
        nacc_tmp++;
        nacc_all++;
      } else if (tid == 0) {
        pend_s[0] = 0;  // a deferred update, if any, was applied and stored by this pass
      }
      __syncthreads();
    }
    if (status(c)) break;
    if (i0 > 0) {  // make_sample.f90:228-232
      size_t sidx = (size_t)w * d.ns + (i0 - 1);
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
  if (!status(c) && pend_s[0]) {  // leave Y consistent with the final state
    const Move mk{pend_s[1], pend_s[2], pend_s[3], pend_s[4]};
    run_pass<KPL, NP>(c, sm, pp, true, mk, false, &cand_flag, ++pass_id, mv, &abort_flag);
  }
  // every bulk copy of this CTA has landed before the CTA exits (bounded waits)
  if (tid == kProducerThread)
    for (int k = 0; k < sm.ST && k < kMaxStages; k++)
      if (pp.last_issued[k] >= 0) (void)mbar_wait(&sm.full[k], ((uint32_t)pp.last_issued[k] / sm.ST) & 1u);
  bulk_wait_all();
  __syncthreads();
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

}  // namespace

// Stage count and shared memory of the streaming sampler; 0 when it does not apply.
int rbmpp_stream_stages(const DevDims& d, int max_smem) {
  // As many stages as fit, up to two per pair (a pair's next tile then loads while it computes the
  // current one) and no more than there are projections; at least one per pair, else the direct sampler
  // takes the shape.  The stage tickets keep the mbarrier phases unambiguous for any count.
  if (d.Np != 8 && d.Np != 18 && d.Np != 32 && d.Np != 50) return 0;  // the compiled block sizes
  int hi = 2 * kPairs < kMaxStages ? 2 * kPairs : kMaxStages;
  if (d.n_qp < hi) hi = d.n_qp;
  const int lo = d.n_qp < kPairs ? d.n_qp : kPairs;
  for (int st = hi; st >= lo; st--)
    if ((long long)stream_layout(d, st, nullptr, nullptr, nullptr) <= max_smem) return st;
  return 0;
}

size_t rbmpp_stream_smem(const DevDims& d, int st) { return stream_layout(d, st, nullptr, nullptr, nullptr); }

cudaError_t rbmpp_launch_sampler_stream(const DevDims& d, const DevTables& t, const DevParams& p, const DevWalkers& W,
                                        int first, int st, cudaStream_t stream) {
  size_t smem = rbmpp_stream_smem(d, st);
#define LAUNCH(K, NPC)                                                                                        \
  do {                                                                                                        \
    cudaError_t e = cudaFuncSetAttribute(sampler_stream_kernel<K, NPC>,                                       \
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);             \
    if (e != cudaSuccess) return e;                                                                           \
    rbmpp_note_launch(); sampler_stream_kernel<K, NPC><<<d.nw, kWarps * 32, smem, stream>>>(d, t, p, W, first, st); \
    return cudaGetLastError();                                                                                \
  } while (0)
  switch (d.Np) {  // block sizes of the even-L lattices with a compile-time specialisation
    case 8: LAUNCH(1, 8);
    case 18: LAUNCH(1, 18);
    case 32: LAUNCH(1, 32);
    case 50: LAUNCH(2, 50);
    default: break;
  }
#undef LAUNCH
  return cudaErrorInvalidValue;
}

/*
 * rbmpp.h -- C ABI of the B200 (sm_100a) implementation of RBM_PP's variational-Monte-Carlo hot path
 * (Metropolis sampling with Pfaffian fast updates, local energy, O_k, stochastic reconfiguration).
 *
 * Conventions
 *  - Plain C types only.  Every array argument is a HOST pointer to a column-major array with the
 *    Fortran layout of the reference's module variable it replaces (module.f90), 1-based index values
 *    where the reference stores indices (W_map, Orbital_Idx).  Complex values are (re, im) pairs.
 *  - The library owns all device memory.  One host thread drives one context.
 *  - Every call returns 0 on success or an RBMPP_E_* code naming the violated invariant (the
 *    reference `stop`s on the same conditions); rbmpp_last_error() returns the message.
 *  - Emulated MPI ranks are "walkers": walker w behaves exactly like rank w of the reference
 *    (own MT19937 stream seeded iseed0 + w, own Nfastup, Nsample/Nmpi stored samples).
 *
 * Reference-side binding: a Fortran ISO_C_BINDING interface block over these functions replaces the
 * bodies of make_sample, calc_phys_quantity_opt and the SR_pdposv include.
 */
#ifndef RBMPP_H
#define RBMPP_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rbmpp_ctx rbmpp_ctx;

enum {
  RBMPP_OK = 0,
  RBMPP_E_ARG = 1,          /* bad argument / unsupported configuration                          */
  RBMPP_E_CONFIG = 2,       /* x / Ele_Idx / Ele_Cfg bookkeeping (interface_for_PP.f90:26-65)     */
  RBMPP_E_SIGN = 3,         /* sign_PP inconsistency (interface_for_PP.f90:101-103)               */
  RBMPP_E_THETA = 4,        /* theta drift > 1e-5 (make_sample.f90:84-89)                          */
  RBMPP_E_CANDIDATE = 5,    /* exchange-candidate search exhausted (make_sample.f90:290-291)      */
  RBMPP_E_INITX = 6,        /* make_initial_x fails (make_sample.f90:337,359)                     */
  RBMPP_E_SKEW = 7,         /* Slater_Elm / InvM skew checks (slater.f90:51-56, matrix.f90:103)    */
  RBMPP_E_SINGULAR = 8,     /* singular Pfaffian matrix (matrix.f90:145-148,171-174)              */
  RBMPP_E_SDIAG = 9,        /* S-matrix diagonal checks (SR_pdposv.f90:32-33,78-100,140)           */
  RBMPP_E_CHOL = 10,        /* Cholesky breakdown (pdposv info /= 0, SR_pdposv.f90:233-236)       */
  RBMPP_E_SLATER_NORM = 11, /* f renormalisation check (SR_pdposv.f90:414)                        */
  RBMPP_E_LAMBDA = 12,      /* lambda block split check (SR_pdposv.f90:308)                       */
  RBMPP_E_CUDA = 20,        /* CUDA runtime error                                                 */
  RBMPP_E_STATE = 21,       /* call out of order (e.g. measure before make_sample)                */
  RBMPP_E_TIMEOUT = 22,     /* a bounded device-side wait ran out (copy pipeline did not progress) */
  RBMPP_E_COMM = 23         /* the host all-reduce of rbmpp_set_allreduce returned non-zero         */
};

/* Sizes (RBM.input, sym_info.txt, orbitalidx.def; main.f90:75-141). */
typedef struct {
  int L;            /* linear lattice size; N = L*L sites (main.f90:85)                          */
  int n_mp_trans;   /* N_MP_Trans: number of symmetry operations in sym_info.txt (main.f90:91)  */
  int alphac;       /* complex RBM density; must be 0 (real-RBM branch)                          */
  int alphar;       /* real RBM density                                                           */
  int n_slater;     /* N_Slater (orbitalidx.def, main.f90:128)                                    */
  int nsample;      /* stored samples per walker = Nsample/Nmpi (main.f90:138)                    */
  int n_walkers;    /* number of emulated ranks                                                   */
  int spin_parity;  /* +1 / -1 (spin_projection.f90:56-62)                                        */
  double J1, J2;    /* couplings (main.f90:83)                                                    */
  int device;       /* CUDA device ordinal                                                        */
  int walker_offset;/* global rank of walker 0 (multi-GPU sharding: rank r holds walkers r*n_walkers..) */
} rbmpp_dims;

/* Inputs of one SR step (main.f90 locals used by the SR_pdposv.f90 include). */
enum { RBMPP_SR_FP64 = 0, RBMPP_SR_SPLIT_BF16 = 1 };
typedef struct {
  int iteration;      /* optimisation step (1-based)                                             */
  int precision;      /* RBMPP_SR_FP64: FP64 S build; RBMPP_SR_SPLIT_BF16: 3-term split-BF16 S on the
                         tensor cores + FP64 Cholesky, refined against the exact S                 */
  int refine_steps;   /* RBMPP_SR_SPLIT_BF16: at most this many conjugate-gradient iterations on the
                         exact FP64 S (applied through O), preconditioned by the split-precision
                         Cholesky factor; they stop at relative residual 1e-13.  0 = no refinement */
  int reserved;
  double delta_tau;   /* RBM.input                                                               */
  double s_factor0;   /* current stabilisation factor (main.f90:439 schedule applied by caller)   */
  double s_cut;       /* RBM.input                                                               */
} rbmpp_sr_in;

typedef struct {
  double Etot, Etot2, norm, wf_av;   /* normalised as in main.f90:351-361                        */
  double accept_ratio;               /* main.f90:349                                              */
  double lambda;                     /* step norm after the 5/L scaling (SR_pdposv.f90:309)       */
  double lambda_rbm_rbm, lambda_pp_pp, lambda_rbm_pp;
  double delW_max, s_factor, sdiag_av, smat_scaling;
  double refine_residual;            /* relative residual ||g - S x|| / ||g|| against the exact S
                                        (RBMPP_SR_SPLIT_BF16 with refinement; 0 otherwise)      */
  double precond_shift;              /* extra diagonal added to the split-precision S before its
                                        Cholesky when S + shift was not positive definite at
                                        working precision (0 when none was needed)              */
  int kmax, k_nonzero, nSmat;
  int refine_iterations;             /* conjugate-gradient iterations taken                       */
} rbmpp_sr_out;

/* Lifecycle -------------------------------------------------------------------------------- */
int rbmpp_create(const rbmpp_dims* dims, rbmpp_ctx** out);
int rbmpp_destroy(rbmpp_ctx* ctx);
const char* rbmpp_last_error(const rbmpp_ctx* ctx);
/* what: 0 = Nv, 1 = Nv_RBM, 2 = Mr, 3 = N_QP_Full, 4 = N, 5 = device bytes held,
 * 6 = kernel launches issued by the library so far (all contexts of the process) */
int rbmpp_query(const rbmpp_ctx* ctx, int what, long long* value);

/* Tables: W_map(N, 1, N_MP_Trans) (main.f90:94-122; also MP_Trans_Idx, parameter.f90:105-109),
 * para_mp_trans(N_MP_Trans) complex, Orbital_Idx(N,N) (parameter.f90:88-100),
 * Orbital_Sgn(N,N) or NULL (all +1; l_AP = .false.),
 * subB(N) = 1 for sites of sublattice B, 0 otherwise (subB_or_not, define_sublattice interface_for_PP.f90:110-136)
 * or NULL (derived: site i = i2 L + i1 + 1 is on B when i1 + i2 is odd),
 * sp_weights(3, 2) = {SP_GL_Cos, SP_GL_Sin, para_spin_proj} of the two spin-projection points
 * (InitSPWeight, spin_projection.f90:5-79) or NULL (beta = 0 and pi, para_spin_proj = (1, spin_parity)).
 * Where SP_GL_Cos * SP_GL_Sin vanishes (relative 1e-12) at both points, the Pfaffian matrix is block
 * off-diagonal and the library carries its Np x Np up-down block; otherwise (the transverse code's
 * beta = -pi/2, pi/2 with sqrt(2)-scaled weights, transverse_code/spin_projection.f90:30-38) it carries the full
 * N x N skew matrix (N <= 128), and rbmpp_iteration uses the transverse shift schedule
 * (transverse_code/main.f90:451).  The skew form has no batched sampler, no correlation measurement and no
 * allocation-free evaluation.
 * Replaces the module setup of main.f90:89-300. */
int rbmpp_set_tables(rbmpp_ctx* ctx, const int* W_map, const double* para_mp_trans, const int* Orbital_Idx,
                     const int* Orbital_Sgn, const int* subB, const double* sp_weights);

/* Parameters: Wrirr(N, alphar), brirr(alphar), Slater(N_Slater), shift (module.f90 mod_RBM, mod_PP,
 * mod_main); Wcirr(N, alphac), bcirr(alphac) complex as (re, im) pairs or NULL (kept).  Also rebuilds
 * Slater_Elm on the device (update_slater_elements, slater.f90:7-64). */
int rbmpp_set_params(rbmpp_ctx* ctx, const double* Wr, const double* br, const double* Wc, const double* bc,
                     const double* Slater, double shift);
int rbmpp_get_params(rbmpp_ctx* ctx, double* Wr, double* br, double* Slater, double* shift);
/* Complex RBM parameters Wcirr(N, alphac), bcirr(alphac) (complex, as (re, im) pairs) after SR steps; set them with
 * rbmpp_set_params' Wc and bc.  Complex units (RBM.f90 thetac; sub.f90:37-41 multiplies psi_x_wo_pf by
 * 0.5^alphac prod cosh(thetac)) make psi complex: O then has two rows per sample as with complex para_mp_trans, and
 * the parameters are ordered as main.f90:136 and SR_pdposv.f90:385-413 order them (complex pairs first). */
int rbmpp_get_params_c(rbmpp_ctx* ctx, double* Wc, double* bc);
/* Sets mod_main's shift alone (main.f90:451), keeping the other parameters. */
int rbmpp_set_shift(rbmpp_ctx* ctx, double shift);
/* Precision of S builds that happen before rbmpp_sr_step names one: rbmpp_measure with Smat != NULL and
 * rbmpp_exchange_measurement (RBMPP_SR_FP64 default, or RBMPP_SR_SPLIT_BF16).  rbmpp_sr_step builds S
 * in its own in->precision when no S exists yet.  Replaces the dgemm of calc_phys_quantity.f90:240. */
int rbmpp_set_s_precision(rbmpp_ctx* ctx, int precision);

/* RNG: walker w (global rank g = walker_offset + w) is seeded sgrnd(iseed0 + g) and skips
 * Nsample*g + 1 draws (main.f90:224-234). */
int rbmpp_seed_walkers(rbmpp_ctx* ctx, int iseed0);
/* n draws from walker 0's stream (rank 0's draws in initialize_parameters, parameter.f90:21-41). */
int rbmpp_rank0_grnd(rbmpp_ctx* ctx, int n, double* out);

/* make_sample(myrank, first_iteration, naccept) for every walker (make_sample.f90:4-240).
 * naccept: per-walker counts (n_walkers ints) or NULL; naccept_total: sum or NULL. */
int rbmpp_make_sample(rbmpp_ctx* ctx, int first_iteration, int* naccept, long long* naccept_total);
/* x_sample(N, Nsample, n_walkers), psi_x_sample(0:N_QP, Nsample, n_walkers) complex,
 * PfM_sample(N_QP, Nsample, n_walkers); any pointer may be NULL (mod_sample, module.f90:37-42). */
int rbmpp_get_samples(rbmpp_ctx* ctx, int* x_sample, double* psi_x_sample, double* PfM_sample);
int rbmpp_set_samples(rbmpp_ctx* ctx, const int* x_sample);

/* calc_phys_quantity_opt (calc_phys_quantity.f90:20-246) over all walkers, summed as the MPI
 * reductions of main.f90:348-369 do (before division by norm): scal = {Etot, Etot2, norm, wf_av}.
 * gvec, Ovec (Nv) and Smat (Nv x Nv, = sum O O^T) are copied to the host when non-NULL; they also
 * stay on the device for rbmpp_sr_step. */
int rbmpp_measure(rbmpp_ctx* ctx, double* scal, double* gvec, double* Ovec, double* Smat);
/* calc_phys_quantity_after_opt (calc_phys_quantity.f90:250-302): scal = {Etot, Etot2, norm, wf_av}. */
int rbmpp_measure_energy(rbmpp_ctx* ctx, double* scal);
/* calc_phys_quantity_after_opt of the Calc_Correlation program (Calc_Correlation/calc_phys_quantity.f90:264-344,
 * with calc_local_energy_correlation :348-424 and calc_local_correlation :477-550) over all walkers, summed as
 * the MPI_REDUCE calls of Calc_Correlation/main.f90:553-581 (before division by norm):
 * scal = {Etot, Etot2, norm, wf_av, Re wf_sgn}; chi_sp = Chi_sp(2, Nchi) (SzSz, exchange part) and
 * chi_vbs = Chi_vbs(Nchi, 4) (bond types (1,0), (0,1), (1,1), (1,-1)), column-major, Nchi = N (N + 1) / 2,
 * pair i0 = i2 (i2 - 1) / 2 + i1 for 1 <= i1 <= i2 <= N.  Any pointer may be NULL.  Each walker's stream
 * advances by one draw per sample, antiparallel bond and antiparallel site pair, as the reference's
 * amplitude calls do (sub.f90:72). */
int rbmpp_measure_correlation(rbmpp_ctx* ctx, double* scal, double* chi_sp, double* chi_vbs);

/* Cross-GPU reduction of the measurement (the MPI_ALLREDUCE calls of main.f90:348-369).
 * direction 0: copy this context's sums into caller DEVICE buffers d_S (Nv*Nv), d_g, d_ov (Nv) and
 *              host scal6 = {Etot, Etot2, norm, wf_av, naccept_total, n_samples};
 * direction 1: load reduced sums (same layout) back for rbmpp_sr_step. */
int rbmpp_exchange_measurement(rbmpp_ctx* ctx, int direction, double* d_S, double* d_g, double* d_ov, double* scal6);

/* Cross-rank sums done by the library itself, through a host-supplied all-reduce: fn(user, buf, n) must sum
 * n doubles at the DEVICE address buf over all ranks, in place, and return 0 when the result is in buf (the
 * library's stream is synchronised before the call and its next launch follows the return).  Every rank
 * must get bit-identical sums (NCCL and MPI all-reduces do).  With it set:
 *  - rbmpp_measure reduces {Etot, Etot2, norm, wf_av, naccept_total, n_samples}, gvec and Ovec in one call,
 *    and rbmpp_measure_energy the scalars: the MPI_ALLREDUCE calls of main.f90:348-369;
 *  - the S build reduces each rank's S (Nv x Nv): S_raw in FP64, or, in split-BF16, the centred product of the
 *    rank's samples about the global mean plus the exact FP64 diagonal, before the global mean is added back;
 *  - the split-BF16 refinement reduces O^T (O x) (Nv doubles) once per conjugate-gradient iteration, so it
 *    runs on the exact S of all ranks' samples (SR_pdposv.f90:232 distributed as pdposv is);
 *  - rbmpp_exchange_measurement is refused (the context reduces by itself).
 * Every rank then takes identical SR steps (the parameter broadcast of main.f90:427-438 is not needed).
 * fn = NULL switches it off. */
typedef int (*rbmpp_allreduce_fn)(void* user, double* buf, long long n);
int rbmpp_set_allreduce(rbmpp_ctx* ctx, rbmpp_allreduce_fn fn, void* user);

/* SR block (SR_pdposv.f90:1-432 with the normalisation of main.f90:351-369) on the device-resident
 * measurement of the last rbmpp_measure; replaces pdposv.  Updates the parameters in place.
 * dx (Nv, nullable) receives the SR direction after scaling (gvec at SR_pdposv.f90:327). */
int rbmpp_sr_step(rbmpp_ctx* ctx, const rbmpp_sr_in* in, rbmpp_sr_out* out, double* dx);

/* One optimisation iteration of main.f90:311-453: update_slater_elements, make_sample, measure,
 * reductions, SR step, and the s_factor0 / shift bookkeeping (main.f90:439-453), which the
 * context keeps between calls.  s_factor_scale multiplies s_factor0 after the step. */
int rbmpp_iteration(rbmpp_ctx* ctx, int precision, double delta_tau, double s_factor_scale, double s_cut,
                    double s_factor0_initial, rbmpp_sr_out* out);

/* Device-side statistics of the last calls, timed with CUDA events on the library's stream:
 * out[0] make_sample kernel ms, [1] estimator kernel ms, [2] gvec/Ovec GEMV ms, [3] S build ms,
 * [4] Cholesky factor(s) + first solve ms, [5] accepted moves in all sweeps of the last make_sample,
 * [6] proposals of the last make_sample, [7] last rbmpp_iteration ms, [8] refinement ms (conjugate
 * gradients on the exact S and the final lambda products), [9] Cholesky attempts of the last SR step.
 * n = number of entries wanted (at most 10). */
int rbmpp_get_stats(const rbmpp_ctx* ctx, double* out, int n);

/* Copies the whole sampling state of src into dst (same shape, same device, tables set on both): every
 * walker's configuration, inverse blocks, amplitudes, random stream, Nfastup and stored samples, the
 * parameters and shift, and the iteration bookkeeping of rbmpp_iteration.  dst then continues exactly as src
 * would (no counterpart in the reference, whose state is the rank's memory; used to run two SR variants
 * from one state). */
int rbmpp_copy_state(rbmpp_ctx* dst, const rbmpp_ctx* src);

/* Per-walker sampler state: Nfastup (adaptive recompute interval, make_sample.f90:120-127) and the
 * accepted moves of the last make_sample over all sweeps.  Either pointer may be NULL. */
int rbmpp_get_walker_state(const rbmpp_ctx* ctx, int* nfastup, int* naccept_all);

/* Per-walker diagnostics of the last make_sample (the events of make_sample.f90, recorded on the device).
 * events(5, n_walkers) = {global spin flips tried (:135), flips accepted (:145-157), make_initial_x re-seeds
 * of a continued chain (:61), Nfastup checkpoints (:74-128), trace records produced (possibly more than were
 * kept)}.  trace(6, max_records, n_walkers), filled when rbmpp_set_trace enabled it, lists the chain's
 * random decisions in draw order:
 *   {0, i1, i2, ratio^2, u, accepted}  exchange proposal of sites i1, i2 (0-based), accepted = u < ratio^2
 *                                      with ratio = (|psi'| + shift) / (|psi| + shift) (:160-220);
 *   {1, i0, inverse drift, Pf drift, Nfastup before, Nfastup after}  checkpoint at sweep i0 (:74-128; the
 *                                      inverse drift is measured on the Np x Np block inverse);
 *   {2, 0, 0, ratio^2, u, accepted}    global spin flip (:135-158);
 *   {3, 0, 0, 0, 0, 0}                 make_initial_x re-seed of a continued chain (:61).
 * Records beyond max_records are dropped.  Either pointer may be NULL. */
int rbmpp_get_walker_events(const rbmpp_ctx* ctx, int* events, double* trace);
/* Enables (max_records > 0) or disables (0) the per-walker chain trace of later make_sample calls. */
int rbmpp_set_trace(rbmpp_ctx* ctx, int max_records);
/* Verification replay (no counterpart in the reference): decisions(2, max_checkpoints, n_walkers) =
 * {Nfastup after, 1 if the extra draw of make_sample.f90:122 is taken} replace the drift test of the first
 * max_checkpoints checkpoints of each walker in later make_sample calls (the draw of :116 still happens).
 * It lets a chain follow another implementation's recompute schedule; 0 turns it off. */
int rbmpp_set_replay(rbmpp_ctx* ctx, const int* decisions, int max_checkpoints);
/* Verification hooks of the failure paths (no counterpart in the reference; off by default):
 * what 1: walker 0 of the streaming sampler never issues its bulk load number `value` (1-based, 0 = off), so
 *         the consumer's bounded wait on it runs out: make_sample returns RBMPP_E_TIMEOUT and the context
 *         stays usable (the next make_sample rebuilds every walker's state);
 * what 2: poll bound of the streaming sampler's pipeline waits (0 = the default, 2^22 polls). */
int rbmpp_debug_hook(rbmpp_ctx* ctx, int what, int value);

/* Adjoint O_k kernel: for n configurations x(N, n): psi(0:N_QP, n) complex, hpsi(n) complex
 * (sum_x' <x|H|x'> psi(x'), calc_local_energy_correlation), and O(Nv, n) = d psi(x) / d theta_k
 * (Ovec_loc_x before reweighting, calc_phys_quantity.f90:115-220).  With complex para_mp_trans, O is complex and
 * comes as O(Nv, 2, n): real part, then imaginary part, per configuration (the Ovec_Store columns of
 * calc_phys_quantity.f90:227-228).  Any output may be NULL. */
int rbmpp_eval_configs(rbmpp_ctx* ctx, int n, const int* x, double* psi, double* hpsi, double* O);

/* Batched sampling: one persistent launch over the walkers of several contexts on one device (different
 * lattice sizes L, couplings J1/J2 and parameters; the Pfaffian block size may differ per context).  No
 * counterpart in the reference, which runs one lattice per job.  Each context keeps its own walkers,
 * random streams and stored samples, exactly as its own rbmpp_make_sample would produce them. */
typedef struct rbmpp_batch rbmpp_batch;
int rbmpp_batch_create(rbmpp_ctx* const* ctxs, int n, rbmpp_batch** out);
int rbmpp_batch_destroy(rbmpp_batch* b);
const char* rbmpp_batch_last_error(const rbmpp_batch* b);
/* Autotuner: times probe launches (up to 8 walkers per context, 2 sweeps) for each block size in
 * {128, 256, 512} threads, measures every context's per-walker cost, and picks the block size and walker
 * order (context-major, round robin, or longest-first) with the smallest predicted makespan.  Call after
 * seeding and before the first rbmpp_batch_make_sample; the probed walkers' random streams and Nfastup
 * are restored.  Outputs (nullable): threads, order (0, 1, 2), probe time in ms of the chosen shape. */
int rbmpp_batch_tune(rbmpp_batch* b, int* threads, int* order, double* probe_ms);
/* make_sample (make_sample.f90:4-240) for every walker of every context in one launch;
 * naccept_total: per-context accepted moves of the stored sweeps (n values) or NULL. */
int rbmpp_batch_make_sample(rbmpp_batch* b, int first_iteration, long long* naccept_total);

/* rbmpp_eval_configs without any device allocation.  No counterpart in the reference: it exists for
 * callers that can't call cudaMalloc/cudaFree, such as a host code whose own pool allocator holds the
 * GPU's memory, or a loop that must not be stalled by cudaFree's device-wide wait.
 * x, psi, hpsi, O have the layouts of rbmpp_eval_configs but are DEVICE pointers on the context's
 * device, owned by the caller (psi, hpsi, O may be NULL).  Scratch comes from one fixed array of
 * about 2 MiB in the library's device image: at most 4096 configurations per call (more returns
 * RBMPP_E_ARG).  Each call looks up that array's device address on the context's device.  All calls share
 * the array, so calls whose GPU work overlaps race: issue them one at a time.  Returns after the results are
 * complete on the device. */
int rbmpp_eval_configs_noalloc(rbmpp_ctx* ctx, int n, const int* d_x, double* d_psi, double* d_hpsi, double* d_O);

#ifdef __cplusplus
}
#endif
#endif /* RBMPP_H */

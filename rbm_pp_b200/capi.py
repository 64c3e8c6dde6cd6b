"""ctypes binding of the C ABI in include/rbmpp.h (the CUDA library ``librbmpp.so``).

This is the host-side mirror of the reference's module interface for the sampling/SR loop:
``make_sample`` (make_sample.f90:4), ``calc_phys_quantity_opt`` (calc_phys_quantity.f90:20),
the SR_pdposv.f90 block, and the seeding/initialisation of main.f90:224-300.  There is no CPU
fallback: if the library is missing or no GPU is present, construction fails with an error.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librbmpp.so")
_lib = None

EXPORTS = ["rbmpp_create", "rbmpp_destroy", "rbmpp_last_error", "rbmpp_query", "rbmpp_set_tables",
           "rbmpp_set_params", "rbmpp_get_params", "rbmpp_seed_walkers", "rbmpp_rank0_grnd", "rbmpp_make_sample",
           "rbmpp_get_samples", "rbmpp_set_samples", "rbmpp_measure", "rbmpp_measure_energy", "rbmpp_sr_step",
           "rbmpp_iteration", "rbmpp_eval_configs", "rbmpp_get_stats", "rbmpp_exchange_measurement",
           "rbmpp_set_shift", "rbmpp_get_walker_state", "rbmpp_eval_configs_noalloc",
           "rbmpp_set_s_precision", "rbmpp_batch_create", "rbmpp_batch_destroy", "rbmpp_batch_last_error",
           "rbmpp_batch_tune", "rbmpp_batch_make_sample", "rbmpp_measure_correlation",
           "rbmpp_get_walker_events", "rbmpp_set_trace", "rbmpp_set_replay", "rbmpp_debug_hook",
           "rbmpp_copy_state", "rbmpp_set_allreduce", "rbmpp_get_params_c"]

SR_FP64 = 0
SR_SPLIT_BF16 = 1

# int (*)(void* user, double* device_buffer, long long n): the host all-reduce of rbmpp_set_allreduce
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_longlong)


def allreduce_callback(fn, on_error=None):
    """The C function pointer rbmpp_set_allreduce takes, around fn(pointer: int, n: int) -> None: returns 0,
    or 1 after an exception (passed to on_error)."""

    def _cb(user, ptr, n):
        try:
            fn(int(ptr), int(n))
            return 0
        except Exception as e:
            if on_error is not None:
                on_error(e)
            return 1

    return ALLREDUCE_FN(_cb)


class Dims(C.Structure):
    _fields_ = [("L", C.c_int), ("n_mp_trans", C.c_int), ("alphac", C.c_int), ("alphar", C.c_int),
                ("n_slater", C.c_int), ("nsample", C.c_int), ("n_walkers", C.c_int), ("spin_parity", C.c_int),
                ("J1", C.c_double), ("J2", C.c_double), ("device", C.c_int), ("walker_offset", C.c_int)]


class SrIn(C.Structure):
    _fields_ = [("iteration", C.c_int), ("precision", C.c_int), ("refine_steps", C.c_int), ("reserved", C.c_int),
                ("delta_tau", C.c_double), ("s_factor0", C.c_double), ("s_cut", C.c_double)]


class SrOut(C.Structure):
    _fields_ = [("Etot", C.c_double), ("Etot2", C.c_double), ("norm", C.c_double), ("wf_av", C.c_double),
                ("accept_ratio", C.c_double), ("lambda_", C.c_double), ("lambda_rbm_rbm", C.c_double),
                ("lambda_pp_pp", C.c_double), ("lambda_rbm_pp", C.c_double), ("delW_max", C.c_double),
                ("s_factor", C.c_double), ("sdiag_av", C.c_double), ("smat_scaling", C.c_double),
                ("refine_residual", C.c_double), ("precond_shift", C.c_double), ("kmax", C.c_int), ("k_nonzero", C.c_int), ("nSmat", C.c_int),
                ("refine_iterations", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class RbmppError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"rbmpp error {code}: {msg}")
        self.code = code


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RbmppError(-1, f"CUDA library not built: {LIB_PATH} (run rbm_pp_b200/build.py)")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.rbmpp_create.argtypes = [C.POINTER(Dims), C.POINTER(P)]
        L.rbmpp_destroy.argtypes = [P]
        L.rbmpp_last_error.restype = C.c_char_p
        L.rbmpp_last_error.argtypes = [P]
        L.rbmpp_query.argtypes = [P, C.c_int, C.POINTER(C.c_longlong)]
        L.rbmpp_set_tables.argtypes = [P, P, P, P, P, P, P]
        L.rbmpp_set_params.argtypes = [P, P, P, P, P, P, C.c_double]
        L.rbmpp_get_params.argtypes = [P, P, P, P, P]
        L.rbmpp_get_params_c.argtypes = [P, P, P]
        L.rbmpp_seed_walkers.argtypes = [P, C.c_int]
        L.rbmpp_rank0_grnd.argtypes = [P, C.c_int, P]
        L.rbmpp_make_sample.argtypes = [P, C.c_int, P, P]
        L.rbmpp_get_samples.argtypes = [P, P, P, P]
        L.rbmpp_set_samples.argtypes = [P, P]
        L.rbmpp_measure.argtypes = [P, P, P, P, P]
        L.rbmpp_measure_energy.argtypes = [P, P]
        L.rbmpp_measure_correlation.argtypes = [P, P, P, P]
        L.rbmpp_sr_step.argtypes = [P, C.POINTER(SrIn), C.POINTER(SrOut), P]
        L.rbmpp_iteration.argtypes = [P, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.POINTER(SrOut)]
        L.rbmpp_eval_configs.argtypes = [P, C.c_int, P, P, P, P]
        L.rbmpp_get_stats.argtypes = [P, P, C.c_int]
        L.rbmpp_exchange_measurement.argtypes = [P, C.c_int, P, P, P, P]
        L.rbmpp_set_shift.argtypes = [P, C.c_double]
        L.rbmpp_get_walker_state.argtypes = [P, P, P]
        L.rbmpp_get_walker_events.argtypes = [P, P, P]
        L.rbmpp_set_trace.argtypes = [P, C.c_int]
        L.rbmpp_set_replay.argtypes = [P, P, C.c_int]
        L.rbmpp_debug_hook.argtypes = [P, C.c_int, C.c_int]
        L.rbmpp_copy_state.argtypes = [P, P]
        L.rbmpp_set_allreduce.argtypes = [P, ALLREDUCE_FN, P]
        L.rbmpp_eval_configs_noalloc.argtypes = [P, C.c_int, P, P, P, P]
        L.rbmpp_set_s_precision.argtypes = [P, C.c_int]
        L.rbmpp_batch_create.argtypes = [P, C.c_int, C.POINTER(P)]
        L.rbmpp_batch_destroy.argtypes = [P]
        L.rbmpp_batch_last_error.restype = C.c_char_p
        L.rbmpp_batch_last_error.argtypes = [P]
        L.rbmpp_batch_tune.argtypes = [P, P, P, P]
        L.rbmpp_batch_make_sample.argtypes = [P, C.c_int, P]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f(a, dtype):
    return np.ascontiguousarray(np.asarray(a, dtype=dtype).reshape(-1, order="F"))


class Context:
    """One library context: ``n_walkers`` emulated MPI ranks on one GPU."""

    def __init__(self, problem, n_walkers: int, nsample_per_walker: int, device: int = 0, walker_offset: int = 0,
                 subB=None, sp_weights=None):
        self.p = problem
        inp = problem.inp
        self.N = inp.L * inp.L
        self.n_mp = problem.sym.n_mp
        self.n_qp = 2 * self.n_mp
        self.nw = n_walkers
        self.ns = nsample_per_walker
        self.alphac = getattr(inp, "alphac", 0)
        d = Dims(inp.L, self.n_mp, self.alphac, inp.alphar, problem.n_slater, nsample_per_walker, n_walkers,
                 inp.spin_parity, inp.J1, inp.J2, device, walker_offset)
        h = C.c_void_p()
        rc = lib().rbmpp_create(C.byref(d), C.byref(h))
        self.h = h
        self._chk(rc)
        v = C.c_longlong()
        lib().rbmpp_query(self.h, 0, C.byref(v))
        self.Nv = v.value
        para = np.zeros(2 * self.n_mp)
        para[0::2] = problem.sym.para_mp.real
        para[1::2] = problem.sym.para_mp.imag
        self._w = _f(problem.sym.W_map, np.int32)
        self._o = _f(problem.orbital_idx, np.int32)
        self._sb = None if subB is None else np.ascontiguousarray(subB, dtype=np.int32)
        self._spw = None if sp_weights is None else _f(sp_weights, np.float64)
        self._chk(lib().rbmpp_set_tables(self.h, _p(self._w), _p(para), _p(self._o), None, _p(self._sb),
                                         _p(self._spw)))
        # complex para_mp_trans or complex units: psi, H psi and O_k are complex (O comes as a real and an
        # imaginary row)
        self.complex_weights = bool(np.any(para[1::2] != 0.0)) or self.alphac > 0

    def close(self):
        if getattr(self, "h", None):
            lib().rbmpp_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _chk(self, rc):
        if rc != 0:
            raise RbmppError(rc, lib().rbmpp_last_error(self.h).decode())

    def kernel_launches(self) -> int:
        """Kernel launches the library has issued so far (process-wide counter)."""
        v = C.c_longlong()
        lib().rbmpp_query(self.h, 6, C.byref(v))
        return v.value

    def device_bytes(self) -> int:
        v = C.c_longlong()
        lib().rbmpp_query(self.h, 5, C.byref(v))
        return v.value

    def set_params(self, br, Wr, slater, shift=0.0, bc=None, Wc=None):
        """Real units (br, Wr(N, alphar)), f_ij, shift and, with complex units, bc (alphac) and Wc (N, alphac)
        complex (None keeps the current ones)."""
        Wr = _f(Wr, np.float64)
        br = np.ascontiguousarray(br, np.float64)
        sl = np.ascontiguousarray(slater, np.float64)
        Wcp = None if Wc is None else _f(np.asarray(Wc, np.complex128), np.complex128).view(np.float64)
        bcp = None if bc is None else np.ascontiguousarray(bc, np.complex128).view(np.float64)
        self._chk(lib().rbmpp_set_params(self.h, _p(Wr), _p(br), _p(Wcp), _p(bcp), _p(sl), float(shift)))

    def get_params_c(self):
        """(bc, Wc(N, alphac)) complex."""
        Wc = np.zeros(self.N * max(self.alphac, 1), np.complex128)
        bc = np.zeros(max(self.alphac, 1), np.complex128)
        self._chk(lib().rbmpp_get_params_c(self.h, _p(Wc.view(np.float64)), _p(bc.view(np.float64))))
        return bc[:self.alphac], Wc[:self.N * self.alphac].reshape((self.N, self.alphac), order="F")

    def get_params(self):
        a = self.p.inp.alphar
        Wr = np.zeros(self.N * a)
        br = np.zeros(max(a, 1))
        sl = np.zeros(self.p.n_slater)
        sh = np.zeros(1)
        self._chk(lib().rbmpp_get_params(self.h, _p(Wr), _p(br), _p(sl), _p(sh)))
        return br[:a], Wr.reshape((self.N, a), order="F"), sl, float(sh[0])

    def seed(self, iseed0: int):
        self._chk(lib().rbmpp_seed_walkers(self.h, int(iseed0)))

    def rank0_grnd(self, n: int):
        out = np.zeros(max(n, 1))
        self._chk(lib().rbmpp_rank0_grnd(self.h, n, _p(out)))
        return out[:n]

    def make_sample(self, first: bool):
        nacc = np.zeros(self.nw, dtype=np.int32)
        self._chk(lib().rbmpp_make_sample(self.h, 1 if first else 0, _p(nacc), None))
        return nacc

    def samples(self):
        x = np.zeros(self.N * self.ns * self.nw, dtype=np.int32)
        psi = np.zeros(2 * (self.n_qp + 1) * self.ns * self.nw)
        pf = np.zeros(self.n_qp * self.ns * self.nw)
        self._chk(lib().rbmpp_get_samples(self.h, _p(x), _p(psi), _p(pf)))
        return (x.reshape(self.nw, self.ns, self.N), psi.view(np.complex128).reshape(self.nw, self.ns, self.n_qp + 1),
                pf.reshape(self.nw, self.ns, self.n_qp))

    def set_samples(self, x):
        x = np.ascontiguousarray(x, dtype=np.int32).reshape(-1)
        self._chk(lib().rbmpp_set_samples(self.h, _p(x)))

    def measure(self, want_S=True, want_vectors=True):
        scal = np.zeros(4)
        g = np.zeros(self.Nv) if want_vectors else None
        ov = np.zeros(self.Nv) if want_vectors else None
        S = np.zeros(self.Nv * self.Nv) if want_S else None
        self._chk(lib().rbmpp_measure(self.h, _p(scal), _p(g), _p(ov), _p(S)))
        out = dict(Etot=scal[0], Etot2=scal[1], norm=scal[2], wf_av=scal[3], gvec=g, Ovec=ov)
        if S is not None:
            out["S"] = S.reshape((self.Nv, self.Nv), order="F")
        return out

    def measure_energy(self):
        scal = np.zeros(4)
        self._chk(lib().rbmpp_measure_energy(self.h, _p(scal)))
        return dict(Etot=scal[0], Etot2=scal[1], norm=scal[2], wf_av=scal[3])

    def measure_correlation(self):
        """Calc_Correlation's calc_phys_quantity_after_opt: scalars, Chi_sp (2, Nchi), Chi_vbs (Nchi, 4)."""
        nchi = self.N * (self.N + 1) // 2
        scal = np.zeros(5)
        sp = np.zeros(2 * nchi)
        vb = np.zeros(4 * nchi)
        self._chk(lib().rbmpp_measure_correlation(self.h, _p(scal), _p(sp), _p(vb)))
        return dict(Etot=scal[0], Etot2=scal[1], norm=scal[2], wf_av=scal[3], wf_sgn=scal[4],
                    chi_sp=sp.reshape((2, nchi), order="F"), chi_vbs=vb.reshape((nchi, 4), order="F"))

    def sr_step(self, iteration, delta_tau, s_factor0, s_cut, precision=SR_FP64, refine_steps=50):
        sin = SrIn(iteration, precision, refine_steps, 0, delta_tau, s_factor0, s_cut)
        sout = SrOut()
        dx = np.zeros(self.Nv)
        self._chk(lib().rbmpp_sr_step(self.h, C.byref(sin), C.byref(sout), _p(dx)))
        return sout, dx

    def iteration(self, precision, delta_tau, s_factor_scale, s_cut, s_factor0):
        sout = SrOut()
        self._chk(lib().rbmpp_iteration(self.h, precision, delta_tau, s_factor_scale, s_cut, s_factor0,
                                        C.byref(sout)))
        return sout

    def nfastup(self):
        out = np.zeros(self.nw, dtype=np.int32)
        self._chk(lib().rbmpp_get_walker_state(self.h, _p(out), None))
        return out

    def set_trace(self, max_records: int):
        self._chk(lib().rbmpp_set_trace(self.h, int(max_records)))
        self.trace_max = int(max_records)

    def set_replay(self, decisions):
        """decisions: int array (n_walkers, max_checkpoints, 2) of {Nfastup after, extra draw}, or None."""
        if decisions is None:
            self._chk(lib().rbmpp_set_replay(self.h, None, 0))
            return
        d = np.ascontiguousarray(decisions, dtype=np.int32)
        self._chk(lib().rbmpp_set_replay(self.h, _p(d), int(d.shape[1])))

    def events(self):
        """Per walker {global flips tried, accepted, make_initial_x re-seeds, checkpoints, trace records} of
        the last make_sample, and the chain trace (n_walkers, max_records, 6) when one is enabled."""
        ev = np.zeros(5 * self.nw, dtype=np.int32)
        m = getattr(self, "trace_max", 0)
        tr = np.zeros(6 * m * self.nw) if m > 0 else None
        self._chk(lib().rbmpp_get_walker_events(self.h, _p(ev), _p(tr)))
        return ev.reshape(self.nw, 5), (tr.reshape(self.nw, m, 6) if tr is not None else None)

    def debug_hook(self, what: int, value: int):
        self._chk(lib().rbmpp_debug_hook(self.h, int(what), int(value)))

    def copy_state_from(self, other: "Context"):
        """Continue from other's sampling state, parameters and iteration bookkeeping."""
        self._chk(lib().rbmpp_copy_state(self.h, other.h))

    def set_s_precision(self, precision):
        self._chk(lib().rbmpp_set_s_precision(self.h, int(precision)))

    def set_shift(self, shift):
        self._chk(lib().rbmpp_set_shift(self.h, float(shift)))

    def set_allreduce(self, fn):
        """fn(device_pointer: int, n: int) -> None sums n float64 at the device address over all ranks in place
        (None switches the library's own reductions off).  An exception in fn becomes RBMPP_E_COMM; the
        exception itself is kept in self.allreduce_error."""
        if fn is None:
            self._allreduce = None
            self._chk(lib().rbmpp_set_allreduce(self.h, ALLREDUCE_FN(), None))
            return

        def on_error(e):
            self.allreduce_error = e

        self._allreduce = allreduce_callback(fn, on_error)  # kept alive while the context uses it
        self._chk(lib().rbmpp_set_allreduce(self.h, self._allreduce, None))

    def exchange_measurement(self, direction, S_ptr, g_ptr, ov_ptr, scal6):
        """Device pointers (ints) for S, gvec, Ovec; scal6 a float64 array of 6."""
        self._chk(lib().rbmpp_exchange_measurement(self.h, direction, C.c_void_p(S_ptr), C.c_void_p(g_ptr),
                                                   C.c_void_p(ov_ptr), _p(scal6)))

    def stats(self):
        out = np.zeros(10)
        self._chk(lib().rbmpp_get_stats(self.h, _p(out), 10))
        keys = ["sampler_ms", "estimator_ms", "gemv_ms", "sbuild_ms", "solve_ms", "accepts_all", "proposals",
                "iteration_ms", "refine_ms", "cholesky_attempts"]
        return dict(zip(keys, out.tolist()))

    def eval_configs(self, x, want_h=True, want_O=False):
        x = np.ascontiguousarray(x, dtype=np.int32)
        n = x.shape[0]
        psi = np.zeros(2 * (self.n_qp + 1) * n)
        hp = np.zeros(2 * n) if want_h else None
        rows = 2 if self.complex_weights else 1
        O = np.zeros(self.Nv * n * rows) if want_O else None
        self._chk(lib().rbmpp_eval_configs(self.h, n, _p(x.reshape(-1)), _p(psi), _p(hp), _p(O)))
        out = dict(psi=psi.view(np.complex128).reshape(n, self.n_qp + 1))
        if hp is not None:
            out["hpsi"] = hp.view(np.complex128)
        if O is not None:
            O = O.reshape(n, rows, self.Nv)
            out["O"] = O[:, 0] + 1j * O[:, 1] if rows == 2 else O[:, 0]
        return out

    def eval_configs_noalloc(self, n: int, d_x: int, d_psi: int, d_hpsi: int, d_O: int):
        """rbmpp_eval_configs_noalloc on caller-owned device buffers (integer device addresses, 0 for
        an output that is not wanted); the library allocates nothing for this call."""
        self._chk(lib().rbmpp_eval_configs_noalloc(self.h, int(n), C.c_void_p(d_x or None),
                                                   C.c_void_p(d_psi or None), C.c_void_p(d_hpsi or None),
                                                   C.c_void_p(d_O or None)))


class Batch:
    """One launch of make_sample over several contexts (rbmpp_batch_*)."""

    def __init__(self, contexts):
        self.ctxs = list(contexts)
        arr = (C.c_void_p * len(self.ctxs))(*[c.h.value for c in self.ctxs])
        h = C.c_void_p()
        rc = lib().rbmpp_batch_create(C.cast(arr, C.c_void_p), len(self.ctxs), C.byref(h))
        self.h = h
        self._chk(rc)

    def _chk(self, rc):
        if rc != 0:
            raise RbmppError(rc, lib().rbmpp_batch_last_error(self.h).decode())

    def tune(self):
        th, order, ms = C.c_int(), C.c_int(), C.c_double()
        self._chk(lib().rbmpp_batch_tune(self.h, C.byref(th), C.byref(order), C.byref(ms)))
        return th.value, order.value, ms.value

    def make_sample(self, first: bool):
        out = np.zeros(len(self.ctxs), dtype=np.int64)
        self._chk(lib().rbmpp_batch_make_sample(self.h, 1 if first else 0, _p(out)))
        return out

    def close(self):
        if getattr(self, "h", None):
            lib().rbmpp_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def initial_params_c(ctx: Context, problem):
    """initialize_parameters (parameter.f90:21-41) with complex units: rank 0 draws, in this order, for every
    complex unit f the pair (re, im) of bcirr(f) and then of each Wcirr(iw, f), all U(-0.05, 0.05) (bcirr x10 for
    spin_parity = -1), then the real units as initial_params does.  Returns (bc, Wc, br, Wr); W.input (the
    problem's br, Wr and, when present, bc, Wc) overrides the draws."""
    inp = problem.inp
    N = inp.L * inp.L
    ac = getattr(inp, "alphac", 0)
    u = ctx.rank0_grnd(2 * ac * (N + 1) + inp.alphar * (N + 1))
    k = 0
    bc = np.zeros(ac, np.complex128)
    Wc = np.zeros((N, ac), np.complex128)
    for f in range(ac):
        bc[f] = 0.1 * (u[k] - 0.5) + 0.1j * (u[k + 1] - 0.5)
        k += 2
        if inp.spin_parity == -1:
            bc[f] *= 10.0
        for iw in range(N):
            Wc[iw, f] = 0.1 * (u[k] - 0.5) + 0.1j * (u[k + 1] - 0.5)
            k += 2
    br = np.zeros(inp.alphar)
    Wr = np.zeros((N, inp.alphar))
    for f in range(inp.alphar):
        br[f] = 0.1 * (u[k] - 0.5)
        k += 1
        if inp.spin_parity == -1:
            br[f] *= 10.0
        for iw in range(N):
            Wr[iw, f] = 0.1 * (u[k] - 0.5)
            k += 1
    if problem.Wr is not None:
        br, Wr = problem.br, problem.Wr
    if getattr(problem, "Wc", None) is not None:
        bc, Wc = problem.bc, problem.Wc
    return bc, Wc, br, Wr


def initial_params(ctx: Context, problem):
    """initialize_parameters (parameter.f90:21-75): rank 0 draws U(-0.05, 0.05) RBM parameters from its
    stream (consuming alphar*(N+1) draws), then W.input overrides them when present."""
    inp = problem.inp
    N = inp.L * inp.L
    u = ctx.rank0_grnd(inp.alphar * (N + 1))
    br = np.zeros(inp.alphar)
    Wr = np.zeros((N, inp.alphar))
    k = 0
    for f in range(inp.alphar):
        br[f] = 0.1 * (u[k] - 0.5)
        k += 1
        if inp.spin_parity == -1:
            br[f] *= 10.0
        for iw in range(N):
            Wr[iw, f] = 0.1 * (u[k] - 0.5)
            k += 1
    if problem.Wr is not None:
        br, Wr = problem.br, problem.Wr
    return br, Wr

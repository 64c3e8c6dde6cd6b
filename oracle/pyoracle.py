"""ctypes wrapper of the CPU oracle (oracle/rbmpp_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline / reference arm as the checker.  The product package never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None


def build() -> str:
    src = os.path.join(_HERE, "rbmpp_oracle.cpp")
    if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(src):
        subprocess.check_call(["make", "-C", _HERE, "-s"])
    return _LIB


class SrIn(C.Structure):
    _fields_ = [("iteration", C.c_int), ("delta_tau", C.c_double), ("s_factor0", C.c_double),
                ("s_cut", C.c_double), ("Etot", C.c_double), ("Etot2", C.c_double)]


class SrOut(C.Structure):
    _fields_ = [("lambda_", C.c_double), ("lambda_rbm_rbm", C.c_double), ("lambda_pp_pp", C.c_double),
                ("lambda_rbm_pp", C.c_double), ("delW_max", C.c_double), ("s_factor", C.c_double),
                ("sdiag_av", C.c_double), ("smat_scaling", C.c_double), ("kmax", C.c_int),
                ("k_nonzero", C.c_int), ("nSmat", C.c_int)]


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB)
        P = C.c_void_p
        dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
        ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
        up = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
        L.orc_create.restype = P
        L.orc_create.argtypes = [C.c_int] * 8 + [C.c_double, C.c_double]
        L.orc_destroy.argtypes = [P]
        L.orc_errmsg.restype = C.c_char_p
        L.orc_errmsg.argtypes = [P]
        L.orc_nv.argtypes = [P]
        L.orc_set_tables.argtypes = [P, ip, dp, ip, P]
        L.orc_set_params.argtypes = [P, dp, dp, dp, C.c_double]
        L.orc_set_sp_weights.argtypes = [P, dp]
        L.orc_set_params_c.argtypes = [P, dp, dp]
        L.orc_get_params_c.argtypes = [P, dp, dp]
        L.orc_get_params.argtypes = [P, dp, dp, dp, P]
        L.orc_get_slater_elements.argtypes = [P, dp]
        L.orc_seed.argtypes = [P, C.c_int]
        L.orc_seed_offset.argtypes = [P, C.c_int, C.c_int]
        L.orc_rank_grnd.argtypes = [P, C.c_int, C.c_int, P]
        L.orc_get_rng_state.argtypes = [P, C.c_int, up, ip]
        L.orc_get_nfastup.argtypes = [P, ip]
        L.orc_make_sample.argtypes = [P, C.c_int, ip, C.c_int]
        L.orc_get_samples.argtypes = [P, P, P, P]
        L.orc_set_trace.argtypes = [P, C.c_int]
        L.orc_get_events.argtypes = [P, P, P]
        L.orc_set_samples.argtypes = [P, ip]
        L.orc_measure.argtypes = [P, dp, dp, dp, P, P, P, C.c_int]
        L.orc_measure_energy.argtypes = [P, dp, C.c_int]
        L.orc_measure_correlation.argtypes = [P, dp, dp, dp, C.c_int]
        L.orc_eval_configs.argtypes = [P, C.c_int, ip, P, P, P, P]
        L.orc_proposal_pf.argtypes = [P, ip, C.c_int, C.c_int, dp, dp]
        L.orc_sr_step.argtypes = [P, C.POINTER(SrIn), dp, C.c_double, dp, dp, C.POINTER(SrOut), P]
        L.orc_pfaffian.restype = C.c_double
        L.orc_pfaffian.argtypes = [C.c_int, dp]
        L.orc_inverse.argtypes = [C.c_int, dp]
        L.orc_mt_u32.argtypes = [C.c_int, C.c_int, C.c_int, up]
        L.orc_mt_state.argtypes = [C.c_int, up]
        L.orc_grnd.argtypes = [C.c_int, C.c_int, C.c_int, dp]
        L.orc_max_threads.restype = C.c_int
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def fortran_array(a, dtype):
    """Column-major flat copy (the Fortran layout the C API expects)."""
    return np.ascontiguousarray(np.asarray(a, dtype=dtype).reshape(-1, order="F"))


class OracleError(RuntimeError):
    pass


class Oracle:
    """One oracle context: nranks emulated MPI ranks (walkers), each with its own MT19937 stream."""

    def __init__(self, problem, nranks: int, nsample_per_rank: int, nthreads: int = 1, sp_weights=None):
        self.p = problem
        inp = problem.inp
        self.L = inp.L
        self.N = inp.L * inp.L
        self.n_mp = problem.sym.n_mp
        self.n_qp = 2 * self.n_mp
        self.nranks = nranks
        self.nsample = nsample_per_rank
        self.nthreads = nthreads
        L = lib()
        self.alphac = getattr(inp, "alphac", 0)
        self.h = L.orc_create(inp.L, self.n_mp, self.alphac, inp.alphar, problem.n_slater, nsample_per_rank,
                              nranks, inp.spin_parity, inp.J1, inp.J2)
        if not self.h:
            raise OracleError("orc_create failed")
        self.Nv = L.orc_nv(self.h)
        para = np.zeros(2 * self.n_mp)
        para[0::2] = problem.sym.para_mp.real
        para[1::2] = problem.sym.para_mp.imag
        self._chk(L.orc_set_tables(self.h, fortran_array(problem.sym.W_map, np.int32), para,
                                   fortran_array(problem.orbital_idx, np.int32), None))
        if sp_weights is not None:  # (3, 2): SP_GL_Cos, SP_GL_Sin, para_spin_proj per point
            self._chk(L.orc_set_sp_weights(self.h, fortran_array(sp_weights, np.float64)))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def _chk(self, rc):
        if rc != 0:
            raise OracleError(f"oracle error {rc}: {lib().orc_errmsg(self.h).decode()}")

    def set_params(self, br, Wr, slater, shift=0.0):
        self._chk(lib().orc_set_params(self.h, fortran_array(Wr, np.float64), np.ascontiguousarray(br, np.float64),
                                       np.ascontiguousarray(slater, np.float64), float(shift)))

    def set_params_c(self, bc, Wc):
        """Complex units: bc (alphac), Wc (N, alphac) complex."""
        Wcp = fortran_array(np.asarray(Wc, np.complex128), np.complex128).view(np.float64)
        bcp = np.ascontiguousarray(bc, np.complex128).view(np.float64)
        self._chk(lib().orc_set_params_c(self.h, np.ascontiguousarray(Wcp), np.ascontiguousarray(bcp)))

    def get_params_c(self):
        ac = self.alphac
        Wc = np.zeros(2 * self.N * ac)
        bc = np.zeros(2 * ac)
        lib().orc_get_params_c(self.h, Wc, bc)
        return bc.view(np.complex128), Wc.view(np.complex128).reshape((self.N, ac), order="F")

    def get_params(self):
        inp = self.p.inp
        Wr = np.zeros(self.N * inp.alphar)
        br = np.zeros(inp.alphar)
        sl = np.zeros(self.p.n_slater)
        sh = C.c_double(0)
        lib().orc_get_params(self.h, Wr, br, sl, C.cast(C.pointer(sh), C.c_void_p))
        return br, Wr.reshape((self.N, inp.alphar), order="F"), sl, sh.value

    def slater_elements(self):
        out = np.zeros(4 * self.N * self.N * self.n_qp)
        lib().orc_get_slater_elements(self.h, out)
        return out.reshape((2 * self.N, 2 * self.N, self.n_qp), order="F")

    def seed(self, iseed0: int, offset: int = 0):
        """main.f90:224-234 for global ranks offset .. offset + nranks - 1."""
        self.rank0 = int(offset)
        self._chk(lib().orc_seed_offset(self.h, int(iseed0), int(offset)))

    def rank_grnd(self, rank: int, n: int):
        out = np.zeros(max(n, 1))
        self._chk(lib().orc_rank_grnd(self.h, rank, n, _ptr(out)))
        return out[:n]

    def rng_state(self, rank: int):
        mt = np.zeros(624, dtype=np.uint32)
        mti = np.zeros(1, dtype=np.int32)
        lib().orc_get_rng_state(self.h, rank, mt, mti)
        return mt, int(mti[0])

    def nfastup(self):
        out = np.zeros(self.nranks, dtype=np.int32)
        lib().orc_get_nfastup(self.h, out)
        return out

    def make_sample(self, first: bool):
        nacc = np.zeros(self.nranks, dtype=np.int32)
        self._chk(lib().orc_make_sample(self.h, 1 if first else 0, nacc, self.nthreads))
        return nacc

    def set_trace(self, max_records: int):
        self.trace_max = int(max_records)
        lib().orc_set_trace(self.h, self.trace_max)

    def events(self):
        """Per rank {global flips tried, accepted, make_initial_x re-seeds, checkpoints, trace records} of the
        last make_sample, and the chain trace (nranks, trace_max, 6) when one is kept (the library's layout)."""
        ev = np.zeros(5 * self.nranks, dtype=np.int32)
        m = getattr(self, "trace_max", 0)
        tr = np.zeros(6 * m * self.nranks) if m > 0 else None
        lib().orc_get_events(self.h, _ptr(ev), _ptr(tr))
        return ev.reshape(self.nranks, 5), (tr.reshape(self.nranks, m, 6) if tr is not None else None)

    def samples(self):
        x = np.zeros(self.N * self.nsample * self.nranks, dtype=np.int32)
        psi = np.zeros(2 * (self.n_qp + 1) * self.nsample * self.nranks)
        pf = np.zeros(self.n_qp * self.nsample * self.nranks)
        lib().orc_get_samples(self.h, _ptr(x), _ptr(psi), _ptr(pf))
        x = x.reshape((self.nranks, self.nsample, self.N))
        psi = psi.view(np.complex128).reshape((self.nranks, self.nsample, self.n_qp + 1))
        pf = pf.reshape((self.nranks, self.nsample, self.n_qp))
        return x, psi, pf

    def set_samples(self, x):
        lib().orc_set_samples(self.h, np.ascontiguousarray(x, dtype=np.int32).reshape(-1))

    def measure(self, want_S=True, want_O=False, want_eloc=False):
        scal = np.zeros(4)
        g = np.zeros(self.Nv)
        ov = np.zeros(self.Nv)
        S = np.zeros(self.Nv * self.Nv) if want_S else None
        O = np.zeros(self.Nv * 2 * self.nsample * self.nranks) if want_O else None
        E = np.zeros(2 * self.nsample * self.nranks) if want_eloc else None
        self._chk(lib().orc_measure(self.h, scal, g, ov, _ptr(S), _ptr(O), _ptr(E), self.nthreads))
        out = dict(Etot=scal[0], Etot2=scal[1], norm=scal[2], wf_av=scal[3], gvec=g, Ovec=ov)
        if S is not None:
            out["S"] = S.reshape((self.Nv, self.Nv), order="F")
        if O is not None:
            out["O"] = O.reshape((self.Nv, 2 * self.nsample * self.nranks), order="F")
        if E is not None:
            out["eloc"] = E.view(np.complex128)
        return out

    def measure_energy(self):
        scal = np.zeros(4)
        self._chk(lib().orc_measure_energy(self.h, scal, self.nthreads))
        return dict(Etot=scal[0], Etot2=scal[1], norm=scal[2], wf_av=scal[3])

    def measure_correlation(self):
        """Calc_Correlation's calc_phys_quantity_after_opt: scalars, Chi_sp (2, Nchi), Chi_vbs (Nchi, 4)."""
        nchi = self.N * (self.N + 1) // 2
        scal = np.zeros(5)
        sp = np.zeros(2 * nchi)
        vb = np.zeros(4 * nchi)
        self._chk(lib().orc_measure_correlation(self.h, scal, sp, vb, self.nthreads))
        return dict(Etot=scal[0], Etot2=scal[1], norm=scal[2], wf_av=scal[3], wf_sgn=scal[4],
                    chi_sp=sp.reshape((2, nchi), order="F"), chi_vbs=vb.reshape((nchi, 4), order="F"))

    def eval_configs(self, x, want_h=True, want_O=False):
        x = np.ascontiguousarray(x, dtype=np.int32)
        n = x.shape[0]
        psi = np.zeros(2 * (self.n_qp + 1) * n)
        hp = np.zeros(2 * n) if want_h else None
        O = np.zeros(2 * self.Nv * n) if want_O else None
        pf = np.zeros(self.n_qp * n)
        self._chk(lib().orc_eval_configs(self.h, n, x.reshape(-1), _ptr(psi), _ptr(hp), _ptr(O), _ptr(pf)))
        out = dict(psi=psi.view(np.complex128).reshape(n, self.n_qp + 1), pf=pf.reshape(n, self.n_qp))
        if hp is not None:
            out["hpsi"] = hp.view(np.complex128)
        if O is not None:
            out["O"] = O.view(np.complex128).reshape(n, self.Nv)
        return out

    def proposal_pf(self, x, i1, i2):
        pf_old = np.zeros(self.n_qp)
        pf_new = np.zeros(self.n_qp)
        self._chk(lib().orc_proposal_pf(self.h, np.ascontiguousarray(x, dtype=np.int32), i1, i2, pf_old, pf_new))
        return pf_old, pf_new

    def sr_step(self, iteration, delta_tau, s_factor0, s_cut, Etot, Etot2, S_raw, norm, gvec, Ovec):
        sin = SrIn(iteration, delta_tau, s_factor0, s_cut, Etot, Etot2)
        sout = SrOut()
        g = np.ascontiguousarray(gvec, dtype=np.float64).copy()
        dx = np.zeros(self.Nv)
        self._chk(lib().orc_sr_step(self.h, C.byref(sin), fortran_array(S_raw, np.float64), float(norm), g,
                                    np.ascontiguousarray(Ovec, np.float64), C.byref(sout), _ptr(dx)))
        return sout, dx, g


def pfaffian(A):
    A = np.asarray(A, dtype=np.float64)
    return lib().orc_pfaffian(A.shape[0], fortran_array(A, np.float64))


def mt_u32(seed, n, skip=0):
    out = np.zeros(n, dtype=np.uint32)
    lib().orc_mt_u32(seed, skip, n, out)
    return out


def mt_state(seed):
    out = np.zeros(624, dtype=np.uint32)
    lib().orc_mt_state(seed, out)
    return out


def grnd(seed, n, skip=0):
    out = np.zeros(n)
    lib().orc_grnd(seed, skip, n, out)
    return out


def max_threads():
    return lib().orc_max_threads()


class VMCLoop:
    """main.f90:300-455 restated around an Oracle: one call of ``iteration`` is one SR step
    (update_slater_elements, make_sample, calc_phys_quantity_opt, MPI reductions, SR_pdposv,
    and the s_factor0 / shift bookkeeping of main.f90:439-453).  With ``offset`` > 0 the oracle holds
    the shard of global ranks offset.. and ``allreduce`` (called with scal6, S, g, ov) sums the
    measurement over the shards, as the MPI_ALLREDUCE calls of main.f90:348-369 do."""

    def __init__(self, orc: Oracle, problem, iseed0: int, offset: int = 0, allreduce=None, shift_coef=0.001):
        self.o = orc
        self.shift_coef = shift_coef  # main.f90:451 (0.003 in transverse_code/main.f90:451)
        self.p = problem
        inp = problem.inp
        self.s_factor0 = inp.s_factor0
        self.wf_av_list = [0.0] * 10
        self.shift = 0.0
        self.iteration = 0
        self.allreduce = allreduce
        orc.seed(iseed0, offset)
        # initialize_parameters (parameter.f90:21-41): rank 0 draws the random RBM init, which W.input
        # (when present) then overrides.
        if offset != 0 and problem.Wr is None:
            raise OracleError("a shard without global rank 0 needs W.input (rank 0's random init is broadcast)")
        ac = orc.alphac
        nd = 2 * ac * (self.o.N + 1) + inp.alphar * (self.o.N + 1)
        u = orc.rank_grnd(0, nd) if offset == 0 else np.zeros(nd)
        k = 0
        bc = np.zeros(ac, np.complex128)
        Wc = np.zeros((self.o.N, ac), np.complex128)
        for f in range(ac):  # complex units first (parameter.f90:22-31)
            bc[f] = 0.1 * (u[k] - 0.5) + 0.1j * (u[k + 1] - 0.5)
            k += 2
            if inp.spin_parity == -1:
                bc[f] *= 10.0
            for iw in range(self.o.N):
                Wc[iw, f] = 0.1 * (u[k] - 0.5) + 0.1j * (u[k + 1] - 0.5)
                k += 2
        if getattr(problem, "Wc", None) is not None:
            bc, Wc = problem.bc, problem.Wc
        if ac:
            orc.set_params_c(bc, Wc)
        br = np.zeros(inp.alphar)
        Wr = np.zeros((self.o.N, inp.alphar))
        for f in range(inp.alphar):
            br[f] = 0.1 * (u[k] - 0.5)
            k += 1
            if inp.spin_parity == -1:
                br[f] *= 10.0
            for iw in range(self.o.N):
                Wr[iw, f] = 0.1 * (u[k] - 0.5)
                k += 1
        if problem.Wr is not None:
            br, Wr = problem.br, problem.Wr
        orc.set_params(br, Wr, problem.slater, 0.0)
        self.history = []

    def iteration_step(self):
        o, inp = self.o, self.p.inp
        self.iteration += 1
        nacc = o.make_sample(self.iteration == 1)
        m = o.measure(want_S=True)
        scal6 = np.array([m["Etot"], m["Etot2"], m["norm"], m["wf_av"], float(nacc.sum()), float(o.nsample * o.nranks)])
        S, gsum, osum = m["S"], m["gvec"], m["Ovec"]
        if self.allreduce is not None:
            scal6, S, gsum, osum = self.allreduce(scal6, S, gsum, osum)
        ntot = scal6[5]
        accept_ratio = float(scal6[4]) / ntot / o.N
        wf_av = scal6[3] / ntot
        norm = scal6[2]
        Etot = scal6[0] / norm
        Etot2 = scal6[1] / norm
        g = gsum / norm
        ov = osum / norm
        sout, dx, _ = o.sr_step(self.iteration, inp.delta_tau, self.s_factor0, inp.s_cut, Etot, Etot2, S, norm,
                                g, ov)
        self.s_factor0 *= inp.s_factor_scale
        self.wf_av_list = self.wf_av_list[1:] + [wf_av]
        wf = 0.0
        for v in self.wf_av_list:
            wf = wf + v
        wf = wf / 10.0
        self.shift = wf * self.shift_coef / float(o.N) / float(o.N)
        br, Wr, sl, _ = o.get_params()
        o.set_params(br, Wr, sl, self.shift)
        rec = dict(iteration=self.iteration, Etot=Etot, Etot2=Etot2, accept=accept_ratio, wf_av=wf_av,
                   shift=self.shift, lam=sout.lambda_, delW=sout.delW_max)
        self.history.append(rec)
        return rec

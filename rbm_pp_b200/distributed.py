"""SR iterations over one or several GPUs (one process per GPU, walkers sharded across ranks).

Rank r holds global walkers r*nw .. r*nw+nw-1 (the reference's MPI ranks).  Each SR step runs
make_sample and the estimators locally, then the one exchange of the reference -- the
MPI_ALLREDUCE of Etot, Etot2, norm, wf_av, naccept, gvec, Ovec and the full S matrix
(main.f90:348-369) -- as NCCL all-reduces over NVLink, then the identical SR solve on every rank
(so the parameter broadcast of main.f90:427-438 is not needed), then the s_factor0 / shift
bookkeeping of main.f90:439-453.
"""
from __future__ import annotations

import numpy as np

from . import capi


class Bookkeeping:
    """main.f90:439-453: s_factor0 schedule and the 10-step moving average of wf_av -> shift."""

    def __init__(self, inp, N):
        self.s_factor0 = inp.s_factor0
        self.scale = inp.s_factor_scale
        self.wf_av_list = [0.0] * 10
        self.N = N

    def after_step(self, wf_av):
        self.s_factor0 = self.s_factor0 * self.scale
        self.wf_av_list = self.wf_av_list[1:] + [wf_av]
        wf = 0.0
        for v in self.wf_av_list:
            wf = wf + v
        wf = wf / 10.0
        return wf * 0.001 / float(self.N) / float(self.N)


def allreduce_measurement(S, g, ov, scal6, group=None):
    """The MPI_ALLREDUCE(SUM) calls of main.f90:348-369, in place on torch tensors: the partial S
    matrix, gvec, Ovec and scal6 = (Etot, Etot2, norm, wf_av, naccept, n_samples) of every rank.
    NCCL over NVLink for CUDA tensors; the same call runs over gloo for CPU tensors."""
    import torch.distributed as dist
    for t in (S, g, ov, scal6):
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)


def reduce_measurement(parts):
    """Host-side reference of the cross-rank sum: parts is a list of (scal6, S, g, ov)."""
    scal = np.sum([p[0] for p in parts], axis=0)
    S = np.sum([p[1] for p in parts], axis=0)
    g = np.sum([p[2] for p in parts], axis=0)
    ov = np.sum([p[3] for p in parts], axis=0)
    return scal, S, g, ov


class SRRunner:
    def __init__(self, ctx: "capi.Context", problem, iseed0: int, precision=capi.SR_FP64, world=1, rank=0):
        self.ctx = ctx
        self.p = problem
        self.world = world
        self.rank = rank
        self.precision = precision
        self.iteration = 0
        inp = problem.inp
        ctx.seed(iseed0)
        if rank == 0:
            br, Wr = capi.initial_params(ctx, problem)
        else:
            br, Wr = problem.br, problem.Wr
        ctx.set_params(br, Wr, problem.slater, 0.0)
        self.book = Bookkeeping(inp, ctx.N)
        self._bufs = None

    @classmethod
    def attach(cls, ctx: "capi.Context", problem, precision=capi.SR_FP64):
        """A one-GPU runner over a context whose state is already set (seeded, parameters loaded, possibly
        copied from another context with Context.copy_state_from): it continues from that state."""
        r = cls.__new__(cls)
        r.ctx, r.p, r.world, r.rank, r.precision, r.iteration = ctx, problem, 1, 0, precision, 0
        r.book = Bookkeeping(problem.inp, ctx.N)
        r._bufs = None
        return r

    def step(self):
        import torch
        inp = self.p.inp
        if self.world == 1:
            out = self.ctx.iteration(self.precision, inp.delta_tau, inp.s_factor_scale, inp.s_cut, inp.s_factor0)
            rec = out.as_dict()
            rec["device_ms"] = self.ctx.stats()["iteration_ms"]
            return rec
        self.iteration += 1
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record()
        self.ctx.make_sample(self.iteration == 1)
        self.ctx.measure(want_S=False, want_vectors=False)
        nv = self.ctx.Nv
        if self._bufs is None:
            self._bufs = (torch.empty((nv, nv), dtype=torch.float64, device="cuda"),
                          torch.empty(nv, dtype=torch.float64, device="cuda"),
                          torch.empty(nv, dtype=torch.float64, device="cuda"))
        S, g, ov = self._bufs
        scal = np.zeros(6)
        torch.cuda.synchronize()
        self.ctx.exchange_measurement(0, S.data_ptr(), g.data_ptr(), ov.data_ptr(), scal)
        sc = torch.tensor(scal, dtype=torch.float64, device="cuda")
        allreduce_measurement(S, g, ov, sc)
        torch.cuda.synchronize()
        scal = sc.cpu().numpy()
        self.ctx.exchange_measurement(1, S.data_ptr(), g.data_ptr(), ov.data_ptr(), scal)
        out, _ = self.ctx.sr_step(self.iteration, inp.delta_tau, self.book.s_factor0, inp.s_cut, self.precision)
        self.ctx.set_shift(self.book.after_step(out.wf_av))
        ev1.record()
        torch.cuda.synchronize()
        rec = out.as_dict()
        rec["device_ms"] = ev0.elapsed_time(ev1)
        return rec

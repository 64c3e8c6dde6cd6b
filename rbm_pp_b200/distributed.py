"""SR iterations over one or several GPUs (one process per GPU, walkers sharded across ranks).

Rank r holds global walkers r*nw .. r*nw+nw-1 (the reference's MPI ranks).  The library does the
cross-rank sums itself through a host all-reduce handed to it once (rbmpp_set_allreduce): the
MPI_ALLREDUCE of Etot, Etot2, norm, wf_av, naccept, gvec and Ovec (main.f90:348-369), the S matrix,
and, on the split-BF16 path, one Nv-vector per conjugate-gradient iteration of the refinement on the
exact S.  Here that all-reduce is NCCL over NVLink on the library's own device buffers.  Every rank
then takes the identical SR step (so the parameter broadcast of main.f90:427-438 is not needed), and
the s_factor0 / shift bookkeeping of main.f90:439-453.
"""
from __future__ import annotations

import ctypes as C

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


class _DeviceVector:
    """n float64 at a raw device address, seen by torch without a copy (CUDA array interface v3, no stream:
    the library has drained its stream before it hands the buffer out)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                         "strides": None}


def allreduce_fn(group=None, where="cuda"):
    """The host all-reduce for Context.set_allreduce: fn(ptr, n) sums n float64 at ptr over the ranks of
    `group`, in place, and returns when the sum is there.
      where="cuda": ptr is a device address; with NCCL torch.distributed all-reduces it in place over NVLink,
                    with gloo a host copy is reduced and copied back;
      where="host": ptr is a host address (the same call over gloo, for CPU tests of this adapter)."""
    import torch
    import torch.distributed as dist
    nccl = dist.get_backend(group) == "nccl"

    def fn(ptr, n):
        if where == "cuda":
            t = torch.as_tensor(_DeviceVector(ptr, n), device="cuda")
            if nccl:
                dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
            else:
                h = t.cpu()
                dist.all_reduce(h, op=dist.ReduceOp.SUM, group=group)
                t.copy_(h)
            torch.cuda.current_stream().synchronize()
        else:
            t = torch.from_numpy(np.ctypeslib.as_array((C.c_double * n).from_address(ptr)))
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)

    return fn


def broadcast_initial_params(br, Wr, group=None):
    """The MPI_BCAST of rank 0's initial RBM parameters (parameter.f90:21-75): only rank 0 draws them."""
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.from_numpy(np.concatenate([np.ravel(br), np.ravel(Wr, order="F")])).to(dev)
    dist.broadcast(t, src=0, group=group)
    v = t.cpu().numpy()
    nb = np.size(br)
    return v[:nb].copy(), v[nb:].reshape(np.shape(Wr), order="F").copy()


class SRRunner:
    """main.f90:311-455 on this rank's context: one rbmpp_iteration per step.  With world > 1 the context
    sums over the ranks by itself (allreduce_fn on the process group)."""

    def __init__(self, ctx: "capi.Context", problem, iseed0: int, precision=capi.SR_FP64, world=1, rank=0,
                 group=None):
        self.ctx = ctx
        self.p = problem
        self.world = world
        self.rank = rank
        self.precision = precision
        inp = problem.inp
        ctx.seed(iseed0)
        ac = getattr(ctx, "alphac", 0)
        if rank == 0:
            bc, Wc, br, Wr = capi.initial_params_c(ctx, problem)
        else:
            bc, Wc = np.zeros(ac, np.complex128), np.zeros((ctx.N, ac), np.complex128)
            br = np.zeros(inp.alphar) if problem.br is None else problem.br
            Wr = np.zeros((ctx.N, inp.alphar)) if problem.Wr is None else problem.Wr
        if world > 1:
            br, Wr = broadcast_initial_params(br, Wr, group)
            if ac:
                bcf, Wcf = broadcast_initial_params(np.asarray(bc, np.complex128).view(np.float64),
                                                    np.asarray(Wc, np.complex128).reshape(-1, order="F")
                                                    .view(np.float64), group)
                bc, Wc = bcf.view(np.complex128), Wcf.view(np.complex128).reshape((ctx.N, ac), order="F")
            ctx.set_allreduce(allreduce_fn(group))
        if ac:
            ctx.set_params(br, Wr, problem.slater, 0.0, bc=bc, Wc=Wc)
        else:
            ctx.set_params(br, Wr, problem.slater, 0.0)
        self.book = Bookkeeping(inp, ctx.N)

    @classmethod
    def attach(cls, ctx: "capi.Context", problem, precision=capi.SR_FP64):
        """A one-GPU runner over a context whose state is already set (seeded, parameters loaded, possibly
        copied from another context with Context.copy_state_from): it continues from that state."""
        r = cls.__new__(cls)
        r.ctx, r.p, r.world, r.rank, r.precision = ctx, problem, 1, 0, precision
        r.book = Bookkeeping(problem.inp, ctx.N)
        return r

    def step(self):
        inp = self.p.inp
        out = self.ctx.iteration(self.precision, inp.delta_tau, inp.s_factor_scale, inp.s_cut, inp.s_factor0)
        rec = out.as_dict()
        rec["device_ms"] = self.ctx.stats()["iteration_ms"]
        return rec

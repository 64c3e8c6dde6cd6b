"""Walker sharding and the cross-rank sums of an SR step, run as 2 gloo ranks on the CPU.

Each rank holds half of the walkers (global ranks offset..offset+nw-1, seeded by the rule of
main.f90:224-234), measures them, sums the measurement over the ranks (the MPI_ALLREDUCE calls of
main.f90:348-369), and takes the SR step and the shift bookkeeping on the reduced sums.  The CPU oracle
stands in for the per-GPU context; the sums go through the product's host all-reduce
(``distributed.allreduce_fn`` behind the C function pointer ``capi.allreduce_callback`` builds for
rbmpp_set_allreduce, called through that pointer on buffers packed as the library packs them:
{Etot, Etot2, norm, wf_av, naccept, n_samples, gvec, Ovec}, then S).  Rank 0's random initial RBM
parameters reach the other rank through ``distributed.broadcast_initial_params``.  The result must
equal one process holding all walkers: the same parameters, energies and shift.
"""
import datetime
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

STEPS = 2
NW_TOTAL = 8
NS = 16


def _problem():
    from rbm_pp_b200 import formats as fm
    return fm.synthetic_problem(4, translations=True, alphar=1, nsample=NW_TOTAL * NS, seed=31)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    try:
        import torch
        import torch.distributed as dist

        import ctypes as C

        import pyoracle as po
        from rbm_pp_b200 import capi
        from rbm_pp_b200.distributed import allreduce_fn, broadcast_initial_params
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        p = _problem()
        nw = NW_TOTAL // world
        # rank 0's initial parameters, broadcast (rank 1 starts from zeros)
        br0 = np.arange(3.0) + 1.0 if rank == 0 else np.zeros(3)
        Wr0 = np.arange(12.0).reshape(4, 3) if rank == 0 else np.zeros((4, 3))
        bb, wb = broadcast_initial_params(br0, Wr0)
        assert np.array_equal(bb, np.arange(3.0) + 1.0) and np.array_equal(wb, np.arange(12.0).reshape(4, 3))
        # the C function pointer the library would hold, called through that pointer
        cb = capi.allreduce_callback(allreduce_fn(where="host"))
        native = capi.ALLREDUCE_FN(C.cast(cb, C.c_void_p).value)

        def call(buf):
            rc = native(None, buf.ctypes.data, buf.size)
            assert rc == 0, rc

        def reduce(scal6, S, g, ov):
            nv = g.size
            packed = np.concatenate([np.asarray(scal6, dtype=np.float64), g, ov])
            call(packed)
            Sr = np.array(S, dtype=np.float64, order="F")
            call(Sr.reshape(-1, order="F"))
            return packed[:6].copy(), Sr, packed[6:6 + nv].copy(), packed[6 + nv:].copy()

        o = po.Oracle(p, nranks=nw, nsample_per_rank=NS, nthreads=2)
        loop = po.VMCLoop(o, p, iseed0=4242, offset=rank * nw, allreduce=reduce)
        recs = [loop.iteration_step() for _ in range(STEPS)]
        br, Wr, sl, sh = o.get_params()
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, "ok", (recs, br, Wr, sl, sh)))
    except Exception as e:  # report to the parent instead of hanging it
        q.put((rank, "error", repr(e)))


def test_two_gloo_ranks_match_one_process():
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import pyoracle as po
    p = _problem()
    o = po.Oracle(p, nranks=NW_TOTAL, nsample_per_rank=NS, nthreads=4)
    loop = po.VMCLoop(o, p, iseed0=4242)
    want = [loop.iteration_step() for _ in range(STEPS)]
    wbr, wWr, wsl, wsh = o.get_params()

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    got = {}
    try:
        for _ in range(2):
            rank, status, payload = q.get(timeout=240)
            assert status == "ok", payload
            got[rank] = payload
    finally:
        for pr in procs:
            pr.join(timeout=30)
            if pr.is_alive():
                pr.kill()
    for rank in (0, 1):
        recs, br, Wr, sl, sh = got[rank]
        for a, b in zip(recs, want):
            for k in ("Etot", "Etot2", "accept", "wf_av", "shift", "lam", "delW"):
                assert abs(a[k] - b[k]) <= 1e-10 * max(abs(b[k]), 1e-300), (rank, k, a[k], b[k])
        assert np.allclose(Wr, wWr, rtol=1e-10, atol=1e-14)
        assert np.allclose(br, wbr, rtol=1e-10, atol=1e-14)
        assert np.allclose(sl, wsl, rtol=1e-10, atol=1e-14)
        assert abs(sh - wsh) <= 1e-10 * abs(wsh)

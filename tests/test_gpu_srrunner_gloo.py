"""The product's multi-rank driver on one GPU: two processes, each a rank with half of the walkers, running
distributed.SRRunner with world = 2 over a gloo process group.  SRRunner broadcasts rank 0's random initial RBM
parameters (parameter.f90:21-41) and hands the library distributed.allreduce_fn, so the context sums the
measurement, S and (split-BF16) the refinement's O^T O x over the ranks by itself (main.f90:348-369).  gloo reduces
the library's device buffers through the host here; the bench's multi-GPU runs use the same function over NCCL.
The ranks wait for one another on the host only.  Three SR steps must equal one process holding all walkers.
"""
import datetime
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NW, NS, STEPS, SEED = 4, 16, 3, 2468


def _problem():
    from rbm_pp_b200 import formats as fm
    p = fm.synthetic_problem(4, translations=True, alphar=1, nsample=2 * NW * NS, seed=71)
    p.br, p.Wr = None, None  # no W.input: rank 0 draws the initial RBM parameters
    return p


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, precision, q):
    try:
        import torch
        import torch.distributed as dist

        from rbm_pp_b200 import capi
        from rbm_pp_b200 import distributed as rdist
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
        torch.cuda.set_device(0)
        p = _problem()
        ctx = capi.Context(p, n_walkers=NW, nsample_per_walker=NS, walker_offset=rank * NW)
        runner = rdist.SRRunner(ctx, p, iseed0=SEED, precision=precision, world=world, rank=rank)
        recs = [runner.step() for _ in range(STEPS)]
        out = (recs, ctx.get_params())
        ctx.close()
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, "ok", out))
    except Exception as e:  # report to the parent instead of hanging it
        q.put((rank, "error", repr(e)))


@pytest.mark.parametrize("precision", [0, 1])
def test_srrunner_two_ranks_equal_one_context(precision):
    from rbm_pp_b200 import capi
    from rbm_pp_b200 import distributed as rdist
    p = _problem()
    one = capi.Context(p, n_walkers=2 * NW, nsample_per_walker=NS)
    r1 = rdist.SRRunner(one, p, iseed0=SEED, precision=precision)
    want = [r1.step() for _ in range(STEPS)]
    wparams = one.get_params()
    one.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, precision, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    got = {}
    try:
        for _ in range(2):
            rank, status, payload = q.get(timeout=300)
            assert status == "ok", payload
            got[rank] = payload
    finally:
        for pr in procs:
            pr.join(timeout=60)
            if pr.is_alive():
                pr.kill()
    for rank in (0, 1):
        recs, params = got[rank]
        for a, b in zip(recs, want):
            assert abs(a["Etot"] - b["Etot"]) <= 1e-12 * abs(b["Etot"])
            assert a["accept_ratio"] == b["accept_ratio"]
            assert abs(a["lambda_"] - b["lambda_"]) <= 1e-8 * abs(b["lambda_"])
        for x, y in zip(params[:3], wparams[:3]):
            x, y = np.asarray(x), np.asarray(y)
            assert np.abs(x - y).max() <= 1e-8 * np.abs(y).max()
    # the two ranks hold bit-identical parameters
    for x, y in zip(got[0][1][:3], got[1][1][:3]):
        assert np.array_equal(np.asarray(x), np.asarray(y))

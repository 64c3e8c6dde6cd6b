"""The product's multi-GPU path on one GPU: walkers sharded over two contexts.

1. The exchange of an SR step through caller buffers (rbmpp_exchange_measurement, the MPI_ALLREDUCE block of
   main.f90:348-369) done by summing the two contexts' device buffers, then the SR step on the reduced sums.
2. The library's own cross-rank sums (rbmpp_set_allreduce), which the split-BF16 path needs: the measurement,
   S, and O^T (O x) once per conjugate-gradient iteration.  The two ranks are two host threads, each driving
   its context through rbmpp_iteration; the all-reduce copies each rank's buffer to the host, waits for the
   other rank on a host barrier and writes back the sum taken in rank order.  No kernel waits on another.
Both must equal one context holding all walkers.  Also: rbmpp_copy_state makes a second context continue
exactly as the first.
"""
import threading

import numpy as np
import pytest

from rbm_pp_b200 import capi
from rbm_pp_b200 import distributed as rdist
from rbm_pp_b200 import formats as fm

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def test_two_shards_equal_one_context():
    import torch

    L, nw, ns = 4, 4, 8
    p = fm.synthetic_problem(L, translations=True, alphar=1, nsample=2 * nw * ns, seed=61)
    inp = p.inp
    one = capi.Context(p, n_walkers=2 * nw, nsample_per_walker=ns)
    shards = [capi.Context(p, n_walkers=nw, nsample_per_walker=ns, walker_offset=r * nw) for r in range(2)]
    for c in [one] + shards:
        c.set_params(p.br, p.Wr, p.slater, 0.0)
        c.seed(4242)
    book = rdist.Bookkeeping(inp, L * L)
    nv = one.Nv
    for it in range(1, 4):
        na1 = one.make_sample(it == 1)
        nas = [c.make_sample(it == 1) for c in shards]
        assert np.array_equal(na1, np.concatenate(nas))
        one.measure(want_S=False, want_vectors=False)
        for c in shards:
            c.measure(want_S=False, want_vectors=False)
        bufs = [(torch.empty((nv, nv), dtype=torch.float64, device="cuda"),
                 torch.empty(nv, dtype=torch.float64, device="cuda"),
                 torch.empty(nv, dtype=torch.float64, device="cuda")) for _ in shards]
        scal = [np.zeros(6) for _ in shards]
        torch.cuda.synchronize()
        for c, (S, g, ov), sc in zip(shards, bufs, scal):
            c.exchange_measurement(0, S.data_ptr(), g.data_ptr(), ov.data_ptr(), sc)
        S = bufs[0][0] + bufs[1][0]
        g = bufs[0][1] + bufs[1][1]
        ov = bufs[0][2] + bufs[1][2]
        sc = scal[0] + scal[1]
        torch.cuda.synchronize()
        for c in shards:
            c.exchange_measurement(1, S.data_ptr(), g.data_ptr(), ov.data_ptr(), sc.copy())
        o1, dx1 = one.sr_step(it, inp.delta_tau, book.s_factor0, inp.s_cut)
        outs = [c.sr_step(it, inp.delta_tau, book.s_factor0, inp.s_cut) for c in shards]
        shift = book.after_step(o1.wf_av)
        for c in [one] + shards:
            c.set_shift(shift)
        for o, dx in outs:
            assert abs(o.Etot - o1.Etot) <= 1e-12 * abs(o1.Etot)
            assert abs(o.lambda_ - o1.lambda_) <= 1e-9 * abs(o1.lambda_)
            assert _rel(dx, dx1) < 1e-9
        for c in shards:
            # the two summation orders of S differ by rounding, which the solve amplifies by cond(S)
            for a, b in zip(c.get_params()[:3], one.get_params()[:3]):
                assert _rel(a, b) < 1e-8
    for c in [one] + shards:
        c.close()


@pytest.mark.parametrize("precision", [capi.SR_FP64, capi.SR_SPLIT_BF16])
def test_copy_state_continues_identically(precision):
    L, nw, ns = 6, 4, 4
    p = fm.synthetic_problem(L, translations=True, alphar=1, nsample=nw * ns, seed=62)
    a = capi.Context(p, n_walkers=nw, nsample_per_walker=ns)
    ra = rdist.SRRunner(a, p, iseed0=99, precision=precision)
    for _ in range(2):
        ra.step()
    b = capi.Context(p, n_walkers=nw, nsample_per_walker=ns)
    b.copy_state_from(a)
    rb = rdist.SRRunner.attach(b, p, precision)
    for _ in range(2):
        ea, eb = ra.step(), rb.step()
        assert ea["Etot"] == eb["Etot"] and ea["lambda_"] == eb["lambda_"]
    assert np.array_equal(a.samples()[0], b.samples()[0])
    for x, y in zip(a.get_params(), b.get_params()):
        assert np.array_equal(np.asarray(x), np.asarray(y))
    a.close()
    b.close()


class ThreadAllreduce:
    """Ranks as threads of this process: rank r's fn(ptr, n) copies its device buffer to the host, waits for
    every rank, and writes back the sum in rank order (the same bits on every rank, as NCCL gives)."""

    def __init__(self, world):
        self.world = world
        self.parts = [None] * world
        self.bar = threading.Barrier(world, timeout=120)
        self.calls = [0] * world

    def fn(self, rank):
        import torch

        def f(ptr, n):
            t = torch.as_tensor(rdist._DeviceVector(ptr, n), device="cuda")
            self.parts[rank] = t.cpu().numpy()
            self.bar.wait()
            s = self.parts[0].copy()
            for r in range(1, self.world):
                s += self.parts[r]
            self.bar.wait()
            t.copy_(torch.from_numpy(s))
            torch.cuda.synchronize()
            self.calls[rank] += 1

        return f


def _run_threads(ctxs, body):
    out = [None] * len(ctxs)
    errs = []

    def run(r):
        try:
            out[r] = body(ctxs[r])
        except Exception as e:  # noqa: BLE001 - reported below
            errs.append((r, e))

    th = [threading.Thread(target=run, args=(r,)) for r in range(len(ctxs))]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=600)
    assert not errs, errs
    return out


@pytest.mark.parametrize("precision", [capi.SR_FP64, capi.SR_SPLIT_BF16])
def test_library_allreduce_shards_equal_one_context(precision):
    import torch

    L, nw, ns, steps = 4, 8, 16, 3
    p = fm.synthetic_problem(L, translations=True, alphar=1, nsample=2 * nw * ns, seed=63)
    inp = p.inp
    one = capi.Context(p, n_walkers=2 * nw, nsample_per_walker=ns)
    shards = [capi.Context(p, n_walkers=nw, nsample_per_walker=ns, walker_offset=r * nw) for r in range(2)]
    red = ThreadAllreduce(2)
    for r, c in enumerate(shards):
        c.set_allreduce(red.fn(r))
    for c in [one] + shards:
        c.set_params(p.br, p.Wr, p.slater, 0.0)
        c.seed(4343)
    torch.cuda.synchronize()

    def body(c):
        return [c.iteration(precision, inp.delta_tau, inp.s_factor_scale, inp.s_cut, inp.s_factor0).as_dict()
                for _ in range(steps)]

    want = body(one)
    got = _run_threads(shards, body)
    # the measurement, S, and per refinement iteration one O^T O x; lambda needs two more
    assert red.calls[0] == red.calls[1] and red.calls[0] >= 2 * steps
    for recs in got:
        for a, b in zip(recs, want):
            assert abs(a["Etot"] - b["Etot"]) <= 1e-12 * abs(b["Etot"])
            assert abs(a["accept_ratio"] - b["accept_ratio"]) == 0.0
            assert abs(a["lambda_"] - b["lambda_"]) <= 1e-8 * abs(b["lambda_"])
            if precision == capi.SR_SPLIT_BF16:
                assert a["refine_iterations"] > 0 and a["refine_residual"] < 1e-12
    pw = one.get_params()
    for c in shards:
        for a, b in zip(c.get_params()[:3], pw[:3]):
            assert _rel(a, b) < 1e-8
        assert np.array_equal(c.get_params()[0], shards[0].get_params()[0])  # ranks bit-identical
    for c in [one] + shards:
        c.close()


def test_failing_allreduce_is_reported():
    """A host all-reduce that raises (a rank that has gone away) ends the call with RBMPP_E_COMM, and the
    context is usable again once the all-reduce is removed."""
    L, nw, ns = 4, 4, 8
    p = fm.synthetic_problem(L, translations=True, alphar=1, nsample=nw * ns, seed=64)
    inp = p.inp
    g = capi.Context(p, n_walkers=nw, nsample_per_walker=ns)
    g.set_params(p.br, p.Wr, p.slater, 0.0)
    g.seed(11)

    def gone(ptr, n):
        raise ConnectionError("peer rank left")

    g.make_sample(True)
    m0 = g.measure(want_S=False)
    # a world of one rank: the sum is the buffer itself, so the measurement is unchanged
    g.set_allreduce(lambda ptr, n: None)
    m1 = g.measure(want_S=False)
    assert m1["Etot"] == m0["Etot"] and np.array_equal(m1["gvec"], m0["gvec"])
    # the context reduces by itself: the caller-buffer exchange is refused
    with pytest.raises(capi.RbmppError) as ei:
        g.exchange_measurement(0, 0, 0, 0, np.zeros(6))
    assert ei.value.code == 21, str(ei.value)
    g.set_allreduce(gone)
    with pytest.raises(capi.RbmppError) as ei:
        g.measure(want_S=False)
    assert ei.value.code == 23 and "all-reduce" in str(ei.value)
    assert isinstance(g.allreduce_error, ConnectionError)
    g.set_allreduce(None)
    m = g.measure(want_S=False)
    assert np.isfinite(m["Etot"])
    g.close()

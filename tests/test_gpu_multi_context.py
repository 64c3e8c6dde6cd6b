"""The product's multi-GPU path on one GPU: walkers sharded over two contexts, the one exchange of an SR step
(rbmpp_exchange_measurement, the MPI_ALLREDUCE block of main.f90:348-369) done by summing the two contexts'
device buffers, then the SR step on the reduced sums.  It must equal one context holding all walkers.
Also: rbmpp_copy_state makes a second context continue exactly as the first.
"""
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

"""Split-BF16 tensor-core S build and the refined SR step against the all-FP64 path.

S = sum_s O_s O_s^T is built as H^T H + H^T L + L^T H with O = H + L split into BF16 parts (FP32
accumulation on the tensor cores) and an exact FP64 diagonal.  The SR solve is then refined by conjugate
gradients on the exact FP64 S (applied through O), preconditioned by the split-precision Cholesky
factor.  Stated tolerances: S entries within 5e-5 of max|S| (diagonal within 1e-12 relative), and after
refinement the SR direction and lambda within 1e-8 relative and the updated parameters within 1e-9 of the
FP64 path's.
"""
import numpy as np
import pytest

from rbm_pp_b200 import capi
from rbm_pp_b200 import formats as fm

pytestmark = pytest.mark.gpu


def _ctx(L, trans, alphar, nw, ns, seed=5):
    p = fm.synthetic_problem(L, translations=trans, alphar=alphar, nsample=nw * ns, seed=seed)
    g = capi.Context(p, n_walkers=nw, nsample_per_walker=ns)
    g.set_params(p.br, p.Wr, p.slater, 0.0)
    g.seed(99)
    return p, g


@pytest.mark.parametrize("L,trans,alphar,nw,ns", [(6, True, 2, 32, 8), (4, False, 1, 20, 7)])
def test_split_bf16_s_matrix_error(L, trans, alphar, nw, ns):
    p, g = _ctx(L, trans, alphar, nw, ns)
    g.make_sample(True)
    g.set_s_precision(capi.SR_FP64)
    S64 = g.measure(want_S=True)["S"]
    g.set_s_precision(capi.SR_SPLIT_BF16)
    Ssp = g.measure(want_S=True)["S"]
    scale = np.abs(S64).max()
    d64, dsp = np.diag(S64), np.diag(Ssp)
    assert np.all(np.abs(dsp - d64) <= 1e-12 * np.maximum(np.abs(d64), 1e-300))
    assert np.array_equal(Ssp, Ssp.T)
    err = np.abs(Ssp - S64).max() / scale
    assert err < 5e-5, err
    assert err > 0.0  # the split path really ran in reduced precision
    g.close()


@pytest.mark.parametrize("L,trans,alphar,nw,ns", [(6, True, 2, 32, 8), (4, True, 1, 16, 8)])
def test_split_bf16_sr_step_matches_fp64(L, trans, alphar, nw, ns):
    p, a = _ctx(L, trans, alphar, nw, ns)
    _, b = _ctx(L, trans, alphar, nw, ns)
    for c in (a, b):
        c.make_sample(True)
        c.measure(want_S=False)
    oa, dxa = a.sr_step(1, 0.05, 1e-3, 1e-3, precision=capi.SR_FP64)
    ob, dxb = b.sr_step(1, 0.05, 1e-3, 1e-3, precision=capi.SR_SPLIT_BF16, refine_steps=50)
    assert ob.refine_residual < 1e-12, (ob.refine_residual, ob.refine_iterations)
    assert np.abs(dxb - dxa).max() <= 1e-8 * np.abs(dxa).max(), np.abs(dxb - dxa).max() / np.abs(dxa).max()
    assert abs(ob.lambda_ - oa.lambda_) <= 1e-8 * abs(oa.lambda_)
    assert ob.nSmat == oa.nSmat and ob.kmax == oa.kmax
    for xa, xb in zip(a.get_params()[:3], b.get_params()[:3]):
        assert np.abs(xb - xa).max() <= 1e-9 * max(np.abs(xa).max(), 1e-300)
    a.close()
    b.close()

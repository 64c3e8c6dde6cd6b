"""rbmpp_eval_configs_noalloc against rbmpp_eval_configs.

The allocation-free entry point serves callers that can't call cudaMalloc (a host code whose pool
allocator owns the GPU's memory, or a loop that must not be stalled by cudaFree).  It keeps its scratch
in one fixed device array shared by every call, so the test runs two calls in a row with different
configurations and checks each against the allocating entry point.  The test allocates the caller's
device buffers with torch; the library allocates nothing for the call.
"""
import numpy as np
import pytest

from rbm_pp_b200 import capi
from rbm_pp_b200 import formats as fm

pytestmark = pytest.mark.gpu

RTOL = 1e-10
MAX_CONFIGS = 4096


def _configs(N, n, seed):
    rng = np.random.default_rng(seed)
    x = -np.ones((n, N), dtype=np.int32)
    for r in x:
        r[rng.choice(N, N // 2, replace=False)] = 1
    return x


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_noalloc_matches_eval_configs_on_consecutive_calls():
    import torch

    p = fm.synthetic_problem(6, translations=True, alphar=2, nsample=8, seed=21)
    g = capi.Context(p, n_walkers=1, nsample_per_walker=8)
    g.set_params(p.br, p.Wr, p.slater, 0.0)
    dev = torch.device("cuda", 0)
    N, nq, Nv = g.N, g.n_qp, g.Nv
    for call, (n, seed) in enumerate([(24, 5), (17, 6)]):
        x = _configs(N, n, seed)
        want = g.eval_configs(x, want_h=True, want_O=True)
        d_x = torch.from_numpy(x.reshape(-1)).to(dev)
        d_psi = torch.full((n * (nq + 1) * 2,), float("nan"), dtype=torch.float64, device=dev)
        d_h = torch.full((n * 2,), float("nan"), dtype=torch.float64, device=dev)
        d_O = torch.full((n * Nv,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        g.eval_configs_noalloc(n, d_x.data_ptr(), d_psi.data_ptr(), d_h.data_ptr(), d_O.data_ptr())
        psi = d_psi.cpu().numpy().view(np.complex128).reshape(n, nq + 1)
        hpsi = d_h.cpu().numpy().view(np.complex128)
        O = d_O.cpu().numpy().reshape(n, Nv)
        assert _rel(psi, want["psi"]) < RTOL, call
        assert _rel(hpsi, want["hpsi"]) < RTOL, call
        assert _rel(O, want["O"]) < RTOL, call
    # sizes beyond the fixed scratch are refused before any device work
    with pytest.raises(capi.RbmppError) as ei:
        g.eval_configs_noalloc(MAX_CONFIGS + 1, d_x.data_ptr(), 0, 0, 0)
    assert ei.value.code == 1 and "scratch limit" in str(ei.value)
    g.close()


def test_noalloc_refuses_what_eval_configs_refuses():
    """A lattice whose estimator workspace does not fit one block's shared memory is refused with the
    same code and message as the allocating entry point, before any device work."""
    import torch

    p = fm.synthetic_problem(18, translations=False, alphar=1, nsample=1, seed=3)
    g = capi.Context(p, n_walkers=1, nsample_per_walker=1)
    g.set_params(p.br, p.Wr, p.slater, 0.0)
    x = _configs(g.N, 1, 1)
    try:
        g.eval_configs(x, want_h=True)
    except capi.RbmppError as e:
        want = e
    else:
        want = None
    if want is not None:
        d_x = torch.from_numpy(x.reshape(-1)).to(torch.device("cuda", 0))
        with pytest.raises(capi.RbmppError) as ei:
            g.eval_configs_noalloc(1, d_x.data_ptr(), 0, 0, 0)
        assert ei.value.code == want.code and str(ei.value) == str(want)
    g.close()

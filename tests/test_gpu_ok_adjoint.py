"""The adjoint O_k kernel (rbmpp_eval_configs) as the backward of ln psi, checked against central finite
differences.

ln|psi(x; theta)| is wrapped in a torch.autograd.Function whose forward evaluates psi on the GPU and whose
backward returns d ln psi / d theta_k = O_k(x) / psi(x) from the same launch (O_k is the reweighting-free
d psi / d theta_k of calc_phys_quantity.f90:115-220).  The gradient of a random linear functional of ln psi
over a batch of uniform Sz = 0 configurations is compared with central differences (h = 1e-6) on 64
randomly chosen parameters, at the 10x10 translation-symmetric shape (alpha = 4, full f_ij).  Tolerance:
1e-7 of the largest derivative of the batch, the resolution that central differences of ln psi with
h = 1e-6 have when psi itself is accurate to ~1e-14.
"""
import numpy as np
import pytest

from rbm_pp_b200 import capi
from rbm_pp_b200 import formats as fm

pytestmark = pytest.mark.gpu


def _unpack(theta, N, alphar):
    br = theta[:alphar]
    Wr = theta[alphar:alphar + N * alphar].reshape((N, alphar), order="F")
    sl = theta[alphar + N * alphar:]
    return br, Wr, sl


class LnPsi:
    """torch.autograd.Function over the C ABI: theta (Nv, float64) -> ln|psi| (batch)."""

    @staticmethod
    def make(ctx, x, N, alphar):
        import torch

        class _F(torch.autograd.Function):
            @staticmethod
            def forward(fctx, theta):
                br, Wr, sl = _unpack(theta.detach().cpu().numpy(), N, alphar)
                ctx.set_params(br, Wr, sl, 0.0)
                r = ctx.eval_configs(x, want_h=False, want_O=True)
                psi = r["psi"][:, 0].real
                fctx.save_for_backward(torch.from_numpy(r["O"] / psi[:, None]))
                return torch.from_numpy(np.log(np.abs(psi)))

            @staticmethod
            def backward(fctx, gout):
                (dlog,) = fctx.saved_tensors
                return gout @ dlog

        return _F.apply


def _configs(N, n, seed):
    rng = np.random.default_rng(seed)
    x = -np.ones((n, N), dtype=np.int32)
    for r in x:
        r[rng.choice(N, N // 2, replace=False)] = 1
    return x


@pytest.mark.parametrize("L,trans,alphar,n", [(10, True, 4, 128), (6, False, 2, 256)])
def test_ok_adjoint_matches_central_differences(L, trans, alphar, n):
    import torch
    N = L * L
    p = fm.synthetic_problem(L, translations=trans, alphar=alphar, orbital="full", nsample=8, seed=777)
    g = capi.Context(p, n_walkers=1, nsample_per_walker=8)
    x = _configs(N, n, seed=777)
    theta0 = np.concatenate([p.br, p.Wr.reshape(-1, order="F"), p.slater])
    assert theta0.size == g.Nv
    f = LnPsi.make(g, x, N, alphar)
    w = torch.from_numpy(np.random.default_rng(1).normal(size=n))
    theta = torch.from_numpy(theta0.copy()).requires_grad_(True)
    (w * f(theta)).sum().backward()
    ad = theta.grad.numpy()
    # per-configuration derivatives of the chosen parameters, for the per-entry check
    br, Wr, sl = _unpack(theta0, N, alphar)
    g.set_params(br, Wr, sl, 0.0)
    r0 = g.eval_configs(x, want_h=False, want_O=True)
    dlog = r0["O"] / r0["psi"][:, 0].real[:, None]
    assert np.allclose(ad, w.numpy() @ dlog, rtol=1e-12, atol=1e-12 * np.abs(ad).max())
    rng = np.random.default_rng(2)
    ks = rng.choice(g.Nv, 64, replace=False)
    h = 1e-6
    worst = 0.0
    for k in ks:
        tp, tm = theta0.copy(), theta0.copy()
        tp[k] += h
        tm[k] -= h
        with torch.no_grad():
            fd = (f(torch.from_numpy(tp)) - f(torch.from_numpy(tm))).numpy() / (2 * h)
        scale = max(np.abs(dlog[:, k]).max(), 1e-300)
        err = np.abs(fd - dlog[:, k]).max() / max(np.abs(dlog).max(), 1e-300)
        worst = max(worst, err)
        assert err < 1e-7, (k, err, scale)
    print(f"max |FD - O/psi| / max|O/psi| over 64 parameters: {worst:.3e}")
    g.close()

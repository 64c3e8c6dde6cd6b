"""The adjoint O_k kernel (rbmpp_eval_configs) as the backward of ln psi, checked against central finite
differences and against the oracle's O_k.

ln|psi(x; theta)| is wrapped in a torch.autograd.Function whose forward evaluates psi on the GPU and whose
backward returns d ln psi / d theta_k = O_k(x) / psi(x) from the same launch (O_k is the reweighting-free
d psi / d theta_k of calc_phys_quantity.f90:115-220).

Workload: 10x10, J2 = 0.5, translation-symmetric RBM with alpha = 4 and the full f_ij (N^2 = 10^4 pair
amplitudes): Nv = 10404 parameters; 16384 configurations drawn uniformly from the Sz = 0 sector with a seed.
  - the gradient of a random linear functional of ln psi over the batch (autograd through the adjoint) equals
    the same functional of the per-configuration derivatives;
  - central differences (h = 1e-6) on 64 randomly chosen parameters, every O_k within 1e-8 relative (the
    largest |difference - O_k| over the batch <= 1e-8 times the largest |O_k| over the batch, for each k):
      of psi itself against O_k, on every configuration.  psi is exactly linear in each pair amplitude f_ij
      here (every f_ij fills one entry of each projection's X) and smooth in the RBM parameters, so these
      differences carry rounding only (and an h^2 term of about 1e-12 for the RBM parameters);
      of ln psi against O_k / psi, on the configurations where those differences resolve 1e-8.  They err in
      two ways the first comparison does not: near a node of psi the log-derivative a = O_k / psi grows and
      the differences of ln|psi| err by about (h a)^2 / 3 relative (exactly so for a linear dependence),
      which reaches 1e-3 on some of 16384 random configurations; and where the projection sum psi =
      sum_qp psi_qp cancels (c = sum |psi_qp| / |psi| large; its median is about 9 at 10x10) the rounding of
      psi, about c * 1e-16 relative, divided by h reaches 1e-7.  Entries with (h a)^2 / 3 > 1e-9 or c > 10 are
      counted and left to the first comparison;
  - the oracle's O_k (its full 2N Pfaffian form) on the first 16 configurations of the batch within 1e-10 of
    each configuration's largest derivative.
A smaller 6x6 case without translations runs the generic (runtime block size) kernels the same way.
"""
import numpy as np
import pytest

import pyoracle as po
from rbm_pp_b200 import capi
from rbm_pp_b200 import formats as fm

pytestmark = pytest.mark.gpu

H = 1e-6
TOL_FD = 1e-8


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


def _psi(g, theta, N, alphar, x):
    br, Wr, sl = _unpack(theta, N, alphar)
    g.set_params(br, Wr, sl, 0.0)
    return g.eval_configs(x, want_h=False)["psi"][:, 0].real


@pytest.mark.parametrize("L,trans,alphar,n", [(10, True, 4, 16384), (6, False, 2, 1024)])
def test_ok_adjoint(L, trans, alphar, n, capsys):
    import torch
    N = L * L
    p = fm.synthetic_problem(L, translations=trans, alphar=alphar, orbital="full", nsample=8, seed=777)
    g = capi.Context(p, n_walkers=1, nsample_per_walker=8)
    x = _configs(N, n, seed=777)
    theta0 = np.concatenate([p.br, p.Wr.reshape(-1, order="F"), p.slater])
    assert theta0.size == g.Nv
    # autograd through the adjoint kernel
    f = LnPsi.make(g, x, N, alphar)
    w = torch.from_numpy(np.random.default_rng(1).normal(size=n))
    theta = torch.from_numpy(theta0.copy()).requires_grad_(True)
    (w * f(theta)).sum().backward()
    ad = theta.grad.numpy()
    br, Wr, sl = _unpack(theta0, N, alphar)
    g.set_params(br, Wr, sl, 0.0)
    r0 = g.eval_configs(x, want_h=False, want_O=True)
    psi0 = r0["psi"][:, 0].real
    canc = np.abs(r0["psi"][:, 1:]).sum(axis=1) / np.abs(psi0)  # cancellation of the projection sum
    assert np.abs(r0["psi"][:, 1:].sum(axis=1).real - psi0).max() <= 1e-12 * np.abs(r0["psi"][:, 1:]).sum(axis=1).max()
    dlog = r0["O"] / psi0[:, None]
    del r0
    assert np.allclose(ad, w.numpy() @ dlog, rtol=1e-12, atol=1e-12 * np.abs(ad).max())
    # the oracle's O_k on the first 16 configurations
    o = po.Oracle(p, nranks=1, nsample_per_rank=8, nthreads=8)
    o.set_params(br, Wr, sl, 0.0)
    ro = o.eval_configs(x[:16], want_h=False, want_O=True)
    for k in range(16):
        ref = ro["O"][k].real
        assert np.abs(dlog[k] * psi0[k] - ref).max() <= 1e-10 * np.abs(ref).max(), k
    # central differences, every O_k relative to its own scale over the batch.  The f_ii amplitudes never enter
    # the Pfaffian (a site is not both up and down), so their O_k vanish: two of them are checked to have
    # vanishing differences too, and the 64 are drawn from the others.
    scales = np.abs(dlog).max(axis=0)
    zero = np.flatnonzero(scales == 0)
    assert 0 < zero.size <= N, zero.size
    rng = np.random.default_rng(2)
    for k in zero[:2]:
        tp, tm = theta0.copy(), theta0.copy()
        tp[k] += H
        tm[k] -= H
        assert np.array_equal(_psi(g, tp, N, alphar, x), _psi(g, tm, N, alphar, x)), k
    ks = rng.choice(np.flatnonzero(scales > 0), 64, replace=False)
    err_psi, err_log, err_log_all, near_node = [], [], [], 0
    for k in ks:
        tp, tm = theta0.copy(), theta0.copy()
        tp[k] += H
        tm[k] -= H
        pp, pm = _psi(g, tp, N, alphar, x), _psi(g, tm, N, alphar, x)
        ok = dlog[:, k] * psi0
        err_psi.append(float(np.abs((pp - pm) / (2 * H) - ok).max() / np.abs(ok).max()))
        fd = (np.log(np.abs(pp)) - np.log(np.abs(pm))) / (2 * H)
        a = np.abs(dlog[:, k])
        off = ((H * a) ** 2 / 3 <= 1e-9) & (canc <= 10.0)
        near_node += int((~off).sum())
        err_log.append(float(np.abs(fd - dlog[:, k])[off].max() / a[off].max()))
        err_log_all.append(float(np.abs(fd - dlog[:, k]).max() / scales[k]))
    err_psi, err_log = np.array(err_psi), np.array(err_log)
    with capsys.disabled():
        print(f"\nOK_FD L={L} n={n} parameters={len(ks)}: psi differences max {err_psi.max():.3e} "
              f"(median {np.median(err_psi):.3e}); ln psi differences off nodes max {err_log.max():.3e} "
              f"(median {np.median(err_log):.3e}), {near_node} of {n * len(ks)} entries near a node or cancelling, "
              f"all entries max {max(err_log_all):.3e}")
    assert err_psi.max() <= TOL_FD, (ks[err_psi.argmax()], err_psi.max())
    assert err_log.max() <= TOL_FD, (ks[err_log.argmax()], err_log.max())
    assert near_node <= 0.75 * n * len(ks)
    g.close()

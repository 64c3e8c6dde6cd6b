"""Pins of the oracle's correlation measurement (the Calc_Correlation program's calc_phys_quantity_after_opt).

No reference outputs exist to pin against, so these are identities that the reference's formulas imply:
- its scalars equal those of the plain final-energy measurement on the same samples;
- the energy is the bond sum of the pair correlations, Etot = sum_b J_b (Chi_sp(1, b) + 2 Chi_sp(2, b)):
  a J1 bond joins the two sublattices (sign -1 times the exchange sign -1), a J2 bond stays on one (+1 times +1);
- every diagonal pair (i, i) has Chi_sp(1) = Chi_sp(2) = norm, since x_i^2 = 1 and Chi_loc(2, ii) = psi;
- each Chi_vbs(ii, t) is a sum of squares.
"""
import numpy as np
import pytest

import pyoracle as po
from rbm_pp_b200 import formats as fm


def _bond_pairs(L):
    """(type, i1, i2) of bond_map (calc_phys_quantity.f90:428-473), 0-based sites."""
    out = []
    for t in range(4):
        for i1 in range(L * L):
            ix, iy = divmod(i1, L)
            if t == 0:
                ix = (ix + 1) % L
            elif t == 1:
                iy = (iy + 1) % L
            elif t == 2:
                ix, iy = (ix + 1) % L, (iy + 1) % L
            else:
                ix, iy = (ix + 1) % L, (iy - 1) % L
            out.append((t, i1, ix * L + iy))
    return out


def _pair_index(a, b):
    a, b = min(a, b), max(a, b)
    return b * (b + 1) // 2 + a


@pytest.mark.parametrize("L,trans,alphar", [(4, False, 1), (4, True, 1), (6, False, 2)])
def test_correlation_identities(L, trans, alphar):
    nw, ns = 2, 3
    p = fm.synthetic_problem(L, translations=trans, alphar=alphar, nsample=nw * ns, seed=21, J2=0.45)
    outs = []
    for kind in ("corr", "energy"):
        o = po.Oracle(p, nranks=nw, nsample_per_rank=ns, nthreads=2)
        o.set_params(p.br, p.Wr, p.slater, 0.0)
        o.seed(314)
        o.make_sample(True)
        outs.append(o.measure_correlation() if kind == "corr" else o.measure_energy())
    mc, me = outs
    for k in ("Etot", "Etot2", "norm", "wf_av"):
        assert abs(mc[k] - me[k]) <= 1e-12 * abs(me[k]), k
    assert abs(mc["wf_sgn"]) <= nw * ns + 1e-12
    chi = mc["chi_sp"]
    J = (p.inp.J1, p.inp.J1, p.inp.J2, p.inp.J2)
    e_bonds = sum(J[t] * (chi[0, _pair_index(a, b)] + 2.0 * chi[1, _pair_index(a, b)]) for t, a, b in _bond_pairs(L))
    assert abs(e_bonds - mc["Etot"]) <= 1e-10 * abs(mc["Etot"])
    diag = [_pair_index(i, i) for i in range(L * L)]
    assert np.allclose(chi[0, diag], mc["norm"], rtol=1e-12)
    assert np.allclose(chi[1, diag], mc["norm"], rtol=1e-12)
    assert (mc["chi_vbs"][diag, :] >= 0.0).all()

"""Pins of the CPU oracle against independent known answers (no GPU needed).

The reference has no tests, fixtures or golden vectors, and cannot be compiled here, so the oracle
is checked against: brute-force Pfaffians, numpy's MT19937 core, numpy LAPACK inverses, exact
diagonalisation of the J1-J2 Hamiltonian, finite differences of ln psi, and its own scratch
recomputation along a Markov chain.
"""
import numpy as np
import pytest

import ed
import pyoracle as po
from rbm_pp_b200 import formats as fm


def pf_brute(A):
    n = A.shape[0]
    if n == 0:
        return 1.0
    s = 0.0
    for j in range(1, n):
        idx = [k for k in range(n) if k not in (0, j)]
        s += (-1) ** (j + 1) * A[0, j] * pf_brute(A[np.ix_(idx, idx)])
    return s


@pytest.mark.parametrize("n", [2, 4, 6, 8, 10])
def test_pfaffian_brute_force(n):
    rng = np.random.default_rng(n)
    B = rng.normal(size=(n, n))
    A = B - B.T
    assert abs(po.pfaffian(A) - pf_brute(A)) <= 1e-12 * max(1.0, abs(pf_brute(A)))


def test_pfaffian_squared_is_det():
    rng = np.random.default_rng(7)
    B = rng.normal(size=(40, 40))
    A = B - B.T
    pf = po.pfaffian(A)
    sign, logdet = np.linalg.slogdet(A)
    assert sign > 0
    assert abs(2 * np.log(abs(pf)) - logdet) < 1e-10


def test_mt19937_matches_numpy_core():
    """mt.f twist + tempering equals numpy's MT19937 when both start from the Knuth-69069 state."""
    for seed in (1, 4357, 12345, 2**31 - 1):
        st = po.mt_state(seed)
        bg = np.random.MT19937(0)
        bg.state = {"bit_generator": "MT19937", "state": {"key": st, "pos": 624}}
        raw = bg.random_raw(5000).astype(np.uint32)
        assert np.array_equal(raw, po.mt_u32(seed, 5000))


def test_grnd_mapping():
    """grnd = y / (2^32 - 1) (mt.f:95-99), computed in double with IEEE division."""
    u32 = po.mt_u32(99, 1000)
    g = po.grnd(99, 1000)
    assert np.array_equal(g, u32.astype(np.float64) / 4294967295.0)
    # Knuth seeding: mt(i) = 69069 * mt(i-1) mod 2^32 (mt.f:23-26)
    st = po.mt_state(3)
    assert st[0] == 3 and st[1] == (69069 * 3) % 2**32 and st[2] == (69069 * int(st[1])) % 2**32


def test_inverse_matches_numpy():
    rng = np.random.default_rng(3)
    A = rng.normal(size=(30, 30))
    B = po.fortran_array(A, np.float64)
    assert po.lib().orc_inverse(30, B) == 0
    inv = B.reshape((30, 30), order="F")
    assert np.allclose(inv, np.linalg.inv(A), rtol=1e-11, atol=1e-12)


@pytest.fixture(scope="module")
def small_oracle():
    p = fm.synthetic_problem(4, translations=False, alphar=1, nsample=64, seed=5)
    o = po.Oracle(p, nranks=2, nsample_per_rank=32)
    o.set_params(p.br, p.Wr, p.slater, 0.0)
    return p, o


@pytest.mark.parametrize("translations", [False, True])
def test_local_energy_matches_exact_hamiltonian(translations):
    """(H psi)(x) from the fast-update local energy equals the ED Hamiltonian applied to the oracle's
    psi vector over the whole Sz = 0 sector of the 4x4 lattice."""
    p = fm.synthetic_problem(4, translations=translations, alphar=1, nsample=64, seed=11)
    o = po.Oracle(p, nranks=1, nsample_per_rank=8)
    o.set_params(p.br, p.Wr, p.slater, 0.0)
    basis = ed.sz0_basis(16)
    if translations:
        basis = basis[::7]  # subset: the dense projection sum is slower
        r = o.eval_configs(basis, want_h=True)
        full = ed.sz0_basis(16)
        psi_all = o.eval_configs(full, want_h=False)["psi"][:, 0]
        H = ed.hamiltonian(4, 1.0, 0.5, full)
        hp = (H @ psi_all)[::7]
    else:
        r = o.eval_configs(basis, want_h=True)
        H = ed.hamiltonian(4, 1.0, 0.5, basis)
        hp = H @ r["psi"][:, 0]
    scale = np.abs(hp).max()
    assert np.abs(hp - r["hpsi"]).max() <= 1e-10 * scale


@pytest.mark.parametrize("spin_parity", [1, -1])
def test_transverse_local_energy_matches_exact_hamiltonian(spin_parity):
    """The transverse code's projection (beta = -pi/2, pi/2, transverse_code/spin_projection.f90:30-38): every
    block of the Pfaffian matrix is non-zero, and (H psi)(x) from the fast-update local energy still equals the
    ED Hamiltonian applied to the oracle's psi over the whole Sz = 0 sector."""
    p = fm.synthetic_problem(4, translations=False, alphar=1, nsample=64, seed=13, spin_parity=spin_parity)
    o = po.Oracle(p, nranks=1, nsample_per_rank=8, sp_weights=fm.spin_projection_weights(spin_parity, True))
    o.set_params(p.br, p.Wr, p.slater, 0.0)
    SE = o.slater_elements()
    N = 16
    assert np.abs(SE[:N, :N, 0]).max() > 0.01  # same-spin block present
    basis = ed.sz0_basis(16)
    r = o.eval_configs(basis, want_h=True)
    H = ed.hamiltonian(4, 1.0, 0.5, basis)
    hp = H @ r["psi"][:, 0]
    assert np.abs(hp - r["hpsi"]).max() <= 1e-10 * np.abs(hp).max()


def test_transverse_chain_and_ok():
    """Transverse projection: stored Pf along a chain (skew rank-4 fast updates) against scratch, and O_k
    against central differences of psi."""
    p = fm.synthetic_problem(4, translations=True, alphar=1, nsample=16, seed=21)
    w = fm.spin_projection_weights(1, True)
    o = po.Oracle(p, nranks=2, nsample_per_rank=8, sp_weights=w)
    o.set_params(p.br, p.Wr, p.slater, 0.0)
    o.seed(78)
    o.make_sample(True)
    x, psi, pf = o.samples()
    r = o.eval_configs(x.reshape(-1, 16), want_h=False)
    # the fast-update products drift; the reference bounds that drift by 1e-5 between recomputes
    assert np.allclose(np.abs(psi.reshape(-1, psi.shape[-1])[:, 0]), np.abs(r["psi"][:, 0]), rtol=1e-6)
    xs = x.reshape(-1, 16)[:3]
    base = o.eval_configs(xs, want_h=False, want_O=True)
    theta0 = np.concatenate([p.br, p.Wr.reshape(-1, order="F"), p.slater])
    rng = np.random.default_rng(3)
    h = 1e-6
    for k in list(rng.choice(o.Nv, 16, replace=False)) + [0, 5]:
        def psi_at(delta):
            t = theta0.copy()
            t[k] += delta
            o.set_params(t[:1], t[1:17].reshape((16, 1), order="F"), t[17:], 0.0)
            return o.eval_configs(xs, want_h=False)["psi"][:, 0].real
        fd = (psi_at(h) - psi_at(-h)) / (2 * h)
        an = base["O"][:, k].real
        assert np.all(np.abs(fd - an) <= 1e-6 * np.abs(base["psi"][:, 0]) + 1e-8 * np.abs(an)), (k, fd, an)
    o.set_params(p.br, p.Wr, p.slater, 0.0)


def test_ed_gauge_invariance_and_value():
    E_g = ed.ground_state_energy(4, 1.0, 0.5, gauge=True)
    E_u = ed.ground_state_energy(4, 1.0, 0.5, gauge=False)
    assert abs(E_g - E_u) < 1e-9
    # E0/N in S.S units = E0/(4N) for the 4x4 J1-J2 model at J2 = 0.5
    assert -0.53 < E_g / 64 < -0.52


def test_proposal_ratio_matches_scratch(small_oracle):
    """calculate_new_PfM_two (fast ratio) equals Pf of the exchanged configuration from scratch, up to
    the electron-relabelling sign, for random exchanges."""
    p, o = small_oracle
    rng = np.random.default_rng(1)
    N = 16
    for _ in range(20):
        x = -np.ones(N, dtype=np.int32)
        x[rng.choice(N, 8, replace=False)] = 1
        ups = np.where(x == 1)[0]
        dns = np.where(x == -1)[0]
        i1, i2 = int(rng.choice(ups)), int(rng.choice(dns))
        pf_old, pf_new = o.proposal_pf(x, i1, i2)
        y = x.copy()
        y[i1], y[i2] = -1, 1
        pf_scratch = o.eval_configs(y[None, :], want_h=False)["pf"][0]
        # fast update keeps electron labels; scratch sorts them: the ratio differs by a sign per qp
        ratio = np.abs(pf_new) / np.abs(pf_scratch)
        assert np.allclose(ratio, 1.0, rtol=1e-10)


def test_chain_fast_update_matches_scratch():
    """Along a Metropolis chain the stored Pf values (fast updates) agree with scratch recomputation."""
    p = fm.synthetic_problem(4, translations=True, alphar=1, nsample=16, seed=2)
    o = po.Oracle(p, nranks=2, nsample_per_rank=8)
    o.set_params(p.br, p.Wr, p.slater, 0.0)
    o.seed(77)
    o.make_sample(True)
    x, psi, pf = o.samples()
    xs = x.reshape(-1, 16)
    r = o.eval_configs(xs, want_h=False)
    assert np.allclose(np.abs(psi.reshape(-1, psi.shape[-1])[:, 0]), np.abs(r["psi"][:, 0]), rtol=1e-9)


def test_ok_against_finite_differences():
    """O_k (raw d psi / d theta_k) against central differences of psi, h = 1e-6 (config 3 check)."""
    p = fm.synthetic_problem(4, translations=True, alphar=2, nsample=16, seed=4)
    o = po.Oracle(p, nranks=1, nsample_per_rank=4)
    o.set_params(p.br, p.Wr, p.slater, 0.0)
    rng = np.random.default_rng(9)
    x = -np.ones((3, 16), dtype=np.int32)
    for r_ in x:
        r_[rng.choice(16, 8, replace=False)] = 1
    base = o.eval_configs(x, want_h=False, want_O=True)
    Nv = o.Nv
    ks = list(rng.choice(Nv, 24, replace=False)) + [0, 2, 2 + 16 * 2 + 5]
    h = 1e-6
    theta0 = np.concatenate([p.br, p.Wr.reshape(-1, order="F"), p.slater])
    for k in ks:
        def psi_at(delta):
            t = theta0.copy()
            t[k] += delta
            br = t[:2]
            Wr = t[2:2 + 32].reshape((16, 2), order="F")
            o.set_params(br, Wr, t[2 + 32:], 0.0)
            return o.eval_configs(x, want_h=False)["psi"][:, 0]
        fd = (psi_at(h) - psi_at(-h)) / (2 * h)
        an = base["O"][:, k]
        scale = np.abs(base["psi"][:, 0])
        assert np.all(np.abs(fd - an) <= 1e-6 * scale + 1e-8 * np.abs(an)), (k, fd, an)
    o.set_params(p.br, p.Wr, p.slater, 0.0)


def test_vmc_energy_decreases_toward_ed():
    """Config-1 shape: 4x4, J2 = 0.5, 1024 samples over 8 walkers; 40 SR steps lower the energy and
    it stays above the exact ground state."""
    p = fm.synthetic_problem(4, translations=False, alphar=1, nsample=1024, seed=12345)
    o = po.Oracle(p, nranks=8, nsample_per_rank=128, nthreads=4)
    loop = po.VMCLoop(o, p, iseed0=12345)
    E = [loop.iteration_step()["Etot"] for _ in range(40)]
    E0 = ed.ground_state_energy(4, 1.0, 0.5)
    assert E[-1] < E[0] - 5.0
    assert min(E) > E0 - 1.0


def test_formats_round_trip(tmp_path):
    p = fm.synthetic_problem(4, translations=True, alphar=2, orbital="sublattice2", nsample=32, seed=3)
    fm.write_problem(str(tmp_path), p)
    q = fm.read_problem(str(tmp_path))
    assert q.inp == p.inp
    assert np.array_equal(q.sym.W_map, p.sym.W_map)
    assert np.array_equal(q.orbital_idx, p.orbital_idx)
    assert np.allclose(q.slater, p.slater, rtol=1e-14)
    assert np.allclose(q.Wr, p.Wr, atol=1e-15) and np.allclose(q.br, p.br, atol=1e-15)
    assert abs(np.abs(q.slater).mean() - 0.25) < 1e-12


def _complex_problem(L, trans, alphar, seed):
    p = fm.synthetic_problem(L, translations=trans, alphar=alphar, nsample=16, seed=seed)
    p.inp.alphac = 1
    rng = np.random.default_rng(seed + 1)
    N = L * L
    p.bc = 0.05 * (rng.normal(size=1) + 1j * rng.normal(size=1))
    p.Wc = 0.05 * (rng.normal(size=(N, 1)) + 1j * rng.normal(size=(N, 1)))
    return p


def test_complex_units_local_energy_and_ok():
    """Complex RBM units (alpha_c = 1, RBM.f90 thetac; sub.f90:37-41): H psi from the fast-update local energy
    equals the ED Hamiltonian applied to psi over the Sz = 0 sector, and O_k equals central differences of psi for
    the complex parameters' real and imaginary parts (the pairs of calc_phys_quantity.f90:115-160)."""
    p = _complex_problem(4, False, 1, 31)
    o = po.Oracle(p, nranks=1, nsample_per_rank=8)
    o.set_params_c(p.bc, p.Wc)
    o.set_params(p.br, p.Wr, p.slater, 0.0)
    basis = ed.sz0_basis(16)
    r = o.eval_configs(basis, want_h=True)
    assert np.abs(r["psi"][:, 0].imag).max() > 1e-3 * np.abs(r["psi"][:, 0]).max()
    H = ed.hamiltonian(4, 1.0, 0.5, basis)
    hp = H @ r["psi"][:, 0]
    assert np.abs(hp - r["hpsi"]).max() <= 1e-10 * np.abs(hp).max()
    xs = basis[::997][:4]
    base = o.eval_configs(xs, want_h=False, want_O=True)
    h = 1e-6
    # parameter order: bc (re, im), Wc(iw) (re, im), br, Wr, f
    for k in [0, 1, 2, 3, 2 + 2 * 7, 2 + 2 * 7 + 1, 34, 35 + 4]:
        def psi_at(delta):
            bc, Wc, br, Wr = p.bc.copy(), p.Wc.copy(), p.br.copy(), p.Wr.copy()
            if k < 2:
                bc[0] += delta * (1.0 if k == 0 else 1j)
            elif k < 34:
                iw, part = divmod(k - 2, 2)
                Wc[iw, 0] += delta * (1.0 if part == 0 else 1j)
            elif k == 34:
                br[0] += delta
            else:
                Wr[k - 35, 0] += delta
            o.set_params_c(bc, Wc)
            o.set_params(br, Wr, p.slater, 0.0)
            return o.eval_configs(xs, want_h=False)["psi"][:, 0]
        fd = (psi_at(h) - psi_at(-h)) / (2 * h)
        an = base["O"][:, k]
        assert np.all(np.abs(fd - an) <= 1e-7 * np.abs(base["psi"][:, 0]) + 1e-8 * np.abs(an)), (k, fd, an)
    o.set_params_c(p.bc, p.Wc)
    o.set_params(p.br, p.Wr, p.slater, 0.0)

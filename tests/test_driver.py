"""The C++ main.f90 host program (rbm_pp_b200/rbmpp_driver) over the C ABI.

CPU: its readers of RBM.input, sym_info.txt, orbitalidx.def, zqp_orbital_initial.dat and W.input agree
with the Python readers on files written in the reference's formats.
GPU: a short optimisation run (Nstep = 3, Nav = 2, 8 emulated ranks) reproduces the oracle's energies,
averaged parameters and final-energy measurement (main.f90:300-575) on the same seed.
"""
import os
import subprocess

import numpy as np
import pytest

from rbm_pp_b200 import build
from rbm_pp_b200 import formats as fm


def _driver():
    build.build()
    return build.DRIVER


@pytest.mark.parametrize("trans,orbital", [(False, "full"), (True, "sublattice2")])
def test_driver_reads_reference_inputs(tmp_path, trans, orbital):
    p = fm.synthetic_problem(4, translations=trans, alphar=2, orbital=orbital, nsample=64, seed=3)
    fm.write_problem(str(tmp_path), p)
    out = subprocess.run([_driver(), "--dir", str(tmp_path), "--walkers", "8", "--check-inputs"],
                         capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    t = out.stdout.split()
    kv = {t[i]: t[i + 1] for i in range(0, len(t) - 1, 2)}
    q = fm.read_problem(str(tmp_path))
    assert int(kv["N"]) == 16 and int(kv["ns"]) == 8 and int(kv["alphar"]) == 2
    assert int(kv["n_mp"]) == q.sym.n_mp and int(kv["n_slater"]) == q.n_slater
    assert int(kv["W.input"]) == 1
    assert abs(float(kv["mean|f|"]) - 0.25) < 1e-12
    assert int(kv["W_map(1,last)"]) == int(q.sym.W_map[0, -1])
    assert int(kv["orbital_idx(N,N)"]) == int(q.orbital_idx[-1, -1])


def test_driver_rejects_bad_walker_split(tmp_path):
    p = fm.synthetic_problem(4, translations=False, alphar=1, nsample=64, seed=3)
    fm.write_problem(str(tmp_path), p)
    out = subprocess.run([_driver(), "--dir", str(tmp_path), "--walkers", "7", "--check-inputs"],
                         capture_output=True, text=True, timeout=60)
    assert out.returncode != 0 and "multiple of --walkers" in out.stderr


@pytest.mark.gpu
def test_driver_run_matches_oracle(tmp_path):
    import pyoracle as po
    nw, ns, nstep, nav, seed = 8, 8, 3, 2, 4242
    p = fm.synthetic_problem(4, translations=False, alphar=1, nsample=nw * ns, seed=17, Nstep=nstep, Nav=nav)
    fm.write_problem(str(tmp_path), p)
    out = subprocess.run([_driver(), "--dir", str(tmp_path), "--walkers", str(nw), "--seed", str(seed)],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr + out.stdout
    got = np.loadtxt(os.path.join(tmp_path, "Energy_vs_Iteration.txt"))
    # oracle: the same loop (VMCLoop restates main.f90:300-455), then the averaging and final energy
    o = po.Oracle(p, nranks=nw, nsample_per_rank=ns, nthreads=4)
    loop = po.VMCLoop(o, p, iseed0=seed)
    acc = None
    shift_av = 0.0
    for it in range(1, nstep + 1):
        shift_now = loop.shift
        rec = loop.iteration_step()
        assert abs(got[it - 1, 1] - rec["Etot"]) <= 1e-9 * abs(rec["Etot"]), (it, got[it - 1, 1], rec["Etot"])
        if it > nstep - nav:
            br, Wr, sl, _ = o.get_params()
            shift_av += shift_now
            acc = (br, Wr, sl) if acc is None else (acc[0] + br, acc[1] + Wr, acc[2] + sl)
    br, Wr, sl = (a / nav for a in acc)
    q = fm.read_W(os.path.join(tmp_path, "optimized_W.txt"), 16, 1)
    assert np.allclose(q[0], br, rtol=1e-9, atol=1e-13) and np.allclose(q[1], Wr, rtol=1e-9, atol=1e-13)
    f = fm.read_zqp(os.path.join(tmp_path, "zqp_orbital_opt.dat"), p.n_slater, rescale=False)
    assert np.allclose(f, sl, rtol=1e-9, atol=1e-13)
    o.set_params(br, Wr, sl, shift_av / nav)
    o.make_sample(True)
    for _ in range(2):
        o.make_sample(False)
    fin = np.loadtxt(os.path.join(tmp_path, "energy_after_opt.txt"))
    for it in range(nav):
        o.make_sample(False)
        m = o.measure_energy()
        E = m["Etot"] / m["norm"]
        assert abs(fin[it, 1] - E) <= 1e-8 * abs(E), (it, fin[it, 1], E)


@pytest.mark.gpu
def test_driver_correlation_files(tmp_path):
    """--correlation: Calc_Correlation's final measurement writes fort.<60000+it> (Chi_sp / norm) and
    fort.<70000+it> (Chi_vbs / norm).  Each round obeys Chi_sp(1, ii) = Chi_sp(2, ii) = 1 and the bond sum
    rule E = sum_b J_b (Chi_sp(1, b) + 2 Chi_sp(2, b)) against its own line of energy_after_opt.txt."""
    L, nw, ns, nav = 4, 8, 4, 2
    p = fm.synthetic_problem(L, translations=False, alphar=1, nsample=nw * ns, seed=19, Nstep=2, Nav=nav, J2=0.5)
    fm.write_problem(str(tmp_path), p)
    out = subprocess.run([_driver(), "--dir", str(tmp_path), "--walkers", str(nw), "--seed", "99", "--correlation"],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr + out.stdout
    fin = np.loadtxt(os.path.join(tmp_path, "energy_after_opt.txt"))
    N = L * L
    nchi = N * (N + 1) // 2

    def pair(a, b):
        a, b = min(a, b), max(a, b)
        return b * (b + 1) // 2 + a

    bonds = []
    for t in range(4):
        for i1 in range(N):
            ix, iy = divmod(i1, L)
            dx, dy = ((1, 0), (0, 1), (1, 1), (1, -1))[t]
            bonds.append((t, i1, ((ix + dx) % L) * L + (iy + dy) % L))
    J = (p.inp.J1, p.inp.J1, p.inp.J2, p.inp.J2)
    for it in range(1, nav + 1):
        sp = np.loadtxt(os.path.join(tmp_path, f"fort.{60000 + it}"), comments="#")
        vb = np.loadtxt(os.path.join(tmp_path, f"fort.{70000 + it}"), comments="#")
        assert sp.shape == (nchi, 3) and vb.shape == (nchi, 5)
        diag = [pair(i, i) for i in range(N)]
        assert np.allclose(sp[diag, 1], 1.0, rtol=1e-12) and np.allclose(sp[diag, 2], 1.0, rtol=1e-12)
        e = sum(J[t] * (sp[pair(a, b), 1] + 2.0 * sp[pair(a, b), 2]) for t, a, b in bonds)
        assert abs(e - fin[it - 1, 1]) <= 1e-9 * abs(fin[it - 1, 1]), (it, e, fin[it - 1, 1])
    # the measurement block of Calc_Correlation/main.f90:587-594 on standard output, in its order and formats
    lines = out.stdout.splitlines()
    heads = [k for k, ln in enumerate(lines) if ln.startswith("Iteration (Energy Measuement) :")]
    assert len(heads) == nav
    for h in heads:
        blk = lines[h:h + 7]
        keys = ["   total energy         :", "   energy variance      :", "   acceptance ratio     :",
                "   wf_av, shift         :", "   norm                 :", "   wf_sgn               :"]
        for ln, key in zip(blk[1:], keys):
            assert ln.startswith(key), (ln, key)
        wf = blk[4][len(keys[3]):]
        assert len(wf) == 40 and wf[:20].strip().startswith("0.") and "E" in wf[:20]  # 2E20.5
        sg = blk[6][len(keys[5]):]
        assert len(sg) == 60
        a, re_, im = (float(sg[i:i + 20]) for i in (0, 20, 40))
        assert a == abs(re_) and im == 0.0 and a <= 1.0
        assert abs(float(blk[5][len(keys[4]):]) - 1.0) < 1.0  # norm / (Nsample Nmpi), weights <= 1


def test_driver_writes_input_checks(tmp_path):
    """chk_orbitalidx.def, chk_qptransidx.def and chk_zqp_orbital_opt.dat (parameter.f90:177-207) echo the
    inputs the driver read, in the reference's record layout and Fortran E format."""
    p = fm.synthetic_problem(4, translations=True, alphar=1, nsample=16, seed=8)
    fm.write_problem(str(tmp_path), p)
    out = subprocess.run([_driver(), "--dir", str(tmp_path), "--walkers", "2", "--check-inputs"],
                         capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    q = fm.read_problem(str(tmp_path))
    N = 16
    lines = open(os.path.join(tmp_path, "chk_orbitalidx.def")).read().splitlines()
    assert int(lines[0]) == q.n_slater
    rows = np.array([[int(v) for v in ln.split()] for ln in lines[1:]])
    assert rows.shape == (N * N, 3)
    assert np.array_equal(rows[:, 2].reshape(N, N), q.orbital_idx - 1)  # i1 outer, i2 inner
    lines = open(os.path.join(tmp_path, "chk_qptransidx.def")).read().splitlines()
    n_mp = int(lines[0])
    assert n_mp == q.sym.n_mp
    para = np.array([[float(v) for v in ln.split()[1:]] for ln in lines[1:1 + n_mp]])
    assert np.allclose(para[:, 0] + 1j * para[:, 1], q.sym.para_mp, atol=1e-12)
    idx = np.array([[int(v) for v in ln.split()] for ln in lines[1 + n_mp:]])
    assert np.array_equal(idx[:, 2].reshape(n_mp, N).T, q.sym.W_map)
    lines = open(os.path.join(tmp_path, "chk_zqp_orbital_opt.dat")).read().splitlines()
    assert lines[0].split()[-1] == str(q.n_slater)
    vals = [ln[4:].strip() for ln in lines[1:]]
    assert all(v.lstrip("-").startswith("0.") and "E" in v for v in vals)
    f = np.array([float(v) for v in vals])
    assert np.allclose(f, q.slater, rtol=1e-14, atol=0)
    assert abs(np.abs(f).mean() - 0.25) < 1e-12


@pytest.mark.gpu
def test_driver_transverse_matches_oracle(tmp_path):
    """--transverse: the transverse code's main program (transverse_code/main.f90) over the library's skew form;
    its energies per iteration follow the oracle's loop with the transverse weights and shift schedule.  No RBM
    units: with this projection the bias has no fluctuation (O_b / psi = tanh b), which the reference's S-diagonal
    check stops on."""
    import pyoracle as po
    nw, ns, nstep, seed = 8, 8, 3, 4343
    p = fm.synthetic_problem(4, translations=False, alphar=0, nsample=nw * ns, seed=18, Nstep=nstep, Nav=1)
    fm.write_problem(str(tmp_path), p)
    out = subprocess.run([_driver(), "--dir", str(tmp_path), "--walkers", str(nw), "--seed", str(seed),
                          "--transverse"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr + out.stdout
    got = np.loadtxt(os.path.join(tmp_path, "Energy_vs_Iteration.txt"))
    o = po.Oracle(p, nranks=nw, nsample_per_rank=ns, nthreads=4, sp_weights=fm.spin_projection_weights(1, True))
    loop = po.VMCLoop(o, p, iseed0=seed, shift_coef=0.003)
    for it in range(1, nstep + 1):
        rec = loop.iteration_step()
        assert abs(got[it - 1, 1] - rec["Etot"]) <= 1e-9 * abs(rec["Etot"]), (it, got[it - 1, 1], rec["Etot"])


def _complex_units_problem(nw, ns, nstep, seed):
    p = fm.synthetic_problem(4, translations=False, alphar=1, nsample=nw * ns, seed=seed, Nstep=nstep, Nav=1)
    p.inp.alphac = 1
    rng = np.random.default_rng(seed)
    p.bc = 0.05 * (rng.normal(size=1) + 1j * rng.normal(size=1))
    p.Wc = 0.05 * (rng.normal(size=(16, 1)) + 1j * rng.normal(size=(16, 1)))
    return p


def test_complex_units_w_input_round_trip(tmp_path):
    """W.input with complex units (parameter.f90:42-75: a (re, im) block per complex unit before the real ones)."""
    p = _complex_units_problem(8, 8, 2, 5)
    fm.write_problem(str(tmp_path), p)
    q = fm.read_problem(str(tmp_path))
    assert q.inp.alphac == 1 and np.allclose(q.bc, p.bc, atol=1e-15) and np.allclose(q.Wc, p.Wc, atol=1e-15)
    assert np.allclose(q.br, p.br, atol=1e-15) and np.allclose(q.Wr, p.Wr, atol=1e-15)
    out = subprocess.run([_driver(), "--dir", str(tmp_path), "--walkers", "8", "--check-inputs"],
                         capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr


@pytest.mark.gpu
def test_driver_complex_units_matches_oracle(tmp_path):
    """alpha_c = 1 through the driver (complex W.input in, complex optimized_W.txt out) against the oracle's loop."""
    import pyoracle as po
    nw, ns, nstep, seed = 8, 8, 3, 4545
    p = _complex_units_problem(nw, ns, nstep, 19)
    fm.write_problem(str(tmp_path), p)
    out = subprocess.run([_driver(), "--dir", str(tmp_path), "--walkers", str(nw), "--seed", str(seed)],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr + out.stdout
    got = np.loadtxt(os.path.join(tmp_path, "Energy_vs_Iteration.txt"))
    q = fm.read_problem(str(tmp_path))
    o = po.Oracle(q, nranks=nw, nsample_per_rank=ns, nthreads=4)
    loop = po.VMCLoop(o, q, iseed0=seed)
    for it in range(1, nstep + 1):
        rec = loop.iteration_step()
        assert abs(got[it - 1, 1] - rec["Etot"]) <= 1e-9 * abs(rec["Etot"]), (it, got[it - 1, 1], rec["Etot"])
    br, Wr, bc, Wc = fm.read_W(os.path.join(tmp_path, "optimized_W.txt"), 16, 1, 1)
    bco, Wco = o.get_params_c()
    assert np.allclose(Wc, Wco, rtol=1e-9, atol=1e-13) and np.allclose(bc, bco, rtol=1e-9, atol=1e-13)

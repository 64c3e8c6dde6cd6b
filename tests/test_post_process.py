"""The C++ correlation post-processing program (rbm_pp_b200/rbmpp_post_process, restating
Calc_Correlation/post_process/post_process.f90) on correlation files of the oracle's measurement.

Its translation averages must give the onsite value 1/4 (the program stops otherwise), its Fourier
transforms the reflection symmetry it checks, and its energy check E_chk.txt (four times the bond sum of
the iteration-averaged real-space correlations) must equal the mean of the per-iteration energies Etot/norm:
the bond sum rule E = sum_b J_b (Chi_sp(1, b) + 2 Chi_sp(2, b)) after the average over translations.
"""
import os
import subprocess

import numpy as np

import ed
import pyoracle as po
from rbm_pp_b200 import build
from rbm_pp_b200 import formats as fm


def _write_fort(path, it, m):
    nchi = m["chi_sp"].shape[1]
    sp = m["chi_sp"] / m["norm"]
    vb = m["chi_vbs"] / m["norm"]
    with open(os.path.join(path, f"fort.{60000 + it}"), "w") as f:
        f.write("# chi index,  SzSz,  SpSm\n")
        for i in range(nchi):
            f.write(f"{i + 1:6d}{sp[0, i]:25.15f}{sp[1, i]:25.15f}\n")
    with open(os.path.join(path, f"fort.{70000 + it}"), "w") as f:
        f.write("# chi index, <SSSS> for (1,0), (0,1), (1,1), (1,-1)\n")
        for i in range(nchi):
            f.write(f"{i + 1:6d}" + "".join(f"{vb[i, t]:25.15f}" for t in range(4)) + "\n")


def test_post_process_energy_check(tmp_path):
    build.build()
    L, nw, ns, nav = 4, 4, 4, 3
    p = fm.synthetic_problem(L, translations=True, alphar=1, nsample=nw * ns, seed=23, Nav=nav, J2=0.5)
    fm.write_problem(str(tmp_path), p)
    o = po.Oracle(p, nranks=nw, nsample_per_rank=ns, nthreads=2)
    o.set_params(p.br, p.Wr, p.slater, 0.0)
    o.seed(5)
    o.make_sample(True)
    energies = []
    for it in range(1, nav + 1):
        o.make_sample(False)
        m = o.measure_correlation()
        energies.append(m["Etot"] / m["norm"])
        _write_fort(str(tmp_path), it, m)
    out = subprocess.run([build.POST, "--dir", str(tmp_path)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    e_chk = float(open(os.path.join(tmp_path, "E_chk.txt")).read())
    assert abs(e_chk - np.mean(energies)) <= 1e-9 * abs(np.mean(energies))
    # onsite real-space correlation 1/4 + 2 * 1/4 = 3/4 in the first row of Chi_SS_R.txt
    first = open(os.path.join(tmp_path, "Chi_SS_R.txt")).readline().split()
    assert first[:2] == ["0", "0"] and abs(float(first[2]) - 0.75) < 1e-12
    # every output of the reference program exists, one row per iteration where it keeps one
    for name in ("m2_SS_vs_iteration.txt", "Chi_VBS_vs_iteration.txt", "sub_Chi_VBS_vs_iteration.txt"):
        assert len(open(os.path.join(tmp_path, name)).read().splitlines()) == nav
    for name in ("Chi_SS_q.txt", "total_S.txt", "m2_SS_pipi.txt", "m2_SS_pi0.txt", "m2_SS_0pi.txt",
                 "Chi_VBS_R.txt", "sub_Chi_VBS_R.txt", "Chi_VBS_q.txt", "sub_Chi_VBS_q.txt", "m2_VBS_pipi.txt",
                 "sub_m2_VBS_0pi.txt", "SS_correlation_ratio_1.txt", "SS_correlation_length_2.txt",
                 "VBS_correlation_ratio_0.txt", "VBS_correlation_length_1.txt", "VBS_correlation_ratio_2.txt",
                 "Chi_SS_10.txt", "Chi_SS_01.txt", "Chi_SS_11.txt"):
        assert os.path.getsize(os.path.join(tmp_path, name)) > 0, name
    # the total spin of an Sz = 0 state: S(q = 0) = N * sum_R Chi_R, 0 <= <S^2> <= (N/2)(N/2 + 1)
    tot = float(open(os.path.join(tmp_path, "total_S.txt")).read().splitlines()[1].split()[0])
    N = L * L
    assert -1e-9 <= tot <= (N / 2) * (N / 2 + 1) + 1e-9


def _numpy_post(L, meas):
    """A numpy restatement of post_process.f90:103-247 (translation averages, the <B><B> correction of the
    VBS correlations, the Fourier sums) for the iterations' measurements, and the ratios of :423-467 and
    :583-620 (SS_correlation_ratio_1, VBS_correlation_ratio_0)."""
    N = L * L
    nav = len(meas)
    bmap = {}
    for k, (i1, i2, _, _) in enumerate(ed.bonds(L)):
        bmap[(k // N, i1)] = i2
    Rzz = np.zeros((nav, L, L))
    Rpm = np.zeros((nav, L, L))
    Rvb = np.zeros((nav, L, L, 4))
    for it, m in enumerate(meas):
        sp = m["chi_sp"] / m["norm"]
        vb = m["chi_vbs"] / m["norm"]
        tmp1 = np.zeros((N, N))
        i0 = 0
        for i2 in range(N):
            for i1 in range(i2 + 1):
                tmp1[i1, i2] = tmp1[i2, i1] = 0.25 * (sp[0, i0] + 2.0 * sp[1, i0])
                x = (i2 // L - i1 // L) % L
                y = (i2 % L - i1 % L) % L
                for (a, b) in ((x, y), ((-x) % L, (-y) % L)):
                    Rzz[it, a, b] += sp[0, i0]
                    Rpm[it, a, b] += sp[1, i0]
                    Rvb[it, a, b] += vb[i0]
                i0 += 1
        Rzz[it] *= 0.25 / N
        Rpm[it] *= 0.25 / N
        Rvb[it] *= 0.0625 / N
        Rzz[it, 0, 0] = 0.25
        Rpm[it, 0, 0] = 0.25
        Rvb[it, 0, 0] *= 0.5
        for t in range(4):
            for x in range(L):
                for y in range(L):
                    for i1 in range(N):
                        i2 = ((i1 // L + x) % L) * L + (i1 % L + y) % L
                        Rvb[it, x, y, t] -= tmp1[i1, bmap[(t, i1)]] * tmp1[i2, bmap[(t, i2)]] / N
    k = np.arange(L + 1)
    r = np.arange(L)
    c1 = np.cos(2.0 * np.pi * np.outer(k, r) / L)
    s1 = np.sin(2.0 * np.pi * np.outer(k, r) / L)
    cosq = c1[:, None, :, None] * c1[None, :, None, :] - s1[:, None, :, None] * s1[None, :, None, :]
    Qzz = np.einsum("ixy,abxy->iab", Rzz, cosq)
    Qpm = np.einsum("ixy,abxy->iab", Rpm, cosq)
    Qvb = np.einsum("ixyt,abxy->iabt", Rvb, cosq)
    h = L // 2
    S = Qzz + 2.0 * Qpm
    out = {"Chi_SS_q_pipi": S[:, h, h].mean(), "Chi_VBS_q_pi0_1": Qvb[:, h, 0, 0].mean()}
    r6 = 0.25 * (S[:, h + 1, h] + S[:, h, h + 1] + S[:, h - 1, h] + S[:, h, h - 1])
    out["SS_ratio_1"] = (1.0 - r6 / S[:, h, h]).mean()
    t1 = 1.0 - 0.25 * (Qvb[:, h + 1, 0, 0] + Qvb[:, h - 1, 0, 0] + Qvb[:, h, 1, 0] + Qvb[:, h, L - 1, 0]) \
        / Qvb[:, h, 0, 0]
    c = Qvb[:, :, :, 0] + Qvb[:, :, :, 1].transpose(0, 2, 1)  # type 1 at (kx, ky) + type 2 at (ky, kx)
    t4 = 1.0 - 0.25 * (c[:, h + 1, 0] + c[:, h - 1, 0] + c[:, h, 1] + c[:, h, L - 1]) / c[:, h, 0]
    out["VBS_ratio_0_combined"] = t4.mean()
    out["VBS_ratio_0_type1"] = t1.mean()
    return out


def test_post_process_values_match_numpy(tmp_path):
    """Structure factor at (pi, pi), VBS structure factor at (pi, 0), the spin correlation ratio and the VBS
    correlation ratio written by the program equal a numpy restatement of the same formulae on the same
    files (the outputs carry 10 decimals, hence the absolute tolerance)."""
    build.build()
    L, nw, ns, nav = 4, 4, 4, 3
    p = fm.synthetic_problem(L, translations=True, alphar=1, nsample=nw * ns, seed=23, Nav=nav, J2=0.5)
    fm.write_problem(str(tmp_path), p)
    o = po.Oracle(p, nranks=nw, nsample_per_rank=ns, nthreads=2)
    o.set_params(p.br, p.Wr, p.slater, 0.0)
    o.seed(5)
    o.make_sample(True)
    for it in range(1, nav + 1):
        o.make_sample(False)
        _write_fort(str(tmp_path), it, o.measure_correlation())
    out = subprocess.run([build.POST, "--dir", str(tmp_path)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    want = _numpy_post(L, [dict(chi_sp=np.loadtxt(os.path.join(tmp_path, f"fort.{60000 + i}"))[:, 1:].T,
                                chi_vbs=np.loadtxt(os.path.join(tmp_path, f"fort.{70000 + i}"))[:, 1:], norm=1.0)
                           for i in range(1, nav + 1)])

    def row(name, kx, ky):
        for ln in open(os.path.join(tmp_path, name)):
            f = ln.split()
            if len(f) > 2 and int(f[0]) == kx and int(f[1]) == ky:
                return [float(v) for v in f[2:]]
        raise AssertionError((name, kx, ky))

    tol = 2e-10
    assert abs(row("Chi_SS_q.txt", L // 2, L // 2)[0] - want["Chi_SS_q_pipi"]) < tol
    assert abs(row("Chi_VBS_q.txt", L // 2, 0)[0] - want["Chi_VBS_q_pi0_1"]) < tol
    ss1 = [float(v) for v in open(os.path.join(tmp_path, "SS_correlation_ratio_1.txt")).read().split()]
    assert abs(ss1[0] - want["SS_ratio_1"]) < tol
    vb0 = [float(v) for v in open(os.path.join(tmp_path, "VBS_correlation_ratio_0.txt")).read().split()]
    assert abs(vb0[0] - want["VBS_ratio_0_combined"]) < tol
    assert abs(vb0[2] - want["VBS_ratio_0_type1"]) < tol

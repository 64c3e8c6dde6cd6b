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

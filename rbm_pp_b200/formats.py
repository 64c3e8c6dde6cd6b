"""Readers, writers and generators for RBM_PP's input/parameter files.

These keep the reference's on-disk formats so the CUDA path is a drop-in for its sampling/SR
loop.  Each reader follows the Fortran list-directed reads it replaces:

* ``RBM.input``                main.f90:75-84
* ``sym_info.txt``             main.f90:89-124
* ``orbitalidx.def``           parameter.f90:81-101 (and main.f90:126-129 for N_Slater)
* ``zqp_orbital_initial.dat``  parameter.f90:114-141 (rescaled to mean |f| = 0.25)
* ``W.input``                  parameter.f90:42-75 (optional initial RBM parameters)

Writers produce the layouts of parameter.f90:148-314 (``optimized_W.txt`` has the W.input layout,
``zqp_orbital_opt.dat`` the zqp_orbital_initial.dat layout, so outputs can be fed back to resume).

Arrays use the Fortran layouts: ``W_map`` is (N, N_MP_Trans) with 1-based site values,
``orbital_idx`` is (N, N) with 1-based parameter indices, ``Wr`` is (N, alphar).
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

SLATER_ABS_AV = 0.25  # module.f90:66


def _fortran_float(tok: str) -> float:
    return float(tok.replace("d", "e").replace("D", "e"))


def _tokens(line: str) -> list[str]:
    return line.replace(",", " ").split()


def _complex_tok(toks: list[str]) -> complex:
    # list-directed complex input is "(re,im)"; also accept "re im"
    s = " ".join(toks).replace("(", " ").replace(")", " ").replace(",", " ").split()
    return complex(_fortran_float(s[0]), _fortran_float(s[1]) if len(s) > 1 else 0.0)


@dataclass
class RBMInput:
    """Contents of RBM.input (main.f90:75-84)."""
    L: int
    Nsample: int
    spin_parity: int
    alphac: int
    alphar: int
    Nstep: int
    Nav: int
    delta_tau: float
    s_factor0: float
    s_factor_scale: float
    s_cut: float
    J1: float
    J2: float


def write_rbm_input(path: str, p: RBMInput) -> None:
    with open(path, "w") as f:
        f.write("# L  Nsample  spin_parity\n")
        f.write(f"{p.L} {p.Nsample} {p.spin_parity}\n")
        f.write("# alphac  alphar  Nstep  Nav  delta_tau\n")
        f.write(f"{p.alphac} {p.alphar} {p.Nstep} {p.Nav} {float(p.delta_tau)!r}\n")
        f.write("# s_factor0  s_factor_scale  s_cut\n")
        f.write(f"{float(p.s_factor0)!r} {float(p.s_factor_scale)!r} {float(p.s_cut)!r}\n")
        f.write("# J1  J2\n")
        f.write(f"{float(p.J1)!r} {float(p.J2)!r}\n")


def read_rbm_input(path: str) -> RBMInput:
    with open(path) as f:
        lines = f.read().splitlines()
    a = _tokens(lines[1])
    b = _tokens(lines[3])
    c = _tokens(lines[5])
    d = _tokens(lines[7])
    return RBMInput(L=int(a[0]), Nsample=int(a[1]), spin_parity=int(a[2]), alphac=int(b[0]), alphar=int(b[1]),
                    Nstep=int(b[2]), Nav=int(b[3]), delta_tau=_fortran_float(b[4]),
                    s_factor0=_fortran_float(c[0]), s_factor_scale=_fortran_float(c[1]),
                    s_cut=_fortran_float(c[2]), J1=_fortran_float(d[0]), J2=_fortran_float(d[1]))


@dataclass
class SymInfo:
    """sym_info.txt: projections (translations) used both by the RBM and the Pfaffian part."""
    n_mp: int
    para_mp: np.ndarray  # complex (n_mp,)
    W_map: np.ndarray    # int32 (N, n_mp), 1-based


def lattice_translations(L: int) -> np.ndarray:
    """All L*L translations of the periodic L x L lattice, site i = ix*L + iy + 1 (bond_map,
    calc_phys_quantity.f90:394-422).  Returns W_map (N, L*L), 1-based, mp = dx*L + dy + 1."""
    N = L * L
    W = np.zeros((N, N), dtype=np.int32)
    for dx in range(L):
        for dy in range(L):
            mp = dx * L + dy
            for ix in range(L):
                for iy in range(L):
                    i = ix * L + iy
                    j = ((ix + dx) % L) * L + (iy + dy) % L
                    W[i, mp] = j + 1
    return W


def make_sym_info(L: int, translations: bool) -> SymInfo:
    N = L * L
    if translations:
        W = lattice_translations(L)
    else:
        W = np.arange(1, N + 1, dtype=np.int32).reshape(N, 1)
    n_mp = W.shape[1]
    return SymInfo(n_mp=n_mp, para_mp=np.ones(n_mp, dtype=np.complex128), W_map=W)


def write_sym_info(path: str, s: SymInfo) -> None:
    N = s.W_map.shape[0]
    with open(path, "w") as f:
        f.write("# N_MP_Trans  Ncopy\n")
        f.write(f"{s.n_mp} 1\n")
        f.write("# mpidx  para_mp_trans\n")
        for mp in range(s.n_mp):
            z = s.para_mp[mp]
            f.write(f"{mp + 1} ({float(z.real)!r},{float(z.imag)!r})\n")
        f.write("# mpidx  icopy  i  W_map\n")
        for mp in range(s.n_mp):
            for i in range(N):
                f.write(f"{mp + 1} 1 {i + 1} {int(s.W_map[i, mp])}\n")


def read_sym_info(path: str, N: int) -> SymInfo:
    """main.f90:89-124, including the permutation checks of :110-119."""
    with open(path) as f:
        lines = [ln for ln in f.read().splitlines()]
    t = _tokens(lines[1])
    n_mp, ncopy = int(t[0]), int(t[1])
    if ncopy != 1:
        raise ValueError("i1/=Ncopy (sym_info.txt)")
    para = np.zeros(n_mp, dtype=np.complex128)
    pos = 3
    for mp in range(n_mp):
        t = lines[pos].replace("(", " ").replace(")", " ").replace(",", " ").split()
        pos += 1
        if int(t[0]) != mp + 1:
            raise ValueError("i1/=mpidx")
        para[mp] = complex(_fortran_float(t[1]), _fortran_float(t[2]) if len(t) > 2 else 0.0)
    pos += 1
    W = np.zeros((N, n_mp), dtype=np.int32)
    for mp in range(n_mp):
        for i in range(N):
            t = _tokens(lines[pos])
            pos += 1
            if int(t[0]) != mp + 1 or int(t[1]) != 1 or int(t[2]) != i + 1:
                raise ValueError("index mismatch (sym_info.txt)")
            w = int(t[3])
            if w < 1 or w > N:
                raise ValueError("W_map wrong 1 (sym_info.txt)")
            W[i, mp] = w
        if len(set(W[:, mp].tolist())) != N:
            raise ValueError("W_map wrong 2 (sym_info.txt)")
    return SymInfo(n_mp=n_mp, para_mp=para, W_map=W)


def make_orbital_idx(L: int, kind: str = "full") -> tuple[int, np.ndarray]:
    """Orbital_Idx(N, N), 1-based.  ``full``: one f_ij per ordered site pair (N_Slater = N^2).
    ``sublattice2``: translation-invariant f resolved by the sublattice of i (N_Slater = 2N).
    Both give N_Slater/N distinct f_ii indices, as SR_pdposv.f90:78-100 requires."""
    N = L * L
    idx = np.zeros((N, N), dtype=np.int32)
    if kind == "full":
        for i in range(N):
            for j in range(N):
                idx[i, j] = i * N + j + 1
        return N * N, idx
    if kind == "sublattice2":
        for i in range(N):
            ix, iy = divmod(i, L)
            sub = (ix + iy) % 2
            for j in range(N):
                jx, jy = divmod(j, L)
                d = ((jx - ix) % L) * L + (jy - iy) % L
                idx[i, j] = sub * N + d + 1
        return 2 * N, idx
    raise ValueError(kind)


def write_orbital_idx(path: str, n_slater: int, idx: np.ndarray) -> None:
    N = idx.shape[0]
    with open(path, "w") as f:
        f.write("=============================================\n")
        f.write(f"NOrbitalIdx {n_slater}\n")
        f.write("ComplexType 0\n")
        f.write("=============================================\n")
        f.write("=============================================\n")
        for i in range(N):
            for j in range(N):
                f.write(f"{i:5d} {j:5d} {int(idx[i, j]) - 1:7d}\n")


def read_orbital_idx(path: str, N: int) -> tuple[int, np.ndarray]:
    """parameter.f90:81-101 (l_AP = .false.: no sign column)."""
    with open(path) as f:
        lines = f.read().splitlines()
    n_slater = int(_tokens(lines[1])[1])
    idx = np.zeros((N, N), dtype=np.int32)
    pos = 5
    for i in range(N):
        for j in range(N):
            t = _tokens(lines[pos])
            pos += 1
            if int(t[0]) != i or int(t[1]) != j:
                raise ValueError("error2/3, orbitalidx")
            v = int(t[2]) + 1
            if v < 1 or v > n_slater:
                raise ValueError("error4, orbitalidx")
            idx[i, j] = v
    return n_slater, idx


def write_zqp(path: str, slater: np.ndarray, header_blank: bool = False) -> None:
    """zqp_orbital_initial.dat / zqp_orbital_opt.dat layout (parameter.f90:266-275)."""
    with open(path, "w") as f:
        f.write("\n" if header_blank else "=============================================\n")
        f.write(f" Slater {len(slater):10d}\n")
        for _ in range(3):
            f.write("\n" if header_blank else "=============================================\n")
        for k, v in enumerate(slater):
            f.write(f"{k:5d} {float(v): .15e} {0.0: .15e}\n")


def read_zqp(path: str, n_slater: int, rescale: bool = True) -> np.ndarray:
    """parameter.f90:114-141: reads f, rejects imaginary parts, rescales to mean |f| = 0.25."""
    with open(path) as f:
        lines = f.read().splitlines()
    if int(_tokens(lines[1])[1]) != n_slater:
        raise ValueError("error in zqp_orbital_initial 1")
    out = np.zeros(n_slater)
    r3 = 0.0
    for k in range(n_slater):
        t = _tokens(lines[5 + k])
        if int(t[0]) + 1 != k + 1:
            raise ValueError("error in zqp_orbital_initial 2")
        out[k] = _fortran_float(t[1])
        r3 = r3 + abs(out[k])
        if len(t) > 2 and abs(_fortran_float(t[2])) > 1e-10:
            raise ValueError("imaginary zqp_orbital_initial, not implemented")
    if rescale:
        r3 = r3 / float(n_slater)
        out = np.array([v * SLATER_ABS_AV / r3 for v in out])
    return out


def write_W(path: str, br: np.ndarray, Wr: np.ndarray, bc=None, Wc=None) -> None:
    """W.input / initial_W.txt / optimized_W.txt layout (parameter.f90:159-175): the complex units bc, Wc(N, alphac)
    first (when given), then the real ones."""
    N, alphar = Wr.shape
    with open(path, "w") as f:
        f.write("# index for independent neurons (f), index for interaction (iw), irreducible interaction Wirr(iw,f)\n")
        if Wc is not None:
            for fi in range(Wc.shape[1]):
                f.write(f"# bias{fi + 1:6d}{complex(bc[fi]).real:22.15f}{complex(bc[fi]).imag:22.15f}\n")
                for iw in range(N):
                    w = complex(Wc[iw, fi])
                    f.write(f"{fi + 1:6d}{iw + 1:6d}{w.real:22.15f}{w.imag:22.15f}\n")
                f.write("\n")
        for fi in range(alphar):
            f.write(f"# bias{fi + 1:6d}{float(br[fi]):22.15f}{0.0:22.15f}\n")
            for iw in range(N):
                f.write(f"{fi + 1:6d}{iw + 1:6d}{float(Wr[iw, fi]):22.15f}{0.0:22.15f}\n")
            f.write("\n")


def read_W(path: str, N: int, alphar: int, alphac: int = 0):
    """parameter.f90:42-75: (br, Wr), or (br, Wr, bc, Wc) when alphac > 0 (the complex units come first)."""
    with open(path) as f:
        lines = f.read().splitlines()
    br = np.zeros(alphar)
    Wr = np.zeros((N, alphar))
    bc = np.zeros(alphac, np.complex128)
    Wc = np.zeros((N, alphac), np.complex128)
    pos = 1
    for fi in range(alphac):
        t = _tokens(lines[pos])
        pos += 1
        if int(t[2]) != fi + 1:
            raise ValueError("i1/=f (W.input)")
        bc[fi] = complex(_fortran_float(t[3]), _fortran_float(t[4]))
        for iw in range(N):
            t = _tokens(lines[pos])
            pos += 1
            if int(t[0]) != fi + 1 or int(t[1]) != iw + 1:
                raise ValueError("index mismatch (W.input)")
            Wc[iw, fi] = complex(_fortran_float(t[2]), _fortran_float(t[3]))
        pos += 1
    for fi in range(alphar):
        t = _tokens(lines[pos])
        pos += 1
        if int(t[2]) != fi + 1:
            raise ValueError("i1/=f (W.input)")
        br[fi] = _fortran_float(t[3])
        if abs(_fortran_float(t[4])) > 1e-15:
            raise ValueError("r2 /= 0 (W.input)")
        for iw in range(N):
            t = _tokens(lines[pos])
            pos += 1
            if int(t[0]) != fi + 1 or int(t[1]) != iw + 1:
                raise ValueError("index mismatch (W.input)")
            Wr[iw, fi] = _fortran_float(t[2])
            if abs(_fortran_float(t[3])) > 1e-15:
                raise ValueError("r2 /= 0 (W.input)")
        pos += 1
    return (br, Wr, bc, Wc) if alphac > 0 else (br, Wr)


def spin_projection_weights(spin_parity: int = 1, transverse: bool = False) -> np.ndarray:
    """InitSPWeight's values for the two Gauss-Legendre points as the (3, 2) array {SP_GL_Cos, SP_GL_Sin,
    para_spin_proj} per point that rbmpp_set_tables takes.  The normal code sets beta = 0, pi
    (spin_projection.f90:29-32, :37-38); the transverse code beta = -pi/2, pi/2 with sqrt(2)-scaled cosines and
    sines (transverse_code/spin_projection.f90:30-31, :37-38).  para_spin_proj = (1, spin_parity)
    (spin_projection.f90:55-62)."""
    if transverse:
        beta = np.array([-0.5 * np.pi, 0.5 * np.pi])
        scale = np.sqrt(2.0)
    else:
        beta = np.array([0.0, np.pi])
        scale = 1.0
    w = np.zeros((3, 2))
    w[0] = scale * np.cos(0.5 * beta)
    w[1] = scale * np.sin(0.5 * beta)
    w[2] = [1.0, 1.0 if spin_parity == 1 else -1.0]
    return w


@dataclass
class Problem:
    """Everything the sampling/SR loop needs, in the reference's layouts."""
    inp: RBMInput
    sym: SymInfo
    n_slater: int
    orbital_idx: np.ndarray
    slater: np.ndarray
    br: np.ndarray | None = None
    Wr: np.ndarray | None = None
    extra: dict = field(default_factory=dict)
    bc: np.ndarray | None = None  # complex units (alphac > 0), from W.input
    Wc: np.ndarray | None = None

    @property
    def N(self) -> int:
        return self.inp.L * self.inp.L

    @property
    def Nv(self) -> int:
        return 2 * self.inp.alphac * (self.N + 1) + self.inp.alphar * (self.N + 1) + self.n_slater


def synthetic_problem(L: int, *, translations: bool, alphar: int, orbital: str = "full", nsample: int = 1024,
                      J1: float = 1.0, J2: float = 0.5, seed: int = 12345, w_sigma: float = 0.01,
                      f_sigma: float = 0.1, Nstep: int = 100, Nav: int = 10, delta_tau: float = 0.05,
                      s_factor0: float = 1e-3, s_factor_scale: float = 1.0, s_cut: float = 1e-3,
                      spin_parity: int = 1) -> Problem:
    """Seeded synthetic inputs: RBM weights ~ N(0, w_sigma^2) (written as W.input), f_ij ~ N(0, f_sigma^2)
    rescaled to mean |f| = 0.25 as the reference does on load (parameter.f90:131-140)."""
    rng = np.random.default_rng(seed)
    N = L * L
    sym = make_sym_info(L, translations)
    n_slater, idx = make_orbital_idx(L, orbital)
    f = rng.normal(0.0, f_sigma, size=n_slater)
    f = f * SLATER_ABS_AV / (np.abs(f).sum() / n_slater)
    br = rng.normal(0.0, w_sigma, size=alphar)
    Wr = rng.normal(0.0, w_sigma, size=(N, alphar))
    inp = RBMInput(L=L, Nsample=nsample, spin_parity=spin_parity, alphac=0, alphar=alphar, Nstep=Nstep, Nav=Nav,
                   delta_tau=delta_tau, s_factor0=s_factor0, s_factor_scale=s_factor_scale, s_cut=s_cut, J1=J1,
                   J2=J2)
    return Problem(inp=inp, sym=sym, n_slater=n_slater, orbital_idx=idx, slater=f, br=br, Wr=Wr)


def write_problem(dirname: str, p: Problem) -> None:
    os.makedirs(dirname, exist_ok=True)
    write_rbm_input(os.path.join(dirname, "RBM.input"), p.inp)
    write_sym_info(os.path.join(dirname, "sym_info.txt"), p.sym)
    write_orbital_idx(os.path.join(dirname, "orbitalidx.def"), p.n_slater, p.orbital_idx)
    write_zqp(os.path.join(dirname, "zqp_orbital_initial.dat"), p.slater)
    if p.Wr is not None:
        write_W(os.path.join(dirname, "W.input"), p.br, p.Wr, p.bc, p.Wc)


def read_problem(dirname: str) -> Problem:
    inp = read_rbm_input(os.path.join(dirname, "RBM.input"))
    N = inp.L * inp.L
    sym = read_sym_info(os.path.join(dirname, "sym_info.txt"), N)
    n_slater, idx = read_orbital_idx(os.path.join(dirname, "orbitalidx.def"), N)
    slater = read_zqp(os.path.join(dirname, "zqp_orbital_initial.dat"), n_slater)
    br = Wr = bc = Wc = None
    wpath = os.path.join(dirname, "W.input")
    if os.path.exists(wpath):
        if inp.alphac > 0:
            br, Wr, bc, Wc = read_W(wpath, N, inp.alphar, inp.alphac)
        else:
            br, Wr = read_W(wpath, N, inp.alphar)
    return Problem(inp=inp, sym=sym, n_slater=n_slater, orbital_idx=idx, slater=slater, br=br, Wr=Wr, bc=bc, Wc=Wc)

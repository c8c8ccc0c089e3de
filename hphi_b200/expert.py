"""Expert-mode input writer for HPhi-format ``.def`` files.

Writes ``namelist.def`` and the per-keyword files that HPhi's expert mode reads
(``HPhi -e namelist.def``).  The formats follow the reference reader:
namelist keywords ``src/readdef.c:46-71``; ``calcmod.def`` keys
``src/readdef.c:233-330``; ``modpara.def`` (8 header lines, then ``key value``
lines) ``src/readdef.c:513-640``; interaction files (5 header lines whose second
line is ``N<Kind> <count>``, then one entry per line) ``src/readdef.c:1006-1400``.

Lattice helpers produce the bond lists used in this project's workloads
(periodic chains, J1-J2 chains, square lattices, the Kitaev honeycomb).  Site
labels are ``x + W*y`` with ``x`` fastest.
"""
from __future__ import annotations

import os
import random
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

CALC_TYPE = {"Lanczos": 0, "TPQ": 1, "FullDiag": 2, "CG": 3, "TimeEvolution": 4, "cTPQ": 5}
CALC_MODEL = {"Hubbard": 0, "Spin": 1, "Kondo": 2, "HubbardGC": 3, "SpinGC": 4, "KondoGC": 5}

_SEP = "=" * 30


@dataclass
class ExpertModel:
    """An expert-mode HPhi input: model, sector and interaction lists.

    Interaction tuples use HPhi's column order:
      trans        (i, s1, j, s2, t_re, t_im)       H += -t c+_{i s1} c_{j s2}
      coulombintra (i, U)                           H += U n_{i up} n_{i dn}
      coulombinter (i, j, V)                        H += V n_i n_j
      hund         (i, j, J)                        H += -J (n_{i up} n_{j up} + n_{i dn} n_{j dn})
      exchange     (i, j, J)                        spin: H += J (S+_i S-_j + S-_i S+_j)
      ising        (i, j, J)                        H += J Sz_i Sz_j
      pairhop      (i, j, J)                        H += J (c+_{i up} c_{j up} c+_{i dn} c_{j dn} + h.c.)
      pairlift     (i, j, J)                        SpinGC: H += J (S+_i S+_j + S-_i S-_j)
      interall     (i, s1, j, s2, k, s3, l, s4, V_re, V_im)
    """

    model: str = "Spin"
    nsite: int = 2
    calc_type: str = "Lanczos"
    two_sz: Optional[int] = 0
    ncond: Optional[int] = None
    nup: Optional[int] = None
    ndown: Optional[int] = None
    locspin: Optional[List[int]] = None
    lanczos_max: int = 2000
    initial_iv: int = -1
    exct: int = 1
    lanczos_eps: int = 14
    lanczos_target: int = 2
    large_value: float = 4.5
    num_ave: int = 5
    expec_interval: int = 20
    calc_eigenvec: int = -1
    initial_vec_type: int = 1
    output_eigenvec: int = 0
    restart: int = 0
    pre_cg: int = 0
    trans: List[Tuple] = field(default_factory=list)
    coulombintra: List[Tuple] = field(default_factory=list)
    coulombinter: List[Tuple] = field(default_factory=list)
    hund: List[Tuple] = field(default_factory=list)
    exchange: List[Tuple] = field(default_factory=list)
    ising: List[Tuple] = field(default_factory=list)
    pairhop: List[Tuple] = field(default_factory=list)
    pairlift: List[Tuple] = field(default_factory=list)
    interall: List[Tuple] = field(default_factory=list)
    # Green's function requests: OneBodyG rows (i, s1, j, s2) and TwoBodyG rows
    # (i, s1, j, s2, k, s3, l, s4) (src/readdef.c:1441-1523)
    greenone: List[Tuple] = field(default_factory=list)
    greentwo: List[Tuple] = field(default_factory=list)
    # ThreeBodyG / FourBodyG / SixBodyG rows: 3, 4, 6 site pairs (i, s, j, t) flattened
    greenthree: List[Tuple] = field(default_factory=list)
    greenfour: List[Tuple] = field(default_factory=list)
    greensix: List[Tuple] = field(default_factory=list)
    # time evolution (calc_type "TimeEvolution"): per time index (time, rows), TEOneBody rows
    # (i, s1, j, s2, t_re, t_im) or TETwoBody rows (i, s1, j, s2, k, s3, l, s4, V_re, V_im)
    # (src/readdef.c:1752-1840); the start state is <spectrum_vec>_rank_0.dat
    te_onebody: List[Tuple[float, List[Tuple]]] = field(default_factory=list)
    te_twobody: List[Tuple[float, List[Tuple]]] = field(default_factory=list)
    spectrum_vec: Optional[str] = None
    input_eigenvec: int = 0
    expand_coef: int = 0
    output_interval: int = 0
    # dynamical Green's function (calc_spec 1, src/CalcSpectrum.c): SingleExcitation rows
    # (i, s, type, re, im) or PairExcitation rows (i, s1, j, s2, type, re, im)
    # (src/readdef.c:1943-2007) and the frequency grid (complex OmegaMax / OmegaMin, OmegaIm)
    calc_spec: int = 0
    single_excitation: List[Tuple] = field(default_factory=list)
    pair_excitation: List[Tuple] = field(default_factory=list)
    omega_max: Optional[complex] = None
    omega_min: Optional[complex] = None
    omega_im: Optional[float] = None
    n_omega: Optional[int] = None
    output_exvec: int = 0

    # ------------------------------------------------------------------ writers
    def write(self, directory: str) -> str:
        """Write all files into ``directory``; return the path of namelist.def."""
        os.makedirs(directory, exist_ok=True)
        names: List[Tuple[str, str]] = [("CalcMod", "calcmod.def"), ("ModPara", "modpara.def"),
                                        ("LocSpin", "locspn.def")]
        self._write_calcmod(os.path.join(directory, "calcmod.def"))
        self._write_modpara(os.path.join(directory, "modpara.def"))
        self._write_locspn(os.path.join(directory, "locspn.def"))
        tables = [
            ("Trans", "trans.def", "NTransfer", self.trans, "{:d} {:d} {:d} {:d} {:.17g} {:.17g}"),
            ("CoulombIntra", "coulombintra.def", "NCoulombIntra", self.coulombintra, "{:d} {:.17g}"),
            ("CoulombInter", "coulombinter.def", "NCoulombInter", self.coulombinter, "{:d} {:d} {:.17g}"),
            ("Hund", "hund.def", "NHund", self.hund, "{:d} {:d} {:.17g}"),
            ("Exchange", "exchange.def", "NExchange", self.exchange, "{:d} {:d} {:.17g}"),
            ("Ising", "ising.def", "NIsing", self.ising, "{:d} {:d} {:.17g}"),
            ("PairHop", "pairhop.def", "NPairhop", self.pairhop, "{:d} {:d} {:.17g}"),
            ("PairLift", "pairlift.def", "NPairlift", self.pairlift, "{:d} {:d} {:.17g}"),
            ("InterAll", "interall.def", "NInterAll", self.interall,
             "{:d} {:d} {:d} {:d} {:d} {:d} {:d} {:d} {:.17g} {:.17g}"),
            ("OneBodyG", "greenone.def", "NCisAjs", self.greenone, "{:d} {:d} {:d} {:d}"),
            ("TwoBodyG", "greentwo.def", "NCisAjsCktAltDC", self.greentwo,
             "{:d} {:d} {:d} {:d} {:d} {:d} {:d} {:d}"),
            ("ThreeBodyG", "greenthree.def", "NThreeBody", self.greenthree, " ".join(["{:d}"] * 12)),
            ("FourBodyG", "greenfour.def", "NFourBody", self.greenfour, " ".join(["{:d}"] * 16)),
            ("SixBodyG", "greensix.def", "NSixBody", self.greensix, " ".join(["{:d}"] * 24)),
            ("SingleExcitation", "single.def", "NSingle", self.single_excitation,
             "{:d} {:d} {:d} {:.17g} {:.17g}"),
            ("PairExcitation", "pair.def", "NPair", self.pair_excitation,
             "{:d} {:d} {:d} {:d} {:d} {:.17g} {:.17g}"),
        ]
        for kw, fname, head, rows, fmt in tables:
            if not rows:
                continue
            with open(os.path.join(directory, fname), "w") as f:
                f.write(f"{_SEP}\n{head} {len(rows)}\n{_SEP}\n{_SEP}\n{_SEP}\n")
                for r in rows:
                    f.write(fmt.format(*r) + "\n")
            names.append((kw, fname))
        for kw, fname, steps, fmt in (
                ("TEOneBody", "teonebody.def", self.te_onebody, "{:d} {:d} {:d} {:d} {:.17g} {:.17g}"),
                ("TETwoBody", "tetwobody.def", self.te_twobody,
                 "{:d} {:d} {:d} {:d} {:d} {:d} {:d} {:d} {:.17g} {:.17g}")):
            if not steps:
                continue
            with open(os.path.join(directory, fname), "w") as f:
                f.write(f"{_SEP}\nAllTimeStep {len(steps)}\n{_SEP}\n{_SEP}\n{_SEP}\n")
                for t, rows in steps:
                    f.write(f"{t!r} {len(rows)}\n")
                    for r in rows:
                        f.write(fmt.format(*r) + "\n")
            names.append((kw, fname))
        if self.spectrum_vec:
            names.append(("SpectrumVec", self.spectrum_vec))
        path = os.path.join(directory, "namelist.def")
        with open(path, "w") as f:
            for kw, fname in names:
                f.write(f"{kw} {fname}\n")
        return path

    def _write_calcmod(self, path: str) -> None:
        with open(path, "w") as f:
            f.write("#CalcType = 0:Lanczos, 1:TPQCalc, 2:FullDiag, 3:CG, 4:Time-evolution\n")
            f.write("#CalcModel = 0:Hubbard, 1:Spin, 2:Kondo, 3:HubbardGC, 4:SpinGC, 5:KondoGC\n")
            f.write(f"CalcType   {CALC_TYPE[self.calc_type]}\n")
            f.write(f"CalcModel  {CALC_MODEL[self.model]}\n")
            f.write(f"CalcEigenVec {self.calc_eigenvec}\n")
            f.write(f"InitialVecType {self.initial_vec_type}\n")
            if self.output_eigenvec:
                f.write(f"OutputEigenVec {self.output_eigenvec}\n")
            if self.input_eigenvec:
                f.write(f"InputEigenVec {self.input_eigenvec}\n")
            if self.restart:
                f.write(f"ReStart {self.restart}\n")
            if self.calc_spec:
                f.write(f"CalcSpec {self.calc_spec}\n")
            if self.output_exvec:
                f.write(f"OutputExVec {self.output_exvec}\n")

    def _write_modpara(self, path: str) -> None:
        lines = ["--------------------", "Model_Parameters   0", "--------------------",
                 "HPhi_Cal_Parameters", "--------------------", "CDataFileHead  zvo",
                 "CParaFileHead  zqp", "--------------------", f"Nsite          {self.nsite}"]
        if self.nup is not None:
            lines.append(f"Nup            {self.nup}")
        if self.ndown is not None:
            lines.append(f"Ndown          {self.ndown}")
        if self.ncond is not None:
            lines.append(f"Ncond          {self.ncond}")
        if self.two_sz is not None and not self.model.endswith("GC"):
            lines.append(f"2Sz            {self.two_sz}")
        lines += [f"Lanczos_max    {self.lanczos_max}", f"initial_iv     {self.initial_iv}",
                  f"exct           {self.exct}", f"LanczosEps     {self.lanczos_eps}",
                  f"LanczosTarget  {self.lanczos_target}", f"LargeValue     {self.large_value}",
                  f"NumAve         {self.num_ave}", f"ExpecInterval  {self.expec_interval}"]
        if self.pre_cg:
            lines.append(f"PreCG          {self.pre_cg}")
        if self.expand_coef:
            lines.append(f"ExpandCoef     {self.expand_coef}")
        if self.output_interval:
            lines.append(f"OutputInterval {self.output_interval}")
        if self.omega_max is not None:
            lines.append(f"OmegaMax       {complex(self.omega_max).real!r} {complex(self.omega_max).imag!r}")
        if self.omega_min is not None:
            lines.append(f"OmegaMin       {complex(self.omega_min).real!r} {complex(self.omega_min).imag!r}")
        if self.omega_im is not None:
            lines.append(f"OmegaIm        {self.omega_im!r}")
        if self.n_omega is not None:
            lines.append(f"NOmega         {self.n_omega}")
        with open(path, "w") as f:
            f.write("\n".join(lines) + "\n")

    def _write_locspn(self, path: str) -> None:
        if self.locspin is not None:
            loc = list(self.locspin)
        elif self.model.startswith("Spin"):
            loc = [1] * self.nsite
        else:
            loc = [0] * self.nsite
        nloc = sum(1 for x in loc if x != 0)
        with open(path, "w") as f:
            f.write(f"{_SEP}\nNlocalSpin {nloc}\n{_SEP}\n{_SEP}\n{_SEP}\n")
            for i, s in enumerate(loc):
                f.write(f"{i} {s}\n")


# ---------------------------------------------------------------------- lattices
def chain_bonds(L: int, dist: int = 1) -> List[Tuple[int, int]]:
    """Periodic chain bonds (i, i+dist mod L)."""
    return [(i, (i + dist) % L) for i in range(L)]


def square_bonds(W: int, L: int) -> List[Tuple[int, int]]:
    """Nearest-neighbour bonds of a W x L periodic square lattice (site = x + W*y)."""
    bonds = []
    for y in range(L):
        for x in range(W):
            s = x + W * y
            bonds.append((s, (x + 1) % W + W * y))
            bonds.append((s, x + W * ((y + 1) % L)))
    return bonds


def honeycomb_bonds(W: int, L: int) -> List[Tuple[int, int, int]]:
    """Bonds (i, j, gamma) of a W x L-cell periodic honeycomb lattice.

    Two sites per cell: A = 2*(x + W*y), B = A + 1.  gamma = 0 (x-bond, inside the
    cell), 1 (y-bond, to the cell at x+1), 2 (z-bond, to the cell at y+1).
    """
    bonds = []
    for y in range(L):
        for x in range(W):
            a = 2 * (x + W * y)
            bonds.append((a, a + 1, 0))
            bonds.append((a + 1, 2 * ((x + 1) % W + W * y), 1))
            bonds.append((a + 1, 2 * (x + W * ((y + 1) % L)), 2))
    return bonds


def heisenberg(nsite: int, bonds: Sequence[Tuple[int, int]], J: float | Sequence[float] = 1.0,
               two_sz: int = 0, **kw) -> ExpertModel:
    """Spin-1/2 Heisenberg model: H = sum J S_i.S_j = Ising(J) + Exchange(J/2)."""
    Js = [J] * len(bonds) if isinstance(J, (int, float)) else list(J)
    m = ExpertModel(model="Spin", nsite=nsite, two_sz=two_sz, **kw)
    m.ising = [(i, j, float(c)) for (i, j), c in zip(bonds, Js)]
    m.exchange = [(i, j, 0.5 * float(c)) for (i, j), c in zip(bonds, Js)]
    return m


def _spin_raise(two_s: int, d: int) -> float:
    """<d+1| S+ |d> for spin S = two_s/2, digit d <-> m = d - S."""
    S, m = 0.5 * two_s, d - 0.5 * two_s
    return (S * (S + 1) - m * (m + 1)) ** 0.5


def general_heisenberg(two_s: Sequence[int], bonds: Sequence[Tuple[int, int]], J: float | Sequence[float] = 1.0,
                       two_sz: Optional[int] = 0, D: float = 0.0, hx: float = 0.0, **kw) -> ExpertModel:
    """Spin-S Heisenberg model with site spins two_s[i]/2 (general spin: InterAll only),
    H = sum J S_i.S_j + D sum (Sz_i)^2 - hx sum Sx_i.  A site's state is its digit
    d = 0 .. 2S (2Sz = 2d - 2S); InterAll (i a i b j c j d V) is V |a><b|_i |c><d|_j, listed
    with its Hermitian partner (j d j c i b i a V*).  hx needs two_sz=None (SpinGC); it is
    written as site-diagonal Trans rows (H += -t |a><b|)."""
    n = len(two_s)
    Js = [J] * len(bonds) if isinstance(J, (int, float)) else list(J)
    m = ExpertModel(model="Spin" if two_sz is not None else "SpinGC", nsite=n, two_sz=two_sz,
                    locspin=list(two_s), **kw)
    rows = []
    for (i, j), c in zip(bonds, Js):
        for a in range(two_s[i] + 1):
            for b in range(two_s[j] + 1):
                v = c * (a - 0.5 * two_s[i]) * (b - 0.5 * two_s[j])
                if v != 0.0:
                    rows.append((i, a, i, a, j, b, j, b, v, 0.0))
        for a in range(two_s[i]):
            for b in range(1, two_s[j] + 1):
                v = 0.5 * c * _spin_raise(two_s[i], a) * _spin_raise(two_s[j], b - 1)
                rows.append((i, a + 1, i, a, j, b - 1, j, b, v, 0.0))
                rows.append((j, b, j, b - 1, i, a, i, a + 1, v, 0.0))
    if D != 0.0:
        for i in range(n):
            for a in range(two_s[i] + 1):
                mz = a - 0.5 * two_s[i]
                if mz != 0.0:
                    # (Sz_i)^2 = sum_a mz^2 |a><a|_i, written as |a><a|_i |a><a|_i
                    rows.append((i, a, i, a, i, a, i, a, D * mz * mz, 0.0))
    m.interall = rows
    if hx != 0.0:
        if two_sz is not None:
            raise ValueError("a transverse field needs the grand-canonical SpinGC model (two_sz=None)")
        for i in range(n):
            for a in range(two_s[i]):
                t = 0.5 * hx * _spin_raise(two_s[i], a)   # -hx Sx = -(hx/2)(S+ + S-): Trans t = hx/2 * <|S+|>
                m.trans += [(i, a + 1, i, a, t, 0.0), (i, a, i, a + 1, t, 0.0)]
    return m


def j1j2_chain(L: int, J1: float, J2: float, **kw) -> ExpertModel:
    bonds = chain_bonds(L, 1) + chain_bonds(L, 2)
    return heisenberg(L, bonds, [J1] * L + [J2] * L, **kw)


def hubbard(nsite: int, bonds: Sequence[Tuple[int, int]], t: float, U: float,
            nup: int, ndown: int, **kw) -> ExpertModel:
    """Canonical Hubbard model with hopping t on every bond (both spins, both directions)."""
    m = ExpertModel(model="Hubbard", nsite=nsite, ncond=nup + ndown, two_sz=nup - ndown, **kw)
    for i, j in bonds:
        for s in (0, 1):
            m.trans.append((i, s, j, s, float(t), 0.0))
            m.trans.append((j, s, i, s, float(t), 0.0))
    m.coulombintra = [(i, float(U)) for i in range(nsite)]
    return m


def kitaev_heisenberg(W: int, L: int, K: float, J: float, **kw) -> ExpertModel:
    """Kitaev-Heisenberg honeycomb in the SpinGC sector (no Sz conservation).

    H = sum_<ij>_gamma K S^gamma_i S^gamma_j + J S_i.S_j, written as
    S^x S^x = (Exchange + PairLift)/4 and S^y S^y = (Exchange - PairLift)/4 in HPhi's
    Exchange / PairLift conventions, S^z S^z = Ising.
    """
    bonds = honeycomb_bonds(W, L)
    m = ExpertModel(model="SpinGC", nsite=2 * W * L, two_sz=None, **kw)
    for i, j, g in bonds:
        kx, ky, kz = (K if g == 0 else 0.0), (K if g == 1 else 0.0), (K if g == 2 else 0.0)
        m.ising.append((i, j, kz + J))
        m.exchange.append((i, j, 0.25 * (kx + ky) + 0.5 * J))
        if kx - ky != 0.0:
            m.pairlift.append((i, j, 0.25 * (kx - ky)))
    return m


def random_interall_spin(nsite: int, nterms: int, seed: int) -> List[Tuple]:
    """Random Hermitian spin InterAll terms (each with its Hermitian partner)."""
    rng = random.Random(seed)
    out = []
    for _ in range(nterms):
        i, k = rng.sample(range(nsite), 2)
        s1, s2, s3, s4 = (rng.randint(0, 1) for _ in range(4))
        v = complex(rng.uniform(-1, 1), rng.uniform(-1, 1))
        if s1 == s2 and s3 == s4:
            v = complex(v.real, 0.0)
            out.append((i, s1, i, s2, k, s3, k, s4, v.real, 0.0))
        else:
            out.append((i, s1, i, s2, k, s3, k, s4, v.real, v.imag))
            out.append((k, s4, k, s3, i, s2, i, s1, v.real, -v.imag))
    return out


def sector_dim_estimate(m: ExpertModel) -> int:
    """Dimension of the model's sector (idim_max) without building it."""
    from math import comb
    if m.model.endswith("GC"):
        return 2 ** (m.nsite if m.model == "SpinGC" else 2 * m.nsite)
    if m.model == "Spin":
        nup = (m.nsite + (m.two_sz or 0)) // 2
        return comb(m.nsite, nup)
    if m.nup is not None and m.ndown is not None:
        return comb(m.nsite, m.nup) * comb(m.nsite, m.ndown)
    ne = m.ncond
    if m.two_sz is None:
        return comb(2 * m.nsite, ne)
    nup = (ne + m.two_sz) // 2
    return comb(m.nsite, nup) * comb(m.nsite, ne - nup)


def kondo_chain(cells: int, t: float, J: float, U: float = 0.0, ncond: Optional[int] = None, two_sz: int = 0,
                gc: bool = False, **kw) -> ExpertModel:
    """1D Kondo lattice: conduction site 2c (hopping t around the ring of cells, on-site U)
    and local spin 2c+1 per cell, coupled by J S_loc . s_cond written as InterAll terms:
    J/4 sum n n (sign by spins) + J/2 (c+_{l up} c_{l dn} c+_{c dn} c_{c up} + h.c.)."""
    n = 2 * cells
    m = ExpertModel(model="KondoGC" if gc else "Kondo", nsite=n, two_sz=None if gc else two_sz,
                    ncond=None if gc else (cells if ncond is None else ncond),
                    locspin=[(i % 2) for i in range(n)], **kw)
    for c in range(cells):
        a, b = 2 * c, 2 * ((c + 1) % cells)
        if cells > 1 and a != b:
            for s in (0, 1):
                m.trans += [(a, s, b, s, t, 0.0), (b, s, a, s, t, 0.0)]
    if U:
        m.coulombintra = [(2 * c, U) for c in range(cells)]
    for c in range(cells):
        l, e = 2 * c + 1, 2 * c
        for s1 in (0, 1):
            for s2 in (0, 1):
                sg = (1 if s1 == 0 else -1) * (1 if s2 == 0 else -1)
                m.interall.append((l, s1, l, s1, e, s2, e, s2, 0.25 * J * sg, 0.0))
        m.interall.append((l, 0, l, 1, e, 1, e, 0, 0.5 * J, 0.0))
        m.interall.append((l, 1, l, 0, e, 0, e, 1, 0.5 * J, 0.0))
    return m

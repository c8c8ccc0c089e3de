"""CPU oracle for the H*v / Lanczos / TPQ path (TEST INFRASTRUCTURE ONLY).

A numpy restatement of the reference's algorithms, used by the tests and by
bench.py's cpu_baseline leg as the checker.  The product (hphi_b200/) never imports
this module.  Each function mirrors the reference routine it cites, structured as the
reference is: one vectorised pass over all rows per Hamiltonian term, push form
``v0[off(j)] += coef * sgn * v1[j]``.

Its outputs are pinned against dumps of the reference itself (oracle/_ref/HPhi_ref,
built by oracle/Makefile from the reference sources) through the fixtures in
tests/golden/.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from math import comb
from typing import Dict, List, Tuple

import numpy as np

HUBBARD, SPIN, KONDO, HUBBARDGC, SPINGC, KONDOGC, HUBBARD_NCONS = 0, 1, 2, 3, 4, 5, 6


# ----------------------------------------------------------------------------- input
@dataclass
class Def:
    """What ReadDefFileNInt / ReadDefFileIdxPara (src/readdef.c:463, 1006) store."""
    calc_type: int = 0
    calc_model: int = 0
    calc_eigenvec: int = 0
    initial_vec_type: int = 0
    nsite: int = 0
    nup: int = 0
    ndown: int = 0
    ne: int = 0
    total_2sz: int = 0
    ncond: int = 0
    nlocspn: int = 0
    lanczos_max: int = 0
    initial_iv: int = 0
    k_exct: int = 1
    lanczos_eps: int = 14
    lanczos_target: int = 2
    large_value: float = 0.0
    num_ave: int = 1
    pre_cg: int = 0
    expand_coef: int = 0              # ExpandCoef of cTPQ (0: 10)
    locspn: List[int] = field(default_factory=list)   # 0 itinerant, 1 local spin (Kondo)
    trans: List[Tuple[int, int, int, int, complex]] = field(default_factory=list)   # off-diagonal, Hermitian pairs
    chemi: List[Tuple[int, int, float]] = field(default_factory=list)                # (site, spin, mu): -mu n
    coulomb_intra: List[Tuple[int, float]] = field(default_factory=list)
    coulomb_inter: List[Tuple[int, int, float]] = field(default_factory=list)
    hund: List[Tuple[int, int, float]] = field(default_factory=list)
    exchange: List[Tuple[int, int, float]] = field(default_factory=list)
    pairhop: List[Tuple[int, int, float]] = field(default_factory=list)
    pairlift: List[Tuple[int, int, float]] = field(default_factory=list)
    interall_diag: List[Tuple[int, int, int, int, float]] = field(default_factory=list)
    interall_off: List[Tuple[int, int, int, int, int, int, int, int, complex]] = field(default_factory=list)
    sz_conserved: bool = False        # iFlgSzConserved: a 2Sz line (src/readdef.c:570-573)
    green_one: List[Tuple[int, int, int, int]] = field(default_factory=list)      # OneBodyG rows
    green_two: List[Tuple[int, int, int, int, int, int, int, int]] = field(default_factory=list)  # TwoBodyG rows
    green_multi: Dict[int, List[Tuple[int, ...]]] = field(default_factory=dict)  # 3/4/6: ThreeBodyG ... rows
    expec_interval: int = 1
    # time evolution (CalcType 4): TEOneBody (te_kind 1) / TETwoBody (te_kind 2) rows per time index
    te_kind: int = 0
    te_time: List[float] = field(default_factory=list)
    te_rows: List[List[Tuple]] = field(default_factory=list)


def _table(path: str) -> List[List[float]]:
    with open(path) as f:
        lines = f.read().splitlines()
    n = int(lines[1].split()[1])
    rows = [list(map(float, l.split())) for l in lines[5:] if l.strip()]
    return rows[:n]


def _int_table(path: str) -> List[List[int]]:
    with open(path) as f:
        lines = f.read().splitlines()
    n = int(lines[1].split()[1])
    rows = [list(map(int, l.split())) for l in lines[5:] if l.strip()]
    return rows[:n]


def read_expert(namelist: str) -> Def:
    """Expert-mode reader (src/readdef.c).  Diagonal transfers become chemical terms and
    Ising becomes Hund(-J/2) + CoulombInter(-J/4) (src/readdef.c:1320-1327); InterAll
    terms with i=j, k=l and equal spins per pair are diagonal (GetDiagonalInterAll,
    src/readdef.c:2415-2549), the others stay as written."""
    base = os.path.dirname(os.path.abspath(namelist))
    files: Dict[str, str] = {}
    for line in open(namelist):
        p = line.split()
        if len(p) >= 2 and not p[0].startswith("#"):
            files[p[0].lower()] = os.path.join(base, p[1])
    d = Def()
    for line in open(files["calcmod"]):
        p = line.split()
        if len(p) < 2 or p[0].startswith("#"):
            continue
        k, v = p[0].lower(), int(p[1])
        if k == "calctype": d.calc_type = v
        elif k == "calcmodel": d.calc_model = v
        elif k == "calceigenvec": d.calc_eigenvec = v
        elif k == "initialvectype": d.initial_vec_type = v
    sz_cons, read_ncond = False, False
    for line in open(files["modpara"]).read().splitlines()[8:]:
        p = line.split()
        if len(p) < 2:
            continue
        k, v = p[0].lower(), float(p[1])
        if k == "nsite": d.nsite = int(v)
        elif k == "nup": d.nup = int(v)
        elif k == "ndown": d.ndown = int(v); d.total_2sz = d.nup - d.ndown
        elif k == "2sz": d.total_2sz = int(v); sz_cons = True
        elif k == "ncond": d.ncond = int(v); read_ncond = True
        elif k == "lanczos_max": d.lanczos_max = int(v)
        elif k == "initial_iv": d.initial_iv = int(v)
        elif k == "exct": d.k_exct = int(v)
        elif k == "precg": d.pre_cg = int(v)
        elif k == "expandcoef": d.expand_coef = int(v)
        elif k == "lanczoseps": d.lanczos_eps = int(v)
        elif k == "lanczostarget": d.lanczos_target = int(v)
        elif k == "largevalue": d.large_value = v
        elif k == "numave": d.num_ave = int(v)
        elif k == "expecinterval": d.expec_interval = int(v)
    loc_lines = open(files["locspin"]).read().splitlines()
    d.nlocspn = int(loc_lines[1].split()[1])
    d.locspn = [0] * d.nsite
    for l in loc_lines[5:]:
        p = l.split()
        if len(p) >= 2 and 0 <= int(p[0]) < d.nsite:
            d.locspn[int(p[0])] = int(p[1])
    if d.calc_model in (SPIN, HUBBARD, KONDO):
        if read_ncond:
            if sz_cons:
                d.nup = (d.nlocspn + d.ncond + d.total_2sz) // 2
                d.ndown = (d.nlocspn + d.ncond - d.total_2sz) // 2
            else:
                d.ne = d.ncond
                d.calc_model = HUBBARD_NCONS
        elif sz_cons:
            d.nup = (d.nlocspn + d.total_2sz) // 2
            d.ndown = (d.nlocspn - d.total_2sz) // 2
        if d.calc_model == SPIN:
            d.ne = d.nup
        elif d.ne == 0:
            d.ne = d.nup + d.ndown
    if d.lanczos_target < d.k_exct:
        d.lanczos_target = d.k_exct
    if "trans" in files:
        acc: Dict[Tuple[int, int, int, int], complex] = {}
        for r in _table(files["trans"]):
            key = (int(r[0]), int(r[1]), int(r[2]), int(r[3]))
            acc[key] = acc.get(key, 0) + complex(r[4], r[5] if len(r) > 5 else 0.0)
        for (i, s1, j, s2), t in acc.items():
            if i == j and s1 == s2:
                d.chemi.append((i, s1, t.real))
            else:
                d.trans.append((i, s1, j, s2, t))
    if "coulombintra" in files:
        d.coulomb_intra = [(int(r[0]), r[1]) for r in _table(files["coulombintra"])]
    if "coulombinter" in files:
        d.coulomb_inter = [(int(r[0]), int(r[1]), r[2]) for r in _table(files["coulombinter"])]
    if "hund" in files:
        d.hund = [(int(r[0]), int(r[1]), r[2]) for r in _table(files["hund"])]
    if "ising" in files:
        for r in _table(files["ising"]):
            d.hund.append((int(r[0]), int(r[1]), -r[2] / 2.0))
            d.coulomb_inter.append((int(r[0]), int(r[1]), -r[2] / 4.0))
    if "exchange" in files:
        d.exchange = [(int(r[0]), int(r[1]), r[2]) for r in _table(files["exchange"])]
    if "pairhop" in files:
        for r in _table(files["pairhop"]):
            d.pairhop.append((int(r[0]), int(r[1]), r[2]))
            d.pairhop.append((int(r[1]), int(r[0]), r[2]))
    if "pairlift" in files:
        d.pairlift = [(int(r[0]), int(r[1]), r[2]) for r in _table(files["pairlift"])]
    if "interall" in files:
        for r in _table(files["interall"]):
            i, s1, j, s2, k, s3, l, s4 = (int(x) for x in r[:8])
            v = complex(r[8], r[9] if len(r) > 9 else 0.0)
            if i == j and k == l and s1 == s2 and s3 == s4:
                d.interall_diag.append((i, s1, k, s3, v.real))
            else:
                d.interall_off.append((i, s1, j, s2, k, s3, l, s4, v))
    d.sz_conserved = sz_cons
    # Green's function rows (src/readdef.c:1441-1523)
    if "onebodyg" in files:
        for r in _int_table(files["onebodyg"]):
            if d.calc_model == SPIN and r[0] != r[2]:   # skipped with a warning (:1455-1460)
                continue
            d.green_one.append(tuple(r[:4]))
    if "twobodyg" in files:
        for r in _int_table(files["twobodyg"]):
            if _is_spin(d) and (r[0] != r[2] or r[4] != r[6]):   # CheckFormatForSpinInt (:1497-1503)
                raise ValueError("spin two-body Green's function rows need i == j and k == l")
            d.green_two.append(tuple(r[:8]))
    for key, npairs in (("threebodyg", 3), ("fourbodyg", 4), ("sixbodyg", 6)):   # :1525-1700
        if key in files:
            d.green_multi[npairs] = [tuple(r[:4 * npairs]) for r in _int_table(files[key])]
    # TEOneBody / TETwoBody (src/readdef.c:755-797, 1752-1840), read for CalcType 4 only:
    # 5 header lines (2nd: "AllTimeStep n"), then per time index "time count" and count rows
    for key, kind in (("teonebody", 1), ("tetwobody", 2)):
        if key in files and d.calc_type == 4:
            lines = [l for l in open(files[key]).read().splitlines()[5:] if l.strip()]
            pos = 0
            while pos < len(lines):
                t, n = lines[pos].split()[:2]
                rows = [tuple(float(x) for x in l.split()) for l in lines[pos + 1: pos + 1 + int(n)]]
                d.te_time.append(float(t))
                d.te_rows.append(rows)
                pos += 1 + int(n)
            d.te_kind = kind
    return d


# ------------------------------------------------------------------------- helpers
def _is_spin(d: Def) -> bool:
    return d.calc_model in (SPIN, SPINGC)


def _is_gc(d: Def) -> bool:
    return d.calc_model in (HUBBARDGC, SPINGC, KONDOGC)


def _rows_are_configs(d: Def) -> bool:
    """Grand-canonical models without lists (KondoGC keeps lists: its local spins stay
    singly occupied, src/sz.c:1342-1420)."""
    return d.calc_model in (HUBBARDGC, SPINGC)


def _general(d: Def) -> bool:
    """General spin: a spin model with some site 2S > 1 (CheckLocSpin, src/readdef.c:2735-2760)."""
    return _is_spin(d) and any(x > 1 for x in d.locspn)


def _tpow(d: Def) -> List[int]:
    """Mixed-radix place values (check, src/check.c:171-178): Tpow[i] = prod_{j<i} (2S_j + 1)."""
    t = [1]
    for x in d.locspn:
        t.append(t[-1] * (x + 1))
    return t


def _digit(d: Def, c: np.ndarray, site: int) -> np.ndarray:
    """GetBitGeneral (src/bitcalc.c:421-432): digit of `site` in mixed-radix configurations."""
    t = _tpow(d)
    return ((c // np.uint64(t[site])) % np.uint64(d.locspn[site] + 1)).astype(np.int64)


def _general_split(d: Def) -> Tuple[int, int]:
    """GetSplitBitForGeneralSpin (src/bitcalc.c:124-150): (ihfbit, number of lower sites)."""
    total = _tpow(d)[-1]
    isq = int(np.sqrt(float(total)))
    t = 1
    for i, x in enumerate(d.locspn):
        t *= x + 1
        if t >= isq:
            return t, i + 1
    return t, d.nsite


def nbits(d: Def) -> int:
    return d.nsite if _is_spin(d) else 2 * d.nsite


def split_bits(d: Def) -> Tuple[int, int, int]:
    """GetSplitBit (src/bitcalc.c:45-62): (ihfbit, irght, ilft)."""
    nb = nbits(d)
    ihfbit = 1 << ((nb + 1) // 2)
    irght = ihfbit - 1
    ilft = ((1 << nb) - 1) ^ irght
    return ihfbit, irght, ilft


def sdim(d: Def) -> int:
    """check() (src/check.c:296-328)."""
    return (1 << d.nsite) if not _is_spin(d) else (1 << (d.nsite // 2))


def _popcount(x: np.ndarray) -> np.ndarray:
    x = x.astype(np.uint64)
    c = np.zeros(x.shape, dtype=np.int64)
    while np.any(x):
        c += (x & np.uint64(1)).astype(np.int64)
        x = x >> np.uint64(1)
    return c


def _parity(x: np.ndarray) -> np.ndarray:
    """SgnBit (src/bitcalc.c:338-352) as 0/1 parity."""
    x = x.astype(np.uint64)
    for s in (1, 2, 4, 8, 16, 32):
        x = x ^ (x >> np.uint64(s))
    return (x & np.uint64(1)).astype(np.int64)


# ---------------------------------------------------------------------------- sz
def sz(d: Def):
    """sz (src/sz.c:62-832), hacker enumeration omp_sz_hacker (:993-1094) /
    omp_sz_spin_hacker (:1495-1546): blocks by upper half ib ascending, each block the
    ascending lower halves ia whose particle numbers complete the sector."""
    if _rows_are_configs(d):
        raise ValueError("grand-canonical models have no lists")
    if d.calc_model in (KONDO, KONDOGC):
        return _sz_kondo(d)
    if _general(d):
        return _sz_general(d)
    ihfbit, irght, ilft = split_bits(d)
    sd = sdim(d)
    lo = (nbits(d) + 1) // 2
    size21 = sd * 2 + 2 if (d.calc_model == SPIN and d.nsite % 2 == 1) else sd + 2
    list_2_1 = np.zeros(size21, dtype=np.uint64)
    list_2_2 = np.zeros(sd + 2, dtype=np.uint64)
    ia = np.arange(ihfbit, dtype=np.uint64)
    even = np.uint64(0x5555555555555555)
    if d.calc_model == HUBBARD:
        a_up, a_dn = _popcount(ia & even), _popcount(ia & ~even)
    else:
        a_up, a_dn = _popcount(ia), np.zeros(ihfbit, dtype=np.int64)
    blocks = []
    jb = 0
    cache: Dict[Tuple[int, int], np.ndarray] = {}
    for ib in range(sd):
        i = np.uint64(ib) * np.uint64(ihfbit)
        if d.calc_model == HUBBARD:
            nu, nd = int(_popcount(np.array([i & even]))[0]), int(_popcount(np.array([i & ~even]))[0])
            key = (d.nup - nu, d.ndown - nd)
            if key not in cache:
                cache[key] = np.nonzero((a_up == key[0]) & (a_dn == key[1]))[0].astype(np.uint64)
        else:
            nu = int(_popcount(np.array([i]))[0])
            target = d.ne
            key = (target - nu, 0)
            if key not in cache:
                cache[key] = np.nonzero(a_up == key[0])[0].astype(np.uint64) if key[0] >= 0 else np.zeros(0, np.uint64)
        sel = cache[key]
        if sel.size:
            blocks.append(sel + np.uint64(ib) * np.uint64(ihfbit))
            list_2_1[sel] = np.arange(sel.size, dtype=np.uint64) + np.uint64(2)
            list_2_2[ib] = jb + 1
            jb += sel.size
    list_1 = np.concatenate([np.zeros(1, dtype=np.uint64)] + blocks)
    return list_1, list_2_1, list_2_2


def _sz_general(d: Def):
    """General spin (src/sz.c:795-830 with omp_sz_GeneralSpin :1564-1590): 2Sz of every lower
    index ia < ihfbit and upper index ib; blocks by ib ascending, each the ascending ia whose
    2Sz completes Total2Sz; list_2_1[ia] = rank in its 2Sz class + 2 (classes some block
    uses), list_2_2[ib] = block offset + 1; list_1 holds mixed-radix configurations."""
    ihfbit, k = _general_split(d)
    total = _tpow(d)[-1]
    nhi = total // ihfbit
    ia = np.arange(ihfbit, dtype=np.uint64)
    sz_lo = np.zeros(ihfbit, dtype=np.int64)
    for site in range(k):
        sz_lo += 2 * _digit(d, ia, site) - d.locspn[site]
    ib_cfg = np.arange(nhi, dtype=np.uint64) * np.uint64(ihfbit)
    sz_hi = np.zeros(nhi, dtype=np.int64)
    for site in range(k, d.nsite):
        sz_hi += 2 * _digit(d, ib_cfg, site) - d.locspn[site]
    list_2_1 = np.zeros(ihfbit + 2, dtype=np.uint64)
    list_2_2 = np.zeros(nhi + 2, dtype=np.uint64)
    blocks, jb = [], 0
    for ib in range(nhi):
        sel = np.nonzero(sz_lo == d.total_2sz - sz_hi[ib])[0].astype(np.uint64)
        if sel.size:
            blocks.append(sel + np.uint64(ib * ihfbit))
            list_2_1[sel] = np.arange(sel.size, dtype=np.uint64) + np.uint64(2)
            list_2_2[ib] = jb + 1
            jb += sel.size
    list_1 = np.concatenate([np.zeros(1, dtype=np.uint64)] + blocks)
    return list_1, list_2_1, list_2_2


def _sz_kondo(d: Def):
    """omp_sz_Kondo / omp_sz_KondoGC (src/sz.c:1110-1220, 1342-1420) for even Nsite: a half
    is admissible when its local spins are singly occupied; blocks by ascending upper half,
    each block the ascending admissible lower halves with the missing (up, down) counts
    (KondoGC: all admissible lower halves)."""
    if d.nsite % 2:
        raise ValueError("odd Nsite Kondo is not restated")
    N, half = d.nsite, d.nsite // 2
    nh = 1 << N
    x = np.arange(nh, dtype=np.uint64)

    def admissible(site0):
        ok = np.ones(nh, dtype=bool)
        for j in range(half):
            if d.locspn[site0 + j]:
                u = (x >> np.uint64(2 * j)) & np.uint64(1)
                dn = (x >> np.uint64(2 * j + 1)) & np.uint64(1)
                ok &= (u != dn)
        return ok

    even = np.uint64(0x5555555555555555)
    up, dn = _popcount(x & even), _popcount(x & ~even)
    lo_ok, hi_ok = admissible(0), admissible(half)
    list_2_1 = np.zeros(nh + 2, dtype=np.uint64)
    list_2_2 = np.zeros(nh + 2, dtype=np.uint64)
    gc = d.calc_model == KONDOGC
    blocks, jb = [], 0
    for ib in range(nh):
        if not hi_ok[ib]:
            continue
        if gc:
            sel = np.nonzero(lo_ok)[0]
        else:
            nu, nd = d.nup - int(up[ib]), d.ndown - int(dn[ib])
            sel = np.nonzero(lo_ok & (up == nu) & (dn == nd))[0]
        if sel.size:
            blocks.append(sel.astype(np.uint64) + np.uint64(ib << N))
            list_2_1[sel] = np.arange(sel.size, dtype=np.uint64) + np.uint64(2)
            list_2_2[ib] = jb + 1
            jb += sel.size
    list_1 = np.concatenate([np.zeros(1, dtype=np.uint64)] + blocks)
    return list_1, list_2_1, list_2_2


def configs(d: Def, lists) -> np.ndarray:
    """Configuration of every row (1-based arrays: element 0 unused)."""
    if _rows_are_configs(d):
        n = _tpow(d)[-1] if _general(d) else 1 << nbits(d)
        return np.concatenate([np.zeros(1, np.uint64), np.arange(n, dtype=np.uint64)])
    return lists[0]


def get_off(d: Def, lists, c: np.ndarray) -> np.ndarray:
    """GetOffComp (src/bitcalc.c:195-223): 1-based row of configuration c, 0 if absent."""
    if _rows_are_configs(d):
        return c.astype(np.int64) + 1
    if _general(d):   # ConvertToList1GeneralSpin (src/bitcalc.c:285-300)
        ihfbit = np.uint64(_general_split(d)[0])
        a = lists[1][(c % ihfbit).astype(np.int64)].astype(np.int64)
        b = lists[2][(c // ihfbit).astype(np.int64)].astype(np.int64)
        return np.where((a == 0) | (b == 0), 0, a + b - 2)
    ihfbit, irght, ilft = split_bits(d)
    lo = (nbits(d) + 1) // 2
    a = lists[1][(c & np.uint64(irght)).astype(np.int64)].astype(np.int64)
    b = lists[2][(c >> np.uint64(lo)).astype(np.int64)].astype(np.int64)
    return np.where((a == 0) | (b == 0), 0, a + b - 2)


# ------------------------------------------------------------------------ diagonal
def diagonalcalc(d: Def, lists) -> np.ndarray:
    """diagonalcalc (src/diagonalcalc.c:84-187) in the reference's term order:
    CoulombIntra, Chemi, CoulombInter, Hund, InterAll-diagonal."""
    c = configs(d, lists)
    diag = np.zeros(c.size)
    if _general(d):
        # general spin: Chemi -mu [digit_i == s] (:425-433), InterAll-diagonal
        # V [digit_i == s1][digit_k == s3] (:1180-1202)
        for i, s_, mu in d.chemi:
            diag += -mu * (_digit(d, c, i) == s_)
        for i, s1, k, s3, V in d.interall_diag:
            diag += V * ((_digit(d, c, i) == s1) & (_digit(d, c, k) == s3))
        diag[0] = 0.0
        return diag
    bit = lambda pos: ((c >> np.uint64(pos)) & np.uint64(1)).astype(np.int64)
    spin = _is_spin(d)
    for i, U in d.coulomb_intra:   # SetDiagonalCoulombIntra :260-355 (zero for spin)
        if not spin:
            diag += U * (bit(2 * i) & bit(2 * i + 1))
    for i, s, mu in d.chemi:       # SetDiagonalChemi :373-527, tmp_V = -mu
        n = (bit(i) ^ (1 - s)) if spin else bit(2 * i + s)
        diag += -mu * n
    for i, j, V in d.coulomb_inter:  # SetDiagonalCoulombInter :543-787
        if spin:
            diag += V
        else:
            diag += V * (bit(2 * i) + bit(2 * i + 1)) * (bit(2 * j) + bit(2 * j + 1))
    for i, j, J in d.hund:         # SetDiagonalHund :788-1112, tmp_V = -J
        if spin:
            diag += -J * (bit(i) == bit(j))
        else:
            diag += -J * (bit(2 * i) * bit(2 * j) + bit(2 * i + 1) * bit(2 * j + 1))
    for i, s1, k, s3, V in d.interall_diag:  # SetDiagonalInterAll :1113-1415
        if spin:
            diag += V * ((bit(i) == s1) & (bit(k) == s3))
        else:
            diag += V * (bit(2 * i + s1) * bit(2 * k + s3))
    diag[0] = 0.0
    return diag


# -------------------------------------------------------------------------- mltply
def _hop(c: np.ndarray, b_to: int, b_from: int):
    """c+_{to} c_{from} on configurations c (CisAjt, src/mltplyHubbardCore.c:305-347):
    allowed iff 'to' empty and 'from' occupied (or to == from: n_from); returns
    (allowed mask, new configurations, sign) with sign = (-1)^(occupied strictly between)."""
    if b_to == b_from:
        ok = ((c >> np.uint64(b_from)) & np.uint64(1)).astype(bool)
        return ok, c, np.ones(c.size, dtype=np.int64)
    m_to, m_from = np.uint64(1 << b_to), np.uint64(1 << b_from)
    ok = ((c & m_to) == 0) & ((c & m_from) != 0)
    lo_b, hi_b = min(b_to, b_from), max(b_to, b_from)
    between = np.uint64(((1 << hi_b) - 1) ^ ((1 << (lo_b + 1)) - 1))
    sgn = 1 - 2 * _parity(c & between)
    return ok, c ^ (m_to | m_from), sgn


def _spin_flip(c: np.ndarray, site: int, to: int, frm: int):
    """|to><from| on spin site (child_exchange_spin_element / child_SpinGC_CisAit,
    src/mltplySpinCore.c:203-266): sigma equals the bit value."""
    b = (c >> np.uint64(site)) & np.uint64(1)
    ok = b == np.uint64(frm)
    if to == frm:
        return ok, c
    return ok, c ^ np.uint64(1 << site)


def mltply(d: Def, lists, diag: np.ndarray, v0: np.ndarray, v1: np.ndarray):
    """mltply (src/mltply.c:56-132): v0 += H v1 (1-based complex arrays) and
    prdct = <v1|H|v1>; the diagonal pass first, then one pass per off-diagonal term in
    the reference's order (mltplyHubbard src/mltplyHubbard.c:150-340, mltplyHalfSpin /
    mltplyHalfSpinGC src/mltplySpin.c:192-703)."""
    v0 = v0.astype(np.complex128).copy()
    v1 = v1.astype(np.complex128)
    c = configs(d, lists)
    rows = np.arange(1, c.size, dtype=np.int64)
    cj = c[1:]
    x = v1[1:]
    v0[1:] += diag[1:] * x
    prdct = np.sum(diag[1:] * np.abs(x) ** 2)
    spin = _is_spin(d)

    def scatter(ok, target, coef):
        nonlocal prdct
        off = np.zeros(cj.size, dtype=np.int64)
        off[ok] = get_off(d, lists, target[ok])
        ok = ok & (off > 0)
        dmv = coef[ok] * x[ok]
        np.add.at(v0, off[ok], dmv)
        prdct += np.sum(np.conj(v1[off[ok]]) * dmv)

    if spin and _general(d):
        tp = _tpow(d)

        def dflip(cc, site, to, frm):
            """GetOffCompGeneralSpin (src/bitcalc.c:243-275): digit frm -> to."""
            ok = _digit(d, cc, site) == frm
            return ok, (cc.astype(np.int64) + (to - frm) * tp[site]).astype(np.uint64)
        # Trans (GC, |s1><s2| with -t; mltplyGeneralSpinGC src/mltplySpin.c:738-770)
        for (i, s1, j, s2, t) in d.trans:
            ok, t1 = dflip(cj, i, s1, s2)
            scatter(ok, np.where(ok, t1, cj), np.full(cj.size, -t))
        # InterAll (mltplyGeneralSpin src/mltplySpin.c:351-381): site k first, then site i
        for (i, s1, j, s2, k, s3, l, s4, V) in d.interall_off:
            ok2, t2 = dflip(cj, k, s3, s4)
            t2 = np.where(ok2, t2, cj)
            ok1, t1 = dflip(t2, i, s1, s2)
            ok = ok1 & ok2
            scatter(ok, np.where(ok, t1, cj), np.full(cj.size, V))
    elif spin:
        # InterAll off-diagonal (general_int_spin :1020-1051 / GC_general_int_spin :1058-1112)
        for (i, s1, j, s2, k, s3, l, s4, V) in d.interall_off:
            ok2, t2 = _spin_flip(cj, k, s3, s4)
            ok1, t1 = _spin_flip(t2, i, s1, s2)
            scatter(ok1 & ok2, t1, np.full(cj.size, V))
        # transverse field (SpinGC Trans with s1 != s2; GC_CisAit, src/mltplySpin.c:500-560)
        for (i, s1, j, s2, t) in d.trans:
            ok, t1 = _spin_flip(cj, i, s1, s2)
            scatter(ok, t1, np.full(cj.size, -t))
        # Exchange (exchange_spin_element, src/mltplySpinCore.c:273-307): flip antiparallel pair
        for (i, j, J) in d.exchange:
            bi = (cj >> np.uint64(i)) & np.uint64(1)
            bj = (cj >> np.uint64(j)) & np.uint64(1)
            ok = bi != bj
            scatter(ok, cj ^ np.uint64((1 << i) | (1 << j)), np.full(cj.size, complex(J)))
        # PairLift (GC_pairlift_spin_element, src/mltplySpinCore.c:352-382): flip parallel pair
        for (i, j, J) in d.pairlift:
            bi = (cj >> np.uint64(i)) & np.uint64(1)
            bj = (cj >> np.uint64(j)) & np.uint64(1)
            ok = bi == bj
            scatter(ok, cj ^ np.uint64((1 << i) | (1 << j)), np.full(cj.size, complex(J)))
    else:
        fb = lambda site, s: 2 * site + s
        # Transfer (general_hopp / CisAjt): tmp_trans = -t  (src/mltplyHubbard.c:202)
        for (i, s1, j, s2, t) in d.trans:
            ok, t1, sg = _hop(cj, fb(i, s1), fb(j, s2))
            scatter(ok, t1, -t * sg)
        # InterAll off-diagonal: c+_i c_j c+_k c_l = (c+_i c_j)(c+_k c_l), right pair first
        for (i, s1, j, s2, k, s3, l, s4, V) in d.interall_off:
            ok2, t2, sg2 = _hop(cj, fb(k, s3), fb(l, s4))
            ok1, t1, sg1 = _hop(t2, fb(i, s1), fb(j, s2))
            scatter(ok1 & ok2, t1, V * sg1 * sg2)
        # PairHop (pairhopp_element :533-575): J, i both empty, j both occupied
        for (i, j, J) in d.pairhop:
            if i == j:
                continue
            b = lambda p: ((cj >> np.uint64(p)) & np.uint64(1)).astype(bool)
            ok = ~b(fb(i, 0)) & ~b(fb(i, 1)) & b(fb(j, 0)) & b(fb(j, 1))
            m = np.uint64((1 << fb(i, 0)) | (1 << fb(i, 1)) | (1 << fb(j, 0)) | (1 << fb(j, 1)))
            scatter(ok, cj ^ m, np.full(cj.size, complex(J)))
        # Exchange (exchange_element :472-526): tmp_J = -J, (i dn, j up) <-> (i up, j dn)
        for (i, j, J) in d.exchange:
            if i == j:
                continue
            b = lambda p: ((cj >> np.uint64(p)) & np.uint64(1)).astype(bool)
            ok = (~b(fb(i, 0)) & b(fb(i, 1)) & b(fb(j, 0)) & ~b(fb(j, 1))) | \
                 (b(fb(i, 0)) & ~b(fb(i, 1)) & ~b(fb(j, 0)) & b(fb(j, 1)))
            m = np.uint64((1 << fb(i, 0)) | (1 << fb(i, 1)) | (1 << fb(j, 0)) | (1 << fb(j, 1)))
            scatter(ok, cj ^ m, np.full(cj.size, complex(-J)))
    return v0, complex(prdct)


# ------------------------------------------------------------------------- drivers
def lanczos_eigenvalues(d: Def, lists, diag, v_init: np.ndarray, max_steps: int = None):
    """Lanczos_EigenValue (src/Lanczos_EigenValue.c:50-310): two-vector recurrence,
    dense tridiagonal eigenvalues every step, stop at |dE/E| < 10^-LanczosEps or
    beta < 1e-14.  Returns (converged step, E_target, lowest eigenvalues, alpha, beta)."""
    dim = v_init.size - 1
    maxs = min(d.lanczos_max if max_steps is None else max_steps, dim)
    eps = 10.0 ** (-d.lanczos_eps)
    target = d.lanczos_target
    v1 = v_init.astype(np.complex128).copy()
    v0 = np.zeros_like(v1)
    v0, pr = mltply(d, lists, diag, v0, v1)
    alpha, beta = [0.0, pr.real], [0.0]
    beta.append(float(np.sqrt(np.sum(np.abs(v0[1:] - alpha[1] * v1[1:]) ** 2))))
    ebefor = 0.0
    for stp in range(2, maxs + 1):
        a1, b1 = alpha[-1], beta[-1]
        tmp = v1.copy()
        v1[1:] = (v0[1:] - a1 * v1[1:]) / b1
        v0[1:] = -b1 * tmp[1:]
        v0, pr = mltply(d, lists, diag, v0, v1)
        alpha.append(pr.real)
        beta.append(float(np.sqrt(np.sum(np.abs(v0[1:] - alpha[-1] * v1[1:]) ** 2))))
        T = np.diag(alpha[1:stp + 1]) + np.diag(beta[1:stp], 1) + np.diag(beta[1:stp], -1)
        E = np.linalg.eigvalsh(T)
        if stp == 2 and target < 2:
            ebefor = E[target]
        if stp > 2 and stp > target:
            et = E[target]
            if abs((et - ebefor) / et) < eps or abs(beta[stp]) < 1e-14:
                return stp, et, E, np.array(alpha[1:]), np.array(beta[1:])
            ebefor = et
    raise RuntimeError("Lanczos did not converge")


def lanczos_eigenvector(d: Def, lists, diag, v_init: np.ndarray, alpha, beta, k: int = 0) -> np.ndarray:
    """Lanczos_EigenVector (src/Lanczos_EigenVector.c:46-195): the k-th eigenvector c of the
    tridiagonal matrix, then the recurrence replayed from the start vector with the stored
    alpha / beta, accumulating vg = sum_j c_j q_j; returned normalised (1-based)."""
    n = len(alpha)
    T = np.diag(alpha) + np.diag(beta[:n - 1], 1) + np.diag(beta[:n - 1], -1)
    c = np.linalg.eigh(T)[1][:, k]
    v1 = v_init.astype(np.complex128).copy()
    vg = c[0] * v1
    v0, _ = mltply(d, lists, diag, np.zeros_like(v1), v1)
    for stp in range(1, n):
        a1, b1 = alpha[stp - 1], beta[stp - 1]
        tmp = v1.copy()
        v1[1:] = (v0[1:] - a1 * v1[1:]) / b1
        v0[1:] = -b1 * tmp[1:]
        v0, _ = mltply(d, lists, diag, v0, v1)
        vg[1:] += c[stp] * v1[1:]
    vg[1:] /= np.sqrt(np.sum(np.abs(vg[1:]) ** 2))
    return vg


def expec_energy(d: Def, lists, diag, v: np.ndarray):
    """expec_energy_flct (src/expec_energy_flct.c:60-180) for a normalised vector: energy
    <v|H|v>, var <Hv|Hv>, doublon sum |v|^2 D and Sz sum |v|^2 (N_up - N_dn)/2 (Hubbard bit
    2i + s; spin bit i = up)."""
    hv, _ = mltply(d, lists, diag, np.zeros_like(v), v)
    energy = float(np.vdot(v[1:], hv[1:]).real)
    var = float(np.sum(np.abs(hv[1:]) ** 2))
    w = np.abs(v[1:]) ** 2
    c = configs(d, lists)[1:].astype(np.uint64)
    if _general(d):
        doublon = 0.0
        two_sz = sum(2 * _digit(d, c, i) - d.locspn[i] for i in range(d.nsite))
        sz = float(np.sum(w * 0.5 * two_sz))
    elif _is_spin(d):
        doublon = 0.0
        sz = float(np.sum(w * 0.5 * (2 * _popcount(c) - d.nsite)))
    else:
        even = np.uint64(0x5555555555555555)
        up, dn = _popcount(c & even), _popcount(c & ~even)
        doublon = float(np.sum(w * _popcount(c & (c >> np.uint64(1)) & even)))
        sz = float(np.sum(w * 0.5 * (up - dn)))
    return energy, var, doublon, sz


def cg_eigenvector(d: Def, lists, diag, v: np.ndarray, eig: float, noise: np.ndarray,
                   eps: float = 1e-8, eps_cg: float = 1e-8):
    """CG_EigenVector (src/CG_EigenVector.c:30-255): inverse iteration with conjugate-gradient
    solves of (H - eig + eps_cg) x = b.  b = v + noise, normalised (the reference draws the
    noise, amplitude 1e-3, from per-thread dSFMT streams); each round runs CG from x = 0
    until |r| < eps |b| (at most 500 iterations), normalises x and stops when
    ||<x|b>| - 1| < eps, else restarts from b = x (at most 51 rounds).
    Returns (x normalised, rounds, total CG iterations)."""
    b = v.astype(np.complex128).copy()
    b[1:] += noise
    b[1:] /= np.sqrt(np.sum(np.abs(b[1:]) ** 2))
    total = 0
    for rnd in range(51):
        bnorm = float(np.sum(np.abs(b[1:]) ** 2))
        r, p, x = b.copy(), b.copy(), np.zeros_like(b)
        for _ in range(500):
            y = (-eig + eps_cg) * p
            y, _ = mltply(d, lists, diag, y, p)
            rp = float(np.sum(np.abs(r[1:]) ** 2))
            alpha = rp / np.sum(y[1:] * np.conj(p[1:]))
            x[1:] += alpha * p[1:]
            r[1:] -= alpha * y[1:]
            rnorm2 = float(np.sum(np.abs(r[1:]) ** 2))
            p[1:] = r[1:] + (rnorm2 / rp) * p[1:]
            total += 1
            if np.sqrt(rnorm2) < eps * np.sqrt(bnorm):
                break
        x[1:] /= np.sqrt(np.sum(np.abs(x[1:]) ** 2))
        xb = np.vdot(x[1:], b[1:])
        if abs(abs(xb) - 1.0) < eps:
            return x, rnd + 1, total
        b = x
    return x, 51, total


def tpq_energies(d: Def, lists, diag, v_start: np.ndarray, nsteps: int):
    """CalcByTPQ (src/CalcByTPQ.c:52-294) for one sample: returns the energies of the
    SS_rand lines for steps 0 .. nsteps-1 (step 0 = the start vector itself)."""
    ns = float(d.nsite)
    L = d.large_value
    v = v_start.astype(np.complex128) / np.sqrt(np.sum(np.abs(v_start[1:]) ** 2))
    out = []
    h, _ = mltply(d, lists, diag, np.zeros_like(v), v)
    out.append(np.vdot(v[1:], h[1:]).real)
    for step in range(1, nsteps):
        w = L * v - h / ns
        w[0] = 0
        v = w / np.sqrt(np.sum(np.abs(w[1:]) ** 2))
        h, _ = mltply(d, lists, diag, np.zeros_like(v), v)
        out.append(np.vdot(v[1:], h[1:]).real)
    return np.array(out)


def dense_hamiltonian(d: Def, lists, diag) -> np.ndarray:
    """Dense H from columns H e_j (small dims only)."""
    dim = diag.size - 1
    H = np.zeros((dim, dim), dtype=np.complex128)
    for j in range(dim):
        e = np.zeros(dim + 1, dtype=np.complex128)
        e[j + 1] = 1.0
        col, _ = mltply(d, lists, diag, np.zeros_like(e), e)
        H[:, j] = col[1:]
    return H


# ----------------------------------------------------------------------------- LOBPCG
def _lowdin_eigen(hsub: np.ndarray, ovlp: np.ndarray):
    """diag_ovrp (src/CalcByLOBPCG.c:43-123): Lowdin-orthogonalised H v = mu O v, overlap
    eigenvalues <= 1e-10 dropped.  Returns (mu ascending, vectors as columns)."""
    oe, ov = np.linalg.eigh(ovlp)
    keep = oe > 1.0e-10
    S = ov[:, keep] / np.sqrt(oe[keep])
    mu, phi = np.linalg.eigh(S.conj().T @ hsub @ S)
    return mu, S @ phi


def _preshift(eig: float, res: float, eps: float) -> float:
    """calc_preshift (src/CalcByLOBPCG.c:129-148)."""
    if res >= 1.0:
        return 0.0
    k = np.trunc(np.log10(abs(eig)))
    i = np.ceil(np.log10(eps)) if eps > res else np.ceil(np.log10(res))
    return float(np.trunc(eig / 10.0 ** (k + i)) * 10.0 ** (k + i))


def lobpcg(d: Def, lists, diag, x_init: np.ndarray):
    """LOBPCG_Main (src/CalcByLOBPCG.c:328-632) on a dense H: x_init is (exct, dim+1).
    Returns (step rows [step, max residual, threshold, eig...], final x (exct, dim))."""
    H = dense_hamiltonian(d, lists, diag)
    dg = diag[1:]
    k = x_init.shape[0]
    x = np.array(x_init[:, 1:], dtype=np.complex128)
    x /= np.linalg.norm(x, axis=1)[:, None]
    hx = x @ H.T
    p = np.zeros_like(x)
    hp = np.zeros_like(x)
    eig = np.real(np.sum(x.conj() * hx, axis=1))
    shift0 = d.large_value * d.nsite
    rows = []
    for stp in range(1, d.lanczos_max + 1):
        eps = 10.0 ** (-0.5 * d.lanczos_eps)
        if np.max(np.abs(eig)) > 1.0:
            eps *= np.max(np.abs(eig))
        w = hx - eig[:, None] * x
        dmax = 0.0
        for i in range(k):
            dn = np.linalg.norm(w[i])
            dmax = max(dmax, dn)
            if stp != 1:
                if d.pre_cg == 1:
                    sh = _preshift(eig[i] + shift0, dn, eps) - shift0
                    pc = dg - sh
                    m = np.abs(pc) > eps
                    w[i, m] /= pc[m]
                w[i] /= np.linalg.norm(w[i])
        rows.append([stp, dmax, eps] + list(eig))
        if dmax < eps:
            break
        hw = w @ H.T
        B = np.concatenate([w, x, p])
        HB = np.concatenate([hw, hx, hp])
        hsub = B.conj() @ HB.T
        ovlp = B.conj() @ B.T
        eig = np.real(np.diag(hsub)[k:2 * k]).copy()
        mu, V = _lowdin_eigen(hsub, ovlp)
        eig = 0.5 * (eig + mu[:k])
        C = V[:, :k]
        Cp = C.copy()
        Cp[k:2 * k] = 0.0
        x, hx, p, hp = C.T @ B, C.T @ HB, Cp.T @ B, Cp.T @ HB
        nx = np.linalg.norm(x, axis=1)[:, None]
        np_ = np.linalg.norm(p, axis=1)[:, None]
        x, hx, p, hp = x / nx, hx / nx, p / np_, hp / np_
    return np.array(rows), x


# ------------------------------------------------------------- Green's functions
def _fbit(site: int, s: int) -> int:
    return 2 * site + s


def _sum_pairs(d: Def, lists, ok, target, coef, vec, x):
    """sum over rows j with ok of conj(vec[off(target_j)]) * coef_j * vec[j] (M_CORR mode of
    the element routines: the scatter into v0 is skipped, dam_pr is returned)."""
    off = np.zeros(x.size, dtype=np.int64)
    off[ok] = get_off(d, lists, target[ok])
    ok = ok & (off > 0)
    return complex(np.sum(np.conj(vec[off[ok]]) * coef[ok] * x[ok]))


def expec_cisajs(d: Def, lists, vec: np.ndarray) -> np.ndarray:
    """expec_cisajs (src/expec_cisajs.c:66-641): <vec| c+_{i s1} c_{j s2} |vec> per OneBodyG
    row (spin models: |s1><s2| on site i, zero for i != j); vec is 1-based complex."""
    vec = vec.astype(np.complex128)
    cj = configs(d, lists)[1:]
    x = vec[1:]
    one = np.ones(x.size)
    out = []
    for (i, s1, j, s2) in d.green_one:
        val = 0j
        if d.calc_model == HUBBARDGC:                                   # :193-243
            ok, t, sg = _hop(cj, _fbit(i, s1), _fbit(j, s2))
            val = _sum_pairs(d, lists, ok, t, sg, vec, x)
        elif d.calc_model in (HUBBARD, HUBBARD_NCONS, KONDO, KONDOGC):   # :254-316
            if d.sz_conserved and s1 != s2:
                val = 0j
            elif d.calc_model in (KONDO, KONDOGC) and (
                    (d.locspn[i] == 1 and d.locspn[j] == 0) or (d.locspn[i] == 0 and d.locspn[j] == 1)):
                val = 0j
            elif i == j and s1 == s2:
                n = ((cj >> np.uint64(_fbit(i, s1))) & np.uint64(1)).astype(np.float64)
                val = complex(np.sum(n * np.abs(x) ** 2))
            else:
                ok, t, sg = _hop(cj, _fbit(i, s1), _fbit(j, s2))
                val = _sum_pairs(d, lists, ok, t, sg, vec, x)
        elif d.calc_model == SPIN:                                     # :329-470
            if i == j and s1 == s2:
                hit = (_digit(d, cj, i) if _general(d) else ((cj >> np.uint64(i)) & np.uint64(1)).astype(np.int64)) == s1
                val = complex(np.sum(hit * np.abs(x) ** 2))
        elif d.calc_model == SPINGC:                                   # :496-641
            if i == j:
                if _general(d):
                    dig = _digit(d, cj, i)
                    if s1 == s2:
                        val = complex(np.sum((dig == s1) * np.abs(x) ** 2))
                    else:   # GetOffCompGeneralSpin(j-1, site, s2 -> s1)
                        tp = _tpow(d)
                        ok = dig == s2
                        t = (cj.astype(np.int64) + (s1 - s2) * tp[i]).astype(np.uint64)
                        val = _sum_pairs(d, lists, ok, np.where(ok, t, cj), one, vec, x)
                else:
                    b = ((cj >> np.uint64(i)) & np.uint64(1)).astype(np.int64)
                    if s1 == s2:   # child_SpinGC_CisAis = bit ^ (1 - s1)
                        val = complex(np.sum((b == s1) * np.abs(x) ** 2))
                    else:          # child_SpinGC_CisAit(j, site, s2): bit == s2 flips
                        ok = b == s2
                        val = _sum_pairs(d, lists, ok, cj ^ np.uint64(1 << i), one, vec, x)
        out.append(val)
    return np.array(out, dtype=np.complex128)


def _rearray(r):
    """Rearray_Interactions (src/expec_cisajscktaltdc.c:274-391): on-site pairs ordered by
    site; returns (i, s1, j, s2, k, s3, l, s4, V) or None."""
    i, s1, j, s2, k, s3, l, s4 = r
    if i == j and k == l:
        return (k, s3, l, s4, i, s1, j, s2, 1.0) if i > k else (i, s1, j, s2, k, s3, l, s4, 1.0)
    if i == l and k == j:
        return (k, s3, j, s2, i, s1, l, s4, -1.0) if i > k else (i, s1, l, s4, k, s3, j, s2, -1.0)
    return None


def expec_cisajscktalt(d: Def, lists, vec: np.ndarray) -> np.ndarray:
    """expec_cisajscktaltdc (src/expec_cisajscktaltdc.c:87-1647): <vec| c+_{i s1} c_{j s2}
    c+_{k s3} c_{l s4} |vec> per TwoBodyG row; spin models through Rearray_Interactions and
    the per-model branches."""
    vec = vec.astype(np.complex128)
    cj = configs(d, lists)[1:]
    x = vec[1:]
    one = np.ones(x.size)
    out = []
    general = _general(d)
    tp = _tpow(d) if general else None

    def sbit(c, site):
        return _digit(d, c, site) if general else ((c >> np.uint64(site)) & np.uint64(1)).astype(np.int64)

    def sflip(c, site, to, frm):
        """|to><frm| on a site: (ok, new configurations)."""
        ok = sbit(c, site) == frm
        if general:
            return ok, (c.astype(np.int64) + (to - frm) * tp[site]).astype(np.uint64)
        return ok, (c ^ np.uint64(1 << site)) if to != frm else c

    for row in d.green_two:
        val = 0j
        if not _is_spin(d):
            i, s1, j, s2, k, s3, l, s4 = row
            if d.calc_model in (HUBBARD, HUBBARD_NCONS, KONDO, KONDOGC) and d.sz_conserved and s1 + s3 != s2 + s4:
                out.append(0j)                                          # :535-541
                continue
            # general_int_GetInfo + CisAjtCkuAlv_element and its relatives (:393-618):
            # c+_k c_l first, then c+_i c_j on the intermediate configuration
            ok2, t2, sg2 = _hop(cj, _fbit(k, s3), _fbit(l, s4))
            ok1, t1, sg1 = _hop(t2, _fbit(i, s1), _fbit(j, s2))
            val = _sum_pairs(d, lists, ok1 & ok2, t1, (sg1 * sg2).astype(np.float64), vec, x)
            out.append(val)
            continue
        rr = _rearray(row)
        if rr is None:
            out.append(0j)
            continue
        i, s1, j, s2, k, s3, l, s4, V = rr
        if d.calc_model == SPIN and not general:                       # :652-770
            if s1 == s2 and s3 == s4:
                val = complex(V * np.sum(((sbit(cj, i) == s2) & (sbit(cj, k) == s4)) * np.abs(x) ** 2))
            elif i == k and s1 == s4 and s3 == s2:
                val = complex(V * np.sum((sbit(cj, i) == s1) * np.abs(x) ** 2))
            elif s1 == s4 and s2 == s3:   # child_exchange_spin_element; tmp_V is not applied
                ok = (sbit(cj, i) == s2) & (sbit(cj, k) == s4)
                val = _sum_pairs(d, lists, ok, cj ^ np.uint64((1 << i) | (1 << k)), one, vec, x)
        elif d.calc_model == SPIN:                                     # :784-890
            two_sz = lambda site, g: 2 * g - d.locspn[site]   # GetLocal2Sz
            o = row
            dsz = two_sz(o[0], o[1]) - two_sz(o[2], o[3]) + two_sz(o[4], o[5]) - two_sz(o[6], o[7])
            if dsz != 0:
                val = 0j
            elif s1 == s2 and s3 == s4:
                val = complex(V * np.sum(((sbit(cj, i) == s1) & (sbit(cj, k) == s3)) * np.abs(x) ** 2))
            elif s1 != s2 and s3 != s4:
                ok2, t2 = sflip(cj, k, s3, s4)
                ok1, t1 = sflip(np.where(ok2, t2, cj), i, s1, s2)
                ok = ok1 & ok2
                val = _sum_pairs(d, lists, ok, np.where(ok, t1, cj), V * one, vec, x)
        else:                                                          # SpinGC :1423-1647
            if s1 == s2 and s3 == s4:
                val = complex(V * np.sum(((sbit(cj, i) == s2) & (sbit(cj, k) == s4)) * np.abs(x) ** 2))
            else:
                # the right pair on the initial configuration, the left pair after it
                ok2, t2 = sflip(cj, k, s3, s4)
                ok1, t1 = sflip(np.where(ok2, t2, cj), i, s1, s2)
                ok = ok1 & ok2
                val = _sum_pairs(d, lists, ok, np.where(ok, t1, cj), V * one, vec, x)
        out.append(val)
    return np.array(out, dtype=np.complex128)


def read_green_file(path: str) -> Tuple[np.ndarray, np.ndarray]:
    """Rows and complex values of a zvo_cisajs*.dat / zvo_cisajscktalt*.dat file."""
    rows, vals = [], []
    for line in open(path):
        p = line.split()
        if not p:
            continue
        rows.append([int(t) for t in p[:-2]])
        vals.append(complex(float(p[-2]), float(p[-1])))
    return np.array(rows, dtype=np.int64), np.array(vals, dtype=np.complex128)


def expec_multibody(d: Def, vec: np.ndarray, npairs: int):
    """expec_Threebody / Fourbody / Sixbody_SpinGCHalf (src/expec_cisajscktaltdc.c:901-1420)
    for the ThreeBodyG / FourBodyG / SixBodyG rows: the pairs after the second act first,
    last pair first, through mltplyHalfSpinGC_mini (src/mltplySpin.c:416-500: |s><t| on one
    site, nothing for a pair on two sites); then Rearray_Interactions on the first two pairs
    (None: the reference prints 8 indices and zero) and <vec| O_12 O_34 |vec_pr>.  Returns
    (values, short) or None when the model is not spin-1/2 SpinGC (the file stays empty)."""
    if d.calc_model != SPINGC or _general(d):
        return None
    vec = vec.astype(np.complex128)
    n = vec.size - 1
    c = np.arange(n, dtype=np.uint64)

    def apply(site, to, frm, x):
        y = np.zeros_like(x)
        ok = ((c >> np.uint64(site)) & np.uint64(1)) == np.uint64(frm)
        tgt = (c ^ np.uint64(1 << site)) if to != frm else c
        y[(tgt[ok] + np.uint64(1)).astype(np.int64)] += x[1:][ok]
        return y

    vals, short = [], []
    for row in d.green_multi.get(npairs, []):
        pairs = [row[4 * k:4 * k + 4] for k in range(npairs)]
        vp = vec.copy()
        for (i, s_, j, t) in reversed(pairs[2:]):
            vp = apply(i, s_, t, vp) if i == j else np.zeros_like(vp)
        rr = _rearray(tuple(row[:8]))
        if rr is None:
            vals.append(0j)
            short.append(True)
            continue
        i1, s1, _, s2, k1, s3, _, s4, V = rr
        w = apply(i1, s1, s2, apply(k1, s3, s4, vp))
        vals.append(complex(V * np.vdot(vec[1:], w[1:])))
        short.append(False)
    return np.array(vals, dtype=np.complex128), np.array(short, dtype=bool)



def _te_def(d: Def, step: int) -> Def:
    """H at time index `step`: the static terms plus that index's TE rows, as MakeTEDTransfer /
    MakeTEDInterAll (src/CalcByTEM.c:237-279) and diagonalcalcForTE (src/diagonalcalc.c:195-245)
    add them: a site-diagonal transfer is -t n (real part), other transfers -t c+c, InterAll
    rows split as the static InterAll."""
    import dataclasses
    e = dataclasses.replace(d, trans=list(d.trans), chemi=list(d.chemi),
                            interall_diag=list(d.interall_diag), interall_off=list(d.interall_off))
    for r in d.te_rows[step]:
        if d.te_kind == 1:
            i, s1, j, s2 = (int(x) for x in r[:4])
            t = complex(r[4], r[5])
            if i == j and s1 == s2:
                e.chemi.append((i, s1, t.real))
            else:
                e.trans.append((i, s1, j, s2, t))
        else:
            i, s1, j, s2, k, s3, l, s4 = (int(x) for x in r[:8])
            v = complex(r[8], r[9])
            if i == j and k == l and s1 == s2 and s3 == s4:
                e.interall_diag.append((i, s1, k, s3, v.real))
            else:
                e.interall_off.append((i, s1, j, s2, k, s3, l, s4, v))
    return e


def te_flct(d: Def, lists, v: np.ndarray):
    """Diagonal observables of expec_energy_flct (src/expec_energy_flct.c:186-666) for a
    normalised vector: (doublon, doublon^2, N, N^2, Sz, Sz^2); a canonical spin model gives
    the constants of :92-101."""
    w = np.abs(v[1:]) ** 2
    if d.calc_model == SPIN:
        sz = 0.5 * d.total_2sz
        return 0.0, 0.0, float(d.nsite), float(d.nsite) ** 2, sz, sz * sz
    c = configs(d, lists)[1:].astype(np.uint64)
    even = np.uint64(0x5555555555555555)
    up, dn = _popcount(c & even).astype(float), _popcount(c & ~even).astype(float)
    dbl = _popcount(c & (c >> np.uint64(1)) & even).astype(float)
    n, sz = up + dn, 0.5 * (up - dn)
    return (float(w @ dbl), float(w @ dbl ** 2), float(w @ n), float(w @ n ** 2), float(w @ sz),
            float(w @ sz ** 2))


def te_run(d: Def, lists, v_init: np.ndarray, step_initial: int = 0, keep_states=()):
    """CalcByTEM (src/CalcByTEM.c:52-234) with MultiplyForTEM (src/Multiply.c:79-139).  Per time
    index: dt = TETime[i] - TETime[i-1] (0 at index 0); for dt >= 1e-14 the state becomes
    psi - i dt H' psi + sum_{k=2}^{ExpandCoef} (-i dt)^k / k! H^k psi, where H' psi is the H psi
    of the previous index (zero before the first one) and H is this index's Hamiltonian; then it
    is normalised (norm = global_norm) and measured: E = <psi|H psi>, var = <H psi|H psi> and the
    Flct observables.  Returns per-index rows (time, E, var, norm, flct...) and the states at
    the indices in keep_states."""
    psi = np.asarray(v_init, dtype=np.complex128).copy()
    hpsi = np.zeros_like(psi)
    rows, states = [], {}
    for step in range(step_initial, d.lanczos_max):
        e = _te_def(d, step)
        diag = diagonalcalc(e, lists)
        dt = 0.0 if step == 0 else d.te_time[step] - d.te_time[step - 1]
        if dt >= 1e-14:
            acc = psi + (-1j * dt) * hpsi
            term, coef = hpsi, -1j * dt
            for k in range(2, d.expand_coef + 1):
                coef *= -1j * dt / k
                term, _ = mltply(e, lists, diag, np.zeros_like(psi), term)
                acc = acc + coef * term
            psi = acc
        psi[0] = 0.0
        norm = float(np.sqrt(np.sum(np.abs(psi[1:]) ** 2)))
        psi = psi / norm
        hpsi, _ = mltply(e, lists, diag, np.zeros_like(psi), psi)
        energy = float(np.vdot(psi[1:], hpsi[1:]).real)
        var = float(np.sum(np.abs(hpsi[1:]) ** 2))
        rows.append((d.te_time[step], energy, var, norm) + te_flct(d, lists, psi) + (step,))
        if step in keep_states:
            states[step] = psi.copy()
    return rows, states

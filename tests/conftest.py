import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden_cases(kind=None):
    out = []
    for name in sorted(os.listdir(GOLDEN)):
        p = os.path.join(GOLDEN, name, "golden.npz")
        if not os.path.exists(p):
            continue
        z = np.load(p)
        large = "sha_list_1" in z.files
        te = "text_SS" in z.files          # time-evolution cases
        if (kind == "te") != te:
            continue
        green = "green_files" in z.files
        if kind != "te" and (kind == "green") != green:
            continue
        if kind == "large" and not large:
            continue
        if kind == "small" and large:
            continue
        if kind == "lanczos" and (large or "steps" not in z.files):
            continue
        if kind == "tpq" and (large or "tpq" not in z.files):
            continue
        if kind == "lobpcg" and (large or "lobpcg_steps" not in z.files):
            continue
        if kind == "lanczos_or_tpq" and (large or ("steps" not in z.files and "tpq" not in z.files)):
            continue
        if kind == "eigenvector" and (large or "energy_state" not in z.files):
            continue
        out.append(name)
    return out


def case_dir(name):
    return os.path.join(GOLDEN, name)


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name, "golden.npz")))


def green_reference(z, fname):
    """(rows, values, text lines) of a reference Green's function file stored in a fixture."""
    lines = str(z["text_" + fname]).splitlines()
    rows = [[int(t) for t in l.split()[:-2]] for l in lines]  # short multi-body lines have 8 indices
    vals = np.array([complex(float(l.split()[-2]), float(l.split()[-1])) for l in lines])
    return rows, vals, lines


def tpq_state(O, d, lists, start, step):
    """The normalised TPQ state of `step` from the normalised start vector (oracle H*v):
    microcanonical v <- (L v - H v / Ns) / |.| (src/Multiply.c:42-68); canonical (CalcType 5)
    v <- sum_{c <= ExpandCoef} (-dtau H / 2)^c / c! v / |.|, dtau = 1 / L (src/Multiply.c:162-203)."""
    v = start.astype(np.complex128).copy()
    diag = O.diagonalcalc(d, lists)
    H = lambda x: O.mltply(d, lists, diag, np.zeros_like(x), x)[0]
    for _ in range(step):
        if d.calc_type == 5:
            a = -0.5 / d.large_value
            acc, term, coef = v.copy(), v.copy(), 1.0
            for c in range(1, (d.expand_coef or 10) + 1):
                term = H(term)
                coef *= a / c
                acc = acc + coef * term
            v = acc
        else:
            v = d.large_value * v - H(v) / d.nsite
        v[0] = 0
        v /= np.linalg.norm(v[1:])
    return v



def oracle_green_file(O, d, lists, v, fname):
    """(rows, values) the reference writes into Green's function file `fname` for the
    vector v, from the oracle: rows as printed (8 indices for rows Rearray_Interactions
    rejects), empty arrays for a file the reference leaves empty."""
    empty = (np.zeros((0,), dtype=np.int64), np.zeros(0, dtype=np.complex128))
    for key, npairs in (("ThreeBody", 3), ("FourBody", 4), ("SixBody", 6)):
        if key in fname:
            res = O.expec_multibody(d, v, npairs)
            if res is None:
                return empty
            vals, short = res
            rows = [list(r[:8]) if sh else list(r) for r, sh in zip(d.green_multi[npairs], short)]
            return rows, vals
    if "cktalt" in fname:
        if not d.green_two:
            return empty
        return [list(r) for r in d.green_two], O.expec_cisajscktalt(d, lists, v)
    return [list(r) for r in d.green_one], O.expec_cisajs(d, lists, v)


def check_green_lines(lines, rows, vals, atol):
    """Parsed lines of a Green's function file against (rows, values)."""
    assert len(lines) == len(rows), (len(lines), len(rows))
    for line, r, v in zip(lines, rows, vals):
        p = line.split()
        assert [int(t) for t in p[:-2]] == list(r), (line, r)
        assert abs(complex(float(p[-2]), float(p[-1])) - v) <= atol, (line, v)

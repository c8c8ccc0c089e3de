"""CPU-side checks of the C-ABI library: it loads, exports every symbol the header
declares, parses expert-mode input on the host, and its compiled terms - evaluated
here in numpy with the kernel's gather rule - reproduce the reference's H*v."""
import os
import re
import shutil

import numpy as np
import pytest

import hphi_b200
from conftest import ROOT, case_dir, golden_cases, load_golden

HEADER = os.path.join(ROOT, "include", "hphi_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hphi_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_header_symbols():
    lib = hphi_b200.load_library()
    syms = declared_symbols()
    assert syms, "no declarations found in include/hphi_b200.h"
    for s in syms:
        assert hasattr(lib, s), f"{s} declared in the header but not exported"
    assert set(syms) == set(hphi_b200.EXPORTED_SYMBOLS)
    assert b"sm_100a" in lib.hphi_version()


def test_open_without_device_or_bad_input_reports_error(tmp_path):
    with pytest.raises(hphi_b200.HPhiError, match="cannot open"):
        hphi_b200.Hamiltonian(str(tmp_path / "missing.def"))
    src = case_dir("chain16")
    for f in os.listdir(src):
        if f.endswith(".def"):
            shutil.copy(os.path.join(src, f), tmp_path)
    with open(tmp_path / "namelist.def", "a") as f:
        f.write("Bogus bogus.def\n")
    with pytest.raises(hphi_b200.HPhiError, match="unknown keyword"):
        hphi_b200.Hamiltonian(str(tmp_path / "namelist.def"))


def test_parser_rejects_non_hermitian_transfer(tmp_path):
    from hphi_b200 import expert
    m = expert.hubbard(4, expert.chain_bonds(4), 1.0, 2.0, 2, 2)
    m.trans.append((0, 0, 2, 0, 0.5, 0.0))  # partner (2,0,0,0) missing
    path = m.write(str(tmp_path))
    with pytest.raises(hphi_b200.HPhiError, match="not Hermitian"):
        hphi_b200.inspect_terms(path)


def _popcount(x):
    x = x.astype(np.uint64)
    c = np.zeros(x.shape, dtype=np.int64)
    for s in range(64):
        c += ((x >> np.uint64(s)) & np.uint64(1)).astype(np.int64)
    return c


def _general_spins(name):
    """2S of every site when the case is a general-spin one (some 2S > 1), else None."""
    lines = open(os.path.join(case_dir(name), "locspn.def")).read().splitlines()[5:]
    two_s = [int(l.split()[1]) for l in lines if len(l.split()) >= 2]
    calc = open(os.path.join(case_dir(name), "calcmod.def")).read()
    spin = any(l.split()[:2] in (["CalcModel", "1"], ["CalcModel", "4"]) for l in calc.splitlines())
    return two_s if spin and any(x > 1 for x in two_s) else None


def _packed(mixed, two_s):
    """Mixed-radix configurations -> the engine's packed digit codes (fixed-width fields)."""
    bits = max(1, int(np.ceil(np.log2(max(two_s) + 1))))
    x = mixed.astype(np.uint64).copy()
    out = np.zeros(x.size, dtype=np.uint64)
    for i, t in enumerate(two_s):
        out |= (x % np.uint64(t + 1)) << np.uint64(bits * i)
        x //= np.uint64(t + 1)
    return out


def emulate_hv(name, v1_1based):
    """H v1 from the compiled terms with the device kernel's gather rule."""
    g = load_golden(name)
    masks, coefs, dmasks, dcoefs = hphi_b200.inspect_terms(os.path.join(case_dir(name), "namelist.def"))
    two_s = _general_spins(name)
    if two_s is not None:
        # packed codes in row order (ascending, as the mixed-radix configurations)
        mixed = g["list_1"][1:] if "list_1" in g else np.arange(v1_1based.size - 1, dtype=np.uint64)
        conf = _packed(mixed, two_s)

        def row(s):
            idx = np.searchsorted(conf, s)
            hit = (idx < conf.size) & (conf[np.minimum(idx, conf.size - 1)] == s)
            return np.where(hit, idx, -1)
    elif "list_1" in g:
        conf = g["list_1"][1:]
        l21, l22 = g["list_2_1"], g["list_2_2"]
        nb = int(np.log2(l22.size - 2)) if l22.size > 2 else 0
        lo_bits = int(np.log2(l21.size - 2))
        # spin with odd Nsite: list_2_1 has 2*sdim+2 entries (ihfbit = 2*sdim)

        def row(s):
            a = l21[(s & np.uint64((1 << lo_bits) - 1)).astype(np.int64)].astype(np.int64)
            b = l22[(s >> np.uint64(lo_bits)).astype(np.int64)].astype(np.int64)
            return np.where((a == 0) | (b == 0), -1, a + b - 3)
    else:
        conf = np.arange(v1_1based.size - 1, dtype=np.uint64)

        def row(s):
            return s.astype(np.int64)
    x = v1_1based[1:]
    d = np.zeros(conf.size)
    for (cm, cv), v in zip(dmasks, dcoefs):
        d += v * ((conf & cm) == cv)
    y = d * x
    for (cm, cv, fl, sm), c in zip(masks, coefs):
        hit = (conf & cm) == cv
        src = conf[hit] ^ fl
        r = row(src)
        ok = r >= 0
        sg = 1 - 2 * (_popcount(conf[hit] & sm) & 1)
        contrib = np.zeros(hit.sum(), dtype=np.complex128)
        contrib[ok] = c * sg[ok] * x[r[ok]]
        y[np.nonzero(hit)[0]] += contrib
    return d, y


@pytest.mark.parametrize("name", golden_cases("small"))
def test_compiled_terms_reproduce_reference_hv(name):
    g = load_golden(name)
    d, y = emulate_hv(name, g["hv0_v1"])
    np.testing.assert_allclose(d, g["diag"][1:], rtol=0, atol=1e-12)
    ref = g["hv0_v0a"][1:]
    assert np.max(np.abs(y - ref)) <= 1e-12 * np.max(np.abs(ref))
    if "hv3_v1" in g:
        _, y3 = emulate_hv(name, g["hv3_v1"])
        ref3 = g["hv3_v0a"][1:] - g["hv3_v0b"][1:]
        assert np.max(np.abs(y3 - ref3)) <= 1e-11 * np.max(np.abs(g["hv3_v0a"][1:]))


@pytest.mark.parametrize("name", golden_cases("green"))
def test_green_rows_read_as_the_reference_keeps_them(name):
    """Green's function rows after the reader: the rows of the reference's output files (a
    canonical Spin model drops one-body rows with i != j; a multi-body line the reference
    cut to 8 indices starts the row)."""
    from conftest import green_reference
    z = load_golden(name)
    nl = os.path.join(case_dir(name), "namelist.def")
    for f in (str(x) for x in z["green_files"]):
        body = 3 if "ThreeBody" in f else 4 if "FourBody" in f else 6 if "SixBody" in f else 2 if "cktalt" in f else 1
        rows = hphi_b200.inspect_green(nl, body)
        _, _, lines = green_reference(z, f)
        if not lines:
            continue  # a file the reference leaves empty for this model
        assert len(lines) == len(rows)
        for line, r in zip(lines, rows):
            idx = [int(t) for t in line.split()[:-2]]
            assert idx == list(r[:len(idx)]), (f, line, r)


def test_green_reader_warnings_and_rejections(tmp_path, capfd):
    src = case_dir("green_spin10")
    d = tmp_path / "in"
    shutil.copytree(src, d)
    n_file = int(open(d / "greenone.def").read().splitlines()[1].split()[1])
    rows = hphi_b200.inspect_green(str(d / "namelist.def"), 1)
    out = capfd.readouterr().out
    # the reference's warning for every skipped off-site row
    assert out.count("Warning: Site component of (i, j) =(") == n_file - len(rows)
    assert (rows[:, 0] == rows[:, 2]).all()
    # a spin two-body row with i != j is a fatal input error (CheckFormatForSpinInt)
    lines = open(d / "greentwo.def").read().splitlines()
    n = int(lines[1].split()[1])
    lines[1] = f"NCisAjsCktAltDC {n + 1}"
    lines.append("0 0 1 0 1 0 0 0")
    open(d / "greentwo.def", "w").write("\n".join(lines) + "\n")
    with pytest.raises(hphi_b200.HPhiError, match="i=j and k=l must be satisfied"):
        hphi_b200.inspect_green(str(d / "namelist.def"), 2)
    # out-of-range spin index
    lines = open(src + "/greenone.def").read().splitlines()
    lines[5] = "0 2 0 2"
    open(d / "greenone.def", "w").write("\n".join(lines) + "\n")
    with pytest.raises(hphi_b200.HPhiError, match="bad index"):
        hphi_b200.inspect_green(str(d / "namelist.def"), 1)


def test_green_inspect_rejects_unknown_body():
    nl = os.path.join(case_dir("green_multi_spingc8"), "namelist.def")
    for body in (0, 5, 7):
        with pytest.raises(hphi_b200.HPhiError):
            hphi_b200.inspect_green(nl, body)
    assert hphi_b200.inspect_green(nl, 6).shape[1] == 24


def test_time_evolution_inputs_are_checked(tmp_path):
    """TEOneBody / TETwoBody are read for CalcType 4: both at once is an error (as the
    reference's CalcByTEM reports), so is a time-dependent term that leaves a canonical sector;
    a valid TETwoBody file reads."""
    from hphi_b200 import expert
    m = expert.hubbard(4, expert.chain_bonds(4), 1.0, 4.0, 2, 2, calc_type="TimeEvolution", lanczos_max=2,
                       input_eigenvec=1, spectrum_vec="zvo_eigenvec_0")
    m.te_twobody = [(0.0, [(0, 0, 1, 0, 1, 1, 0, 1, 1.0, 0.0), (0, 1, 1, 1, 1, 0, 0, 0, 1.0, 0.0)]), (0.1, [])]
    hphi_b200.inspect_terms(m.write(str(tmp_path / "ok")))
    m.te_onebody = [(0.0, [(0, 0, 1, 0, 1.0, 0.0), (1, 0, 0, 0, 1.0, 0.0)]), (0.1, [])]
    with pytest.raises(hphi_b200.HPhiError, match="TEOneBody and TETwoBody at the same time"):
        hphi_b200.inspect_terms(m.write(str(tmp_path / "both")))
    m.te_twobody = []
    m.te_onebody = [(0.0, [(0, 0, 1, 1, 1.0, 0.0), (1, 1, 0, 0, 1.0, 0.0)]), (0.1, [])]
    with pytest.raises(hphi_b200.HPhiError, match="leaves the sector"):
        hphi_b200.inspect_terms(m.write(str(tmp_path / "flip")))

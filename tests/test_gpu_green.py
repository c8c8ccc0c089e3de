"""Green's functions (expec_cisajs / expec_cisajscktaltdc) on the device, through the C-ABI:
against the oracle on the same vector, against the files the reference wrote for its own
eigenvectors and TPQ states, and as the files the drivers write (same rows, same layout)."""
import os
import shutil

import numpy as np
import pytest

import hphi_b200
import hphi_oracle as O
from conftest import case_dir, golden_cases, green_reference, load_golden, tpq_state

pytestmark = pytest.mark.gpu


def _oracle(name):
    d = O.read_expert(os.path.join(case_dir(name), "namelist.def"))
    return d, (None if O._rows_are_configs(d) else O.sz(d))


def _vector(d, lists, z, fname):
    if "step" in fname:
        return tpq_state(O, d, lists, z["start"], int(fname.split("step")[1].split(".")[0]))
    k = int(fname.split("eigen")[1].split(".")[0]) if "eigen" in fname else 0
    return z[f"vec_zvo_eigenvec_{k}_rank_0.dat"]


def _read_eigvec(path):
    with open(path, "rb") as f:
        f.read(4)
        dim = int(np.frombuffer(f.read(8), dtype=np.int64)[0])
        return np.frombuffer(f.read(16 * (dim + 1)), dtype=np.complex128).copy()


def _same_layout(mine, ref, atol):
    """Line for line: the index columns as printed, the line ending, values within atol."""
    assert len(mine) == len(ref)
    for a, b in zip(mine, ref):
        assert a.rsplit(None, 2)[0] == b.rsplit(None, 2)[0], (a, b)
        assert a.endswith(" ") == b.endswith(" "), (a, b)
        va = complex(float(a.split()[-2]), float(a.split()[-1]))
        vb = complex(float(b.split()[-2]), float(b.split()[-1]))
        assert abs(va - vb) <= atol, (a, b)


@pytest.mark.parametrize("name", golden_cases("green"))
def test_green_kernels_match_oracle_and_reference(name, tmp_path):
    z = load_golden(name)
    d, lists = _oracle(name)
    with hphi_b200.Hamiltonian(os.path.join(case_dir(name), "namelist.def")) as H:
        for f in (str(x) for x in z["green_files"]):
            rows, vals, lines = green_reference(z, f)
            v = _vector(d, lists, z, f)
            multi = {"ThreeBody": 3, "FourBody": 4, "SixBody": 6}
            body = next((n for k, n in multi.items() if k in f), 2 if "cktalt" in f else 1)
            if body >= 3:
                full = d.green_multi[body]
                res = O.expec_multibody(d, v, body)
                got = H.expec_green(v, full, body)
                if res is None:
                    np.testing.assert_array_equal(got, 0)   # the reference leaves the file empty
                    assert lines == []
                    continue
                np.testing.assert_allclose(got, res[0], rtol=0, atol=1e-12, err_msg=f)
                np.testing.assert_allclose(got, vals, rtol=0, atol=1e-10, err_msg=f)
                continue
            if not lines:
                continue
            got = H.expec_green(v, rows, body)
            want = O.expec_cisajscktalt(d, lists, v) if body == 2 else O.expec_cisajs(d, lists, v)
            np.testing.assert_allclose(got, want, rtol=0, atol=1e-12, err_msg=f)
            np.testing.assert_allclose(got, vals, rtol=0, atol=1e-10, err_msg=f)
            # the input's rows through the reference-named entry points, and the file they write
            path = str(tmp_path / f)
            g2 = H.expec_cisajscktaltdc(v, path) if body == 2 else H.expec_cisajs(v, path)
            np.testing.assert_array_equal(g2, got)
            _same_layout(open(path).read().splitlines(), lines, 1e-10)


def _run_case(name, tmp_path, monkeypatch, run):
    monkeypatch.setenv("HPHI_B200_REF_THREADS", "1")
    d = tmp_path / "in"
    shutil.copytree(case_dir(name), d)
    os.remove(d / "golden.npz")
    out = tmp_path / "output"
    with hphi_b200.Hamiltonian(str(d / "namelist.def")) as H:
        run(H, str(out))
    return out


@pytest.mark.parametrize("name", [n for n in golden_cases("green") if "tpq" not in n and "lobpcg" not in n])
def test_lanczos_writes_green_files(name, tmp_path, monkeypatch):
    """calc_by_lanczos with Green's function requests: every file of the reference (same
    names, rows, line layout), equal to the oracle on the eigenvector file the engine wrote
    (1e-10) and to the reference's values for the same input and start vector."""
    from conftest import check_green_lines, oracle_green_file
    z = load_golden(name)
    d, lists = _oracle(name)
    out = _run_case(name, tmp_path, monkeypatch, lambda H, o: H.calc_by_lanczos(output_dir=o))
    v = _read_eigvec(out / "zvo_eigenvec_0_rank_0.dat")
    written = sorted(f for f in os.listdir(out) if "cisajs" in f or "Body" in f)
    assert written == sorted(str(x) for x in z["green_files"])
    for f in written:
        _, _, lines = green_reference(z, f)
        mine = open(out / f).read().splitlines()
        rows, want = oracle_green_file(O, d, lists, v, f)
        check_green_lines(mine, rows, want, 1e-10)
        _same_layout(mine, lines, 1e-6)


def test_tpq_writes_green_files(tmp_path, monkeypatch):
    """calc_by_tpq: zvo_cisajs_set0step{0,4,8}.dat (ExpecInterval 4) from the reference's start
    vector, against the reference's files."""
    name = "green_tpq_hub6"
    z = load_golden(name)
    out = _run_case(name, tmp_path, monkeypatch, lambda H, o: H.calc_by_tpq(output_dir=o))
    written = sorted(f for f in os.listdir(out) if "cisajs" in f)
    assert written == sorted(str(x) for x in z["green_files"])
    for f in written:
        _, _, lines = green_reference(z, f)
        _same_layout(open(out / f).read().splitlines(), lines, 1e-9)


def test_lobpcg_writes_green_files(tmp_path, monkeypatch):
    """calc_by_lobpcg: zvo_cisajs_eigen{k}.dat per state and the eigenvector files
    (OutputEigenVec): each file equals the oracle on the written vector; the ground state's
    (non-degenerate) values equal the reference's."""
    name = "green_lobpcg_chain10"
    z = load_golden(name)
    d, lists = _oracle(name)
    out = _run_case(name, tmp_path, monkeypatch, lambda H, o: H.calc_by_lobpcg(output_dir=o))
    written = sorted(f for f in os.listdir(out) if "cisajs" in f)
    assert written == sorted(str(x) for x in z["green_files"])
    for f in written:
        k = int(f.split("eigen")[1].split(".")[0])
        v = _read_eigvec(out / f"zvo_eigenvec_{k}_rank_0.dat")
        _, got = O.read_green_file(str(out / f))
        two = "cktalt" in f
        want = O.expec_cisajscktalt(d, lists, v) if two else O.expec_cisajs(d, lists, v)
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-10, err_msg=f)
        if k == 0:
            _, _, lines = green_reference(z, f)
            _same_layout(open(out / f).read().splitlines(), lines, 1e-6)


def test_green_on_the_full_size_sector():
    """Size-independent checks on the 8+8-electron 4x4 Hubbard sector: on a normalised random
    vector the densities sum to N (sum_i <n_i up + n_i dn> = 16), every <n_i s> lies in
    [0, 1], and <c+_i c_j> = conj(<c+_j c_i>) (Hermiticity)."""
    from hphi_b200 import expert
    import tempfile
    m = expert.hubbard(16, expert.square_bonds(4, 4), 1.0, 8.0, 8, 8, lanczos_max=1)
    m.greenone = [(i, s, i, s) for i in range(16) for s in (0, 1)] + [(0, 0, 5, 0), (5, 0, 0, 0), (3, 1, 2, 1),
                                                                     (2, 1, 3, 1)]
    with tempfile.TemporaryDirectory() as tmp:
        m.write(tmp)
        with hphi_b200.Hamiltonian(os.path.join(tmp, "namelist.def")) as H:
            rng = np.random.default_rng(5)
            v = np.zeros(H.dim + 1, dtype=np.complex128)
            v[1:] = rng.standard_normal(H.dim)
            v[1:] /= np.linalg.norm(v[1:])
            g = H.expec_cisajs(v)
    dens = g[:32].real
    assert abs(dens.sum() - 16.0) < 1e-9
    assert (dens >= -1e-12).all() and (dens <= 1 + 1e-12).all()
    assert abs(g[32] - np.conj(g[33])) < 1e-12 and abs(g[34] - np.conj(g[35])) < 1e-12


def test_lobpcg_input_eigenvectors(tmp_path, monkeypatch):
    """CalcByLOBPCG with InputEigenVec: the reference's stored states replace the iteration;
    phys() of them gives the reference's energies and, per state, the reference's Green's
    function files (same vectors, so the excited state's files compare too)."""
    name = "green_lobpcg_chain10"
    z = load_golden(name)
    d = tmp_path / "in"
    shutil.copytree(case_dir(name), d)
    os.remove(d / "golden.npz")
    txt = open(d / "calcmod.def").read().replace("OutputEigenVec 1", "InputEigenVec 1")
    open(d / "calcmod.def", "w").write(txt)
    out = tmp_path / "output"
    os.makedirs(out)
    for k in range(2):
        v = z[f"vec_zvo_eigenvec_{k}_rank_0.dat"]
        with open(out / f"zvo_eigenvec_{k}_rank_0.dat", "wb") as f:
            f.write(np.array([0], dtype=np.int32).tobytes())
            f.write(np.array([v.size - 1], dtype=np.int64).tobytes())
            f.write(v.astype(np.complex128).tobytes())
    with hphi_b200.Hamiltonian(str(d / "namelist.def")) as H:
        r = H.calc_by_lobpcg(output_dir=str(out))
    assert r["converged"] and r["steps"] == 0
    assert not (out / "zvo_Lanczos_Step.dat").exists()
    np.testing.assert_allclose(r["energy"], z["states"][:, 0], rtol=0, atol=1e-10)
    for f in (str(x) for x in z["green_files"]):
        _, _, lines = green_reference(z, f)
        _same_layout(open(out / f).read().splitlines(), lines, 1e-10)


def test_canonical_tpq_files_match_reference(tmp_path, monkeypatch):
    """calc_by_tpq with CalcType 5 (cTPQ): SS_rand0.dat, Norm_rand0.dat and Flct_rand0.dat (a
    Flct line at step 0, the inverse temperature growing by 1/LargeValue) and the Green's
    function files of steps 0, 4 and 8, against the reference's run from the same start."""
    name = "green_ctpq_hub6"
    z = load_golden(name)
    out = _run_case(name, tmp_path, monkeypatch, lambda H, o: H.calc_by_tpq(output_dir=o))
    for base in ("SS_rand0", "Norm_rand0", "Flct_rand0"):
        mine = [l for l in open(out / f"{base}.dat").read().splitlines()]
        ref = str(z["text_" + base]).splitlines()
        assert len(mine) == len(ref) and mine[0] == ref[0]
        a = np.array([[float(x) for x in l.split()] for l in mine[1:]])
        b = np.array([[float(x) for x in l.split()] for l in ref[1:]])
        np.testing.assert_allclose(a, b, rtol=1e-10, atol=1e-10, err_msg=base)
    written = sorted(f for f in os.listdir(out) if "cisajs" in f)
    assert written == sorted(str(x) for x in z["green_files"])
    for f in written:
        _, _, lines = green_reference(z, f)
        _same_layout(open(out / f).read().splitlines(), lines, 1e-9)

"""Lanczos restart (ReStart 1 / 3) against the reference's own restart runs: the files the
engine writes after an unconverged run (TMComponents with the printed coefficients,
recalcvec with v0 and v1) equal the reference's, and a run continued from the reference's
files converges to the reference's continued energy."""
import os
import shutil

import numpy as np
import pytest

import hphi_b200
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

CASE = os.path.join(GOLDEN, "restart_chain14")


def _copy_inputs(sub, dst):
    os.makedirs(dst, exist_ok=True)
    for f in os.listdir(os.path.join(CASE, sub)):
        shutil.copy(os.path.join(CASE, sub, f), dst)
    return os.path.join(dst, "namelist.def")


def _write_reference_files(z, outdir):
    os.makedirs(outdir, exist_ok=True)
    with open(os.path.join(outdir, "zvo_TMComponents.dat"), "w") as f:
        f.write("%d \n" % int(z["tm_steps"]))
        f.write("%.10f \n" % float(z["tm_dnorm"]))
        for a, b in zip(z["tm_alpha"], z["tm_beta"]):
            f.write("%.10f %.10f \n" % (a, b))
    with open(os.path.join(outdir, "zvo_recalcvec_rank_0.dat"), "wb") as f:
        f.write(np.array([int(z["rv_step"]), z["rv_v0"].size - 1], dtype=np.int64).tobytes())
        f.write(z["rv_v0"].astype(np.complex128).tobytes())
        f.write(z["rv_v1"].astype(np.complex128).tobytes())


def test_restart_files_match_reference(tmp_path, monkeypatch):
    monkeypatch.setenv("HPHI_B200_REF_THREADS", "1")
    z = np.load(os.path.join(CASE, "restart.npz"))
    out = tmp_path / "output"
    with hphi_b200.Hamiltonian(_copy_inputs("a", str(tmp_path / "a"))) as H:
        r = H.calc_by_lanczos(output_dir=str(out))
    assert not r["converged"] and r["steps"] == int(z["tm_steps"])
    lines = open(out / "zvo_TMComponents.dat").read().splitlines()
    assert int(lines[0].split()[0]) == int(z["tm_steps"])
    assert lines[1].strip() == "0.0000000000"
    ab = np.array([[float(x) for x in l.split()] for l in lines[2:]])
    np.testing.assert_allclose(ab[:, 0], z["tm_alpha"], rtol=0, atol=2e-10)
    np.testing.assert_allclose(ab[:, 1], z["tm_beta"], rtol=0, atol=2e-10)
    with open(out / "zvo_recalcvec_rank_0.dat", "rb") as f:
        stp, dim = np.frombuffer(f.read(16), dtype=np.int64)
        v = np.frombuffer(f.read(), dtype=np.complex128)
    assert stp == int(z["rv_step"]) and dim == z["rv_v0"].size - 1
    np.testing.assert_allclose(v[1:dim + 1], z["rv_v0"][1:], rtol=0, atol=1e-10)
    np.testing.assert_allclose(v[dim + 2:], z["rv_v1"][dim + 2 - (dim + 1):], rtol=0, atol=1e-10)
    assert not (out / "zvo_energy.dat").exists()


def test_continue_from_reference_files(tmp_path, monkeypatch):
    monkeypatch.setenv("HPHI_B200_REF_THREADS", "1")
    z = np.load(os.path.join(CASE, "restart.npz"))
    out = tmp_path / "output"
    _write_reference_files(z, str(out))
    with hphi_b200.Hamiltonian(_copy_inputs("b", str(tmp_path / "b"))) as H:
        r = H.calc_by_lanczos(output_dir=str(out))
    assert r["converged"]
    assert abs(r["steps"] - int(z["b_steps"][-1])) <= 1
    assert abs(r["e1"] - z["b_step_vals"][-1][0]) < 1.5e-10
    ref = z["b_energy_state"]
    assert abs(r["energy"] - ref[0]) < 1e-10 * max(1.0, abs(ref[0]))
    # the continued run appends its step lines after the restored ones
    lines = open(out / "zvo_Lanczos_Step.dat").read().splitlines()
    assert lines[0].startswith("stp=21 ") or lines[0].startswith("stp=22 ")


def test_restart_chain_equals_reference(tmp_path, monkeypatch):
    """The engine's own files: stop after 20 steps, continue, same energy as the reference's
    restarted run."""
    monkeypatch.setenv("HPHI_B200_REF_THREADS", "1")
    z = np.load(os.path.join(CASE, "restart.npz"))
    out = tmp_path / "output"
    with hphi_b200.Hamiltonian(_copy_inputs("a", str(tmp_path / "a"))) as H:
        H.calc_by_lanczos(output_dir=str(out))
    with hphi_b200.Hamiltonian(_copy_inputs("b", str(tmp_path / "b"))) as H:
        r = H.calc_by_lanczos(output_dir=str(out))
    assert r["converged"]
    assert abs(r["energy"] - z["b_energy_state"][0]) < 1e-9


TPQ_CASE = os.path.join(GOLDEN, "tpqrestart_hub6")


def _rows(text):
    return np.array([[float(x) for x in l.split()] for l in text.splitlines() if l.strip() and "#" not in l])


def _tpq_inputs(sub, dst):
    os.makedirs(dst, exist_ok=True)
    for f in os.listdir(os.path.join(TPQ_CASE, sub)):
        shutil.copy(os.path.join(TPQ_CASE, sub, f), dst)
    return os.path.join(dst, "namelist.def")


def test_tpq_restart_vectors_match_reference(tmp_path, monkeypatch):
    """ReStart 1: the stored states tmpvec_set%d_rank_0.dat (step, dim, normalised state) and
    the sample files equal the reference's for both samples."""
    monkeypatch.setenv("HPHI_B200_REF_THREADS", "1")
    z = np.load(os.path.join(TPQ_CASE, "restart.npz"))
    out = tmp_path / "output"
    with hphi_b200.Hamiltonian(_tpq_inputs("a", str(tmp_path / "a"))) as H:
        H.calc_by_tpq(output_dir=str(out))
    for r in range(2):
        with open(out / f"tmpvec_set{r}_rank_0.dat", "rb") as f:
            stp = int(np.frombuffer(f.read(4), dtype=np.int32)[0])
            dim = int(np.frombuffer(f.read(8), dtype=np.int64)[0])
            v = np.frombuffer(f.read(), dtype=np.complex128)
        assert stp == int(z[f"a_step{r}"]) and v.size == dim + 1
        np.testing.assert_allclose(v[1:], z[f"a_vec{r}"][1:], rtol=0, atol=1e-10)
        for base in ("SS_rand", "Norm_rand", "Flct_rand"):
            np.testing.assert_allclose(_rows(open(out / f"{base}{r}.dat").read()), _rows(str(z[f"a_{base}{r}"])),
                                       rtol=1e-10, atol=1e-10)


def test_tpq_continues_from_reference_state(tmp_path, monkeypatch):
    """ReStart 3 from the reference's stored states and files: the appended lines (steps
    12..24, global_1st_norm printed as 0) equal the reference's continued run."""
    monkeypatch.setenv("HPHI_B200_REF_THREADS", "1")
    z = np.load(os.path.join(TPQ_CASE, "restart.npz"))
    out = tmp_path / "output"
    os.makedirs(out)
    for r in range(2):
        for base in ("SS_rand", "Norm_rand", "Flct_rand"):
            open(out / f"{base}{r}.dat", "w").write(str(z[f"a_{base}{r}"]))
        with open(out / f"tmpvec_set{r}_rank_0.dat", "wb") as f:
            f.write(np.array([int(z[f"a_step{r}"])], dtype=np.int32).tobytes())
            f.write(np.array([z[f"a_vec{r}"].size - 1], dtype=np.int64).tobytes())
            f.write(z[f"a_vec{r}"].astype(np.complex128).tobytes())
    with hphi_b200.Hamiltonian(_tpq_inputs("b", str(tmp_path / "b"))) as H:
        H.calc_by_tpq(output_dir=str(out))
    for r in range(2):
        for base in ("SS_rand", "Norm_rand", "Flct_rand"):
            mine, ref = _rows(open(out / f"{base}{r}.dat").read()), _rows(str(z[f"b_{base}{r}"]))
            assert mine.shape == ref.shape
            np.testing.assert_allclose(mine, ref, rtol=1e-10, atol=1e-10)


LOBPCG_CASE = os.path.join(GOLDEN, "lobpcgrestart_chain12")


def _lobpcg_inputs(sub, dst):
    os.makedirs(dst, exist_ok=True)
    for f in os.listdir(os.path.join(LOBPCG_CASE, sub)):
        shutil.copy(os.path.join(LOBPCG_CASE, sub, f), dst)
    return os.path.join(dst, "namelist.def")


def _lobpcg_step_rows(path):
    rows = []
    for line in open(path):
        p = line.split()
        if p and p[0].isdigit():
            rows.append([float(x) for x in p])
    return np.array(rows)


def test_lobpcg_restart_vectors_match_reference(tmp_path, monkeypatch):
    """ReStart 1, unconverged after Lanczos_max steps: no error, no energy file, the step
    rows, and tmpvec_set%d_rank_0.dat per state (X->Large.itr = Lanczos_max + 1) spanning the
    reference's vectors."""
    monkeypatch.setenv("HPHI_B200_REF_THREADS", "1")
    z = np.load(os.path.join(LOBPCG_CASE, "restart.npz"))
    out = tmp_path / "output"
    with hphi_b200.Hamiltonian(_lobpcg_inputs("a", str(tmp_path / "a"))) as H:
        r = H.calc_by_lobpcg(output_dir=str(out))
    assert not r["converged"]
    assert not (out / "zvo_energy.dat").exists() and not bool(z["a_energy_exists"])
    np.testing.assert_allclose(_lobpcg_step_rows(out / "zvo_Lanczos_Step.dat"), z["a_steps"], rtol=2e-5, atol=0)
    mine, ref = [], []
    for ie in range(2):
        with open(out / f"tmpvec_set{ie}_rank_0.dat", "rb") as f:
            itr = int(np.frombuffer(f.read(4), dtype=np.int32)[0])
            dim = int(np.frombuffer(f.read(8), dtype=np.int64)[0])
            v = np.frombuffer(f.read(), dtype=np.complex128)
        assert itr == int(z[f"a_itr{ie}"]) and v.size == dim + 1
        mine.append(v[1:])
        ref.append(z[f"a_vec{ie}"][1:])
    # same two-dimensional subspace (the Ritz vectors are fixed up to phases)
    q_m, _ = np.linalg.qr(np.array(mine).T)
    q_r, _ = np.linalg.qr(np.array(ref).T)
    s = np.linalg.svd(q_m.conj().T @ q_r, compute_uv=False)
    assert np.all(s > 1 - 1e-9), s


def test_lobpcg_continues_from_reference_vectors(tmp_path, monkeypatch):
    """ReStart 3 from the reference's stored vectors: the step rows and the energies of the
    reference's continued run."""
    monkeypatch.setenv("HPHI_B200_REF_THREADS", "1")
    z = np.load(os.path.join(LOBPCG_CASE, "restart.npz"))
    out = tmp_path / "output"
    os.makedirs(out)
    for ie in range(2):
        with open(out / f"tmpvec_set{ie}_rank_0.dat", "wb") as f:
            f.write(np.array([int(z[f"a_itr{ie}"])], dtype=np.int32).tobytes())
            f.write(np.array([z[f"a_vec{ie}"].size - 1], dtype=np.int64).tobytes())
            f.write(z[f"a_vec{ie}"].astype(np.complex128).tobytes())
    with hphi_b200.Hamiltonian(_lobpcg_inputs("b", str(tmp_path / "b"))) as H:
        r = H.calc_by_lobpcg(output_dir=str(out))
    assert r["converged"]
    np.testing.assert_allclose(r["energy"], z["b_states"][:, 0], rtol=0, atol=1e-10)
    mine, ref = _lobpcg_step_rows(out / "zvo_Lanczos_Step.dat"), z["b_steps"]
    n = min(len(mine), len(ref))
    assert abs(len(mine) - len(ref)) <= 1
    np.testing.assert_allclose(mine[:n, 1:], ref[:n, 1:], rtol=2e-5, atol=0)


@pytest.mark.parametrize("mode", [1, 2])
def test_lanczos_input_eigenvector(mode, tmp_path, monkeypatch):
    """InputEigenVec 1 / 2: the reference's stored eigenvector replaces the Lanczos run (mode 2
    takes H v / |H v|); the Green's function files equal the reference's for that vector, and
    zvo_energy.dat prints Energy and Doublon as 0 (not computed on this path) with Sz."""
    from conftest import case_dir, green_reference, load_golden
    name = "green_hub6"
    z = load_golden(name)
    d = tmp_path / "in"
    shutil.copytree(case_dir(name), d)
    os.remove(d / "golden.npz")
    txt = open(d / "calcmod.def").read().replace("OutputEigenVec 1", f"InputEigenVec {mode}")
    open(d / "calcmod.def", "w").write(txt)
    out = tmp_path / "output"
    os.makedirs(out)
    v = z["vec_zvo_eigenvec_0_rank_0.dat"]
    with open(out / "zvo_eigenvec_0_rank_0.dat", "wb") as f:
        f.write(np.array([0], dtype=np.int32).tobytes())
        f.write(np.array([v.size - 1], dtype=np.int64).tobytes())
        f.write(v.astype(np.complex128).tobytes())
    with hphi_b200.Hamiltonian(str(d / "namelist.def")) as H:
        H.calc_by_lanczos(output_dir=str(out))
    assert not (out / "zvo_Lanczos_Step.dat").exists()
    e = open(out / "zvo_energy.dat").read().splitlines()
    assert e[0] == "Energy  0.0000000000000000 " and e[1] == "Doublon  0.0000000000000000 "
    assert abs(float(e[2].split()[1])) < 1e-12
    for f in (str(x) for x in z["green_files"]):
        _, vals, _ = green_reference(z, f)
        got = np.array([complex(float(l.split()[-2]), float(l.split()[-1])) for l in open(out / f)])
        np.testing.assert_allclose(got, vals, rtol=0, atol=1e-10 if mode == 1 else 1e-8, err_msg=f)

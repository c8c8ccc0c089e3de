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

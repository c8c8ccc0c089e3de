"""LOBPCG (CalcType 3) on the GPU against the reference's own runs: same number of steps,
the step file's residuals and eigenvalue estimates to its printed precision, converged
energies to 1e-10 and HPhi's output files."""
import os

import numpy as np
import pytest

import hphi_b200
from conftest import case_dir, golden_cases, load_golden

pytestmark = pytest.mark.gpu


def _steps_file(path):
    rows = []
    with open(path) as f:
        for line in f:
            p = line.split()
            if p and p[0].isdigit():
                rows.append([float(x) for x in p])
    return np.array(rows)


@pytest.mark.parametrize("name", golden_cases("lobpcg"))
def test_lobpcg_matches_reference(name, tmp_path, monkeypatch):
    # the reference's own start vectors: single-element ones (initial_iv > 0 on canonical
    # models) or its random ones drawn with one OpenMP thread, as the fixtures were made
    monkeypatch.setenv("HPHI_B200_REF_THREADS", "1")
    g = load_golden(name)
    ref_steps, ref_states = g["lobpcg_steps"], g["lobpcg_states"]
    with hphi_b200.Hamiltonian(os.path.join(case_dir(name), "namelist.def")) as H:
        r = H.calc_by_lobpcg(output_dir=str(tmp_path))
    assert r["converged"]
    assert abs(r["steps"] - ref_steps.shape[0]) <= 1, (r["steps"], ref_steps.shape[0])
    np.testing.assert_allclose(r["energy"], ref_states[:, 0], rtol=0, atol=1e-10)
    np.testing.assert_allclose(r["doublon"], ref_states[:, 1], rtol=0, atol=1e-6)
    np.testing.assert_allclose(r["sz"], ref_states[:, 2], rtol=0, atol=1e-6)
    mine = _steps_file(tmp_path / "zvo_Lanczos_Step.dat")
    n = min(10, mine.shape[0], ref_steps.shape[0])
    np.testing.assert_allclose(mine[:n, 1:], ref_steps[:n, 1:], rtol=2e-5, atol=0)
    text = (tmp_path / "zvo_energy.dat").read_text()
    assert text.startswith("State 0\n  Energy  ")
    assert text.count("State ") == ref_states.shape[0]

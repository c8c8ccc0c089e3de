"""The reference's own known-answer tests (test/*.sh; standard-mode inputs written here in
expert mode, tests/golden/known_answers/make_known_answers.py) through the engine's drivers:
the energies and ground-state doublons those tests check."""
import json
import os
import shutil

import numpy as np
import pytest

import hphi_b200
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

BASE = os.path.join(GOLDEN, "known_answers")
EXPECTED = json.load(open(os.path.join(BASE, "expected.json")))


@pytest.mark.parametrize("name", sorted(EXPECTED))
def test_engine_reproduces_reference_test_values(name, tmp_path, monkeypatch):
    monkeypatch.setenv("HPHI_B200_REF_THREADS", "1")
    d = tmp_path / "in"
    shutil.copytree(os.path.join(BASE, name), d)
    want = np.array(EXPECTED[name])
    with hphi_b200.Hamiltonian(str(d / "namelist.def")) as H:
        if name.startswith("lobcg"):
            r = H.calc_by_lobpcg(output_dir=str(tmp_path / "output"))
            energy, doublon = np.array(r["energy"]), np.array(r["doublon"])
        else:
            r = H.calc_by_lanczos(output_dir=str(tmp_path / "output"))
            assert r["converged"]
            energy, doublon = np.array([r["energy"]]), np.array([r["doublon"]])
    np.testing.assert_allclose(energy, want[:, 0], rtol=0, atol=1e-9)
    assert abs(doublon[0] - want[0, 1]) < 1e-8

"""The oracle's restatement of the real-time evolution (CalcByTEM) against the reference:
its own known-answer tables (test/te_hubbard_chain_interall*.sh, 100 steps from the chain's
ground state) and the files the reference wrote for the te_* golden inputs from a seeded start
(time-dependent TEOneBody / TETwoBody terms, ExpandCoef 0 / 4 / 6 / 10, a repeated time)."""
import json
import os

import numpy as np
import pytest

import hphi_oracle as O
from conftest import GOLDEN, case_dir, golden_cases, load_golden

KNOWN = os.path.join(GOLDEN, "known_answers")


def table(text):
    return np.array([[float(x) for x in l.split()] for l in str(text).splitlines()[1:]])


def ground_state(d, lists):
    """The lowest eigenvector of the static Hamiltonian (dense; the sector is small)."""
    static = O.Def(**{k: getattr(d, k) for k in d.__dataclass_fields__})
    static.te_kind = 0
    H = O.dense_hamiltonian(static, lists, O.diagonalcalc(static, lists))
    w, V = np.linalg.eigh(H)
    assert w[1] - w[0] > 1e-6
    v = np.zeros(len(w) + 1, dtype=np.complex128)
    v[1:] = V[:, 0]
    return v


@pytest.mark.parametrize("name", ["te_hubbard_chain_interall", "te_hubbard_chain_interall_diagonal"])
def test_oracle_te_known_answers(name):
    expected = np.array(json.load(open(os.path.join(KNOWN, "te_expected.json")))[name])
    d = O.read_expert(os.path.join(KNOWN, name, "namelist.def"))
    lists = O.sz(d)
    rows, _ = O.te_run(d, lists, ground_state(d, lists))
    got = np.array(rows)[:, [0, 6, 7, 4, 5, 8, 9, 10]]   # Flct columns
    assert got.shape == expected.shape
    np.testing.assert_allclose(got, expected, rtol=0, atol=1e-10)


@pytest.mark.parametrize("name", golden_cases("te"))
def test_oracle_te_matches_reference(name):
    z = load_golden(name)
    d = O.read_expert(os.path.join(case_dir(name), "namelist.def"))
    lists = None if O._rows_are_configs(d) else O.sz(d)
    green_steps = [s for s in range(d.lanczos_max) if d.green_one and s % d.expec_interval == 0]
    rows, states = O.te_run(d, lists, z["start"], keep_states=green_steps)
    r = np.array(rows)
    ss, norm, flct = table(z["text_SS"]), table(z["text_Norm"]), table(z["text_Flct"])
    np.testing.assert_allclose(r[:, [0, 1, 2, 4, 6, 10]], ss, rtol=0, atol=1e-10)
    np.testing.assert_allclose(r[:, [0, 3, 10]], norm, rtol=0, atol=1e-10)
    np.testing.assert_allclose(r[:, [0, 6, 7, 4, 5, 8, 9, 10]], flct, rtol=0, atol=1e-10)
    for s in green_steps:
        f = f"zvo_cisajs_step{s}.dat"
        path = os.path.join(str(os.environ.get("TMPDIR", "/tmp")), f"{name}_{f}")
        open(path, "w").write(str(z["text_" + f]))
        _, want = O.read_green_file(path)
        os.remove(path)
        np.testing.assert_allclose(O.expec_cisajs(d, lists, states[s]), want, rtol=0, atol=1e-10, err_msg=f)

"""The reference's random start vectors (one dSFMT-19937 generator per OpenMP thread over
its static-schedule rows) against the first mltply input of the reference's own runs: one
thread for every golden case that starts from a random vector, 3 and 4 threads for the
refstart fixtures.  Host code only."""
import os

import numpy as np
import pytest

import hphi_b200
import hphi_oracle as O
from conftest import GOLDEN, case_dir, golden_cases, load_golden

KIND = {0: hphi_b200.REF_LANCZOS, 1: hphi_b200.REF_TPQ, 3: hphi_b200.REF_LOBPCG}


def _random_start(d):
    """SetInitialVector / Initialize_wave take a single element for canonical S=1/2-type
    models with initial_iv > 0 (src/CalcByLanczos.c:66-93), a random vector otherwise."""
    return O._is_gc(d) or O._general(d) or d.initial_iv <= 0 or d.calc_type == 1


def _reproduce(d, dim, threads):
    kind = KIND[d.calc_type]
    v = hphi_b200.reference_start(dim, kind, d.initial_iv, 0, d.initial_vec_type, threads,
                                  max(1, d.k_exct) if kind == hphi_b200.REF_LOBPCG else 1)[0]
    if kind == hphi_b200.REF_TPQ:   # the TPQ vector is returned before its normalisation
        v[1:] /= np.sqrt(np.sum(np.abs(v[1:]) ** 2))
    return v


@pytest.mark.parametrize("name", golden_cases("small"))
def test_start_vector_matches_reference_one_thread(name):
    g = load_golden(name)
    d = O.read_expert(os.path.join(case_dir(name), "namelist.def"))
    if not _random_start(d):
        pytest.skip("single-element start")
    v = _reproduce(d, g["hv0_v1"].size - 1, 1)
    assert np.max(np.abs(v[1:] - g["hv0_v1"][1:])) < 1e-15


STARTS = sorted(n for n in os.listdir(GOLDEN) if os.path.exists(os.path.join(GOLDEN, n, "start.npz")))


@pytest.mark.parametrize("name", STARTS)
def test_start_vector_matches_reference_several_threads(name):
    z = np.load(os.path.join(GOLDEN, name, "start.npz"))
    d = O.read_expert(os.path.join(case_dir(str(z["source"])), "namelist.def"))
    v = _reproduce(d, z["v1"].size - 1, int(z["threads"]))
    assert np.max(np.abs(v[1:] - z["v1"][1:])) < 1e-15
    # another thread count gives another vector
    w = _reproduce(d, z["v1"].size - 1, 1)
    assert np.max(np.abs(w[1:] - z["v1"][1:])) > 1e-3


def test_static_schedule_and_generator_basics():
    # every row is drawn exactly once, in [-1, 1)
    v = hphi_b200.reference_start(1001, hphi_b200.REF_TPQ, -7, 2, 1, 5)[0]
    assert np.all(np.abs(v[1:].real) <= 1.0) and np.all(v[1:].imag == 0) and np.all(v[1:] != 0)
    g = hphi_b200.reference_start(1001, hphi_b200.REF_TPQ, -7, 2, -1, 5)[0]   # Gaussian pairs
    assert abs(np.mean(np.abs(g[1:]) ** 2) - 2.0) < 0.3
    with pytest.raises(hphi_b200.HPhiError):
        hphi_b200.reference_start(0)

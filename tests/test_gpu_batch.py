"""Batched Lanczos engine: every instance of a batch against the plain single-instance
driver on the same start vector and step count, FP32 storage with FP64 refinement
against FP64, graph and non-graph runs, and the autotuner's choice."""
import numpy as np
import pytest

import hphi_b200
from hphi_b200 import expert

pytestmark = pytest.mark.gpu
STEPS = 64


def _complex_hubbard_chain(L):
    m = expert.hubbard(L, expert.chain_bonds(L), 1.0, 4.0, L // 2, L // 2)
    m.trans = []
    for i, j in expert.chain_bonds(L):
        for s in (0, 1):
            m.trans += [(i, s, j, s, 0.8, 0.3), (j, s, i, s, 0.8, -0.3)]
    return m


MODELS = [
    ("heis12", lambda: expert.heisenberg(12, expert.chain_bonds(12), 1.0)),
    ("j1j2_14", lambda: expert.j1j2_chain(14, 1.0, 0.4)),
    ("hub6", lambda: expert.hubbard(6, expert.chain_bonds(6), 1.0, 6.0, 3, 3)),
    ("heis6_small", lambda: expert.heisenberg(6, expert.chain_bonds(6), 1.0)),   # dim 20 < steps
    ("hub6_complex", lambda: _complex_hubbard_chain(6)),
    ("kh_gc", lambda: expert.kitaev_heisenberg(2, 2, -1.0, 0.2, initial_vec_type=0)),
]


@pytest.fixture(scope="module")
def hams(tmp_path_factory):
    hs = []
    for name, make in MODELS:
        d = tmp_path_factory.mktemp(name)
        hs.append(hphi_b200.Hamiltonian(make().write(str(d))))
    yield hs
    for h in hs:
        h.close()


def test_batch_fp64_matches_plain_driver(hams):
    seed = 11
    with hphi_b200.Batch(hams, hphi_b200.FP64) as b:
        r = b.lanczos(STEPS, seed=seed, graph=True)
    for i, h in enumerate(hams):
        steps = min(STEPS, h.dim)
        e_plain = h.lanczos_steps(STEPS, seed=seed + 1000003 * i, nev=1)[0]
        assert r["steps"][i] <= steps
        assert abs(r["e_lanczos"][i] - e_plain) < 1e-10 * max(1.0, abs(e_plain)), (MODELS[i][0], r["e_lanczos"][i],
                                                                                    e_plain)


def test_batch_graph_equals_direct_launches(hams):
    with hphi_b200.Batch(hams, hphi_b200.FP64) as b:
        g = b.lanczos(STEPS, seed=5, graph=True)
        d = b.lanczos(STEPS, seed=5, graph=False)
    assert np.array_equal(g["e_lanczos"], d["e_lanczos"])
    assert np.array_equal(g["steps"], d["steps"])


def test_batch_fp32_refined_energy_within_1e8_of_fp64(hams):
    with hphi_b200.Batch(hams, hphi_b200.FP64) as b64:
        r64 = b64.lanczos(STEPS, seed=3, refine=True)
    with hphi_b200.Batch(hams, hphi_b200.FP32) as b32:
        r32 = b32.lanczos(STEPS, seed=3, refine=True)
    for i, (name, _) in enumerate(MODELS):
        # the FP64 refinement agrees with the FP64 tridiagonal eigenvalue
        assert abs(r64["e_refined"][i] - r64["e_lanczos"][i]) < 1e-9, name
        assert r64["residual"][i] < 1e-4, name
        # FP32 storage: raw Ritz value only to FP32 accuracy, refined energy to 1e-8
        assert abs(r32["e_lanczos"][i] - r64["e_lanczos"][i]) < 1e-4, name
        assert abs(r32["e_refined"][i] - r64["e_lanczos"][i]) < 1e-8, (name, r32["e_refined"][i], r64["e_lanczos"][i])
        assert 1 <= r32["replay_steps"][i] <= r32["steps"][i]


def test_batch_tuning_shape(hams):
    with hphi_b200.Batch(hams[:3], hphi_b200.FP64) as b:
        t = b.tuning()
        assert t["threads"] in (128, 256, 512)
        assert t["rows_per_thread"] in (1, 2, 4, 8)
        assert t["threads"] * t["ctas_per_sm"] <= 2048
        r1 = b.lanczos(20, seed=1)
        t2 = b.tuning(retune=True)
        assert t2["threads"] in (128, 256, 512)
        r2 = b.lanczos(20, seed=1)
    # a different launch shape gives the same eigenvalues to rounding
    assert np.allclose(r1["e_lanczos"], r2["e_lanczos"], rtol=0, atol=1e-11)

"""GPU parity against the reference (golden fixtures made by the reference HPhi) and
against the oracle: lists bit-exact, H*v to 1e-12 relative, Lanczos ground-state
energy to 1e-10, TPQ energies to 1e-10 relative - all through the C-ABI."""
import hashlib
import os
import re
import shutil

import numpy as np
import pytest

import hphi_b200
from conftest import case_dir, golden_cases, load_golden
from test_oracle_golden import check_lanczos_against_reference

pytestmark = pytest.mark.gpu

HV_RTOL = 1e-12      # FP64 H*v, relative to max |v_out|
E_TOL = 1e-10        # eigenvalues / TPQ energies


def open_case(name):
    return hphi_b200.Hamiltonian(os.path.join(case_dir(name), "namelist.def"))


@pytest.mark.parametrize("name", golden_cases("small"))
def test_lists_and_diagonal_match_reference(name):
    g = load_golden(name)
    with open_case(name) as H:
        assert H.dim == g["diag"].size - 1
        if "list_1" in g:
            l1, l21, l22 = H.sz()
            assert np.array_equal(l1, g["list_1"])
            assert np.array_equal(l21, g["list_2_1"])
            assert np.array_equal(l22, g["list_2_2"])
        else:
            with pytest.raises(hphi_b200.HPhiError):
                H.sz()
        np.testing.assert_allclose(H.diagonalcalc(), g["diag"], rtol=0, atol=1e-13)


@pytest.mark.parametrize("name", golden_cases("small"))
def test_mltply_matches_reference(name):
    g = load_golden(name)
    with open_case(name) as H:
        v0 = np.zeros_like(g["hv0_v1"])
        pr = H.mltply(v0, g["hv0_v1"])
        ref = g["hv0_v0a"]
        assert np.max(np.abs(v0 - ref)) <= HV_RTOL * np.max(np.abs(ref))
        assert abs(pr - complex(g["hv0_pr"])) <= HV_RTOL * max(1.0, abs(complex(g["hv0_pr"])))
        if "hv3_v1" in g:  # accumulate into a non-zero v0 (reference's v0 += H v1)
            v0 = g["hv3_v0b"].copy()
            pr = H.mltply(v0, g["hv3_v1"])
            ref = g["hv3_v0a"]
            assert np.max(np.abs(v0 - ref)) <= HV_RTOL * np.max(np.abs(ref))
            assert abs(pr - complex(g["hv3_pr"])) <= 1e-11 * max(1.0, abs(complex(g["hv3_pr"])))


@pytest.mark.parametrize("name", golden_cases("small"))
def test_mltply_device_real_and_complex(name):
    """The device entry point with real FP64 vectors (real Hamiltonians) and complex128."""
    torch = pytest.importorskip("torch")
    g = load_golden(name)
    with open_case(name) as H:
        v1 = g["hv0_v1"][1:]
        ref = g["hv0_v0a"][1:]
        d1 = torch.tensor(v1, device="cuda")
        d0 = torch.full_like(d1, 7.0)  # must be ignored: acc = 0
        H.mltply_device(d0.data_ptr(), d1.data_ptr(), hphi_b200.COMPLEX128, acc=0.0, scale=1.0)
        out = d0.cpu().numpy()
        assert np.max(np.abs(out - ref)) <= HV_RTOL * np.max(np.abs(ref))
        if H.info["vec_type"] == hphi_b200.REAL64 or (np.all(v1.imag == 0) and H.info["n_offdiag"] >= 0
                                                      and np.all(np.isreal(ref))):
            r1 = torch.tensor(v1.real.copy(), device="cuda")
            r0 = torch.zeros_like(r1)
            try:
                H.mltply_device(r0.data_ptr(), r1.data_ptr(), hphi_b200.REAL64, acc=0.0, scale=1.0)
            except hphi_b200.HPhiError as e:
                assert "complex" in str(e)
                return
            assert np.max(np.abs(r0.cpu().numpy() - ref.real)) <= HV_RTOL * np.max(np.abs(ref))


@pytest.mark.parametrize("name", golden_cases("lanczos"))
def test_lanczos_matches_reference(name, tmp_path):
    g = load_golden(name)
    with open_case(name) as H:
        r = H.calc_by_lanczos(v_init=g["hv0_v1"], output_dir=str(tmp_path))
        assert r["converged"]
        alpha, beta = H.lanczos_tridiagonal()
        check_lanczos_against_reference(g, r["e1"], alpha, beta)
        lines = open(tmp_path / "zvo_Lanczos_Step.dat").read().splitlines()
        assert lines[0].startswith("LanczosStep  E[1] E[2] E[3] E[4] Target:E[")
        assert re.match(r"stp = 2 -?\d+\.\d{10} -?\d+\.\d{10} ", lines[1])
        assert re.match(r"stp=3 (-?\d+\.\d{10} ){4}", lines[2])
        assert len(lines) - 1 == r["steps"] - 1


@pytest.mark.parametrize("name", ["chain16", "hubchain8_complex", "kitaev2x2", "gspin1_chain8", "hubgc4"])
def test_lanczos_default_start_matches_reference(name, tmp_path, monkeypatch):
    """Without an injected vector the driver draws the reference's own random start (one
    OpenMP thread, as the fixtures were made), so the run reproduces the reference's."""
    monkeypatch.setenv("HPHI_B200_REF_THREADS", "1")
    g = load_golden(name)
    with open_case(name) as H:
        r = H.calc_by_lanczos(output_dir=str(tmp_path))
        assert r["converged"]
        alpha, beta = H.lanczos_tridiagonal()
        check_lanczos_against_reference(g, r["e1"], alpha, beta)


@pytest.mark.parametrize("name", golden_cases("tpq"))
def test_tpq_default_start_matches_reference(name, tmp_path, monkeypatch):
    monkeypatch.setenv("HPHI_B200_REF_THREADS", "1")
    g = load_golden(name)
    ref = g["tpq"]
    with open_case(name) as H:
        e = H.calc_by_tpq(output_dir=str(tmp_path), nresult=ref.shape[0])
    np.testing.assert_allclose(e, ref[:, 1], rtol=E_TOL, atol=1e-12)


@pytest.mark.parametrize("name", ["chain16", "hub2x4", "kitaev2x2", "hub6_allterms"])
def test_lanczos_eigenvector_energy_and_variance(name, tmp_path):
    g = load_golden(name)
    src = case_dir(name)
    for f in os.listdir(src):
        if f.endswith(".def"):
            shutil.copy(os.path.join(src, f), tmp_path)
    cm = open(tmp_path / "calcmod.def").read().replace("CalcEigenVec -1", "CalcEigenVec 0")
    open(tmp_path / "calcmod.def", "w").write(cm)
    with hphi_b200.Hamiltonian(str(tmp_path / "namelist.def")) as H:
        r = H.calc_by_lanczos(v_init=g["hv0_v1"], output_dir=str(tmp_path / "output"))
        e0 = g["step_vals"][-1][0]
        assert abs(r["energy"] - e0) < 1e-9
        assert abs(r["var"] - r["energy"] ** 2) < 1e-7 * max(1.0, r["energy"] ** 2)
        v = H.lanczos_eigenvector()
        assert abs(np.vdot(v[1:], v[1:]).real - 1.0) < 1e-12
        text = open(tmp_path / "output" / "zvo_energy.dat").read()
        assert re.match(r"Energy  -?\d+\.\d{16} \nDoublon  -?\d+\.\d{16} \nSz  -?\d+\.\d{16} \n", text)


@pytest.mark.parametrize("name", golden_cases("eigenvector"))
def test_lanczos_cg_refinement_matches_reference(name, tmp_path):
    """CalcEigenVec 0 with a Lanczos run stopped early: the accuracy check fails as in the
    reference and the CG refinement gives the reference's Energy / Doublon / Sz."""
    g = load_golden(name)
    ref = g["energy_state"]
    with open_case(name) as H:
        r = H.calc_by_lanczos(v_init=g["hv0_v1"], output_dir=str(tmp_path))
        assert r["converged"]
        assert (r["cg_rounds"] > 0) == bool(g["cg_ran"])
        if g["cg_ran"]:
            assert r["check_var"] >= 1e-12 or r["check_diff"] >= 1e-12
            assert r["cg_var"] < 1e-12 and r["cg_iterations"] >= r["cg_rounds"]
        assert abs(r["energy"] - ref[0]) < E_TOL * max(1.0, abs(ref[0]))
        assert abs(r["doublon"] - ref[1]) < 1e-9
        assert abs(r["sz"] - ref[2]) < 1e-9
        v = H.lanczos_eigenvector()
        assert abs(np.vdot(v[1:], v[1:]).real - 1.0) < 1e-12
    vals = [float(l.split()[1]) for l in open(tmp_path / "zvo_energy.dat")]
    np.testing.assert_allclose(vals, ref, rtol=0, atol=1e-9)


@pytest.mark.parametrize("name", golden_cases("tpq"))
def test_tpq_energies_match_reference(name, tmp_path):
    g = load_golden(name)
    ref = g["tpq"]
    with open_case(name) as H:
        e = H.calc_by_tpq(v_init=[g["hv0_v1"]], output_dir=str(tmp_path), nresult=ref.shape[0])
    np.testing.assert_allclose(e, ref[:, 1], rtol=E_TOL, atol=1e-12)
    rows = np.array([[float(x) for x in l.split()] for l in open(tmp_path / "SS_rand0.dat") if not l.lstrip().startswith("#")])
    assert rows.shape == ref.shape
    np.testing.assert_allclose(rows[:, 0], ref[:, 0], rtol=1e-9, atol=1e-12)   # inverse temperature
    np.testing.assert_allclose(rows[:, 1:5], ref[:, 1:5], rtol=1e-9, atol=1e-10)
    np.testing.assert_array_equal(rows[:, 5], ref[:, 5])


@pytest.mark.parametrize("name", golden_cases("large"))
def test_full_size_lists_bit_exact(name):
    """Full-size sectors (e.g. the half-filled 4x4 Hubbard, dim 165,636,900): SHA-256 of
    list_1 / list_2_1 / list_2_2 equals that of the reference's own sz()."""
    g = load_golden(name)
    with open_case(name) as H:
        assert H.dim == int(g["dim"])
        l1, l21, l22 = H.sz()
        assert l21.size == int(g["n21"]) and l22.size == int(g["n22"])
        for a, key in ((l1, "sha_list_1"), (l21, "sha_list_2_1"), (l22, "sha_list_2_2")):
            assert hashlib.sha256(a.tobytes()).hexdigest() == str(g[key])
        # structural properties: strictly increasing configurations, inverse map
        c = l1[1:]
        assert np.all(c[1:] > c[:-1])

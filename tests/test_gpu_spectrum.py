"""Dynamical Green's functions (CalcSpec 1, Lanczos) against the reference: each fixture of
tests/golden/spectrum_* holds the reference's spectrum run (its inputs, the ground state it
started from and its zvo_DynamicalGreen.dat / zvo_TMComponents.dat, written by
tests/golden/make_spectrum_golden.py).  The engine reads the same input vector, applies the same
excitation operators (Heisenberg S^z-type projectors, a spin flip into the Sz = 1 sector, the
removal of an up electron from a half-filled Hubbard chain, a Hubbard pair excitation with
a 1 - n term, the creation of a down electron in a grand-canonical cluster) and must give the
same excited-state norm, the same leading Lanczos components and the same Green's function at
the printed precision."""
import os
import shutil

import numpy as np
import pytest

import hphi_b200

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(d[len("spectrum_"):] for d in os.listdir(GOLDEN) if d.startswith("spectrum_"))


def _stage(name, tmp_path):
    src = os.path.join(GOLDEN, "spectrum_" + name)
    ind = tmp_path / "in"
    out = tmp_path / "out"
    ind.mkdir()
    out.mkdir()
    for f in os.listdir(src):
        if f.endswith(".def"):
            shutil.copy(os.path.join(src, f), ind / f)
    shutil.copy(os.path.join(src, "zvo_eigenvec_0_rank_0.dat"), out / "zvo_eigenvec_0_rank_0.dat")
    return src, str(ind / "namelist.def"), str(out)


def _tm(path):
    t = open(path).read().split()
    return int(t[0]), float(t[1]), np.array(t[2:], dtype=float).reshape(-1, 2)


@pytest.mark.parametrize("via_run", [False, True])
@pytest.mark.parametrize("name", CASES)
def test_spectrum_matches_reference(name, via_run, tmp_path):
    src, nl, out = _stage(name, tmp_path)
    ref_g = np.loadtxt(os.path.join(src, "ref_DynamicalGreen.dat"))
    with hphi_b200.Hamiltonian(nl) as H:
        if via_run:
            H.run(out)
        else:
            res = H.calc_spectrum(output_dir=out, n_omega=len(ref_g))
            assert res.shape == (len(ref_g), 2)
            np.testing.assert_allclose(res[:, 1].real, ref_g[:, 2], rtol=0, atol=2e-8 * np.abs(ref_g[:, 2:]).max())
    g = np.loadtxt(os.path.join(out, "zvo_DynamicalGreen.dat"))
    assert g.shape == ref_g.shape
    np.testing.assert_allclose(g[:, :2], ref_g[:, :2], rtol=0, atol=1e-10)   # the frequency grid
    scale = np.abs(ref_g[:, 2:]).max()
    assert np.abs(g[:, 2:] - ref_g[:, 2:]).max() <= 2e-8 * scale, np.abs(g[:, 2:] - ref_g[:, 2:]).max()
    L, dn, ab = _tm(os.path.join(out, "zvo_TMComponents.dat"))
    Lr, dnr, abr = _tm(os.path.join(src, "ref_TMComponents.dat"))
    assert L == Lr
    assert abs(dn - dnr) <= 1e-9
    # the leading components at the printed precision: once the recurrence has lost
    # orthogonality (after ~8 steps on the 256-state grand-canonical cluster) rounding
    # differences grow from step to step in both codes
    np.testing.assert_allclose(ab[:6], abr[:6], rtol=0, atol=2e-9)

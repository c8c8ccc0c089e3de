"""The drop-in patch, compiled: the reference HPhi with its mltply replaced at link time by
the engine's hphi_mltply (oracle/_ref/HPhi_ref_b200, built by `make -C oracle shim` from the
reference's sources and oracle/shim_b200.c).  Every other step -- CalcByLanczos, the Lanczos
recurrence and its convergence test, the eigenvector replay, expec_energy_flct, the output
files -- is the reference's own code, so its zvo_Lanczos_Step.dat and zvo_energy.dat must equal
those of the plain reference run on the same input with the same OpenMP thread count (same
random start vector).  Match: src/mltply.c:56, src/CalcByLanczos.c:55."""
import os
import shutil
import subprocess

import pytest

from conftest import GOLDEN
from hphi_b200 import expert
import run_ref

pytestmark = pytest.mark.gpu

SHIM = os.path.join(os.path.dirname(run_ref.REF_BIN), "HPhi_ref_b200")
THREADS = 4


def _input(name, dst):
    if name == "hubbard3x4_4e":
        # product-layout plan with the two-pass kernels for real vectors
        expert.hubbard(12, expert.square_bonds(3, 4), 1.0, 8.0, 4, 4).write(dst)
    else:
        shutil.copytree(os.path.join(GOLDEN, name), dst)
        os.remove(os.path.join(dst, "golden.npz"))
    p = os.path.join(dst, "calcmod.def")
    lines = [("CalcEigenVec 0" if l.startswith("CalcEigenVec") else l) for l in open(p).read().splitlines()]
    open(p, "w").write("\n".join(lines) + "\n")


def _run(binary, workdir):
    env = dict(os.environ, OMP_NUM_THREADS=str(THREADS), OMP_PROC_BIND="close")
    return subprocess.run([binary, "-e", "namelist.def"], cwd=workdir, env=env, capture_output=True, text=True,
                          timeout=900)


def _steps(path):
    out = []
    for line in open(path):
        if line.startswith("stp"):
            head, rest = line.split("=", 1)
            tok = rest.split()
            out.append((int(tok[0]), [None if "x" in t else float(t) for t in tok[1:]]))
    return out


def _energy(path):
    return {l.split()[0]: float(l.split()[1]) for l in open(path) if l.strip()}


@pytest.mark.parametrize("name", ["chain16", "hub2x4", "hubbard3x4_4e"])
def test_reference_with_engine_mltply_matches_reference(name, tmp_path):
    if not (run_ref.available() and os.path.exists(SHIM)):
        pytest.skip("oracle/_ref/HPhi_ref and HPhi_ref_b200 are not built (make -C oracle ref shim)")
    ref_dir, shim_dir = str(tmp_path / "ref"), str(tmp_path / "shim")
    _input(name, ref_dir)
    _input(name, shim_dir)
    pr = _run(run_ref.REF_BIN, ref_dir)
    ps = _run(SHIM, shim_dir)
    assert pr.returncode == 0, pr.stdout[-1500:] + pr.stderr[-1500:]
    assert ps.returncode == 0, ps.stdout[-1500:] + ps.stderr[-1500:]
    ref = _steps(os.path.join(ref_dir, "output", "zvo_Lanczos_Step.dat"))
    got = _steps(os.path.join(shim_dir, "output", "zvo_Lanczos_Step.dat"))
    # LanczosEps 14 stops on a relative change of 1e-14; rounding of the H*v may move the stop
    # by one step, so the common steps are compared
    assert abs(len(ref) - len(got)) <= 1, (len(ref), len(got))
    for (sr, vr), (sg, vg) in zip(ref, got):
        assert sr == sg
        for a, b in zip(vr, vg):
            assert (a is None) == (b is None)
            if a is not None:
                assert abs(a - b) <= 1.5e-10, (sr, vr, vg)
    er = _energy(os.path.join(ref_dir, "output", "zvo_energy.dat"))
    eg = _energy(os.path.join(shim_dir, "output", "zvo_energy.dat"))
    assert set(er) == set(eg) == {"Energy", "Doublon", "Sz"}
    for k in er:
        assert abs(er[k] - eg[k]) <= 1e-10, (k, er[k], eg[k])

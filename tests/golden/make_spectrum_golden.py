"""Generates the dynamical Green's function fixtures tests/golden/spectrum_*/ by running the
reference HPhi (oracle/_ref/HPhi_ref) twice per case:

  1. a Lanczos run with OutputEigenVec 1, which writes the ground state
     output/zvo_eigenvec_0_rank_0.dat;
  2. a spectrum run (CalcSpec 1, SpectrumVec zvo_eigenvec_0) with the case's SingleExcitation /
     PairExcitation operators and frequency grid, which writes output/zvo_DynamicalGreen.dat and
     output/zvo_TMComponents.dat.

Each fixture directory holds the spectrum run's input files, the input vector
(zvo_eigenvec_0_rank_0.dat) and the reference's two output files (ref_DynamicalGreen.dat,
ref_TMComponents.dat).  The sectors are small (dimension below Lanczos_max), so the
reference's tridiagonal components stay inside its arrays.

Run in a container that has oracle/_ref/HPhi_ref (`make -C oracle`):
    python tests/golden/make_spectrum_golden.py [case ...]
"""
from __future__ import annotations

import copy
import os
import shutil
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from hphi_b200 import expert  # noqa: E402
import run_ref  # noqa: E402


def _cases():
    c = {}
    # S^z-like pair excitation on a Heisenberg chain (same sector): n_up at sites 0 and 1 with phases
    m = expert.heisenberg(10, expert.chain_bonds(10), lanczos_max=500)
    c["spin_sz_chain10"] = (m, dict(pair_excitation=[(0, 1, 0, 1, 1, 0.5, 0.0), (1, 1, 1, 1, 1, -0.5, 0.0),
                                                     (2, 0, 2, 0, 0, 0.25, 0.1)],
                                    omega_min=-8.0, omega_max=4.0, omega_im=0.1, n_omega=60))
    # spin flip |up><down| at site 3 (Sz = 0 -> 1 sector)
    m = expert.j1j2_chain(10, 1.0, 0.3, lanczos_max=500)
    c["spin_flip_j1j2_10"] = (m, dict(pair_excitation=[(3, 1, 3, 0, 1, 1.0, 0.0)],
                                      omega_min=-7.0, omega_max=3.0, omega_im=0.05, n_omega=50))
    # removal of an up electron from a half-filled Hubbard chain (N -> N-1 sector)
    m = expert.hubbard(6, expert.chain_bonds(6), 1.0, 4.0, 3, 3, lanczos_max=500)
    c["hub_single_chain6"] = (m, dict(single_excitation=[(0, 0, 0, 1.0, 0.0), (1, 0, 0, -1.0, 0.0)],
                                      omega_min=-6.0, omega_max=6.0, omega_im=0.1, n_omega=48))
    # a pair excitation c+_{0 up} c_{2 up} + c_{1 dn} c+_{1 dn} on a Hubbard chain (same sector)
    m = expert.hubbard(6, expert.chain_bonds(6), 1.0, 4.0, 3, 3, lanczos_max=500)
    c["hub_pair_chain6"] = (m, dict(pair_excitation=[(0, 0, 2, 0, 1, 0.7, 0.2), (1, 1, 1, 1, 0, 0.4, 0.0)],
                                    omega_min=-5.0, omega_max=8.0, omega_im=0.1, n_omega=52))
    # creation of a down electron on a grand-canonical Hubbard cluster (chemical potential)
    m = expert.hubbard(4, expert.square_bonds(2, 2), 1.0, 3.0, 2, 2, lanczos_max=500)
    m.model, m.two_sz, m.nup, m.ndown, m.ncond = "HubbardGC", None, None, None, None
    m.trans += [(i, s, i, s, 1.2, 0.0) for i in range(4) for s in (0, 1)]
    c["hubgc_single_2x2"] = (m, dict(single_excitation=[(2, 1, 1, 1.0, 0.0)],
                                     omega_min=-4.0, omega_max=6.0, omega_im=0.1, n_omega=40))
    # removal of an up electron from a Hubbard chain with the particle number only (HubbardNConserved)
    m = expert.hubbard(6, expert.chain_bonds(6), 1.0, 4.0, 3, 3, lanczos_max=500)
    m.two_sz = None
    c["hubnc_single_chain6"] = (m, dict(single_excitation=[(0, 0, 0, 1.0, 0.0), (3, 1, 0, 0.5, 0.2)],
                                        omega_min=-6.0, omega_max=6.0, omega_im=0.1, n_omega=36))
    return c


def make(name, model, spec):
    out = os.path.join(HERE, f"spectrum_{name}")
    work = tempfile.mkdtemp()
    try:
        gs = copy.deepcopy(model)
        gs.output_eigenvec = 1
        gs.calc_eigenvec = 0
        gs.write(work)
        p = run_ref.run(work, threads=4, timeout=600)
        vec = os.path.join(work, "output", "zvo_eigenvec_0_rank_0.dat")
        if not os.path.exists(vec):
            raise RuntimeError(p.stdout[-2000:] + p.stderr[-2000:])
        sp = copy.deepcopy(model)
        sp.calc_spec = 1
        sp.spectrum_vec = "zvo_eigenvec_0"
        for k, v in spec.items():
            setattr(sp, k, v)
        for f in os.listdir(work):
            if f.endswith(".def"):
                os.remove(os.path.join(work, f))
        sp.write(work)
        p = run_ref.run(work, threads=4, timeout=600)
        green = os.path.join(work, "output", "zvo_DynamicalGreen.dat")
        if not os.path.exists(green):
            raise RuntimeError(p.stdout[-2000:] + p.stderr[-2000:])
        if os.path.isdir(out):
            shutil.rmtree(out)
        os.makedirs(out)
        sp.write(out)
        shutil.copy(vec, os.path.join(out, "zvo_eigenvec_0_rank_0.dat"))
        shutil.copy(green, os.path.join(out, "ref_DynamicalGreen.dat"))
        shutil.copy(os.path.join(work, "output", "zvo_TMComponents.dat"), os.path.join(out, "ref_TMComponents.dat"))
        print(name, "ok")
    finally:
        shutil.rmtree(work, ignore_errors=True)


if __name__ == "__main__":
    cases = _cases()
    for n in (sys.argv[1:] or list(cases)):
        make(n, *cases[n])

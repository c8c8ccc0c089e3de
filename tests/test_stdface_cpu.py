"""Standard-mode generator (hphi_stdface, `HPhi_b200 -s / -sdry`) on the CPU.

The reference's own standard-mode test scripts (test/*.sh, replayed from
tests/golden/stdface/) are run with this generator writing the expert-mode files and the
reference binary (oracle/_ref/HPhi_ref, when it has been built) reading them: their energies,
site-resolved correlation functions, TPQ averages and full-diagonalisation spectra must come
out as the scripts expect.  This pins the generator itself (lattice geometry, site numbering,
bond directions, Hamiltonian conventions, correlation lists) independently of the engine.
"""
import os

import pytest

import hphi_b200
import stdface_runner as R

GENERATOR_CASES = [n for n in R.names() if not n.startswith("te_")]


def _stan_inputs(name):
    return [s for s in R.load(name)["steps"] if s["op"] == "write" and s["file"].endswith(".in")]


@pytest.mark.parametrize("name", GENERATOR_CASES)
def test_generator_writes_expert_files(name, tmp_path):
    st = _stan_inputs(name)[0]
    (tmp_path / st["file"]).write_text(st["text"])
    nl = hphi_b200.standard_mode(str(tmp_path / st["file"]), str(tmp_path))
    listed = [l.split() for l in open(nl) if l.strip()]
    assert {"ModPara", "CalcMod", "LocSpin"} <= {k for k, _ in listed}
    for _, f in listed:
        assert os.path.exists(tmp_path / f), f
    counts = hphi_b200.inspect_terms(nl)
    assert counts is not None


def test_generator_rejects_unknown_and_conflicting_keywords(tmp_path):
    p = tmp_path / "stan.in"
    p.write_text('L = 4\nmodel = "Spin"\nmethod = "Lanczos"\nlattice = "chain"\nJ = 1.0\n2Sz = 0\nJay = 2\n')
    with pytest.raises(hphi_b200.HPhiError, match="jay"):
        hphi_b200.standard_mode(str(p), str(tmp_path))
    p.write_text('L = 4\nW = 2\na0w = 2\nmodel = "Spin"\nmethod = "Lanczos"\nlattice = "square"\nJ = 1.0\n2Sz = 0\n')
    with pytest.raises(hphi_b200.HPhiError, match="not both"):
        hphi_b200.standard_mode(str(p), str(tmp_path))
    p.write_text('L = 4\nmodel = "Spin"\nmethod = "Lanczos"\nlattice = "chain"\nJ = 1.0\nJ0 = 2.0\n2Sz = 0\n')
    with pytest.raises(hphi_b200.HPhiError, match="not both"):
        hphi_b200.standard_mode(str(p), str(tmp_path))
    p.write_text('L = 4\nmodel = "Hubbard"\nmethod = "Lanczos"\nlattice = "chain"\nt = 1.0\n')
    with pytest.raises(hphi_b200.HPhiError, match="nelec"):
        hphi_b200.standard_mode(str(p), str(tmp_path))


def test_cell_enumeration_and_bond_folding(tmp_path):
    """a0 = (3, 0), a1 = (-1, 2) on the triangular lattice: 6 sites, 3 bonds per site of each
    neighbour order; the default LargeValue is the coefficient sum over Nsite."""
    p = tmp_path / "stan.in"
    p.write_text('a0w = 3\na0l = 0\na1w = -1\na1l = 2\nmodel = "HubbardGC"\nmethod = "Lanczos"\n'
                 'lattice = "Triangular"\nt = 1.0\nU = 4.0\nh = 3.0\n')
    hphi_b200.standard_mode(str(p), str(tmp_path))
    rows = [l.split() for l in open(tmp_path / "trans.def").read().split("\n")[5:] if l.strip()]
    hops = [r for r in rows if r[0] != r[2]]
    # sites x directions x (both ways) x spins; on this cluster some site pairs are joined
    # along two directions, and their entries are summed
    assert sum(abs(complex(float(r[4]), float(r[5]))) for r in hops) == pytest.approx(6 * 3 * 2 * 2)
    mod = dict(l.split()[:2] for l in open(tmp_path / "modpara.def") if len(l.split()) >= 2)
    assert int(mod["Nsite"]) == 6
    # |t| per hop entry (72) + |U| per site (24) + |h / 2| per orbital (18), over 6 sites
    assert abs(float(mod["LargeValue"]) - 114.0 / 6) < 1e-12


@pytest.mark.skipif(not os.path.exists(R.REF_EXE), reason="reference binary oracle/_ref/HPhi_ref not built")
@pytest.mark.parametrize("name", GENERATOR_CASES)
def test_reference_reproduces_its_test_values_from_generated_inputs(name, tmp_path):
    problems = R.run(name, str(tmp_path / name), backend="reference", env={"OMP_NUM_THREADS": "4"})
    assert not problems, problems


@pytest.mark.skipif(not os.path.exists(R.REF_EXE), reason="reference binary oracle/_ref/HPhi_ref not built")
def test_reference_reproduces_time_evolution_tests_from_generated_inputs(tmp_path):
    """te_ac_hubbard_square computes the ground state the other three scripts start from."""
    for name in ("te_ac_hubbard_square", "te_dc_hubbard_square", "te_pulse_hubbard_square",
                 "te_quench_hubbard_square"):
        problems = R.run(name, str(tmp_path / name), backend="reference", env={"OMP_NUM_THREADS": "4"})
        assert not problems, (name, problems)

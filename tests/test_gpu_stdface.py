"""The reference's standard-mode test scripts (test/*.sh, replayed from tests/golden/stdface/)
end to end on the engine: `HPhi_b200 -s stan.in` (the standard-mode generator, then the
engine's drivers on the GPU) must print what each script checks, by the script's own
criteria: energies, one- and two-body correlation functions, multi-body Green's functions and
dynamical Green's functions and time-evolution observables summed |difference| < 5e-7 per
block, restarted runs, and TPQ averages within twice the reference's error bars.  The reference computes the spectra of these
scripts (method CG) by shifted BiCG; the engine's Lanczos continued fraction of the same
Green's function matches them to the printed digits.  Full diagonalisation is outside the
engine (its scripts pin the generator on the CPU, tests/test_stdface_cpu.py)."""
import pytest

import stdface_runner as R

pytestmark = pytest.mark.gpu

ENGINE_CASES = [n for n in R.names() if not n.startswith(("fulldiag_", "te_"))]


@pytest.mark.parametrize("name", ENGINE_CASES)
def test_engine_reproduces_standard_mode_test(name, tmp_path):
    problems = R.run(name, str(tmp_path / name), backend="engine")
    assert not problems, problems


def test_engine_reproduces_standard_mode_time_evolution(tmp_path):
    """Quench, pulse, AC and DC lasers on the 3x3 Hubbard cluster: the ground state of
    te_ac_hubbard_square is the initial state of the other three scripts."""
    for name in ("te_ac_hubbard_square", "te_dc_hubbard_square", "te_pulse_hubbard_square",
                 "te_quench_hubbard_square"):
        problems = R.run(name, str(tmp_path / name), backend="engine")
        assert not problems, (name, problems)

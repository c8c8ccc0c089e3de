"""The kernels of the headline workload pinned directly to the reference.

Real vectors on a canonical Hubbard sector whose hops all have one magnitude take the
product-layout two-pass kernels (info["kernel"] == 3).  These tests run the reference itself
(oracle/_ref/HPhi_ref, built from the reference's sources) at test time on sectors where that
plan is selected, and compare:

- a 3x4 periodic Hubbard sector (dim 853,776): one accumulating mltply call of the
  reference's Lanczos (v0 += H v1, src/mltply.c:56-132, with a Lanczos vector as v1 and the
  recurrence's -beta v_prev in v0) against hphi_mltply (complex128 host vectors in HPhi's
  layout, split into two real H*v) and hphi_mltply_device with REAL64 vectors, to 1e-12;
- the half-filled 4x4 periodic Hubbard sector of the headline workload (dim 165,636,900):
  the first Lanczos steps from the reference's deterministic single-element start
  (initial_iv > 0, src/Lanczos_EigenValue.c:499-611), whose zvo_Lanczos_Step.dat lines (Ritz
  values printed to 10 decimals, src/Lanczos_EigenValue.c:202-258) must equal the engine's.
"""
import os

import numpy as np
import pytest

import hphi_b200
from hphi_b200 import expert
import run_ref

pytestmark = pytest.mark.gpu

HV_RTOL = 1e-12


def _ref_threads():
    return max(1, min(os.cpu_count() or 1, 32))


def _need_reference():
    if not run_ref.available():
        pytest.skip("oracle/_ref/HPhi_ref is not built (make -C oracle)")


def _step_lines(path):
    """(step, [printed values]) of each step line; "xxx" placeholders become None."""
    out = []
    with open(path) as f:
        for line in f:
            if not line.startswith("stp"):
                continue
            head, rest = line.split("=", 1)
            tok = rest.split()
            out.append((int(tok[0]), [None if "x" in t else float(t) for t in tok[1:]]))
    return out


def test_two_pass_kernel_accumulating_call_matches_reference(tmp_path):
    _need_reference()
    m = expert.hubbard(12, expert.square_bonds(3, 4), 1.0, 8.0, 6, 6, lanczos_max=5, initial_iv=-1)
    ref_dir = str(tmp_path / "ref")
    m.write(ref_dir)
    p = run_ref.run(ref_dir, threads=_ref_threads(), dump_call=3, timeout=600,
                    extra_env={"HPHI_DUMP_LISTS": "0"})
    assert os.path.exists(os.path.join(ref_dir, "hv.bin")), p.stdout[-2000:] + p.stderr[-2000:]
    v1, v0b, v0a, pr_ref = run_ref.read_hv(ref_dir)
    assert np.max(np.abs(v0b[1:])) > 0  # the call accumulates into a non-zero v0
    H = hphi_b200.Hamiltonian(m.write(str(tmp_path / "eng")))
    try:
        assert H.info["kernel"] == 3  # product layout, two-pass kernels for real vectors
        # HPhi-layout complex128 host vectors (split into real and imaginary H*v)
        v0 = v0b.copy()
        pr = H.mltply(v0, v1)
        err = np.max(np.abs(v0 - v0a)) / np.max(np.abs(v0a))
        assert err <= HV_RTOL, err
        assert abs(pr - pr_ref) <= HV_RTOL * max(1.0, abs(pr_ref)), (pr, pr_ref)
        # device entry point with REAL64 vectors in HPhi order
        torch = pytest.importorskip("torch")
        assert np.all(v1.imag == 0) and np.all(v0b.imag == 0)
        d1 = torch.tensor(v1[1:].real.copy(), device="cuda")
        d0 = torch.tensor(v0b[1:].real.copy(), device="cuda")
        pr = H.mltply_device(d0.data_ptr(), d1.data_ptr(), hphi_b200.REAL64, acc=1.0, scale=1.0)
        out = d0.cpu().numpy()
        err = np.max(np.abs(out - v0a[1:].real)) / np.max(np.abs(v0a[1:]))
        assert err <= HV_RTOL, err
        assert abs(pr - pr_ref) <= HV_RTOL * max(1.0, abs(pr_ref)), (pr, pr_ref)
    finally:
        H.close()


def test_headline_sector_lanczos_steps_match_reference(tmp_path):
    """First Lanczos steps on the 4x4 half-filled sector (the bench workload), both codes from
    the single-element start; the run stops unconverged at Lanczos_max, as the reference's
    does (CalcByLanczos then exits with -3, the engine returns its error)."""
    _need_reference()
    steps = 6
    m = expert.hubbard(16, expert.square_bonds(4, 4), 1.0, 8.0, 8, 8, lanczos_max=steps, initial_iv=1)
    ref_dir = str(tmp_path / "ref")
    m.write(ref_dir)
    p = run_ref.run(ref_dir, threads=_ref_threads(), dump_call=-1, timeout=1800,
                    extra_env={"HPHI_DUMP_LISTS": "0"})
    ref_file = os.path.join(ref_dir, "output", "zvo_Lanczos_Step.dat")
    assert os.path.exists(ref_file), p.stdout[-2000:] + p.stderr[-2000:]
    ref = _step_lines(ref_file)
    assert len(ref) == steps - 1  # stp = 2 .. Lanczos_max
    out = tmp_path / "eng_out"
    with hphi_b200.Hamiltonian(m.write(str(tmp_path / "eng"))) as H:
        assert H.dim == 165636900 and H.info["kernel"] == 3
        with pytest.raises(hphi_b200.HPhiError, match="not converged"):
            H.calc_by_lanczos(output_dir=str(out))
    got = _step_lines(str(out / "zvo_Lanczos_Step.dat"))
    assert [g[0] for g in got] == [r[0] for r in ref]
    for (stp, gv), (_, rv) in zip(got, ref):
        assert [x is None for x in gv] == [x is None for x in rv], (stp, gv, rv)
        for a, b in zip(gv, rv):
            if a is not None:
                assert abs(a - b) <= 1.5e-10, (stp, gv, rv)

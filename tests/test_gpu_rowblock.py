"""Row-block kernels of spin models (row pass over blocks staged in shared memory + column
pass over whole blocks) against the general row kernel (pinned to the reference by
test_gpu_parity), on canonical and grand-canonical sectors, real and complex vectors."""
import os

import numpy as np
import pytest

import hphi_b200
from hphi_b200 import expert

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _open(path, general, simple=False):
    """general: the general row kernel; otherwise the row-block plan (HPHI_B200_KERNEL=rowblock),
    with simple: without its fast row pass (HPHI_B200_RB_SIMPLE), which real vectors of
    Heisenberg-like sectors take by default."""
    saved = {k: os.environ.get(k) for k in ("HPHI_B200_KERNEL", "HPHI_B200_RB_SIMPLE")}
    os.environ.pop("HPHI_B200_KERNEL", None)
    os.environ.pop("HPHI_B200_RB_SIMPLE", None)
    # the plan is built by default from 2^24 rows up; these sectors are smaller
    os.environ["HPHI_B200_KERNEL"] = "general" if general else "rowblock"
    if simple:
        os.environ["HPHI_B200_RB_SIMPLE"] = "1"
    try:
        return hphi_b200.Hamiltonian(path)
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _xxz_field(L):
    m = expert.heisenberg(L, expert.chain_bonds(L), 1.0)
    m.exchange += [(i, (i + 2) % L, 0.3) for i in range(L)]
    return m


MODELS = {
    "chain16": lambda: expert.heisenberg(16, expert.chain_bonds(16)),
    "chain15_sz1": lambda: expert.heisenberg(15, expert.chain_bonds(15), two_sz=1),
    "j1j2_20": lambda: expert.j1j2_chain(20, 1.0, 0.45),
    "square4x4": lambda: expert.heisenberg(16, expert.square_bonds(4, 4)),
    "square4x6": lambda: expert.heisenberg(24, expert.square_bonds(4, 6)),
    "xxz_chain18": lambda: _xxz_field(18),
    "kitaev2x3_gc": lambda: expert.kitaev_heisenberg(2, 3, -1.0, 0.2),
    "kitaev3x4_gc": lambda: expert.kitaev_heisenberg(3, 4, -1.0, 0.25),
}


@pytest.mark.parametrize("simple", [False, True])
@pytest.mark.parametrize("name", list(MODELS))
def test_rowblock_matches_general_kernel(name, simple, tmp_path):
    m = MODELS[name]()
    path = m.write(str(tmp_path))
    Hr = _open(path, general=False, simple=simple)
    Hg = _open(path, general=True)
    try:
        assert Hr.info["kernel"] == 4
        assert Hg.info["kernel"] == 0
        dim = Hr.dim
        g = torch.Generator(device="cuda").manual_seed(3)
        vts = [hphi_b200.REAL64, hphi_b200.COMPLEX128]
        for vt in vts:
            dt = torch.float64 if vt == hphi_b200.REAL64 else torch.complex128
            v1 = (torch.rand(dim, dtype=dt, device="cuda", generator=g) - 0.5)
            v0 = (torch.rand(dim, dtype=dt, device="cuda", generator=g) - 0.5)
            for acc, scale in ((1.0, 1.0), (0.0, 1.0), (0.5, -2.0)):
                yr, yg = v0.clone(), v0.clone()
                torch.cuda.synchronize()  # the engine's stream does not wait for torch's
                pr = Hr.mltply_device(yr.data_ptr(), v1.data_ptr(), vt, acc=acc, scale=scale)
                pg = Hg.mltply_device(yg.data_ptr(), v1.data_ptr(), vt, acc=acc, scale=scale)
                err = (yr - yg).abs().max().item() / max(yg.abs().max().item(), 1e-300)
                assert err < 1e-12, (vt, acc, scale, err)
                assert abs(complex(pr) - complex(pg)) <= 1e-12 * max(1.0, abs(complex(pg))), (pr, pg)
    finally:
        Hr.close()
        Hg.close()


def test_rowblock_lanczos_energy_matches_general(tmp_path):
    """4x6 Heisenberg (dim 2,704,156): the Lanczos ground state through the row-block
    kernels equals the general kernel's (same start vector)."""
    path = MODELS["square4x6"]().write(str(tmp_path))
    out = []
    for general, simple in ((False, False), (False, True), (True, False)):
        H = _open(path, general, simple)
        out.append(H.lanczos_steps(120, seed=5, nev=1)[0])
        H.close()
    assert abs(out[0] - out[2]) < 1e-10 * abs(out[2])
    assert abs(out[1] - out[2]) < 1e-10 * abs(out[2])


# ---------------------------------------------------------------- pinned to the reference
import sys  # noqa: E402

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import run_ref  # noqa: E402

REF_CASES = {
    # fast row pass (one magnitude on every lower-half term)
    "square4x4": lambda: expert.heisenberg(16, expert.square_bonds(4, 4), lanczos_max=5, initial_iv=-1),
    # generic row pass (J1 and J2 lower-half terms)
    "j1j2_18": lambda: expert.j1j2_chain(18, 1.0, 0.4, lanczos_max=5, initial_iv=-1),
    # grand-canonical rows (SpinGC): exchange and pair-lift terms
    "kitaev2x3_gc": lambda: expert.kitaev_heisenberg(2, 3, -1.0, 0.2, lanczos_max=5, initial_iv=-1),
}


@pytest.mark.parametrize("name", list(REF_CASES))
def test_rowblock_accumulating_call_matches_reference(name, tmp_path):
    """One accumulating mltply call of the reference's own Lanczos (v0 += H v1,
    src/mltply.c:56-132; oracle/_ref/HPhi_ref run at test time) against the row-block kernels:
    hphi_mltply on HPhi-layout complex128 host vectors and hphi_mltply_device on real and
    complex device vectors, to 1e-12."""
    if not run_ref.available():
        pytest.skip("oracle/_ref/HPhi_ref is not built (make -C oracle)")
    m = REF_CASES[name]()
    ref_dir = str(tmp_path / "ref")
    m.write(ref_dir)
    p = run_ref.run(ref_dir, threads=4, dump_call=3, timeout=600, extra_env={"HPHI_DUMP_LISTS": "0"})
    assert os.path.exists(os.path.join(ref_dir, "hv.bin")), p.stdout[-2000:] + p.stderr[-2000:]
    v1, v0b, v0a, pr_ref = run_ref.read_hv(ref_dir)
    H = _open(m.write(str(tmp_path / "eng")), general=False)
    try:
        assert H.info["kernel"] == 4
        v0 = v0b.copy()
        pr = H.mltply(v0, v1)
        scale = np.max(np.abs(v0a))
        assert np.max(np.abs(v0 - v0a)) <= 1e-12 * scale
        assert abs(pr - pr_ref) <= 1e-12 * max(1.0, abs(pr_ref))
        vts = [hphi_b200.COMPLEX128]
        if np.all(v1.imag == 0) and np.all(v0b.imag == 0):
            vts.append(hphi_b200.REAL64)
        for vt in vts:
            if vt == hphi_b200.REAL64:
                d1 = torch.tensor(v1[1:].real.copy(), device="cuda")
                d0 = torch.tensor(v0b[1:].real.copy(), device="cuda")
            else:
                d1 = torch.tensor(v1[1:].copy(), device="cuda")
                d0 = torch.tensor(v0b[1:].copy(), device="cuda")
            torch.cuda.synchronize()
            prd = H.mltply_device(d0.data_ptr(), d1.data_ptr(), vt, acc=1.0, scale=1.0)
            out = d0.cpu().numpy()
            assert np.max(np.abs(out - v0a[1:])) <= 1e-12 * scale, vt
            assert abs(prd - pr_ref) <= 1e-12 * max(1.0, abs(pr_ref)), (vt, prd, pr_ref)
    finally:
        H.close()

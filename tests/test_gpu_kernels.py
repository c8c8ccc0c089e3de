"""The specialised Hubbard block kernel against the general kernel (both on the GPU,
the general one pinned to the reference by test_gpu_parity), native-order round trips,
and full-size H*v properties."""
import os

import numpy as np
import pytest

import hphi_b200
from hphi_b200 import expert

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _open(path, general=False, kernel=None):
    """kernel: None (default plan: product layout where it applies, two-pass kernels for real
    vectors), "single" (product layout, one-pass kernel), "block" or "general"."""
    saved = {k: os.environ.get(k) for k in ("HPHI_B200_KERNEL", "HPHI_B200_PROD")}
    if general:
        kernel = "general"
    os.environ.pop("HPHI_B200_KERNEL", None)
    os.environ.pop("HPHI_B200_PROD", None)
    if kernel == "single":
        os.environ["HPHI_B200_PROD"] = "single"
    elif kernel:
        os.environ["HPHI_B200_KERNEL"] = kernel
    try:
        return hphi_b200.Hamiltonian(path)
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _hv_device(H, v1, v0, vt, acc=1.0, scale=1.0):
    out = v0.clone()
    torch.cuda.synchronize()  # the engine's stream does not wait for torch's
    pr = H.mltply_device(out.data_ptr(), v1.data_ptr(), vt, acc=acc, scale=scale)
    return out, pr


MODELS = {
    "hub3x4": lambda: expert.hubbard(12, expert.square_bonds(3, 4), 1.0, 8.0, 6, 6),
    "hub4x2_doped": lambda: expert.hubbard(8, expert.square_bonds(4, 2), 1.0, 4.0, 3, 2),
    "hubchain10_complex_t": lambda: _complex_chain(10),
    "hub_inter": lambda: _with_inter(),
}


def _complex_chain(L):
    m = expert.hubbard(L, expert.chain_bonds(L), 1.0, 3.0, L // 2, L // 2)
    m.trans = []
    for i, j in expert.chain_bonds(L):
        for s in (0, 1):
            m.trans += [(i, s, j, s, 0.8, 0.3), (j, s, i, s, 0.8, -0.3)]
    m.trans += [(0, 0, 0, 0, 0.2, 0.0)]
    return m


def _with_inter():
    m = expert.hubbard(8, expert.square_bonds(2, 4), 1.0, 6.0, 4, 4)
    m.coulombinter = [(i, j, 0.7) for i, j in expert.square_bonds(2, 4)]
    m.hund = [(0, 5, 0.3)]
    return m


@pytest.mark.parametrize("kernel", [None, "single", "block"])
@pytest.mark.parametrize("name", list(MODELS))
def test_block_kernel_matches_general_kernel(name, kernel, tmp_path):
    """Native-order kernels (product layout by default, two-pass for real vectors; the
    one-pass product kernel and the block plan on request) against the general kernel."""
    path = MODELS[name]().write(str(tmp_path))
    Hf = _open(path, kernel=kernel)
    Hg = _open(path, general=True)
    try:
        assert Hf.info["native_order"] == 1, "block kernel should apply to this input"
        assert Hg.info["native_order"] == 0
        dim = Hf.dim
        g = torch.Generator(device="cuda").manual_seed(5)
        cplx = Hf.info["vec_type"] == hphi_b200.COMPLEX128 or "complex" in name
        dt = torch.complex128 if cplx else torch.float64
        vt = hphi_b200.COMPLEX128 if cplx else hphi_b200.REAL64
        v1 = torch.randn(dim, dtype=dt, device="cuda", generator=g)
        v0 = torch.randn(dim, dtype=dt, device="cuda", generator=g)
        # two-pass kernels need real vectors and down hops of one magnitude (a periodic
        # direction of width 2 doubles its hoppings, so only hub3x4 is sure to qualify)
        if kernel is None:
            assert Hf.info["kernel"] in ((3,) if name == "hub3x4" else (2, 3))
        else:
            assert Hf.info["kernel"] == {"single": 2, "block": 1}[kernel]
        for acc, scale in ((1.0, 1.0), (0.0, 1.0), (-0.75, 1.3)):
            yf, pf = _hv_device(Hf, v1, v0, vt, acc, scale)
            yg, pg = _hv_device(Hg, v1, v0, vt, acc, scale)
            err = (yf - yg).abs().max().item() / yg.abs().max().item()
            assert err < 1e-12, (acc, scale, err)
            assert abs(pf - pg) < 1e-10 * abs(pg)
        # vectors that start 8 bytes past a 16-byte boundary (no paired 16-byte loads)
        b1 = torch.empty(dim + 1, dtype=dt, device="cuda")
        b0 = torch.empty(dim + 1, dtype=dt, device="cuda")
        o1, o0 = b1[1:], b0[1:]
        o1.copy_(v1)
        o0.copy_(v0)
        pf = Hf.mltply_device(o0.data_ptr(), o1.data_ptr(), vt, acc=0.5, scale=1.0)
        yg, pg = _hv_device(Hg, v1, v0, vt, 0.5, 1.0)
        assert (o0 - yg).abs().max().item() < 1e-12 * yg.abs().max().item()
        assert abs(pf - pg) < 1e-10 * abs(pg)
        # native order round trip
        nat = torch.empty_like(v1)
        back = torch.empty_like(v1)
        Hf.to_native(v1.data_ptr(), nat.data_ptr(), vt)
        Hf.from_native(nat.data_ptr(), back.data_ptr(), vt)
        assert torch.equal(back, v1)
        assert not torch.equal(nat, v1)
    finally:
        Hf.close()
        Hg.close()


def test_block_kernel_lanczos_energy(tmp_path):
    """Lanczos through the native-order driver gives the general kernel's ground state."""
    path = MODELS["hub3x4"]().write(str(tmp_path))
    rng = np.random.default_rng(3)
    Hf = _open(path)
    v = np.zeros(Hf.dim + 1, dtype=np.complex128)
    v[1:] = rng.uniform(-1, 1, Hf.dim)
    v[1:] /= np.linalg.norm(v[1:])
    rf = Hf.calc_by_lanczos(v_init=v)
    Hf.close()
    Hg = _open(path, general=True)
    rg = Hg.calc_by_lanczos(v_init=v)
    Hg.close()
    assert rf["converged"] and rg["converged"]
    assert abs(rf["e1"] - rg["e1"]) < 1e-10
    assert abs(rf["e1"] - (-5.8334842575)) < 1e-9   # reference HPhi, 3x4 U=8 half filling


def test_product_and_block_plans_agree_full_size_4x4(tmp_path):
    """Half-filled 4x4 Hubbard: product-layout and block plans give the same H*v (1e-12)
    after conversion to HPhi order, and the same <v|H|v>."""
    path = expert.hubbard(16, expert.square_bonds(4, 4), 1.0, 8.0, 8, 8).write(str(tmp_path))
    g = torch.Generator(device="cuda").manual_seed(21)
    out = []
    for kernel in (None, "single", "block"):
        H = _open(path, kernel=kernel)
        if not out:
            v = torch.rand(H.dim, dtype=torch.float64, device="cuda", generator=g) - 0.5
            zero = torch.zeros_like(v)
        y, pr = _hv_device(H, v, zero, hphi_b200.REAL64, acc=0.0)
        out.append((y, pr))
        H.close()
    ref_y, ref_pr = out[-1]   # block plan
    for y, pr in out[:-1]:
        err = (y - ref_y).abs().max().item() / ref_y.abs().max().item()
        assert err < 1e-12
        assert abs(pr - ref_pr) < 1e-11 * abs(ref_pr)


@pytest.mark.parametrize("name", ["hub3x4", "hub3x4_doped", "hub4x4"])
def test_column_pass_kernels_agree(name, tmp_path, monkeypatch):
    """Two-pass plan, real vectors: the warp-task column pass (default) and the CTA-task
    column pass (HPHI_B200_UPPASS=block) give the same v0 += H v1 (1e-12) and prdct, on the
    4x4 sector too (its last 128-column chunk is partial: 12,870 = 100 * 128 + 70)."""
    if name == "hub4x4":
        m = expert.hubbard(16, expert.square_bonds(4, 4), 1.0, 8.0, 8, 8)
    elif name == "hub3x4_doped":   # 495 up x 792 down configurations
        m = expert.hubbard(12, expert.square_bonds(3, 4), 1.0, 8.0, 4, 5)
    else:
        m = MODELS[name]()
    path = m.write(str(tmp_path))
    g = torch.Generator(device="cuda").manual_seed(5)
    res = []
    for mode in (None, "block"):
        if mode:
            monkeypatch.setenv("HPHI_B200_UPPASS", mode)
        else:
            monkeypatch.delenv("HPHI_B200_UPPASS", raising=False)
        H = _open(path)
        if not res:
            assert H.info["kernel"] == 3
            v = torch.rand(H.dim, dtype=torch.float64, device="cuda", generator=g) - 0.5
            w = torch.rand(H.dim, dtype=torch.float64, device="cuda", generator=g) - 0.5
        res.append(_hv_device(H, v, w, hphi_b200.REAL64, acc=0.5, scale=2.0))
        H.close()
    (ya, pa), (yb, pb) = res
    err = (ya - yb).abs().max().item() / yb.abs().max().item()
    assert err < 1e-12, err
    assert abs(pa - pb) < 1e-12 * abs(pb)


def test_full_size_hubbard4x4_block_vs_general(tmp_path):
    """Half-filled 4x4 Hubbard (dim 165,636,900): block kernel == general kernel to 1e-12,
    and H is Hermitian: <u|Hv> = conj(<v|Hu>)."""
    path = expert.hubbard(16, expert.square_bonds(4, 4), 1.0, 8.0, 8, 8).write(str(tmp_path))
    Hf = _open(path)
    assert Hf.info["native_order"] == 1
    dim = Hf.dim
    g = torch.Generator(device="cuda").manual_seed(11)
    u = torch.rand(dim, dtype=torch.float64, device="cuda", generator=g) - 0.5
    v = torch.rand(dim, dtype=torch.float64, device="cuda", generator=g) - 0.5
    zero = torch.zeros_like(u)
    Hu, _ = _hv_device(Hf, u, zero, hphi_b200.REAL64, acc=0.0)
    Hv, _ = _hv_device(Hf, v, zero, hphi_b200.REAL64, acc=0.0)
    a = torch.dot(u, Hv).item()
    b = torch.dot(v, Hu).item()
    assert abs(a - b) < 1e-11 * (abs(a) + abs(b))
    Hf.close()
    Hg = _open(path, general=True)
    Hug, _ = _hv_device(Hg, u, zero, hphi_b200.REAL64, acc=0.0)
    Hg.close()
    err = (Hu - Hug).abs().max().item() / Hug.abs().max().item()
    assert err < 1e-12


@pytest.mark.parametrize("big, small, kernel", [
    # product-layout plan: one-pass kernel on complex vectors stages a 128 KB row of the 6+6 sector
    (lambda: expert.hubbard(16, expert.square_bonds(4, 4), 1.0, 8.0, 6, 6),
     lambda: expert.hubbard(12, expert.square_bonds(3, 4), 1.0, 8.0, 6, 6), None),
    # spin row-block plan: complex vectors of the 4x7 sector (40,116,600 rows) stage 55 KB blocks
    (lambda: expert.heisenberg(28, expert.square_bonds(4, 7)),
     lambda: expert.heisenberg(16, expert.chain_bonds(16)), "rowblock"),
])
def test_shared_memory_limits_survive_a_smaller_sector(big, small, kernel, tmp_path):
    """The kernels' dynamic shared-memory limit is set per kernel, not per sector: opening a
    sector with smaller rows after a larger one must leave the larger one's launches valid."""
    Hb = _open(big().write(str(tmp_path / "big")), kernel=kernel)
    Hs = _open(small().write(str(tmp_path / "small")), kernel=kernel)
    try:
        for H in (Hb, Hs, Hb):
            g = torch.Generator(device="cuda").manual_seed(1)
            v = (torch.rand(H.dim, dtype=torch.complex128, device="cuda", generator=g) - 0.5)
            out = torch.zeros_like(v)
            torch.cuda.synchronize()
            H.mltply_device(out.data_ptr(), v.data_ptr(), hphi_b200.COMPLEX128, acc=0.0)
            assert torch.isfinite(out.abs()).all()
    finally:
        Hb.close()
        Hs.close()

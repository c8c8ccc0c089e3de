"""hphi_mltply_device_noalloc, the H*v entry point for callers that may not allocate device
memory (code under another allocator's memory budget, loops that cannot take cudaMalloc's
synchronisation), against hphi_mltply_device_async on the same native-order vectors.

Its scratch is one static device array shared by every call, so each case makes two calls in
a row with different inputs: the second must not see the first one's counters or partial
sums.  This file is named to be collected last; it passes alone and after the other tests."""
import pytest

import hphi_b200
from hphi_b200 import expert

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _complex_hubbard_chain(L):
    m = expert.hubbard(L, expert.chain_bonds(L), 1.0, 3.0, L // 2, L // 2)  # complex hops below
    m.trans = []
    for i, j in expert.chain_bonds(L):
        for s in (0, 1):
            m.trans += [(i, s, j, s, 0.8, 0.3), (j, s, i, s, 0.8, -0.3)]
    return m


# name: (model, complex vectors, native order flag, kernel plan, environment at sector build)
CASES = {
    # product-layout plan, real vectors: the two-pass kernels (native order differs from HPhi's)
    "hubbard3x4": (lambda: expert.hubbard(12, expert.square_bonds(3, 4), 1.0, 8.0, 6, 6), False, 1, 3, {}),
    # the half-filled 4x4 sector of the headline workload (dim 165,636,900)
    "hubbard4x4": (lambda: expert.hubbard(16, expert.square_bonds(4, 4), 1.0, 8.0, 8, 8), False, 1, 3, {}),
    # product-layout plan, complex vectors: the one-pass kernel
    "hubbard_chain10_complex": (lambda: _complex_hubbard_chain(10), True, 1, 2, {}),
    # block plan of canonical Hubbard sectors (its counter and partial sums live in the array)
    "hubbard3x4_block": (lambda: expert.hubbard(12, expert.square_bonds(3, 4), 1.0, 8.0, 6, 6), False, 1, 1,
                         {"HPHI_B200_KERNEL": "block"}),
    # row-block plan of spin sectors (row pass and column pass partial sums in the array)
    "heisenberg_chain16": (lambda: expert.heisenberg(16, expert.chain_bonds(16), 1.0), False, 0, 4,
                           {"HPHI_B200_KERNEL": "rowblock"}),
    # general kernel (native order is HPhi's order; the default below 2^24 rows)
    "heisenberg_chain16_general": (lambda: expert.heisenberg(16, expert.chain_bonds(16), 1.0), False, 0, 0, {}),
}


def _async_hv(H, v1, v0, vt, acc, scale):
    out = v0.clone()
    coef = torch.tensor([acc, scale], dtype=torch.float64, device="cuda")
    pr = torch.zeros(2, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    H.mltply_device_async(out.data_ptr(), v1.data_ptr(), vt, coef.data_ptr(), pr.data_ptr())
    H.synchronize()
    return out, complex(pr[0].item(), pr[1].item())


def _noalloc_hv(H, v1, v0, vt, acc, scale):
    out = v0.clone()
    torch.cuda.synchronize()
    pr = H.mltply_device_noalloc(out.data_ptr(), v1.data_ptr(), vt, acc=acc, scale=scale)
    return out, pr


@pytest.mark.parametrize("name", list(CASES))
def test_noalloc_matches_async_on_two_calls(name, tmp_path, monkeypatch):
    make, cplx, native, kernel, env = CASES[name]
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    H = hphi_b200.Hamiltonian(make().write(str(tmp_path)))
    try:
        assert H.info["native_order"] == native
        assert H.info["kernel"] == kernel
        dt = torch.complex128 if cplx else torch.float64
        vt = hphi_b200.COMPLEX128 if cplx else hphi_b200.REAL64
        g = torch.Generator(device="cuda").manual_seed(17)
        for acc, scale in ((0.7, -1.3), (0.0, 1.0)):
            v1 = torch.randn(H.dim, dtype=dt, device="cuda", generator=g)
            v0 = torch.randn(H.dim, dtype=dt, device="cuda", generator=g)
            ya, pa = _async_hv(H, v1, v0, vt, acc, scale)
            yn, pn = _noalloc_hv(H, v1, v0, vt, acc, scale)
            err = (yn - ya).abs().max().item() / ya.abs().max().item()
            assert err < 1e-12, (acc, scale, err)
            assert abs(pn - pa) <= 1e-10 * abs(pa), (pn, pa)
    finally:
        H.close()


def test_noalloc_refuses_sector_beyond_fixed_scratch(tmp_path):
    """Complex vectors on the product-layout plan keep one partial sum per up-spin row: with
    11,440 rows (16 sites, 7 up and 1 down electron) that is more than the array holds, so the
    call is refused with an error instead of writing past the array."""
    L = 16
    m = _complex_hubbard_chain(L)
    m.ncond, m.two_sz = 8, 6
    H = hphi_b200.Hamiltonian(m.write(str(tmp_path)))
    try:
        assert H.info["kernel"] == 2
        v1 = torch.zeros(H.dim, dtype=torch.complex128, device="cuda")
        v0 = torch.zeros_like(v1)
        torch.cuda.synchronize()
        with pytest.raises(hphi_b200.HPhiError, match="fixed scratch"):
            H.mltply_device_noalloc(v0.data_ptr(), v1.data_ptr(), hphi_b200.COMPLEX128)
    finally:
        H.close()

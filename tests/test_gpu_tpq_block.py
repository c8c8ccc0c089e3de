"""TPQ samples in lockstep (hphi_tpq groups the NumAve samples of the reference's loop,
src/CalcByTPQ.c:76, into blocks that share one H*V per H application, hv_block_native):
every output file must equal the one-sample-at-a-time run (HPHI_B200_TPQ_BLOCK=0) digit for
digit, since per vector the block kernel does the general kernel's arithmetic in its order.
HPHI_B200_TPQ_BLOCK caps the block size (0: one sample at a time)."""
import os

import pytest

import hphi_b200
from hphi_b200 import expert

pytestmark = pytest.mark.gpu


def _models():
    out = {}
    # microcanonical TPQ, complex vectors (the reference's default), 10 samples: blocks of 8 and 2
    m = expert.heisenberg(12, expert.chain_bonds(12) + expert.chain_bonds(12, 2), J=[1.0] * 12 + [0.4] * 12,
                          calc_type="TPQ", lanczos_max=60, num_ave=10, large_value=3.0, expec_interval=20,
                          initial_vec_type=0)
    out["tpq_j1j2_chain12"] = m
    # canonical TPQ on a grand-canonical spin model, real vectors
    m = expert.kitaev_heisenberg(2, 2, 1.0, 0.3, calc_type="cTPQ", lanczos_max=30, num_ave=3, large_value=5.0)
    out["ctpq_kitaev2x2"] = m
    # a grand-canonical Hubbard sector with Green's functions every ExpecInterval steps
    m = expert.hubbard(5, expert.chain_bonds(5), 1.0, 4.0, 3, 2, calc_type="TPQ", lanczos_max=25, num_ave=4,
                       large_value=4.0, expec_interval=10)
    m.model, m.two_sz, m.ncond = "HubbardGC", None, None
    m.greenone = [(i, s, i, s) for i in range(5) for s in (0, 1)]
    out["tpq_hubbardgc5_green"] = m
    return out


MODELS = _models()


@pytest.mark.parametrize("name", sorted(MODELS))
def test_block_samples_equal_serial_samples(name, tmp_path, monkeypatch):
    d = tmp_path / "in"
    MODELS[name].write(str(d))
    outs = {}
    for mode in ("0", "8", "3"):  # one after another; blocks of up to 8; blocks of up to 3
        monkeypatch.setenv("HPHI_B200_TPQ_BLOCK", mode)
        o = tmp_path / f"out{mode}"
        with hphi_b200.Hamiltonian(str(d / "namelist.def")) as H:
            assert H.info["kernel"] == 0  # the general kernel: samples share block products
            H.calc_by_tpq(output_dir=str(o))
        outs[mode] = o
    files = sorted(os.listdir(outs["0"]))
    assert any(f.startswith("SS_rand") for f in files)
    for mode in ("8", "3"):
        assert files == sorted(os.listdir(outs[mode]))
        for f in files:
            assert (outs["0"] / f).read_text() == (outs[mode] / f).read_text(), (mode, f)

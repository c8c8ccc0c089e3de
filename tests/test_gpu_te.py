"""Real-time evolution (CalcType 4) on the device through the C-ABI: the files of the
reference's runs of the te_* golden inputs from the same start state (SS.dat, Norm.dat,
Flct.dat, Green's function step files, OutputEigenVec files), the reference's own known-answer
tables (test/te_hubbard_chain_interall*.sh), its error cases, and energy / norm conservation on
the full-size 8+8-electron 4x4 Hubbard sector."""
import json
import os
import shutil
import tempfile

import numpy as np
import pytest

import hphi_b200
import hphi_oracle as O
from conftest import GOLDEN, case_dir, golden_cases, load_golden
from test_oracle_te import ground_state, table

pytestmark = pytest.mark.gpu
KNOWN = os.path.join(GOLDEN, "known_answers")


def _write_vec(path, v, step=0):
    with open(path, "wb") as f:
        f.write(np.array([step], dtype=np.int32).tobytes())
        f.write(np.array([v.size - 1], dtype=np.int64).tobytes())
        f.write(np.asarray(v, dtype=np.complex128).tobytes())


def _read_vec(path):
    with open(path, "rb") as f:
        step = int(np.frombuffer(f.read(4), dtype=np.int32)[0])
        dim = int(np.frombuffer(f.read(8), dtype=np.int64)[0])
        return step, np.frombuffer(f.read(16 * (dim + 1)), dtype=np.complex128).copy()


def _setup(src, tmp_path, start):
    d = tmp_path / "in"
    shutil.copytree(src, d)
    if (d / "golden.npz").exists():
        os.remove(d / "golden.npz")
    out = tmp_path / "output"
    os.makedirs(out)
    _write_vec(out / "zvo_eigenvec_0_rank_0.dat", start)
    return d, out


@pytest.mark.parametrize("name", golden_cases("te"))
def test_te_matches_reference(name, tmp_path):
    z = load_golden(name)
    d, out = _setup(case_dir(name), tmp_path, z["start"])
    with hphi_b200.Hamiltonian(str(d / "namelist.def")) as H:
        energy = H.calc_by_tem(output_dir=str(out))
    for base in ("SS", "Norm", "Flct"):
        mine = open(out / f"{base}.dat").read()
        ref = str(z["text_" + base])
        assert mine.splitlines()[0] == ref.splitlines()[0]
        np.testing.assert_allclose(table(mine), table(ref), rtol=0, atol=1e-10, err_msg=base)
    np.testing.assert_allclose(energy, table(z["text_SS"])[:, 1], rtol=0, atol=1e-10)
    written = sorted(f for f in os.listdir(out) if "cisajs" in f)
    assert written == sorted(str(x) for x in z["green_files"])
    for f in written:
        mine, ref = open(out / f).read().splitlines(), str(z["text_" + f]).splitlines()
        assert len(mine) == len(ref)
        for a, b in zip(mine, ref):
            assert a.split()[:-2] == b.split()[:-2] and a.endswith(" ") == b.endswith(" "), (a, b)
            va = complex(float(a.split()[-2]), float(a.split()[-1]))
            vb = complex(float(b.split()[-2]), float(b.split()[-1]))
            assert abs(va - vb) <= 1e-10, (f, a, b)
    for key in (k for k in z if k.startswith("vec_")):
        step, v = _read_vec(out / key[4:])
        np.testing.assert_allclose(v[1:], z[key][1:], rtol=0, atol=1e-10, err_msg=key)


@pytest.mark.parametrize("name", ["te_hubbard_chain_interall", "te_hubbard_chain_interall_diagonal"])
def test_te_known_answers(name, tmp_path):
    expected = np.array(json.load(open(os.path.join(KNOWN, "te_expected.json")))[name])
    od = O.read_expert(os.path.join(KNOWN, name, "namelist.def"))
    d, out = _setup(os.path.join(KNOWN, name), tmp_path, ground_state(od, O.sz(od)))
    with hphi_b200.Hamiltonian(str(d / "namelist.def")) as H:
        H.run(str(out))                                    # CalcType 4 through hphi_run
    np.testing.assert_allclose(table(open(out / "Flct.dat").read()), expected, rtol=0, atol=1e-10)


def test_te_errors(tmp_path):
    name = golden_cases("te")[0]
    z = load_golden(name)
    d, out = _setup(case_dir(name), tmp_path, z["start"])
    with hphi_b200.Hamiltonian(str(d / "namelist.def")) as H:
        with pytest.raises(hphi_b200.HPhiError, match="does not exist"):
            H.calc_by_tem(output_dir=str(tmp_path / "nowhere"))
        _write_vec(tmp_path / "short.dat", z["start"][:-1])
        os.makedirs(tmp_path / "bad")
        shutil.copy(tmp_path / "short.dat", tmp_path / "bad" / "zvo_eigenvec_0_rank_0.dat")
        with pytest.raises(hphi_b200.HPhiError, match="incorrect"):
            H.calc_by_tem(output_dir=str(tmp_path / "bad"))
    txt = open(d / "calcmod.def").read().replace("InputEigenVec 1", "InputEigenVec 0")
    open(d / "calcmod.def", "w").write(txt)
    with hphi_b200.Hamiltonian(str(d / "namelist.def")) as H:
        with pytest.raises(hphi_b200.HPhiError, match="not inputted"):
            H.calc_by_tem(output_dir=str(out))
    import re
    txt = re.sub(r"Lanczos_max\s+(\d+)", lambda g: f"Lanczos_max    {int(g.group(1)) + 1}",
                 open(d / "modpara.def").read())
    open(d / "modpara.def", "w").write(txt)
    with hphi_b200.Hamiltonian(str(d / "namelist.def")) as H:
        with pytest.raises(hphi_b200.HPhiError, match="NTETimeSteps must be larger"):
            H.calc_by_tem(v_init=z["start"], output_dir=str(out))


def test_te_conserves_energy_on_the_full_size_sector():
    """8+8 electrons on the 4x4 Hubbard lattice (dim 165,636,900), no time-dependent terms,
    ExpandCoef 8, dt 1e-3: each step's norm before normalisation stays 1 and the energy stays
    that of the start vector (both to 1e-9)."""
    from hphi_b200 import expert
    m = expert.hubbard(16, expert.square_bonds(4, 4), 1.0, 8.0, 8, 8, calc_type="TimeEvolution", lanczos_max=4,
                       input_eigenvec=1, spectrum_vec="zvo_eigenvec_0", expand_coef=8, expec_interval=100)
    m.te_twobody = [(1e-3 * k, []) for k in range(4)]
    with tempfile.TemporaryDirectory() as tmp:
        m.write(tmp)
        with hphi_b200.Hamiltonian(os.path.join(tmp, "namelist.def")) as H:
            rng = np.random.default_rng(3)
            v = np.zeros(H.dim + 1, dtype=np.complex128)
            v[1:] = rng.standard_normal(H.dim)
            v[1:] /= np.linalg.norm(v[1:])
            e = H.calc_by_tem(v_init=v, output_dir=os.path.join(tmp, "output"))
            norm = table(open(os.path.join(tmp, "output", "Norm.dat")).read())
    assert np.all(np.abs(norm[:, 1] - 1.0) < 1e-9)
    assert np.all(np.abs(e - e[0]) < 1e-9 * abs(e[0]) + 1e-9)


def test_te_restart_continues_from_the_stored_step(tmp_path):
    """ReStart 3 reads the step of <SpectrumVec>_rank_0.dat and starts the loop there with no
    previous H psi (src/CalcByTEM.c:99-102: the first step keeps the stored state), so a run
    continued from the state OutputEigenVec wrote at step 10 repeats the reference's SS and Flct
    rows from step 10 on."""
    name = "te_hub_chain6_two"
    z = load_golden(name)
    d, out = _setup(case_dir(name), tmp_path, z["start"])
    with hphi_b200.Hamiltonian(str(d / "namelist.def")) as H:
        H.calc_by_tem(output_dir=str(out))
    out2 = tmp_path / "output2"
    os.makedirs(out2)
    shutil.copy(out / "zvo_eigenvec_10_rank_0.dat", out2 / "zvo_eigenvec_0_rank_0.dat")
    open(d / "calcmod.def", "a").write("ReStart 3\n")
    with hphi_b200.Hamiltonian(str(d / "namelist.def")) as H:
        H.calc_by_tem(output_dir=str(out2))
    for base in ("SS", "Flct"):
        mine = table(open(out2 / f"{base}.dat").read())
        ref = table(z["text_" + base])
        assert mine[0, -1] == 10 and len(mine) == len(ref) - 10
        np.testing.assert_allclose(mine, ref[10:], rtol=0, atol=1e-10, err_msg=base)

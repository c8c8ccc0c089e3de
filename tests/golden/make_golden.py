"""Generates the golden fixtures in tests/golden/ by running the reference HPhi.

Each case directory holds the expert-mode input the reference ran (the .def files)
and golden.npz with what the reference produced, read through the link-time hooks
of oracle/ref_hooks.c:
  list_1, list_2_1, list_2_2     sz() output (canonical models)
  diag                           list_Diagonal after diagonalcalc()
  hv0_v1, hv0_v0a, hv0_pr        the first mltply call (v0 = 0 before: the start vector in v1)
  hv3_v1, hv3_v0b, hv3_v0a, hv3_pr  the 4th mltply call (accumulates into a non-zero v0)
  steps, step_vals               zvo_Lanczos_Step.dat (Lanczos cases)
  lobpcg_steps, lobpcg_states    zvo_Lanczos_Step.dat rows and zvo_energy.dat states (LOBPCG cases)
  energy_state, cg_ran           zvo_energy.dat of a Lanczos case with CalcEigenVec != -1, and
                                 whether the reference refined the vector by CG
  tpq                            SS_rand0.dat rows (TPQ cases)
refstart_* directories hold start.npz: the first mltply input of a golden case's input rerun
with several OpenMP threads (the reference's per-thread random start vectors).
restart_* directories hold inputs a/ and b/ and restart.npz: the restart files run a wrote
and the steps and energy of run b continued from them.
tpqrestart_* directories hold inputs a/ (ReStart 1) and b/ (ReStart 3, continuing a) and
restart.npz: the TPQ files and the stored states (tmpvec_set%d_rank_0.dat) after each run;
lobpcgrestart_* the same for LOBPCG (step rows of both runs, a's stored vectors, b's states).
green_* directories hold inputs with OneBodyG / TwoBodyG files and golden.npz with the
reference's Green's function files (text_<file>), the eigenvectors it wrote (vec_<file>,
OutputEigenVec), the first mltply input (start) and its energies (states, or tpq rows).
te_* directories hold time-evolution inputs (CalcType 4, TEOneBody / TETwoBody) and golden.npz
with the seeded start state written as zvo_eigenvec_0_rank_0.dat before the run (start), the
reference's SS.dat, Norm.dat, Flct.dat (text_SS ...), its Green's function step files and the
eigenvector files of OutputEigenVec (vec_<file>).
Large cases store only SHA-256 digests of the lists (sha_list_1 ...).

Run in a container that has the reference sources and oracle/_ref/HPhi_ref
(`make -C oracle`):  python tests/golden/make_golden.py [case ...]
"""
from __future__ import annotations

import hashlib
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from hphi_b200 import expert  # noqa: E402
import run_ref  # noqa: E402


def _cases():
    c = {}
    # Heisenberg chain L=16, Sz=0, real vectors, random start (the CPU-runnable workload).
    c["chain16"] = expert.heisenberg(16, expert.chain_bonds(16))
    m = expert.j1j2_chain(14, 1.0, 0.45)
    c["j1j2_14"] = m
    # Odd number of sites: the lower half has more bits than the upper half.
    c["chain13_sz1"] = expert.heisenberg(13, expert.chain_bonds(13), two_sz=1)
    m = expert.hubbard(8, expert.square_bonds(2, 4), 1.0, 8.0, 4, 4)
    c["hub2x4"] = m
    m = expert.hubbard(8, expert.chain_bonds(8), 1.0, 4.0, 4, 4)
    m.initial_vec_type = 0
    c["hubchain8_complex"] = m
    m = expert.hubbard(7, expert.chain_bonds(7), 1.0, 6.0, 3, 4)
    c["hubchain7_odd"] = m
    # Hubbard with Ncond only (HubbardNConserved).
    m = expert.hubbard(6, expert.square_bonds(2, 3), 1.0, 4.0, 3, 3)
    m.two_sz = None
    c["hub2x3_ncons"] = m
    # Grand-canonical Hubbard with chemical potential (diagonal transfers).
    m = expert.ExpertModel(model="HubbardGC", nsite=4, two_sz=None, initial_vec_type=0)
    for i, j in expert.chain_bonds(4):
        for s in (0, 1):
            m.trans += [(i, s, j, s, 1.0, 0.0), (j, s, i, s, 1.0, 0.0)]
    m.trans += [(i, s, i, s, 0.7, 0.0) for i in range(4) for s in (0, 1)]
    m.coulombintra = [(i, 3.0) for i in range(4)]
    c["hubgc4"] = m
    # Kitaev-Heisenberg honeycomb, SpinGC (Exchange + PairLift + Ising), complex vectors.
    m = expert.kitaev_heisenberg(2, 2, -1.0, 0.2)
    m.initial_vec_type = 0
    c["kitaev2x2"] = m
    # SpinGC with a transverse field (site-diagonal Trans with s1 != s2).
    m = expert.heisenberg(8, expert.chain_bonds(8))
    m.model, m.two_sz, m.initial_vec_type = "SpinGC", None, 0
    m.trans = [(i, 0, i, 1, 0.3, 0.0) for i in range(8)] + [(i, 1, i, 0, 0.3, 0.0) for i in range(8)]
    c["spingc_field8"] = m
    # Canonical spin with random InterAll terms (complex coefficients).
    m = expert.heisenberg(10, expert.chain_bonds(10))
    m.initial_vec_type = 0
    inter = [t for t in expert.random_interall_spin(10, 12, seed=7)
             if (t[1] - t[3]) + (t[5] - t[7]) == 0]  # keep Sz-conserving strings
    m.interall = inter
    c["spin_interall10"] = m
    # Hubbard with every two-body keyword and a complex hopping.
    m = expert.hubbard(6, expert.chain_bonds(6), 1.0, 5.0, 3, 3)
    m.initial_vec_type = 0
    m.trans += [(0, 0, 2, 0, 0.3, 0.2), (2, 0, 0, 0, 0.3, -0.2), (0, 1, 2, 1, 0.3, 0.2), (2, 1, 0, 1, 0.3, -0.2)]
    m.coulombinter = [(i, (i + 1) % 6, 0.8) for i in range(6)]
    m.hund = [(i, (i + 1) % 6, 0.4) for i in range(6)]
    m.exchange = [(i, (i + 1) % 6, 0.35) for i in range(6)]
    m.pairhop = [(i, (i + 2) % 6, 0.25) for i in range(6)]
    m.ising = [(0, 3, 0.5)]
    m.interall = [(1, 0, 1, 0, 4, 1, 4, 1, 0.6, 0.0),
                  (0, 0, 1, 0, 3, 1, 4, 1, 0.2, 0.1), (4, 1, 3, 1, 1, 0, 0, 0, 0.2, -0.1)]
    c["hub6_allterms"] = m
    # TPQ on a chain (one sample).
    m = expert.heisenberg(12, expert.chain_bonds(12), calc_type="TPQ", lanczos_max=25, num_ave=1,
                          large_value=4.5)
    c["tpq_chain12"] = m
    m = expert.hubbard(6, expert.chain_bonds(6), 1.0, 4.0, 3, 3, calc_type="TPQ", lanczos_max=20, num_ave=1,
                       large_value=6.0)
    m.initial_vec_type = 0
    c["tpq_hub6"] = m
    # LOBPCG (CalcType 3): single-element starts (initial_iv > 0), with and without PreCG,
    # two states; a grand-canonical case with the reference's random start (its first
    # mltply input is dumped and injected).
    c["lobpcg_chain12"] = expert.heisenberg(12, expert.chain_bonds(12), calc_type="CG", initial_iv=1,
                                            lanczos_max=400)
    m = expert.hubbard(6, expert.chain_bonds(6), 1.0, 4.0, 3, 3, calc_type="CG", initial_iv=2, exct=2,
                       lanczos_max=400, pre_cg=1)
    c["lobpcg_hub6_k2"] = m
    m = expert.kitaev_heisenberg(2, 2, -1.0, 0.2, calc_type="CG", lanczos_max=400, lanczos_eps=12)
    m.initial_vec_type = 0
    c["lobpcg_kitaev2x2"] = m
    # six states (more than one block of the engine's linear-combination kernel), random start
    c["lobpcg_chain10_k6"] = expert.heisenberg(10, expert.chain_bonds(10), calc_type="CG", exct=6,
                                               lanczos_max=600)
    # Kondo lattices (itinerant ring + one local spin per cell, J S.s as InterAll): canonical
    # with real and complex vectors, and the grand-canonical KondoGC sector.
    c["kondo_chain4"] = expert.kondo_chain(4, 1.0, 1.5, lanczos_max=300)
    m = expert.kondo_chain(4, 1.0, 1.2, U=2.0, two_sz=2, lanczos_max=300)
    m.initial_vec_type = 0
    c["kondo_chain4_u"] = m
    m = expert.kondo_chain(2, 1.0, 0.8, gc=True, lanczos_max=200)
    m.initial_vec_type = 0
    c["kondogc_chain2"] = m
    # Lanczos stopped early (LanczosEps 5) with CalcEigenVec 0: the reference's accuracy
    # check fails and CG_EigenVector refines the vector before zvo_energy.dat is written.
    c["lanczos_cg_chain12"] = expert.heisenberg(12, expert.chain_bonds(12), lanczos_eps=5, calc_eigenvec=0)
    m = expert.hubbard(6, expert.chain_bonds(6), 1.0, 4.0, 3, 3, lanczos_eps=3, calc_eigenvec=0)
    m.initial_vec_type = 0
    c["lanczos_cg_hub6"] = m
    # General spin (some 2S > 1; InterAll only): spin-1 chain, mixed spin-1/2 / spin-1 chain
    # with a single-ion term, spin-3/2 chain, and a grand-canonical spin-1 chain in a
    # transverse field (off-diagonal Trans), complex vectors.
    c["gspin1_chain8"] = expert.general_heisenberg([2] * 8, expert.chain_bonds(8), lanczos_max=300)
    c["gspin_mixed6"] = expert.general_heisenberg([1, 2, 1, 2, 1, 2], expert.chain_bonds(6), two_sz=1, D=0.3,
                                                  lanczos_max=300)
    c["gspin32_chain6"] = expert.general_heisenberg([3] * 6, expert.chain_bonds(6), two_sz=2, lanczos_max=300)
    m = expert.general_heisenberg([2] * 5, expert.chain_bonds(5), two_sz=None, D=0.2, hx=0.4, lanczos_max=300)
    m.initial_vec_type = 0
    c["gspingc_field5"] = m
    return c


def _large_cases():
    """Full-size sectors: only list digests are stored (the reference's own sz)."""
    c = {}
    m = expert.hubbard(16, expert.square_bonds(4, 4), 1.0, 8.0, 8, 8, lanczos_max=1)
    c["hub4x4_lists"] = m
    m = expert.heisenberg(24, expert.chain_bonds(24), lanczos_max=1)
    c["chain24_lists"] = m
    c["kondo_chain8_lists"] = expert.kondo_chain(8, 1.0, 1.0, lanczos_max=1)
    c["gspin1_chain14_lists"] = expert.general_heisenberg([2] * 14, expert.chain_bonds(14), lanczos_max=1)
    return c


def _sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint64).tobytes()).hexdigest()


def make_case(name: str, m, large: bool = False) -> None:
    out = os.path.join(HERE, name)
    shutil.rmtree(out, ignore_errors=True)
    m.write(out)
    data = {}
    with tempfile.TemporaryDirectory() as tmp:
        for f in os.listdir(out):
            shutil.copy(os.path.join(out, f), tmp)
        p = run_ref.run(tmp, threads=1 if not large else os.cpu_count(), dump_call=0)
        # large cases stop after sz() output (Lanczos_max=1 does not converge and exits -1)
        if p.returncode != 0 and not (large and os.path.exists(os.path.join(tmp, "lists.bin"))):
            raise RuntimeError(f"{name}: reference failed\n{p.stdout[-3000:]}\n{p.stderr[-3000:]}")
        if os.path.exists(os.path.join(tmp, "lists.bin")):
            l1, l21, l22 = run_ref.read_lists(tmp)
            if large:
                data.update(sha_list_1=_sha(l1), sha_list_2_1=_sha(l21), sha_list_2_2=_sha(l22),
                            dim=l1.size - 1, n21=l21.size, n22=l22.size)
            else:
                data.update(list_1=l1, list_2_1=l21, list_2_2=l22)
        if large:
            np.savez_compressed(os.path.join(out, "golden.npz"), **data)
            return
        data["diag"] = run_ref.read_diag(tmp)
        v1, v0b, v0a, pr = run_ref.read_hv(tmp)
        data.update(hv0_v1=v1, hv0_v0a=v0a, hv0_pr=np.array(pr))
        if m.calc_type == "CG":
            data["lobpcg_steps"] = run_ref.lobpcg_steps(tmp)
            data["lobpcg_states"] = run_ref.energy_states(tmp)
        elif m.calc_type == "Lanczos":
            steps = run_ref.lanczos_steps(tmp)
            data["steps"] = np.array([s for s, _ in steps])
            data["step_vals"] = np.array([[np.nan if v is None else v for v in (vals + [None] * 6)[:6]]
                                          for _, vals in steps])
            if m.calc_eigenvec != -1:
                # zvo_energy.dat (Energy, Doublon, Sz) and whether the CG refinement ran
                data["energy_state"] = run_ref.energy_states(tmp)[0]
                data["cg_ran"] = np.array("Accuracy of Lanczos vectors is NOT enough" in p.stdout)
        else:
            data["tpq"] = run_ref.tpq_table(tmp, 0)
    with tempfile.TemporaryDirectory() as tmp:
        for f in os.listdir(out):
            shutil.copy(os.path.join(out, f), tmp)
        p = run_ref.run(tmp, threads=1, dump_call=3)
        if p.returncode != 0:
            raise RuntimeError(f"{name}: reference failed (call 3)")
        if os.path.exists(os.path.join(tmp, "hv.bin")):
            v1, v0b, v0a, pr = run_ref.read_hv(tmp)
            data.update(hv3_v1=v1, hv3_v0b=v0b, hv3_v0a=v0a, hv3_pr=np.array(pr))
    np.savez_compressed(os.path.join(out, "golden.npz"), **data)


def _start_cases():
    """Reference start vectors drawn with several OpenMP threads (the inputs of golden cases,
    rerun with `threads` threads): only the first mltply input is kept."""
    return {"refstart_chain16_t3": ("chain16", 3), "refstart_kitaev2x2_t4": ("kitaev2x2", 4),
            "refstart_tpq_hub6_t3": ("tpq_hub6", 3)}


def make_start_case(name: str, src: str, threads: int) -> None:
    out = os.path.join(HERE, name)
    shutil.rmtree(out, ignore_errors=True)
    os.makedirs(out)
    with tempfile.TemporaryDirectory() as tmp:
        for f in os.listdir(os.path.join(HERE, src)):
            if f.endswith(".def"):
                shutil.copy(os.path.join(HERE, src, f), tmp)
        p = run_ref.run(tmp, threads=threads, dump_call=0)
        if p.returncode != 0:
            raise RuntimeError(f"{name}: reference failed")
        v1, _, _, _ = run_ref.read_hv(tmp)
    np.savez_compressed(os.path.join(out, "start.npz"), source=np.array(src), threads=np.array(threads), v1=v1)


def _restart_cases():
    """Lanczos restart: input a/ (ReStart 1, Lanczos_max 20: stops unconverged and writes the
    restart files) and b/ (ReStart 3: continues from them to convergence)."""
    def model(restart, lmax):
        m = expert.heisenberg(14, expert.chain_bonds(14), lanczos_max=lmax, calc_eigenvec=0)
        m.restart = restart
        return m
    return {"restart_chain14": (model(1, 20), model(3, 200))}


def make_restart_case(name: str, ma, mb) -> None:
    out = os.path.join(HERE, name)
    shutil.rmtree(out, ignore_errors=True)
    ma.write(os.path.join(out, "a"))
    mb.write(os.path.join(out, "b"))
    data = {}
    with tempfile.TemporaryDirectory() as tmp:
        for f in os.listdir(os.path.join(out, "a")):
            shutil.copy(os.path.join(out, "a", f), tmp)
        if run_ref.run(tmp, threads=1, dump_call=-1).returncode != 0:
            raise RuntimeError(f"{name}: reference run a failed")
        od = os.path.join(tmp, "output")
        lines = open(os.path.join(od, "zvo_TMComponents.dat")).read().split("\n")
        data["tm_steps"] = np.array(int(lines[0].split()[0]))
        data["tm_dnorm"] = np.array(float(lines[1].split()[0]))
        ab = np.array([[float(x) for x in l.split()] for l in lines[2:] if l.strip()])
        data["tm_alpha"], data["tm_beta"] = ab[:, 0], ab[:, 1]
        with open(os.path.join(od, "zvo_recalcvec_rank_0.dat"), "rb") as f:
            stp, dim = np.frombuffer(f.read(16), dtype=np.int64)
            v = np.frombuffer(f.read(), dtype=np.complex128)
        data["rv_step"] = np.array(stp)
        data["rv_v0"], data["rv_v1"] = v[:dim + 1].copy(), v[dim + 1:2 * (dim + 1)].copy()
        data["a_step_lines"] = np.array(open(os.path.join(od, "zvo_Lanczos_Step.dat")).read().splitlines())
        for f in os.listdir(os.path.join(out, "b")):
            shutil.copy(os.path.join(out, "b", f), tmp)
        if run_ref.run(tmp, threads=1, dump_call=-1).returncode != 0:
            raise RuntimeError(f"{name}: reference run b failed")
        steps = run_ref.lanczos_steps(tmp)
        data["b_steps"] = np.array([s for s, _ in steps])
        data["b_step_vals"] = np.array([[np.nan if v is None else v for v in (vals + [None] * 6)[:6]]
                                        for _, vals in steps])
        data["b_energy_state"] = run_ref.energy_states(tmp)[0]
    np.savez_compressed(os.path.join(out, "restart.npz"), **data)


def _green_rows(nsite: int, nsig: int, seed: int, n_one: int, n_two: int, spin: bool):
    """OneBodyG / TwoBodyG rows: every one-body (i, s1, j, s2) (spin models: plus the
    off-site rows the reader drops or zeroes) when n_one < 0, else n_one random rows;
    structured two-body rows (densities, spin flips, overlapping indices) plus n_two
    random rows (spin models: on-site pairs only)."""
    rng = np.random.RandomState(seed)
    sig = range(nsig)
    if n_one < 0:
        one = [(i, a, j, b) for i in range(nsite) for a in sig for j in range(nsite) for b in sig]
    else:
        one = [tuple(int(x) for x in (rng.randint(nsite), rng.randint(nsig), rng.randint(nsite), rng.randint(nsig)))
               for _ in range(n_one)]
    two = []
    if spin:
        for i, k in [(0, 0), (0, 1), (1, 0), (0, nsite - 1), (nsite - 1, 1)]:
            for a in sig:
                for b in sig:
                    for c in sig:
                        for dd in sig:
                            if rng.rand() < (1.0 if nsig == 2 else 0.3):
                                two.append((i, a, i, b, k, c, k, dd))
        for _ in range(n_two):
            i, k = rng.randint(nsite), rng.randint(nsite)
            two.append((int(i), int(rng.randint(nsig)), int(i), int(rng.randint(nsig)), int(k),
                        int(rng.randint(nsig)), int(k), int(rng.randint(nsig))))
    else:
        for i, j in [(0, 1), (1, 0), (0, 0), (0, nsite - 1)]:
            two += [(i, a, i, a, j, b, j, b) for a in sig for b in sig]          # n n
            two += [(i, 0, i, 1, j, 1, j, 0), (i, 1, j, 1, j, 0, i, 0)]          # spin flip / exchange order
            two += [(i, 0, j, 0, j, 0, i, 0), (i, 0, j, 1, j, 1, i, 0)]          # overlapping middle indices
            two += [(i, 0, j, 0, i, 1, j, 1), (i, 0, j, 0, j, 1, i, 1)]          # pair hopping orders
        for _ in range(n_two):
            two.append(tuple(int(rng.randint(m)) for m in (nsite, 2, nsite, 2, nsite, 2, nsite, 2)))
    return one, two


def _green_cases():
    """Lanczos (eigenvector and Green's functions), TPQ and LOBPCG inputs with OneBodyG /
    TwoBodyG files, one per model branch of expec_cisajs / expec_cisajscktaltdc."""
    c = {}

    def lanczos(m, seed, n_one=-1, n_two=40, nsig=2):
        m.calc_eigenvec, m.output_eigenvec = 0, 1
        m.greenone, m.greentwo = _green_rows(m.nsite, nsig, seed, n_one, n_two, m.model.startswith("Spin"))
        return m

    c["green_hub6"] = lanczos(expert.hubbard(6, expert.square_bonds(2, 3), 1.0, 4.0, 3, 3, lanczos_max=300), 1)
    m = expert.ExpertModel(model="HubbardGC", nsite=4, two_sz=None, initial_vec_type=0, lanczos_max=300)
    for i, j in expert.chain_bonds(4):
        for s in (0, 1):
            m.trans += [(i, s, j, s, 1.0, 0.0), (j, s, i, s, 1.0, 0.0)]
    m.trans += [(0, 0, 0, 1, 0.3, 0.2), (0, 1, 0, 0, 0.3, -0.2)]   # a spin-mixing field: complex vectors
    m.coulombintra = [(i, 3.0) for i in range(4)]
    c["green_hubgc4"] = lanczos(m, 2)
    m = expert.hubbard(6, expert.square_bonds(2, 3), 1.0, 4.0, 3, 3, lanczos_max=300)
    m.two_sz = None
    c["green_ncons"] = lanczos(m, 3)
    c["green_kondo3"] = lanczos(expert.kondo_chain(3, 1.0, 1.5, lanczos_max=300), 4)
    c["green_spin10"] = lanczos(expert.heisenberg(10, expert.chain_bonds(10), lanczos_max=300), 5)
    m = expert.kitaev_heisenberg(2, 2, -1.0, 0.2, lanczos_max=300)
    m.initial_vec_type = 0
    c["green_kitaev2x2"] = lanczos(m, 6)
    c["green_gspin6"] = lanczos(expert.general_heisenberg([2] * 6, expert.chain_bonds(6), lanczos_max=300), 7,
                                n_two=60, nsig=3)
    m = expert.general_heisenberg([2] * 5, expert.chain_bonds(5), two_sz=None, D=0.2, hx=0.4, lanczos_max=300)
    m.initial_vec_type = 0
    c["green_gspingc5"] = lanczos(m, 8, n_two=60, nsig=3)
    m = expert.hubbard(6, expert.chain_bonds(6), 1.0, 4.0, 3, 3, calc_type="TPQ", lanczos_max=12, num_ave=1,
                       large_value=6.0, expec_interval=4)
    m.initial_vec_type = 0
    m.greenone, m.greentwo = _green_rows(6, 2, 9, 40, 20, False)
    c["green_tpq_hub6"] = m
    m = expert.heisenberg(10, expert.chain_bonds(10), calc_type="CG", exct=2, lanczos_max=600)
    m.output_eigenvec = 1
    m.greenone, m.greentwo = _green_rows(10, 2, 10, -1, 30, True)
    c["green_lobpcg_chain10"] = m
    # canonical TPQ (CalcType 5): exp(-dtau H / 2) steps, Green's functions every 4 steps
    m = expert.hubbard(6, expert.chain_bonds(6), 1.0, 4.0, 3, 3, calc_type="cTPQ", lanczos_max=12, num_ave=1,
                       large_value=6.0, expec_interval=4)
    m.initial_vec_type = 0
    m.greenone, m.greentwo = _green_rows(6, 2, 13, 30, 10, False)
    c["green_ctpq_hub6"] = m
    # three-, four- and six-body rows (spin-1/2 SpinGC with a transverse field, complex vectors)
    m = expert.heisenberg(8, expert.chain_bonds(8), lanczos_max=300)
    m.model, m.two_sz, m.initial_vec_type = "SpinGC", None, 0
    m.trans = [(i, 0, i, 1, 0.3, 0.0) for i in range(8)] + [(i, 1, i, 0, 0.3, 0.0) for i in range(8)]
    m.calc_eigenvec, m.output_eigenvec = 0, 1
    m.greenthree, m.greenfour, m.greensix = (_multi_rows(8, 11 + k, n, 30) for k, n in enumerate((3, 4, 6)))
    c["green_multi_spingc8"] = m
    # a Hubbard input with ThreeBodyG only: the reference leaves the two- and three-body files empty
    m = expert.hubbard(6, expert.square_bonds(2, 3), 1.0, 4.0, 3, 3, lanczos_max=300)
    m.calc_eigenvec, m.output_eigenvec = 0, 1
    m.greenthree = _multi_rows(6, 12, 3, 5)
    c["green_multi_hub6"] = m
    return c


def _multi_rows(nsite: int, seed: int, npairs: int, n: int):
    """Rows of npairs site pairs (i, s, j, t): the first two pairs on-site, in Rearray's
    exchanged form (i, j)(j, i), or neither; the later pairs on-site except in some rows."""
    rng = np.random.RandomState(seed)
    rows = []
    for r in range(n):
        g = [int(x) for x in rng.randint(2, size=2 * npairs)]
        i, j = (int(x) for x in rng.choice(nsite, 2, replace=False))
        k = int(rng.randint(nsite))
        if r % 5 == 0:
            first = [i, g[0], j, g[1], j, g[2], i, g[3]]
        elif r % 5 == 1:
            first = [i, g[0], j, g[1], k, g[2], int((k + 1) % nsite), g[3]]
        else:
            first = [i, g[0], i, g[1], k, g[2], k, g[3]]
        rest = []
        for q in range(2, npairs):
            a = int(rng.randint(nsite))
            b = int((a + 1) % nsite) if (r % 5 == 4 and q == npairs - 1) else a
            rest += [a, g[2 * q], b, g[2 * q + 1]]
        rows.append(tuple(first + rest))
    return rows


def _read_eigvec(path: str) -> np.ndarray:
    """zvo_eigenvec_%d_rank_%d.dat: int step, long dim, complex128[dim+1] (src/CalcByLanczos.c:262-273)."""
    with open(path, "rb") as f:
        f.read(4)
        dim = int(np.frombuffer(f.read(8), dtype=np.int64)[0])
        return np.frombuffer(f.read(16 * (dim + 1)), dtype=np.complex128).copy()


def make_green_case(name: str, m) -> None:
    out = os.path.join(HERE, name)
    shutil.rmtree(out, ignore_errors=True)
    m.write(out)
    data = {}
    with tempfile.TemporaryDirectory() as tmp:
        for f in os.listdir(out):
            shutil.copy(os.path.join(out, f), tmp)
        p = run_ref.run(tmp, threads=1, dump_call=0)
        if p.returncode != 0:
            raise RuntimeError(f"{name}: reference failed\n{p.stdout[-3000:]}\n{p.stderr[-3000:]}")
        od = os.path.join(tmp, "output")
        v1, _, _, _ = run_ref.read_hv(tmp)
        data["start"] = v1
        files = sorted(f for f in os.listdir(od) if "cisajs" in f or "Body" in f)
        data["green_files"] = np.array(files)
        for f in files:
            text = open(os.path.join(od, f)).read()
            data["text_" + f] = np.array(text)
        for f in sorted(os.listdir(od)):
            if f.startswith("zvo_eigenvec_"):
                data["vec_" + f] = _read_eigvec(os.path.join(od, f))
        if m.calc_type in ("TPQ", "cTPQ"):
            data["tpq"] = run_ref.tpq_table(tmp, 0)
            for base in ("SS_rand0", "Norm_rand0", "Flct_rand0"):
                data["text_" + base] = np.array(open(os.path.join(od, base + ".dat")).read())
        else:
            data["states"] = run_ref.energy_states(tmp)
    np.savez_compressed(os.path.join(out, "golden.npz"), **data)


def _tpq_restart_cases():
    """TPQ restart: input a/ (ReStart 1, Lanczos_max 12, two samples: writes
    tmpvec_set%d_rank_0.dat) and b/ (ReStart 3, Lanczos_max 25: continues both samples; the reference
    divides by (Lanczos_max - step + 1) / 10 for its progress log, so it needs 10 more steps)."""
    def model(restart, lmax):
        m = expert.hubbard(6, expert.chain_bonds(6), 1.0, 4.0, 3, 3, calc_type="TPQ", lanczos_max=lmax,
                           num_ave=2, large_value=6.0, expec_interval=100)
        m.initial_vec_type = 0
        m.restart = restart
        return m
    return {"tpqrestart_hub6": (model(1, 12), model(3, 25))}


def make_tpq_restart_case(name: str, ma, mb) -> None:
    out = os.path.join(HERE, name)
    shutil.rmtree(out, ignore_errors=True)
    ma.write(os.path.join(out, "a"))
    mb.write(os.path.join(out, "b"))
    data = {}
    with tempfile.TemporaryDirectory() as tmp:
        od = os.path.join(tmp, "output")
        for tag, sub in (("a", "a"), ("b", "b")):
            for f in os.listdir(os.path.join(out, sub)):
                shutil.copy(os.path.join(out, sub, f), tmp)
            if run_ref.run(tmp, threads=1, dump_call=-1).returncode != 0:
                raise RuntimeError(f"{name}: reference run {tag} failed")
            for r in range(2):
                for base in ("SS_rand", "Norm_rand", "Flct_rand"):
                    data[f"{tag}_{base}{r}"] = np.array(open(os.path.join(od, f"{base}{r}.dat")).read())
                with open(os.path.join(od, f"tmpvec_set{r}_rank_0.dat"), "rb") as f:
                    data[f"{tag}_step{r}"] = np.array(int(np.frombuffer(f.read(4), dtype=np.int32)[0]))
                    dim = int(np.frombuffer(f.read(8), dtype=np.int64)[0])
                    v = np.frombuffer(f.read(16 * (dim + 1)), dtype=np.complex128).copy()
                    v[0] = 0
                    data[f"{tag}_vec{r}"] = v
    np.savez_compressed(os.path.join(out, "restart.npz"), **data)


def _lobpcg_restart_cases():
    """LOBPCG restart: input a/ (ReStart 1, Lanczos_max 8: stops unconverged and writes
    tmpvec_set%d_rank_0.dat per state) and b/ (ReStart 3: continues from them)."""
    def model(restart, lmax):
        m = expert.heisenberg(12, expert.chain_bonds(12), calc_type="CG", exct=2, lanczos_max=lmax)
        m.restart = restart
        return m
    return {"lobpcgrestart_chain12": (model(1, 8), model(3, 500))}


def make_lobpcg_restart_case(name: str, ma, mb) -> None:
    out = os.path.join(HERE, name)
    shutil.rmtree(out, ignore_errors=True)
    ma.write(os.path.join(out, "a"))
    mb.write(os.path.join(out, "b"))
    data = {}
    with tempfile.TemporaryDirectory() as tmp:
        od = os.path.join(tmp, "output")
        for tag, sub in (("a", "a"), ("b", "b")):
            for f in os.listdir(os.path.join(out, sub)):
                shutil.copy(os.path.join(out, sub, f), tmp)
            p = run_ref.run(tmp, threads=1, dump_call=-1)
            if p.returncode != 0:
                raise RuntimeError(f"{name}: reference run {tag} failed")
            data[f"{tag}_steps"] = run_ref.lobpcg_steps(tmp)
            if tag == "a":
                for ie in range(2):
                    with open(os.path.join(od, f"tmpvec_set{ie}_rank_0.dat"), "rb") as f:
                        data[f"a_itr{ie}"] = np.array(int(np.frombuffer(f.read(4), dtype=np.int32)[0]))
                        dim = int(np.frombuffer(f.read(8), dtype=np.int64)[0])
                        v = np.frombuffer(f.read(16 * (dim + 1)), dtype=np.complex128).copy()
                        v[0] = 0
                        data[f"a_vec{ie}"] = v
                data["a_energy_exists"] = np.array(os.path.exists(os.path.join(od, "zvo_energy.dat")))
            else:
                data["b_states"] = run_ref.energy_states(tmp)
    np.savez_compressed(os.path.join(out, "restart.npz"), **data)


def _te_times(n: int, dt: float, repeat_at: int = -1):
    """Time grid accumulated as t += dt (a repeated time at index repeat_at: a zero step)."""
    out, t = [], 0.0
    for k in range(n):
        out.append(t)
        if k != repeat_at:
            t += dt
    return out


def _te_cases():
    import math
    cases = {}
    # Hubbard chain L=6 (3+3 electrons): a time-dependent exchange-like InterAll on every bond
    # and a time-dependent density-density row, 30 steps of 0.02, ExpandCoef 4, Green's
    # functions every 10 steps, eigenvector files every 10 steps
    L = 6
    m = expert.hubbard(L, expert.chain_bonds(L), 1.0, 4.0, 3, 3, calc_type="TimeEvolution", lanczos_max=30,
                       expec_interval=10, input_eigenvec=1, spectrum_vec="zvo_eigenvec_0", expand_coef=4,
                       output_eigenvec=1, output_interval=10)
    m.greenone = [(i, s, i, s) for i in range(L) for s in (0, 1)] + [(0, 0, 1, 0), (1, 0, 0, 0), (2, 1, 4, 1)]
    m.greentwo = [(i, 0, i, 0, (i + 1) % L, 1, (i + 1) % L, 1) for i in range(L)]
    steps = []
    for k, t in enumerate(_te_times(30, 0.02)):
        v = 0.5 * math.cos(2.0 * t)
        rows = []
        for x in range(L):
            f = (x + 1) % L
            r = (x, 0, f, 0, f, 1, x, 1)
            rows.append(r + (v, 0.0))
            rows.append((r[6], r[7], r[4], r[5], r[2], r[3], r[0], r[1], v, 0.0))
        rows.append((0, 0, 0, 0, 3, 1, 3, 1, 0.3 * t, 0.0))
        steps.append((t, rows))
    m.te_twobody = steps
    cases["te_hub_chain6_two"] = (m, 11)
    # the same chain driven by a Peierls phase on the hoppings, t e^{i A(t)}, with a site
    # potential; non-uniform time steps with one repeated time, ExpandCoef 10
    m = expert.hubbard(L, [], 1.0, 4.0, 3, 3, calc_type="TimeEvolution", lanczos_max=25, expec_interval=6,
                       input_eigenvec=1, spectrum_vec="zvo_eigenvec_0", expand_coef=10)
    m.greenone = [(i, s, i, s) for i in range(L) for s in (0, 1)] + [(0, 0, 1, 0), (1, 0, 0, 0)]
    steps = []
    times = [0.03 * k + 0.002 * k * k for k in range(25)]
    times[7] = times[6]
    for t in times:
        a = 0.8 * math.sin(3.0 * t)
        rows = []
        for x in range(L):
            f = (x + 1) % L
            for sg in (0, 1):
                rows.append((x, sg, f, sg, math.cos(a), math.sin(a)))
                rows.append((f, sg, x, sg, math.cos(a), -math.sin(a)))
        rows.append((2, 0, 2, 0, 0.5 * math.cos(t), 0.0))
        steps.append((t, rows))
    m.te_onebody = steps
    cases["te_hub_chain6_one"] = (m, 12)
    # Heisenberg chain L=10 (Sz=0): the exchange of every bond modulated in time through
    # TETwoBody spin rows plus a time-dependent Ising-type row; ExpandCoef 6
    L = 10
    m = expert.heisenberg(L, expert.chain_bonds(L), 1.0, calc_type="TimeEvolution", lanczos_max=30,
                          input_eigenvec=1, spectrum_vec="zvo_eigenvec_0", expand_coef=6, expec_interval=15)
    m.greenone = [(i, s, i, s) for i in range(L) for s in (0, 1)]
    steps = []
    for t in _te_times(30, 0.05):
        j = 0.5 * (1.0 + 0.5 * math.sin(t))
        rows = []
        for x in range(L):
            f = (x + 1) % L
            rows.append((x, 0, x, 1, f, 1, f, 0, j, 0.0))
            rows.append((f, 0, f, 1, x, 1, x, 0, j, 0.0))
        rows.append((0, 1, 0, 1, 5, 1, 5, 1, 0.2 * t, 0.0))
        steps.append((t, rows))
    m.te_twobody = steps
    cases["te_spin_chain10_two"] = (m, 13)
    # HubbardGC chain L=4 (dim 256): Peierls-phase hoppings and a time-dependent spin-flip
    # transfer on site 1 (grand-canonical: no sector to keep), ExpandCoef 5
    L = 4
    m = expert.ExpertModel(model="HubbardGC", nsite=L, two_sz=None, calc_type="TimeEvolution", lanczos_max=20,
                           input_eigenvec=1, spectrum_vec="zvo_eigenvec_0", expand_coef=5, expec_interval=10)
    m.coulombintra = [(i, 3.0) for i in range(L)]
    m.greenone = [(i, s, i, s) for i in range(L) for s in (0, 1)] + [(1, 0, 1, 1), (1, 1, 1, 0)]
    steps = []
    for t in _te_times(20, 0.05):
        a, h = 0.6 * math.sin(2.0 * t), 0.3 * math.cos(t)
        rows = []
        for x in range(L):
            f = (x + 1) % L
            for sg in (0, 1):
                rows.append((x, sg, f, sg, math.cos(a), math.sin(a)))
                rows.append((f, sg, x, sg, math.cos(a), -math.sin(a)))
        rows += [(1, 0, 1, 1, h, 0.1 * t), (1, 1, 1, 0, h, -0.1 * t)]
        steps.append((t, rows))
    m.te_onebody = steps
    cases["te_hubgc_chain4_one"] = (m, 14)
    # Kondo chain of 3 cells (conduction sites 0, 2, 4; local spins 1, 3, 5; 3 electrons):
    # the local-conduction exchange of every cell modulated in time through TETwoBody, plus a
    # time-dependent density-density row on the conduction sites; ExpandCoef 3
    m = expert.kondo_chain(3, 1.0, 2.0, U=1.0, calc_type="TimeEvolution", lanczos_max=20, input_eigenvec=1,
                           spectrum_vec="zvo_eigenvec_0", expand_coef=3, expec_interval=10)
    m.greenone = [(i, s, i, s) for i in range(6) for s in (0, 1)] + [(0, 0, 2, 0), (2, 0, 0, 0)]
    steps = []
    for t in _te_times(20, 0.05):
        jt = 0.5 + 0.4 * math.sin(3.0 * t)
        rows = []
        for c in range(3):
            l, e = 2 * c + 1, 2 * c
            rows.append((l, 0, l, 1, e, 1, e, 0, jt, 0.0))
            rows.append((l, 1, l, 0, e, 0, e, 1, jt, 0.0))
        rows.append((0, 0, 0, 0, 2, 1, 2, 1, 0.2 * t, 0.0))
        steps.append((t, rows))
    m.te_twobody = steps
    cases["te_kondo_chain3_two"] = (m, 15)
    return cases


def make_te_case(name: str, m, seed: int) -> None:
    import hphi_oracle as O
    out = os.path.join(HERE, name)
    shutil.rmtree(out, ignore_errors=True)
    m.write(out)
    d = O.read_expert(os.path.join(out, "namelist.def"))
    dim = (1 << O.nbits(d)) if O._rows_are_configs(d) else len(O.sz(d)[0]) - 1
    rng = np.random.default_rng(seed)
    v = np.zeros(dim + 1, dtype=np.complex128)
    v[1:] = rng.standard_normal(dim) + 1j * rng.standard_normal(dim)
    v[1:] /= np.linalg.norm(v[1:])
    data = {"start": v}
    with tempfile.TemporaryDirectory() as tmp:
        for f in os.listdir(out):
            shutil.copy(os.path.join(out, f), tmp)
        od = os.path.join(tmp, "output")
        os.makedirs(od)
        with open(os.path.join(od, "zvo_eigenvec_0_rank_0.dat"), "wb") as f:
            f.write(np.array([0], dtype=np.int32).tobytes())
            f.write(np.array([dim], dtype=np.int64).tobytes())
            f.write(v.tobytes())
        p = run_ref.run(tmp, threads=1)
        if p.returncode != 0:
            raise RuntimeError(f"{name}: reference failed\n{p.stdout[-3000:]}\n{p.stderr[-3000:]}")
        for base in ("SS", "Norm", "Flct"):
            data["text_" + base] = np.array(open(os.path.join(od, base + ".dat")).read())
        files = sorted(f for f in os.listdir(od) if "cisajs" in f or "Body" in f)
        data["green_files"] = np.array(files)
        for f in files:
            data["text_" + f] = np.array(open(os.path.join(od, f)).read())
        for f in sorted(os.listdir(od)):
            if f.startswith("zvo_eigenvec_"):
                data["vec_" + f] = _read_eigvec(os.path.join(od, f))
    np.savez_compressed(os.path.join(out, "golden.npz"), **data)


def main(argv) -> None:
    if not run_ref.available():
        raise SystemExit("oracle/_ref/HPhi_ref is missing: run `make -C oracle` first")
    small, large, starts, restarts = _cases(), _large_cases(), _start_cases(), _restart_cases()
    greens, tpq_restarts, lobpcg_restarts = _green_cases(), _tpq_restart_cases(), _lobpcg_restart_cases()
    tes = _te_cases()
    names = argv or (list(small) + list(large) + list(starts) + list(restarts) + list(greens) + list(tpq_restarts)
                     + list(lobpcg_restarts) + list(tes))
    for n in names:
        print("case", n, flush=True)
        if n in small:
            make_case(n, small[n])
        elif n in starts:
            make_start_case(n, *starts[n])
        elif n in restarts:
            make_restart_case(n, *restarts[n])
        elif n in greens:
            make_green_case(n, greens[n])
        elif n in tpq_restarts:
            make_tpq_restart_case(n, *tpq_restarts[n])
        elif n in lobpcg_restarts:
            make_lobpcg_restart_case(n, *lobpcg_restarts[n])
        elif n in tes:
            make_te_case(n, *tes[n])
        else:
            make_case(n, large[n], large=True)


if __name__ == "__main__":
    main(sys.argv[1:])

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


def _neighbours(tmp_path, lattice, extra, model="SpinGC"):
    """Sites and, per site, the set of sites it shares an InterAll (spin) bond with."""
    p = tmp_path / "stan.in"
    # the ladder has no direction-free J (rungs J0, legs J1)
    coupling = "J0 = 1.0\nJ1 = 1.0\n" if lattice == "ladder" else "J = 1.0\n"
    p.write_text(f'model = "{model}"\nmethod = "Lanczos"\nlattice = "{lattice}"\n' + coupling + extra)
    hphi_b200.standard_mode(str(p), str(tmp_path))
    mod = dict(l.split()[:2] for l in open(tmp_path / "modpara.def") if len(l.split()) >= 2)
    n = int(mod["Nsite"])
    nb = {i: set() for i in range(n)}
    for l in open(tmp_path / "interall.def").read().split("\n")[5:]:
        r = l.split()
        if len(r) == 10 and r[0] != r[4]:
            nb[int(r[0])].add(int(r[4]))
            nb[int(r[4])].add(int(r[0]))
    return n, nb


@pytest.mark.parametrize("lattice,extra,nsite,z", [
    ("chain", "L = 8\n", 8, 2),
    ("ladder", "L = 4\nW = 2\n", 8, 3),
    ("square", "W = 4\nL = 4\n", 16, 4),
    ("triangular", "W = 3\nL = 3\n", 9, 6),
    ("honeycomb", "W = 3\nL = 3\n", 18, 3),
    ("kagome", "W = 2\nL = 2\n", 12, 4),
])
def test_nearest_neighbour_coordination(lattice, extra, nsite, z, tmp_path):
    """Every site of the periodic clusters has the lattice's coordination number, and the
    couplings are symmetric (checked through the written InterAll bonds)."""
    n, nb = _neighbours(tmp_path, lattice, extra)
    assert n == nsite
    assert all(len(v) == z for v in nb.values()), {i: len(v) for i, v in nb.items()}


def test_kondo_lattice_layout(tmp_path):
    """Kondo chain: local spins 0..L-1 first, conduction orbitals L..2L-1, local spin n coupled to
    orbital L + n, hoppings only between conduction orbitals."""
    p = tmp_path / "stan.in"
    p.write_text('L = 4\nmodel = "Kondo"\nmethod = "Lanczos"\nlattice = "chain"\nt = 1.0\nJ = 4.0\n'
                 'nelec = 4\n2Sz = 0\n')
    hphi_b200.standard_mode(str(p), str(tmp_path))
    loc = [l.split() for l in open(tmp_path / "locspn.def").read().split("\n")[5:] if l.strip()]
    assert [int(r[1]) for r in loc] == [1, 1, 1, 1, 0, 0, 0, 0]
    hops = [l.split() for l in open(tmp_path / "trans.def").read().split("\n")[5:] if l.strip()]
    assert hops and all(int(r[0]) >= 4 and int(r[2]) >= 4 for r in hops)
    pairs = {tuple(sorted((int(r[0]), int(r[4])))) for r in
             (l.split() for l in open(tmp_path / "interall.def").read().split("\n")[5:]) if len(r) == 10}
    assert pairs == {(n, 4 + n) for n in range(4)}


def test_command_line_dry_run_writes_the_expert_files(tmp_path):
    """`HPhi_b200 -sdry stan.in` only writes the files (no device is touched)."""
    import subprocess
    (tmp_path / "stan.in").write_text('L = 6\nmodel = "Spin"\nmethod = "TPQ"\nlattice = "chain"\nJ = 1.0\n'
                                      '2Sz = 0\nNumAve = 3\n')
    p = subprocess.run([R.ENGINE_EXE, "-sdry", "stan.in"], cwd=tmp_path, capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    names = [l.split()[1] for l in open(tmp_path / "namelist.def") if l.strip()]
    assert {"modpara.def", "calcmod.def", "locspn.def", "trans.def", "interall.def"} <= set(names)
    calc = dict(l.split()[:2] for l in open(tmp_path / "calcmod.def") if l[0] != "#" and len(l.split()) >= 2)
    assert calc["CalcType"] == "1" and calc["CalcModel"] == "1"


def test_geometry_file_matches_the_documented_example(tmp_path):
    """The Fourier utility's geometry.dat for a0 = (2, 2), a1 = (-2, 2) on the square lattice,
    as printed in doc/en/source/fourier/format.rst: unit vectors, phases, the numerical cell
    and the eight cells in the order the standard mode numbers them."""
    p = tmp_path / "stan.in"
    p.write_text('a0W = 2\na0L = 2\na1W = -2\na1L = 2\nmodel = "Hubbard"\nmethod = "Lanczos"\n'
                 'lattice = "square"\nt = 1.0\nU = 4.0\nnelec = 8\n2Sz = 0\n')
    hphi_b200.standard_mode(str(p), str(tmp_path))
    rows = [l.split() for l in open(tmp_path / "geometry.dat") if l.strip()]
    assert [[float(x) for x in r] for r in rows[:4]] == [[1, 0, 0], [0, 1, 0], [0, 0, 1], [0, 0, 0]]
    assert rows[4:7] == [["2", "2", "0"], ["-2", "2", "0"], ["0", "0", "1"]]
    assert [" ".join(r) for r in rows[7:]] == ["0 0 0 0", "-1 1 0 0", "0 1 0 0", "1 1 0 0", "-1 2 0 0",
                                              "0 2 0 0", "1 2 0 0", "0 3 0 0"]


# Lattice geometry (primitive vectors, orbital positions in fractional coordinates) and the
# distances of the first three neighbour shells, from the lattice figures of the reference's
# documentation; used to build hopping matrices independently of the generator's bond tables.
_TRI = [[1.0, 0.0], [0.5, 3 ** 0.5 / 2]]
_GEOMETRY = {
    "chain": ([[1.0, 0.0], [0.0, 1.0]], [[0, 0]], [1.0, 2.0, 3.0]),
    "square": ([[1.0, 0.0], [0.0, 1.0]], [[0, 0]], [1.0, 2 ** 0.5, 2.0]),
    "triangular": (_TRI, [[0, 0]], [1.0, 3 ** 0.5, 2.0]),
    "honeycomb": (_TRI, [[0, 0], [1 / 3, 1 / 3]], [1 / 3 ** 0.5, 1.0, 2 / 3 ** 0.5]),
    "kagome": (_TRI, [[0, 0], [0.5, 0], [0, 0.5]], [0.5, 3 ** 0.5 / 2]),
}


@pytest.mark.parametrize("lattice,cell", [
    ("chain", "L = 7\n"),
    ("square", "W = 4\nL = 3\n"),
    ("square", "a0W = 2\na0L = 2\na1W = -2\na1L = 2\n"),
    ("triangular", "a0W = 3\na0L = 0\na1W = -1\na1L = 2\n"),
    ("triangular", "W = 4\nL = 4\n"),
    ("honeycomb", "W = 3\nL = 2\n"),
    ("honeycomb", "a0W = 2\na0L = 2\na1W = 1\na1L = -2\n"),
    ("kagome", "a0W = 1\na0L = 1\na1W = -1\na1L = 2\n"),
    ("kagome", "W = 3\nL = 2\n"),
])
def test_hoppings_follow_the_lattice_geometry(lattice, cell, tmp_path):
    """The one-body matrix the generator writes (t, t', t'' = 1, 0.3, 0.17) equals the one built
    from the site positions alone: every pair of sites, periodic images included, at the first,
    second or third neighbour distance is joined by -t of that shell."""
    import numpy as np
    prim, orbs, shells = _GEOMETRY[lattice]
    ts = [1.0, 0.3, 0.17][:len(shells)]
    p = tmp_path / "stan.in"
    hop = "".join(f"t{q} = {v}\n" for q, v in zip(["", "'", "''"], ts))
    p.write_text(f'model = "HubbardGC"\nmethod = "Lanczos"\nlattice = "{lattice}"\n' + hop + cell)
    hphi_b200.standard_mode(str(p), str(tmp_path))
    geo = [l.split() for l in open(tmp_path / "geometry.dat") if l.strip()]
    box = np.array([[float(x) for x in r[:2]] for r in geo[4:6]])
    sites = [(float(r[0]), float(r[1]), int(r[3])) for r in geo[7:]]
    n = len(sites)
    h_gen = np.zeros((n, n), dtype=complex)
    for r in open(tmp_path / "trans.def").read().split("\n")[5:]:
        r = r.split()
        if len(r) == 6 and r[1] == "0" and r[3] == "0":
            h_gen[int(r[0]), int(r[2])] -= complex(float(r[4]), float(r[5]))
    prim = np.array(prim)
    pos = np.array([(np.array([w, l]) + np.array(orbs[o])) @ prim for w, l, o in sites])
    h_geo = np.zeros((n, n))
    for i in range(n):
        for j in range(n):
            for n0 in range(-3, 4):
                for n1 in range(-3, 4):
                    if lattice == "chain" and n1 != 0:
                        continue
                    d = np.linalg.norm(pos[j] + (n0 * box[0] + n1 * box[1]) @ prim - pos[i])
                    for shell, t in zip(shells, ts):
                        if abs(d - shell) < 1e-9:
                            h_geo[i, j] -= t
    np.testing.assert_allclose(h_gen, h_geo, atol=1e-12)


# Bond direction of each direction-resolved hopping (t0, t1, t2 and their primed forms) in
# fractional coordinates, as drawn in the reference's lattice figures (doc/figs/*.png).
_LABELS = {
    "square": {"t0": (1, 0), "t1": (0, 1), "t0'": (1, 1), "t1'": (1, -1), "t0''": (2, 0), "t1''": (0, 2)},
    "triangular": {"t0": (1, 0), "t1": (0, 1), "t2": (-1, 1), "t0'": (-1, 2), "t1'": (2, -1), "t2'": (1, 1),
                   "t0''": (2, 0), "t1''": (0, 2), "t2''": (-2, 2)},
    "honeycomb": {"t0": (1 / 3, 1 / 3), "t1": (2 / 3, -1 / 3), "t2": (-1 / 3, 2 / 3)},
    "kagome": {"t0": (-0.5, 0.5), "t1": (0, 0.5), "t2": (0.5, 0)},
}


@pytest.mark.parametrize("lattice", sorted(_LABELS))
def test_direction_resolved_hoppings_follow_the_figures(lattice, tmp_path):
    """Each direction-resolved hopping joins sites displaced along the bond its figure shows."""
    import numpy as np
    prim, orbs, _ = _GEOMETRY[lattice]
    labels = _LABELS[lattice]
    value = {lab: 1.0 + 0.1 * k for k, lab in enumerate(labels)}
    p = tmp_path / "stan.in"
    p.write_text(f'model = "HubbardGC"\nmethod = "Lanczos"\nlattice = "{lattice}"\nW = 5\nL = 5\n' +
                 "".join(f"{lab} = {v}\n" for lab, v in value.items()))
    hphi_b200.standard_mode(str(p), str(tmp_path))
    geo = [l.split() for l in open(tmp_path / "geometry.dat") if l.strip()]
    box = np.array([[float(x) for x in r[:2]] for r in geo[4:6]])
    frac = np.array([[float(r[0]) + orbs[int(r[3])][0], float(r[1]) + orbs[int(r[3])][1]] for r in geo[7:]])
    seen = set()
    for r in open(tmp_path / "trans.def").read().split("\n")[5:]:
        r = r.split()
        if len(r) != 6 or r[1] != "0" or r[3] != "0" or r[0] == r[2]:
            continue
        i, j, t = int(r[0]), int(r[2]), float(r[4])
        d = frac[i] - frac[j]   # the entry is -t c+_i c_j: a hop from j to i
        d = d - np.round(np.linalg.solve(box.T, d)) @ box    # minimal image in the 5x5 cell
        match = [lab for lab, v in labels.items() if np.allclose(np.abs(d), np.abs(v)) and
                 (np.allclose(d, v) or np.allclose(d, -np.array(v)))]
        assert len(match) == 1, (i, j, d)
        assert abs(t - value[match[0]]) < 1e-12, (match[0], t)
        seen.add(match[0])
    assert seen == set(labels)

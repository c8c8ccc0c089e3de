"""Pins the CPU oracle to the reference: every golden fixture was produced by the
reference HPhi itself (tests/golden/make_golden.py); the oracle must reproduce it."""
import numpy as np
import pytest

import hphi_oracle as O
from conftest import case_dir, golden_cases, load_golden


@pytest.mark.parametrize("name", golden_cases("small"))
def test_oracle_lists_and_diagonal(name):
    g = load_golden(name)
    d = O.read_expert(case_dir(name) + "/namelist.def")
    lists = None
    if "list_1" in g:
        lists = O.sz(d)
        for a, b in zip(lists, (g["list_1"], g["list_2_1"], g["list_2_2"])):
            assert a.dtype == np.uint64 and np.array_equal(a, b)
    diag = O.diagonalcalc(d, lists)
    np.testing.assert_allclose(diag, g["diag"], rtol=0, atol=1e-13)


@pytest.mark.parametrize("name", golden_cases("small"))
def test_oracle_mltply(name):
    g = load_golden(name)
    d = O.read_expert(case_dir(name) + "/namelist.def")
    lists = O.sz(d) if "list_1" in g else None
    diag = O.diagonalcalc(d, lists)
    v0, pr = O.mltply(d, lists, diag, np.zeros_like(g["hv0_v1"]), g["hv0_v1"])
    scale = np.max(np.abs(g["hv0_v0a"]))
    assert np.max(np.abs(v0 - g["hv0_v0a"])) <= 1e-12 * scale
    assert abs(pr - complex(g["hv0_pr"])) <= 1e-12 * max(1.0, abs(complex(g["hv0_pr"])))
    if "hv3_v1" in g:
        v0, pr = O.mltply(d, lists, diag, g["hv3_v0b"], g["hv3_v1"])
        scale = np.max(np.abs(g["hv3_v0a"]))
        assert np.max(np.abs(v0 - g["hv3_v0a"])) <= 1e-12 * scale


def ritz_table(alpha, beta, steps):
    """Lowest four eigenvalues of the stp x stp tridiagonal matrix for each stp."""
    out = []
    for s in steps:
        T = np.diag(alpha[:s]) + np.diag(beta[:s - 1], 1) + np.diag(beta[:s - 1], -1)
        e = np.linalg.eigvalsh(T)
        out.append(np.concatenate([e[:4], np.full(4 - min(4, s), np.nan)]))
    return np.array(out)


def check_lanczos_against_reference(g, E1, alpha, beta, nsteps_checked=30):
    """Lanczos without reorthogonalisation amplifies rounding differences once Ritz values
    converge (ghost copies appear at different steps), so parity is checked on the
    ground-state energy at convergence (1e-10) and on the Ritz values E[1..4] of the
    early steps, printed by the reference with 10 decimals."""
    ref_last = g["step_vals"][-1]
    assert abs(E1 - ref_last[0]) < 1e-10 + 5e-11
    steps = [int(s) for s in g["steps"] if s <= min(nsteps_checked, len(alpha))]
    mine = ritz_table(alpha, beta, steps)
    ref = g["step_vals"][: len(steps), :4]
    ok = ~np.isnan(ref) & ~np.isnan(mine)
    assert np.all(np.abs(mine[ok] - ref[ok]) < 1e-9)


@pytest.mark.parametrize("name", golden_cases("lanczos"))
def test_oracle_lanczos_eigenvalue(name):
    g = load_golden(name)
    d = O.read_expert(case_dir(name) + "/namelist.def")
    lists = O.sz(d) if "list_1" in g else None
    diag = O.diagonalcalc(d, lists)
    stp, et, E, alpha, beta = O.lanczos_eigenvalues(d, lists, diag, g["hv0_v1"])
    check_lanczos_against_reference(g, E[0], alpha, beta)


def tridiag_lowest(alpha, beta, k):
    n = len(alpha)
    T = np.diag(alpha) + np.diag(beta[:n - 1], 1) + np.diag(beta[:n - 1], -1)
    return float(np.linalg.eigvalsh(T)[k])


@pytest.mark.parametrize("name", golden_cases("eigenvector"))
def test_oracle_eigenvector_and_cg_refinement(name):
    """Lanczos eigenvector, the accuracy check of CalcByLanczos (eps_Energy 1e-12) and the
    CG refinement against the reference's zvo_energy.dat.  The refined vector does not
    depend on the random components added to b (the reference's come from dSFMT)."""
    g = load_golden(name)
    d = O.read_expert(case_dir(name) + "/namelist.def")
    lists = O.sz(d) if "list_1" in g else None
    diag = O.diagonalcalc(d, lists)
    _, _, _, alpha, beta = O.lanczos_eigenvalues(d, lists, diag, g["hv0_v1"])
    lam = tridiag_lowest(alpha, beta, d.k_exct - 1)
    v = O.lanczos_eigenvector(d, lists, diag, g["hv0_v1"], alpha, beta, d.k_exct - 1)
    e, var, dbl, sz = O.expec_energy(d, lists, diag, v)
    accurate = abs(lam - e) / abs(lam) < 1e-12 and abs(var - e * e) / abs(var) < 1e-12
    assert accurate == (not bool(g["cg_ran"]))
    if not accurate and d.calc_eigenvec == 0:
        noise = 0.002 * (np.random.default_rng(5).random(v.size - 1) - 0.5)
        x, rounds, iters = O.cg_eigenvector(d, lists, diag, v, lam, noise)
        assert 1 <= rounds <= 51 and iters >= 1
        e, var, dbl, sz = O.expec_energy(d, lists, diag, x)
        assert abs(var - e * e) / abs(var) < 1e-12
    ref = g["energy_state"]
    assert abs(e - ref[0]) < 1e-10 * max(1.0, abs(ref[0]))
    assert abs(dbl - ref[1]) < 1e-9
    assert abs(sz - ref[2]) < 1e-9


@pytest.mark.parametrize("name", golden_cases("tpq"))
def test_oracle_tpq_energies(name):
    g = load_golden(name)
    d = O.read_expert(case_dir(name) + "/namelist.def")
    lists = O.sz(d) if "list_1" in g else None
    diag = O.diagonalcalc(d, lists)
    ref = g["tpq"]
    e = O.tpq_energies(d, lists, diag, g["hv0_v1"], ref.shape[0])
    np.testing.assert_allclose(e, ref[:, 1], rtol=1e-10, atol=1e-12)


def lobpcg_start(d, g):
    """The reference's start vectors: single-element ones for initial_iv > 0 on canonical
    models (Initialize_wave, src/CalcByLOBPCG.c:220-251), else its random ones (one thread,
    as the fixtures were made; the first equals the dumped first mltply input)."""
    import hphi_b200
    dim = g["diag"].size - 1
    k = d.k_exct
    if "list_1" not in g or d.initial_iv <= 0:
        x0 = hphi_b200.reference_start(dim, hphi_b200.REF_LOBPCG, d.initial_iv, 0, d.initial_vec_type, 1, k)
        assert np.max(np.abs(x0[0, 1:] - g["hv0_v1"][1:])) < 1e-15
        return x0
    x0 = np.zeros((k, dim + 1), complex)
    for ie in range(k):
        iv = (dim // 2 + d.initial_iv + ie) % dim + 1
        if iv < dim:
            x0[ie, iv + 1] = 1.0 if d.initial_vec_type == 1 else (1 + 1j) / np.sqrt(2)
    return x0


@pytest.mark.parametrize("name", golden_cases("lobpcg"))
def test_oracle_lobpcg_matches_reference(name):
    g = load_golden(name)
    d = O.read_expert(case_dir(name) + "/namelist.def")
    lists = O.sz(d) if "list_1" in g else None
    diag = O.diagonalcalc(d, lists)
    rows, x = O.lobpcg(d, lists, diag, lobpcg_start(d, g))
    ref = g["lobpcg_steps"]
    assert rows.shape[0] == ref.shape[0]
    # the step file prints 6 significant digits; residuals near 1e-7 of degenerate states
    # differ by rounding at the 1e-11 level
    np.testing.assert_allclose(rows[:, 1:], ref[:, 1:], rtol=1e-5, atol=1e-10)
    H = O.dense_hamiltonian(d, lists, diag)
    e = np.real(np.sum(x.conj() * (x @ H.T), axis=1))
    np.testing.assert_allclose(e, g["lobpcg_states"][:, 0], rtol=0, atol=1e-12)


def _green_vector(O, d, lists, z, fname):
    if "step" in fname:
        from conftest import tpq_state
        return tpq_state(O, d, lists, z["start"], int(fname.split("step")[1].split(".")[0]))
    k = int(fname.split("eigen")[1].split(".")[0]) if "eigen" in fname else 0
    return z[f"vec_zvo_eigenvec_{k}_rank_0.dat"]


@pytest.mark.parametrize("name", golden_cases("green"))
def test_oracle_green_functions_match_reference(name):
    """expec_cisajs / expec_cisajscktaltdc (and the three-, four-, six-body functions)
    restated: every value the reference printed (%.10lf) for the eigenvector(s) it wrote, or
    for its TPQ states, with the same rows (and the same empty files)."""
    from conftest import check_green_lines, oracle_green_file
    z = load_golden(name)
    d = O.read_expert(case_dir(name) + "/namelist.def")
    lists = None if O._rows_are_configs(d) else O.sz(d)
    for f in (str(x) for x in z["green_files"]):
        lines = str(z["text_" + f]).splitlines()
        rows, vals = oracle_green_file(O, d, lists, _green_vector(O, d, lists, z, f), f)
        check_green_lines(lines, rows, vals, 1e-10)


def _known_answers():
    import json
    import os
    from conftest import GOLDEN
    base = os.path.join(GOLDEN, "known_answers")
    exp = json.load(open(os.path.join(base, "expected.json")))
    return base, exp


@pytest.mark.parametrize("name", sorted(_known_answers()[1]))
def test_oracle_reproduces_reference_test_values(name):
    """The reference's own known-answer tests (test/*.sh, standard-mode inputs) in expert
    mode: the oracle's lowest eigenvalues of the same Hamiltonian equal the values those
    tests check (1e-10), and so does the ground state's doublon."""
    import os
    base, exp = _known_answers()
    from scipy.sparse.linalg import LinearOperator, eigsh
    d = O.read_expert(os.path.join(base, name, "namelist.def"))
    lists = None if O._rows_are_configs(d) else O.sz(d)
    diag = O.diagonalcalc(d, lists)
    dim = diag.size - 1

    def hv(x):
        v1 = np.zeros(dim + 1, dtype=np.complex128)
        v1[1:] = np.ravel(x)
        return O.mltply(d, lists, diag, np.zeros_like(v1), v1)[0][1:]

    want = np.array(exp[name])
    op = LinearOperator((dim, dim), matvec=hv, dtype=np.complex128)
    w, V = eigsh(op, k=len(want) + 1, which="SA", tol=1e-14, v0=np.ones(dim, dtype=np.complex128))
    order = np.argsort(w)
    w, V = w[order], V[:, order]
    np.testing.assert_allclose(w[:len(want)], want[:, 0], rtol=0, atol=1e-10)
    v = np.zeros(dim + 1, dtype=np.complex128)
    v[1:] = V[:, 0]
    _, _, doublon, _ = O.expec_energy(d, lists, diag, v)
    assert abs(doublon - want[0, 1]) < 1e-10

"""Expert-mode equivalents of standard-mode tests of the reference (test/*.sh), with the
values those tests check (their reference.dat blocks: energy, doublon, Sz per state).

The reference's standard mode (StdFace) is absent here, so each input is written in expert
mode for the same Hamiltonian: the energies do not depend on how the sites are numbered.
  lanczos_kondo_chain    test/lanczos_kondo_chain.sh:6-26     Kondo chain L=4, t=1, J=4, nelec=4, 2Sz=0
  lanczos_kondogc_chain  test/lanczos_kondogc_chain.sh:6-24   the same, KondoGC
  lanczos_genspin_ladder test/lanczos_genspin_ladder.sh:6-27  S=3/2 ladder L=3 W=2, J0=J1=1, 2Sz=0
  lobcg_genspin_ladder   test/lobcg_genspin_ladder.sh:6-34    the same with D=0.2 S_z^2, two states
  lobcg_hubbard_square   test/lobcg_hubbard_square.sh:6-38    Hubbard 4x2 periodic (the length-2
                                                              direction's bond counted twice, as
                                                              the reference's lattice does), t=1,
                                                              U=4, nelec=8, 2Sz=0, three states
  lobcg_kondo_chain      test/lobcg_kondo_chain.sh:6-32       Kondo chain of the first case, two states

Run:  python tests/golden/known_answers/make_known_answers.py   (writes the inputs here)
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(HERE))))
from hphi_b200 import expert  # noqa: E402

# (energy, doublon, Sz) per state, as printed in the reference's test scripts
EXPECTED = {
    "lanczos_kondo_chain": [[-12.6776213781764451, 0.1072445462409946, 0.0]],
    "lanczos_kondogc_chain": [[-12.6776213781764451, 0.1072445462409946, 0.0]],
    "lanczos_genspin_ladder": [[-18.1042786817898147, 0.0, 0.0]],
    "lobcg_genspin_ladder": [[-16.6896771153847965, 0.0, 0.0], [-15.8422975895661722, 0.0, 0.0]],
    "lobcg_hubbard_square": [[-10.2529529552637033, 1.0444442739280635, 0.0],
                             [-9.8328986753266356, 1.1830984216215232, 0.0],
                             [-9.2310650024220635, 1.2843076003322857, 0.0]],
    "lobcg_kondo_chain": [[-12.6776213781764220, 0.1072445462409922, 0.0],
                          [-9.8347989641820277, 0.4289751043491778, 0.0]],
}


def ladder_bonds(L=3, W=2):
    """Legs: periodic rings of L sites; rungs between the W=2 legs."""
    legs = [(y * L + x, y * L + (x + 1) % L) for y in range(W) for x in range(L)]
    return legs + [(x, L + x) for x in range(L)]


def models():
    m = {}
    m["lanczos_kondo_chain"] = expert.kondo_chain(4, 1.0, 4.0, lanczos_max=500, calc_eigenvec=0)
    m["lanczos_kondogc_chain"] = expert.kondo_chain(4, 1.0, 4.0, gc=True, lanczos_max=500, calc_eigenvec=0)
    m["lanczos_genspin_ladder"] = expert.general_heisenberg([3] * 6, ladder_bonds(), lanczos_max=500,
                                                            calc_eigenvec=0)
    m["lobcg_genspin_ladder"] = expert.general_heisenberg([3] * 6, ladder_bonds(), D=0.2, calc_type="CG",
                                                          exct=2, lanczos_max=1000)
    m["lobcg_hubbard_square"] = expert.hubbard(8, expert.square_bonds(4, 2), 1.0, 4.0, 4, 4, calc_type="CG",
                                               exct=3, lanczos_max=1000)
    m["lobcg_kondo_chain"] = expert.kondo_chain(4, 1.0, 4.0, calc_type="CG", exct=2, lanczos_max=1000)
    return m


def main():
    for name, m in models().items():
        m.write(os.path.join(HERE, name))
    with open(os.path.join(HERE, "expected.json"), "w") as f:
        json.dump(EXPECTED, f, indent=1)


if __name__ == "__main__":
    main()

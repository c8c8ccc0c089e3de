"""Time-evolution known answers of the reference's own tests, in expert mode.

test/te_hubbard_chain_interall.sh and test/te_hubbard_chain_interall_diagonal.sh run
test/testTECalc.py: the ground state of the Hubbard chain L=4, t=1, U=4, nelec=4, 2Sz=0
(periodic) is computed first, then evolved for 100 steps of 0.01 under the same chain plus the
TETwoBody InterAll rows of MakeInterAll (test/testTECalc.py:55-73: "Normal"
c+_{x up} c_{x+1 up} c+_{x+1 dn} c_{x dn}, "Diagonal" c+_{x up} c_{x+1 dn} c+_{x+1 dn} c_{x up},
each with its Hermitian partner, value 1) at the times t = 0, 0.01, ... accumulated as
t += 0.01 (PrintTE :101-128).  ExpandCoef is not set in the file the reference reads (the
script appends it to a file named "modpara"), so the step is first order.  The scripts check
Flct.dat (time, N, N^2, D, D^2, Sz, Sz^2, step) against their reference.dat blocks; those rows
are stored here in te_expected.json.  The start state is the chain's ground state, which the
tests compute from the written input (it is non-degenerate).

Run:  python tests/golden/known_answers/make_te_known_answers.py   (reads the reference's
test scripts from $HPHI_REFERENCE/test, by default the checkout beside this repository, and
writes the inputs and te_expected.json here)
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(HERE))))
from hphi_b200 import expert  # noqa: E402

REPO = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))
REF_TEST = os.path.join(os.environ.get("HPHI_REFERENCE", os.path.join(os.path.dirname(REPO), "reference")), "test")
CASES = {"te_hubbard_chain_interall": "Normal", "te_hubbard_chain_interall_diagonal": "Diagonal"}


def reference_rows(script: str):
    lines = open(os.path.join(REF_TEST, script)).read().splitlines()
    start = lines.index("cat > reference.dat <<EOF") + 1
    end = lines.index("EOF", start)
    return [[float(x) for x in l.split()] for l in lines[start:end]]


def model(kind: str):
    L = 4
    m = expert.hubbard(L, expert.chain_bonds(L), 1.0, 4.0, 2, 2, calc_type="TimeEvolution", lanczos_max=100,
                       input_eigenvec=1, spectrum_vec="zvo_eigenvec_0", expec_interval=20)
    pairs = []
    for x in range(L):
        f = (x + 1) % L
        pairs.append((x, 0, f, 0, f, 1, x, 1) if kind == "Normal" else (x, 0, f, 1, f, 1, x, 0))
    rows = []
    for r in pairs:
        rows.append(r + (1.0, 0.0))
        rows.append((r[6], r[7], r[4], r[5], r[2], r[3], r[0], r[1], 1.0, 0.0))
    t, steps = 0.0, []
    for _ in range(100):
        steps.append((t, rows))
        t += 0.01
    m.te_twobody = steps
    return m


def main():
    expected = {}
    for name, kind in CASES.items():
        model(kind).write(os.path.join(HERE, name))
        expected[name] = reference_rows(name + ".sh")
    with open(os.path.join(HERE, "te_expected.json"), "w") as f:
        json.dump(expected, f, indent=1)


if __name__ == "__main__":
    main()

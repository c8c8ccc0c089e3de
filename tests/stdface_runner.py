"""Replays a standard-mode scenario (tests/golden/stdface/<test>.json.gz, made by
tests/golden/make_stdface_golden.py from the reference's test/<test>.sh) in a scratch
directory and checks the values the script checks.

`HPhi -s` / `HPhi -sdry` go through the engine's standard-mode generator (hphi_stdface);
`-e namelist.def` runs on a backend: the engine's command-line program on the GPU, or, as a
check of the generator alone, the reference binary oracle/_ref/HPhi_ref on the CPU.
"""
from __future__ import annotations

import ctypes
import gzip
import json
import os
import shutil
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SCENARIOS = os.path.join(ROOT, "tests", "golden", "stdface")
ENGINE_EXE = os.path.join(ROOT, "hphi_b200", "HPhi_b200")
REF_EXE = os.path.join(ROOT, "oracle", "_ref", "HPhi_ref")


def names():
    return sorted(f[:-8] for f in os.listdir(SCENARIOS) if f.endswith(".json.gz"))


def load(name):
    with gzip.open(os.path.join(SCENARIOS, name + ".json.gz"), "rt") as f:
        return json.load(f)


def _lib():
    lib = ctypes.CDLL(os.path.join(ROOT, "hphi_b200", "libhphi_b200.so"))
    lib.hphi_stdface.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    lib.hphi_stdface.restype = ctypes.c_int
    lib.hphi_last_error.restype = ctypes.c_char_p
    return lib


def generate(stan_in: str, out_dir: str) -> None:
    lib = _lib()
    if lib.hphi_stdface(stan_in.encode(), out_dir.encode()) != 0:
        raise RuntimeError(lib.hphi_last_error().decode())


def _floats(line):
    return [float(t) for t in line.split()]


def compare(path: str, ref: str):
    """(sum of |differences|, problems) between output file `path` and a reference.dat block,
    paired line by line as the script's `paste` does: one-column blocks against the second
    column of the output (zvo_energy.dat), wider blocks column by column (indices exactly)."""
    out = [l for l in open(path).read().split("\n") if l.strip()]
    exp = [l for l in ref.split("\n") if l.strip()]
    problems = []
    if len(out) < len(exp):
        problems.append(f"{os.path.basename(path)}: {len(out)} lines, expected {len(exp)}")
    diff = 0.0
    if "zvo_phys" in path:  # full diagonalisation: eigenvalues (first column) below a header line
        return sum(abs(float(o.split()[0]) - float(e.split()[0])) for o, e in list(zip(out, exp))[1:]), problems
    for o, e in zip(out, exp):
        ef, of = e.split(), o.split()
        if len(ef) == 1:
            diff += abs(float(of[1]) - float(ef[0]))
            continue
        if len(of) != len(ef):
            problems.append(f"columns: {o!r} vs {e!r}")
            continue
        nv = 2 if any("." in t for t in ef[-2:]) else 0
        if "DynamicalGreen" in path:
            nv = 4
        if "flct" in os.path.basename(path).lower():
            nv = len(ef)
        if ef[:len(ef) - nv] != of[:len(of) - nv] and [int(float(t)) for t in ef[:len(ef) - nv]] != \
                [int(float(t)) for t in of[:len(of) - nv]]:
            problems.append(f"indices: {o!r} vs {e!r}")
        diff += sum(abs(a - b) for a, b in zip(_floats(" ".join(of[len(of) - nv:])),
                                               _floats(" ".join(ef[len(ef) - nv:]))))
    return diff, problems


def tpq_average_problems(work: str, ref: str):
    """The reference's TPQ check (test/Ave_SS.py, restated): temperature 1/<beta> and energy
    averaged over the NumAve samples of output/SS_rand*.dat must lie within
    max(2 * the reference's error bar, 1e-8) of the reference's averages."""
    mod = {}
    for line in open(os.path.join(work, "modpara.def")):
        p = line.split()
        if len(p) >= 2:
            mod[p[0]] = p[1]
    nave, nmax = int(mod["NumAve"]), int(mod["Lanczos_max"])
    beta = np.zeros((nave, nmax))
    ene = np.zeros((nave, nmax))
    for s in range(nave):
        rows = [l.split() for l in open(os.path.join(work, "output", f"SS_rand{s}.dat")).read().split("\n")[1:]]
        rows = [r for r in rows if len(r) > 1]
        for k, r in enumerate(rows[:nmax]):
            beta[s, k], ene[s, k] = float(r[0]), float(r[1])
    b_ave, b_err = beta.mean(0), beta.std(0, ddof=1)
    e_ave = ene.mean(0)
    refs = [r.split() for r in ref.split("\n") if len(r.split()) > 1]
    problems = []
    for k, r in enumerate(refs):
        cnt = k + 1
        if cnt >= nmax - 2:
            break
        t = 1.0 / b_ave[cnt]
        rt, rte, re_, ree = float(r[0]), float(r[1]), float(r[2]), float(r[3])
        if abs(rt - t) > max(2 * rte, 1e-8):
            problems.append(f"temperature step {cnt}: {t} vs {rt} +- {rte}")
        if abs(re_ - e_ave[cnt]) > max(2 * ree, 1e-8):
            problems.append(f"energy step {cnt}: {e_ave[cnt]} vs {re_} +- {ree}")
    return problems


def _spectrum_by_lanczos(work: str) -> None:
    """The reference computes spectra of CalcType 3 (CG) inputs by shifted BiCG, a Fortran
    library its binary here is built without; its Lanczos spectrum (CalcType 0) is the same
    Green's function, and the one the engine computes."""
    path = os.path.join(work, "calcmod.def")
    lines = open(path).read().split("\n")
    keys = {l.split()[0]: l.split()[1] for l in lines if len(l.split()) >= 2 and not l.startswith("#")}
    if keys.get("CalcSpec", "0") != "0" and keys.get("CalcType") == "3":
        lines = [("CalcType 0" if l.split()[:1] == ["CalcType"] else l) for l in lines]
        open(path, "w").write("\n".join(lines))


def run(name: str, work: str, backend: str = "engine", env=None, timeout=1200, tol=5e-7):
    """Replays scenario `name` inside `work`; returns a list of problems (empty: it passes).
    The script's own criterion is a summed |difference| that prints as 0.000000 (< 5e-7) per
    reference block."""
    exe = ENGINE_EXE if backend == "engine" else REF_EXE
    sc = load(name)
    os.makedirs(work, exist_ok=True)
    penv = dict(os.environ)
    penv.update(env or {})
    problems = []

    def expert():
        if backend == "reference":
            _spectrum_by_lanczos(work)
        p = subprocess.run([exe, "-e", "namelist.def"], cwd=work, env=penv, capture_output=True, text=True,
                           timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"{backend} run failed: {p.stdout[-1500:]} {p.stderr[-1500:]}")

    for st in sc["steps"]:
        op = st["op"]
        if op == "write":
            open(os.path.join(work, st["file"]), "w").write(st["text"])
        elif op == "append":
            open(os.path.join(work, st["file"]), "a").write(st["text"])
        elif op == "copy":
            shutil.copy(os.path.join(work, st["src"]), os.path.join(work, st["dst"]))
        elif op == "sed":
            p = os.path.join(work, st["file"])
            text = open(p).read()
            open(p, "w").write(text.replace(st["from"], st["to"]))
        elif op == "rm":
            os.remove(os.path.join(work, st["file"]))
        elif op in ("standard", "dry"):
            generate(os.path.join(work, st["file"]), work)
            if op == "standard":
                expert()
        elif op == "expert":
            expert()
        elif op == "drop_first_line":
            lines = open(os.path.join(work, st["src"])).read().split("\n")
            open(os.path.join(work, st["dst"]), "w").write("\n".join(lines[1:]))
        elif op == "import_output":
            src = os.path.join(os.path.dirname(work.rstrip("/")), st["from"], "output")
            shutil.copytree(src, os.path.join(work, "output"), dirs_exist_ok=True)
        elif op == "check":
            path = os.path.join(work, st["file"])
            if not os.path.exists(path):
                problems.append(f"missing {st['file']}")
                continue
            diff, pr = compare(path, st["ref"])
            problems += pr
            # LOBPCG stops at a residual of 10^(-LanczosEps/2) = 1e-7, so every correlation
            # function the reference printed from its eigenvector carries an error of up to
            # ~1e-8; summed over a long file that can exceed the scripts' 5e-7
            limit = max(tol, 2e-8 * len(st["ref"].split("\n"))) if "_eigen" in st["file"] else tol
            if diff >= limit:
                problems.append(f"{st['file']}: summed difference {diff:.3g}")
        elif op == "check_tpq_average":
            problems += tpq_average_problems(work, st["ref"])
        else:
            raise ValueError(op)
    return problems

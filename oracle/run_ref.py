"""Runs the reference HPhi (oracle/_ref/HPhi_ref) on an expert-mode input and reads
back what its link-time hooks (oracle/ref_hooks.c) dumped.  TEST INFRASTRUCTURE ONLY.

Used to generate the golden fixtures (tests/golden/make_golden.py) and as the CPU
baseline of bench.py (the reference timed on the host's cores).
"""
from __future__ import annotations

import os
import subprocess
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "_ref", "HPhi_ref")


def available() -> bool:
    return os.path.exists(REF_BIN)


def run(workdir: str, threads: int = 1, dump_call: int = 0, timeout: Optional[float] = None,
        extra_env: Optional[Dict[str, str]] = None) -> subprocess.CompletedProcess:
    """Runs `HPhi_ref -e namelist.def` inside workdir (which holds the .def files)."""
    env = dict(os.environ)
    env.update({"OMP_NUM_THREADS": str(threads), "HPHI_DUMP_DIR": os.path.abspath(workdir),
                "HPHI_DUMP_CALL": str(dump_call), "OMP_PROC_BIND": "close"})
    if extra_env:
        env.update(extra_env)
    return subprocess.run([REF_BIN, "-e", "namelist.def"], cwd=workdir, env=env, capture_output=True,
                          text=True, timeout=timeout)


def read_lists(workdir: str):
    with open(os.path.join(workdir, "lists.bin"), "rb") as f:
        idim, n21, n22 = np.frombuffer(f.read(24), dtype=np.int64)
        l1 = np.frombuffer(f.read(8 * (idim + 1)), dtype=np.uint64).copy()
        l21 = np.frombuffer(f.read(8 * n21), dtype=np.uint64).copy()
        l22 = np.frombuffer(f.read(8 * n22), dtype=np.uint64).copy()
    return l1, l21, l22


def read_diag(workdir: str) -> np.ndarray:
    with open(os.path.join(workdir, "diag.bin"), "rb") as f:
        idim = int(np.frombuffer(f.read(8), dtype=np.int64)[0])
        return np.frombuffer(f.read(8 * (idim + 1)), dtype=np.float64).copy()


def read_hv(workdir: str):
    """(v1, v0_before, v0_after, prdct) of the dumped mltply call (1-based complex arrays)."""
    with open(os.path.join(workdir, "hv.bin"), "rb") as f:
        idim = int(np.frombuffer(f.read(8), dtype=np.int64)[0])
        n = idim + 1
        v1 = np.frombuffer(f.read(16 * n), dtype=np.complex128).copy()
        v0b = np.frombuffer(f.read(16 * n), dtype=np.complex128).copy()
        v0a = np.frombuffer(f.read(16 * n), dtype=np.complex128).copy()
        pr = complex(np.frombuffer(f.read(16), dtype=np.complex128)[0])
    return v1, v0b, v0a, pr


def read_times(workdir: str) -> np.ndarray:
    with open(os.path.join(workdir, "mltply_times.txt")) as f:
        lines = f.read().split()
    return np.array([float(x) for x in lines[1:]])


def lanczos_steps(workdir: str):
    """Parsed zvo_Lanczos_Step.dat lines: list of (stp, [numbers...])."""
    out = []
    with open(os.path.join(workdir, "output", "zvo_Lanczos_Step.dat")) as f:
        for line in f:
            if not line.startswith("stp"):
                continue
            p = line.replace("stp =", "stp=").replace("=", " ").split()
            stp = int(p[1])
            vals = []
            for tok in p[2:]:
                try:
                    vals.append(float(tok))
                except ValueError:
                    vals.append(None)
            out.append((stp, vals))
    return out


def tpq_table(workdir: str, rand_i: int = 0) -> np.ndarray:
    rows = []
    with open(os.path.join(workdir, "output", f"SS_rand{rand_i}.dat")) as f:
        for line in f:
            if line.lstrip().startswith("#"):
                continue
            rows.append([float(x) for x in line.split()])
    return np.array(rows)


def lobpcg_steps(workdir: str) -> np.ndarray:
    """zvo_Lanczos_Step.dat of a LOBPCG run (src/CalcByLOBPCG.c:445-453): rows of
    (step, largest residual 2-norm, threshold, eigenvalue estimates...)."""
    rows = []
    with open(os.path.join(workdir, "output", "zvo_Lanczos_Step.dat")) as f:
        for line in f:
            p = line.split()
            if not p or not p[0].isdigit():
                continue
            rows.append([float(x) for x in p])
    return np.array(rows)


def energy_states(workdir: str) -> np.ndarray:
    """zvo_energy.dat of a LOBPCG run (src/CalcByLOBPCG.c:736-745): rows (energy, doublon, Sz)."""
    rows, cur = [], {}
    with open(os.path.join(workdir, "output", "zvo_energy.dat")) as f:
        for line in f:
            p = line.split()
            if not p:
                continue
            if p[0] == "State":
                if cur:
                    rows.append([cur["Energy"], cur["Doublon"], cur["Sz"]])
                cur = {}
            elif p[0] in ("Energy", "Doublon", "Sz"):
                cur[p[0]] = float(p[1])
    if cur:
        rows.append([cur["Energy"], cur["Doublon"], cur["Sz"]])
    return np.array(rows)

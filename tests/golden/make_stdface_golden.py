"""Turns the reference's standard-mode test scripts (test/*.sh of HPhi) into fixtures:
tests/golden/stdface/<test>.json.gz holds the script's steps (input files it writes, the HPhi
calls, the sed edits between runs) and the values it checks (its reference.dat blocks with
the output file each is compared against).

The scripts are read as text; nothing of the reference is run.  The subset of shell they use
is interpreted here:

  cat > F <<EOF ... EOF / cat >> F <<EOF ... EOF    write / append a file
  cp A B, sed -i -e "s/X/Y/g" F, rm F               edit between runs
  echo "..." >> F                                    append a line
  HPhi -s F / HPhi -sdry F / HPhi -e namelist.def    the runs
  paste output/X reference.dat                       a check of output/X
  sed -e "1d" output/Flct.dat > flct.dat             (time evolution: Flct.dat without its header)
  python3 .../Ave_SS.py                              the TPQ average check
  cp -rf ../<test>/output .                          output of an earlier test as input

Run where the reference tree is present (REF_TEST overrides its location):
    python tests/golden/make_stdface_golden.py
"""
from __future__ import annotations

import glob
import gzip
import json
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "stdface")
REF_TEST = os.environ.get("REF_TEST", "/root/reference/test")


def parse(path: str):
    lines = open(path).read().split("\n")
    steps = []
    pending_ref = None
    i = 0
    while i < len(lines):
        ln = lines[i].strip()
        i += 1
        m = re.match(r'cat\s+(>>?)\s*(\S+)\s*<<\s*EOF$', ln)
        if m:
            body = []
            while i < len(lines) and lines[i].strip() != "EOF":
                body.append(lines[i])
                i += 1
            i += 1
            text = "\n".join(body) + "\n"
            if m.group(2) == "reference.dat":
                pending_ref = text
            else:
                steps.append({"op": "write" if m.group(1) == ">" else "append", "file": m.group(2), "text": text})
            continue
        if not ln or ln.startswith("#") or ln.startswith("mkdir") or ln.startswith("cd "):
            continue
        m = re.match(r'(?:\$\{MPIRUN\w*\}\s+)?\S*HPhi\s+(-s|-sdry|-e)\s+(\S+)', ln)
        if m:
            op = {"-s": "standard", "-sdry": "dry", "-e": "expert"}[m.group(1)]
            steps.append({"op": op, "file": m.group(2)})
            continue
        m = re.match(r'cp\s+-rf\s+\.\./(\S+)/output\s+\.$', ln)
        if m:
            steps.append({"op": "import_output", "from": m.group(1)})
            continue
        m = re.match(r'cp\s+(\S+)\s+(\S+)$', ln)
        if m:
            steps.append({"op": "copy", "src": m.group(1), "dst": m.group(2)})
            continue
        m = re.match(r'sed\s+-i\s+-e\s+"s/(.*)/(.*)/g"\s+(\S+)$', ln)
        if m:
            steps.append({"op": "sed", "file": m.group(3), "from": m.group(1).replace('\\"', '"'),
                          "to": m.group(2).replace('\\"', '"')})
            continue
        m = re.match(r'sed\s+-e\s+"1d"\s+(\S+)\s*>\s*(\S+)$', ln)
        if m:
            steps.append({"op": "drop_first_line", "src": m.group(1), "dst": m.group(2)})
            continue
        m = re.match(r'rm\s+(\S+)$', ln)
        if m:
            steps.append({"op": "rm", "file": m.group(1)})
            continue
        m = re.match(r'echo\s+"(.*)"\s*>>\s*(\S+)$', ln)
        if m:
            steps.append({"op": "append", "file": m.group(2), "text": m.group(1) + "\n"})
            continue
        m = re.match(r'paste\s+(\S+)\s+reference\.dat', ln)
        if m:
            steps.append({"op": "check", "file": m.group(1), "ref": pending_ref})
            continue
        if "Ave_SS.py" in ln:
            steps.append({"op": "check_tpq_average", "ref": pending_ref})
            continue
        if "testTECalc.py" in ln:
            return None  # driven by a Python script of its own, not a standard-mode input
        # awk / test / exit / diff lines compute the script's own verdict
    return steps


def main():
    os.makedirs(OUT, exist_ok=True)
    n = 0
    for path in sorted(glob.glob(os.path.join(REF_TEST, "*.sh"))):
        name = os.path.basename(path)[:-3]
        steps = parse(path)
        if steps is None or not any(s["op"] in ("standard", "dry") for s in steps):
            continue
        with gzip.open(os.path.join(OUT, name + ".json.gz"), "wt") as f:
            json.dump({"source": "test/" + name + ".sh", "steps": steps}, f)
        n += 1
    print(n, "scenarios")


if __name__ == "__main__":
    main()

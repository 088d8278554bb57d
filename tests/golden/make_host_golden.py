"""Regenerates tests/golden/host/: output files of the reference program mdff20.x that
pin the C host (mdff20gpu.x, libmdffhost).

    make -C oracle ref && python tests/golden/make_host_golden.py

For each case of cases.host_runs() the control file and POSFF (System.write) go into
tests/golden/host/<case>/ together with what oracle/_ref/mdff20.x (the reference's own
main, src/mdff20.c, compiled unchanged) leaves in its working directory: OSZIFF, CONTFF,
TRAJFF, and the thermodynamic blocks of its stdout (stdout_thermo.txt; the rest of its
stdout carries dates and timings).  autoes.json holds alphaES, kES and cutlongrange after
init_field for cases.autoes_cases(), dumped at full precision by the reference harness
(task kmesh).
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from tests.golden import cases  # noqa: E402

OUT = os.path.join(HERE, "host")
EXE = os.path.join(ROOT, "oracle", "_ref", "mdff20.x")
OUTPUTS = ("OSZIFF", "CONTFF", "TRAJFF")


def thermo_blocks(stdout: str) -> str:
    """The info_thermo key-0 blocks (src/thermo.c:36-109) of a stdout stream: from the
    title line to the last "iso" line (one or three stress tensors), plus a blank line."""
    lines = stdout.splitlines(keepends=True)
    out, k = [], 0
    while k < len(lines):
        if not lines[k].startswith("  Thermodynamic information"):
            k += 1
            continue
        j = k
        while j < len(lines):
            if lines[j].startswith("  iso = ") and (j + 3 >= len(lines) or "stress tensor" not in lines[j + 3]):
                break
            j += 1
        out.extend(lines[k:j + 1])
        out.append("\n")
        k = j + 1
    return "".join(out)


def run_case(name, s):
    d = os.path.join(OUT, name)
    os.makedirs(d, exist_ok=True)
    wd = tempfile.mkdtemp(prefix="mdffhost_")
    try:
        s.write(wd)
        env = dict(os.environ, OMP_NUM_THREADS="1")
        p = subprocess.run([EXE, "control.s"], cwd=wd, env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                           timeout=600)
        if p.returncode != 0:
            raise RuntimeError(f"{name}: mdff20.x failed {p.returncode}\n{p.stderr.decode()[-2000:]}")
        for f in ("control.s", "POSFF") + OUTPUTS:
            src = os.path.join(wd, f)
            if os.path.exists(src):
                shutil.copy(src, os.path.join(d, f))
        with open(os.path.join(d, "stdout_thermo.txt"), "w") as fp:
            fp.write(thermo_blocks(p.stdout.decode()))
        print(name, sorted(os.listdir(d)))
    finally:
        shutil.rmtree(wd, ignore_errors=True)


def main():
    if not os.access(EXE, os.X_OK):
        raise SystemExit(f"{EXE} missing: make -C oracle ref")
    for name, s in cases.host_runs().items():
        run_case(name, s)
    auto = {}
    for name, s in cases.autoes_cases().items():
        r = ref.run(s, "kmesh")
        auto[name] = {"alphaES": float(r["alphaES"][0]), "kES": [int(k) for k in r["kES"]],
                      "cutlongrange": float(r["cutlongrange"][0])}
    with open(os.path.join(OUT, "autoes.json"), "w") as fp:
        json.dump(auto, fp, indent=1)
    print(json.dumps(auto))


if __name__ == "__main__":
    main()

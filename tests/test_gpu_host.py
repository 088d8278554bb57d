"""The C host program mdff20gpu.x against the reference program mdff20.x.

Each case of tests/golden/host/ holds a control file, a POSFF and the files the
reference program left after running on them.  mdff20gpu.x runs in a copy of the inputs
and must leave the same files: identical layout (every character except the digits of
the floating-point fields) and numbers within tolerance.  The defaults of mdff20gpu.x
(FP64, the reference's induced-dipole algorithm) are the ones under test, plus one run
with the mixed-precision fused-CG path against the same files at its own tolerance.
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from tests.helpers import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

HOST_GOLDEN = os.path.join(GOLDEN, "host")
EXE = os.path.join(ROOT, "mdff20_b200", "mdff20gpu.x")
NUM = re.compile(r"[-+]?\d+\.\d*(?:[eE][-+]?\d+)?")
MANTISSA_SIGN = re.compile(r"(?<![\deE])-(?=\d)")


def layout(line: str) -> str:
    """The line with every floating-point field masked and mantissa signs blanked (a
    value near zero may change sign)."""
    return NUM.sub("#", MANTISSA_SIGN.sub(" ", line))


CASES = ("pim_nhc", "rigid_equil", "lj_vv", "pim_static", "pim_init")


def run_host(case, wd, *opts):
    for f in ("control.s", "POSFF"):
        shutil.copy(os.path.join(HOST_GOLDEN, case, f), os.path.join(wd, f))
    p = subprocess.run([EXE, *opts, "control.s"], cwd=wd, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                       timeout=600)
    assert p.returncode == 0, p.stderr.decode()[-2000:] + p.stdout.decode()[-2000:]
    return p.stdout.decode()


def thermo_blocks(stdout: str) -> str:
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


def compare_text(got: str, want: str, rtol: float, atol: float, what: str) -> float:
    """Same lines with the same layout; returns the largest relative deviation seen."""
    gl, wl = got.splitlines(), want.splitlines()
    assert len(gl) == len(wl), f"{what}: {len(gl)} lines, reference {len(wl)}"
    worst = 0.0
    for k, (a, b) in enumerate(zip(gl, wl)):
        assert layout(a) == layout(b) and len(a) == len(b), f"{what}:{k + 1}: {a!r} vs {b!r}"
        xa = np.array([float(x) for x in NUM.findall(a)])
        xb = np.array([float(x) for x in NUM.findall(b)])
        if xa.size:
            dev = np.abs(xa - xb)
            assert np.all(dev <= atol + rtol * np.abs(xb)), f"{what}:{k + 1}: {a!r} vs {b!r}"
            worst = max(worst, float(np.max(dev / (atol + rtol * np.abs(xb)))))
    return worst


def compare_case(case, wd, stdout, rtol, atol):
    ref = os.path.join(HOST_GOLDEN, case)
    for f in ("OSZIFF", "CONTFF", "TRAJFF"):
        want_path = os.path.join(ref, f)
        got_path = os.path.join(wd, f)
        assert os.path.exists(got_path) == os.path.exists(want_path), f
        if os.path.exists(want_path):
            compare_text(open(got_path).read(), open(want_path).read(), rtol, atol, f"{case}/{f}")
    want = open(os.path.join(ref, "stdout_thermo.txt")).read()
    compare_text(thermo_blocks(stdout), want, rtol, atol, f"{case}/stdout")


@pytest.mark.parametrize("case", CASES)
def test_host_program_matches_reference(case, tmp_path):
    out = run_host(case, str(tmp_path))
    compare_case(case, str(tmp_path), out, rtol=1e-7, atol=2e-9)


def test_host_program_mixed_fused(tmp_path):
    """The fast path through the same host: layout identical, numbers to the mixed
    precision's force error over six steps."""
    out = run_host("pim_nhc", str(tmp_path), "-p", "mixed", "-s", "cg-fused")
    compare_case("pim_nhc", str(tmp_path), out, rtol=2e-4, atol=2e-5)


def test_host_program_rerun_overwrites(tmp_path):
    """A second run in the same directory starts TRAJFF afresh (check_md removes it) and
    rewrites OSZIFF/CONTFF."""
    run_host("pim_nhc", str(tmp_path))
    first = {f: open(tmp_path / f).read() for f in ("OSZIFF", "CONTFF", "TRAJFF")}
    run_host("pim_nhc", str(tmp_path))
    for f, text in first.items():
        assert open(tmp_path / f).read() == text, f


def test_host_program_restart_continues_exactly(tmp_path):
    """npas 3, then -r RESTART up to npas 6, leaves the files of one 6-step run; a second
    restart from the same step-3 RESTART cuts OSZIFF and TRAJFF back first."""
    full = tmp_path / "full"
    split = tmp_path / "split"
    full.mkdir()
    split.mkdir()
    run_host("pim_nhc", str(full))
    for f in ("control.s", "POSFF"):
        shutil.copy(os.path.join(HOST_GOLDEN, "pim_nhc", f), split / f)
    ctl = (split / "control.s").read_text()
    assert "npas 6" in ctl
    (split / "control.s").write_text(ctl.replace("npas 6", "npas 3"))
    p = subprocess.run([EXE, "control.s"], cwd=split, capture_output=True, timeout=600)
    assert p.returncode == 0, p.stderr.decode()[-2000:]
    shutil.copy(split / "RESTART", split / "RESTART3")
    (split / "control.s").write_text(ctl)
    for attempt in range(2):
        p = subprocess.run([EXE, "-r", "RESTART3", "control.s"], cwd=split, capture_output=True, timeout=600)
        assert p.returncode == 0, p.stderr.decode()[-2000:]
        for f in ("OSZIFF", "CONTFF", "TRAJFF"):
            assert (split / f).read_bytes() == (full / f).read_bytes(), (attempt, f)

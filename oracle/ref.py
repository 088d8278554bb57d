"""Runs the compiled reference mdff20 (oracle/_ref/*.x, built by oracle/Makefile).

Test infrastructure: used by tests/ to pin the oracle restatement and to make the
golden fixtures, and by bench.py's CPU-baseline leg.  Each call runs the harness in a
fresh process and temporary directory (the reference keeps all state in process
globals), feeding it the control file and POSFF written by ``System.write``.
"""
from __future__ import annotations

import os
import shutil
import struct
import subprocess
import tempfile
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


def harness_path(variant: str = "fix") -> str:
    return os.path.join(REF_DIR, f"mdff20_harness_{variant}.x")


def available(variant: str = "fix") -> bool:
    return os.access(harness_path(variant), os.X_OK)


def read_records(path: str) -> Dict[str, np.ndarray]:
    out = {}
    with open(path, "rb") as fp:
        data = fp.read()
    off = 0
    while off < len(data):
        name = data[off:off + 32].split(b"\0", 1)[0].decode()
        kind = chr(data[off + 32])
        (count,) = struct.unpack("<q", data[off + 40:off + 48])
        off += 48
        dt = np.int32 if kind == "i" else np.float64
        nbytes = count * np.dtype(dt).itemsize
        out[name] = np.frombuffer(data[off:off + nbytes], dtype=dt).copy()
        off += nbytes
    return out


def run(system, task: str, *args, variant: str = "fix", threads: Optional[int] = 1,
        extra_files: Optional[Dict[str, np.ndarray]] = None, keep: bool = False,
        timeout: float = 3600.0) -> Dict[str, np.ndarray]:
    """Run one harness task on `system`; returns the dumped records as arrays."""
    exe = harness_path(variant)
    if not os.access(exe, os.X_OK):
        raise FileNotFoundError(f"compiled reference not built: {exe} (make -C oracle ref)")
    wd = tempfile.mkdtemp(prefix="mdffref_")
    try:
        ctl = system.write(wd)
        for name, arr in (extra_files or {}).items():
            np.ascontiguousarray(arr, dtype=np.float64).tofile(os.path.join(wd, name))
        env = dict(os.environ)
        if threads is not None:
            env["OMP_NUM_THREADS"] = str(threads)
        p = subprocess.run([exe, ctl, task, *[str(a) for a in args]], cwd=wd, env=env,
                           stdout=subprocess.PIPE, stderr=subprocess.PIPE, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"reference harness failed ({p.returncode}): "
                               f"{p.stderr.decode()[-2000:]}\n{p.stdout.decode()[-2000:]}")
        rec = read_records(os.path.join(wd, "out.bin"))
        rec["_stdout"] = p.stdout.decode(errors="replace")
        return rec
    finally:
        if not keep:
            shutil.rmtree(wd, ignore_errors=True)

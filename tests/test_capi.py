"""The C ABI library: it loads, exports every function include/mdffgpu.h declares, and
its parameter/thermo blocks have the same layout in C and in the Python binding.
CPU only (no function that needs a GPU is called, except to check it fails cleanly)."""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest
import torch

from mdff20_b200 import engine
from tests.helpers import ROOT

HEADER = os.path.join(ROOT, "include", "mdffgpu.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(mdffgpu_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = engine.load_library()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(engine.EXPORTS)


def test_struct_layout_matches_header():
    src = r"""
#include <stdio.h>
#include <stddef.h>
#include "mdffgpu.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\n", sizeof(mdffgpu_params), offsetof(mdffgpu_params, alphaES),
         offsetof(mdffgpu_params, tauTberendsen), sizeof(mdffgpu_thermo), offsetof(mdffgpu_thermo, scf_iter));
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        x = os.path.join(d, "t.x")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.dirname(HEADER), c, "-o", x], check=True)
        out = subprocess.run([x], capture_output=True, text=True, check=True).stdout.split()
    sizes = [int(v) for v in out]
    assert sizes[0] == ctypes.sizeof(engine.Params)
    assert sizes[1] == engine.Params.alphaES.offset
    assert sizes[2] == engine.Params.tauTberendsen.offset
    assert sizes[3] == ctypes.sizeof(engine.Thermo)
    assert sizes[4] == engine.Thermo.scf_iter.offset


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU failure path")
def test_create_without_gpu_fails_with_status():
    from tests.golden import cases
    s = cases.silica96(False)
    with pytest.raises(engine.MdffgpuError) as ex:
        engine.Engine(s)
    assert ex.value.code in (2, 7)


def test_null_arguments_rejected():
    L = engine.load_library()
    assert L.mdffgpu_create(None, None, None, None, None, None, None, 0, None) == 1
    assert L.mdffgpu_destroy(None) == 1
    assert L.mdffgpu_engforce(None) == 1
    assert L.mdffgpu_md_steps(None, 1, 1, None) == 1
    assert L.mdffgpu_md_steps_host(None, 1, 1, None, None, None) == 1
    assert L.mdffgpu_md_steps_host(None, 1, -1, None, None, None) == 1

"""mdffgpu_build_lists_noalloc: the neighbour-list build that allocates no memory.

Some callers cannot allocate device memory: an application that owns all GPU memory
through its own pool and forbids allocations after start-up, or one that records its
MD step into a CUDA graph.  They pass their own device buffers; the entry point's
scratch is a static device array.  Here the lists it returns (converted to the
reference's half-list form) must equal, pair for pair, the lists of the context-based
mdffgpu_gen_verletlist, on two calls in a row (the second call reuses the static
scratch left by the first).
"""
import ctypes as C

import numpy as np
import pytest

from mdff20_b200.engine import Engine, load_library
from tests.golden import cases
from tests.helpers import load_golden

pytestmark = pytest.mark.gpu


def _half(full, counts, n):
    """Full per-ion rows -> the reference's CSR half list (src/verlet.c:82-83)."""
    point = np.zeros(n + 1, np.int32)
    out = []
    for i in range(n):
        point[i] = len(out)
        row = full[i, :counts[i]]
        keep = [j for j in row if ((i > j) and ((i + j) % 2 == 0)) or ((i < j) and ((i + j) % 2 != 0))]
        out.extend(sorted(keep))
    point[n] = len(out)
    return point, np.array(out, np.int32)


@pytest.mark.parametrize("name", ["silica450_pim", "silica96_rigid"])
def test_noalloc_lists_equal_context_lists(name):
    import torch

    g = load_golden(name)
    s = cases.CASES[name]()
    pos = g["r_in"].reshape(-1, 3)
    n = s.nion
    e = Engine(s, positions=pos)
    e.gen_verletlist()
    ref = [e.verletlist(0), e.verletlist(1)]
    e.close()

    L = load_library()
    dev = torch.device("cuda", torch.cuda.current_device())
    p4 = torch.zeros((n, 4), dtype=torch.float64, device=dev)
    p4[:, :3] = torch.from_numpy(np.ascontiguousarray(pos)).to(dev)
    cap_nb, cap_co = 512, 1024
    nb = torch.full((n, cap_nb), -1, dtype=torch.int32, device=dev)
    nbn = torch.zeros(n, dtype=torch.int32, device=dev)
    co = torch.full((n, cap_co), -1, dtype=torch.int32, device=dev)
    con = torch.zeros(n, dtype=torch.int32, device=dev)
    cell = (C.c_double * 9)(*np.asarray(s.cell, float).reshape(9))
    cut_nb = s.cutshortrange + s.skindiff
    cut_co = s.cutlongrange + s.skindiff
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize()
    for call in range(2):
        st = C.c_int(-1)
        rc = L.mdffgpu_build_lists_noalloc(p4.data_ptr(), n, cell, cut_nb, cut_co, cap_nb, nb.data_ptr(),
                                           nbn.data_ptr(), cap_co, co.data_ptr(), con.data_ptr(),
                                           stream.cuda_stream, C.byref(st))
        assert rc == 0, (call, rc, st.value)
        assert st.value == 0
        for which, (full, cnt) in enumerate(((nb, nbn), (co, con))):
            point, lst = _half(full.cpu().numpy(), cnt.cpu().numpy(), n)
            assert np.array_equal(point, ref[which][0]), (call, which)
            assert np.array_equal(lst, ref[which][1]), (call, which)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    L = load_library()
    cell = (C.c_double * 9)(10.0, 0, 0, 0, 10.0, 0, 0, 0, 10.0)
    # 65537 ions exceed the static scratch: rejected before any device work
    rc = L.mdffgpu_build_lists_noalloc(256, 65537, cell, 5.0, 5.0, 32, 256, 256, 32, 256, 256, None, None)
    assert rc == 1

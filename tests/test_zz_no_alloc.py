"""mdffgpu_build_lists_noalloc: the neighbour-list build that allocates no memory.

Some callers cannot allocate device memory: an application that owns all GPU memory
through its own pool and forbids allocations after start-up, or a host that runs the
engine inside a fixed device-memory budget.  They pass their own device buffers; the
entry point's scratch is a static device array.  Here the lists it returns (converted to
the reference's half-list form) must equal, pair for pair, the reference's own lists
(golden fixtures) and those of the context-based mdffgpu_gen_verletlist, on two calls in
a row (the second call reuses the static scratch left by the first).  A sparse box whose
cell grid exceeds the scratch's 32768 cells is built on a coarser grid and must give the
oracle's pair set.
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


def _noalloc_lists(s, pos, cap_nb=512, cap_co=1024, calls=2):
    """Half lists (nb, coul) from `calls` successive calls of the entry point."""
    import torch

    n = s.nion
    L = load_library()
    dev = torch.device("cuda", torch.cuda.current_device())
    p4 = torch.zeros((n, 4), dtype=torch.float64, device=dev)
    p4[:, :3] = torch.from_numpy(np.ascontiguousarray(pos)).to(dev)
    nb = torch.full((n, cap_nb), -1, dtype=torch.int32, device=dev)
    nbn = torch.zeros(n, dtype=torch.int32, device=dev)
    co = torch.full((n, cap_co), -1, dtype=torch.int32, device=dev)
    con = torch.zeros(n, dtype=torch.int32, device=dev)
    cell = (C.c_double * 9)(*np.asarray(s.cell, float).reshape(9))
    cut_nb = s.cutshortrange + s.skindiff
    cut_co = s.cutlongrange + s.skindiff
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize()
    out = []
    for call in range(calls):
        st = C.c_int(-1)
        rc = L.mdffgpu_build_lists_noalloc(p4.data_ptr(), n, cell, cut_nb, cut_co, cap_nb, nb.data_ptr(),
                                           nbn.data_ptr(), cap_co, co.data_ptr(), con.data_ptr(),
                                           stream.cuda_stream, C.byref(st))
        assert rc == 0, (call, rc, st.value)
        assert st.value == 0
        out.append([_half(full.cpu().numpy(), cnt.cpu().numpy(), n) for full, cnt in ((nb, nbn), (co, con))])
    return out


@pytest.mark.parametrize("name", ["silica450_pim", "silica96_rigid"])
def test_noalloc_lists_equal_reference_lists(name):
    g = load_golden(name)
    s = cases.CASES[name]()
    pos = g["r_in"].reshape(-1, 3)
    e = Engine(s, positions=pos)
    e.gen_verletlist()
    ctx = [e.verletlist(0), e.verletlist(1)]
    e.close()
    golden = [(g["nb_point"], g["nb_list"]), (g["coul_point"], g["coul_list"])]
    for call, lists in enumerate(_noalloc_lists(s, pos)):
        for which, (point, lst) in enumerate(lists):
            assert np.array_equal(point, golden[which][0]), (call, which)
            assert np.array_equal(lst, golden[which][1]), (call, which)
            assert np.array_equal(point, ctx[which][0]) and np.array_equal(lst, ctx[which][1]), (call, which)


def test_noalloc_sparse_box_coarsened_grid():
    """2001 ions in a 210 A box with 6 A lists: the 35^3 grid the context build would use
    exceeds the static scratch's 32768 cells and is coarsened; the pair sets are the
    oracle's."""
    from mdff20_b200 import synth
    from oracle.oracle import Oracle, wrapped_positions

    s = synth.silica(667, seed=31, L=210.0, rc_sr=5.0, rc_lr=5.5, skin=0.5, kmax=2, velocities=False)
    pos = wrapped_positions(s)
    o = Oracle(s)
    o.gen_verletlist()
    ref = [o.verletlist(0), o.verletlist(1)]
    assert ref[1][1].size > 0
    for lists in _noalloc_lists(s, pos, cap_nb=64, cap_co=64):
        for which, (point, lst) in enumerate(lists):
            assert np.array_equal(point, ref[which][0]), which
            assert np.array_equal(lst, ref[which][1]), which


def test_noalloc_rejects_sizes_beyond_its_scratch():
    L = load_library()
    cell = (C.c_double * 9)(10.0, 0, 0, 0, 10.0, 0, 0, 0, 10.0)
    # 65537 ions exceed the static scratch: rejected before any device work
    rc = L.mdffgpu_build_lists_noalloc(256, 65537, cell, 5.0, 5.0, 32, 256, 256, 32, 256, 256, None, None)
    assert rc == 1

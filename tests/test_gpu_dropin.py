"""The drop-in: the reference's own program (its unmodified sources: main, parsers,
run_md, output writers) linked with mdff20_b200/host/mdff_shim.c, which provides
engforce, prop_agate, check_verletlist, gen_pbc_verletlist, multipole_ES and get_dipoles
by their reference names on the engine.  On each case of tests/golden/host/ it must
leave the files the CPU reference program left: the same layout and numbers within
1e-7 relative (the same bar as the repository's own host program).  The program is
built by `make -C mdff20_b200 dropin` where the reference sources are present.
"""
import os
import subprocess

import pytest

from tests.helpers import ROOT
from tests.test_gpu_host import CASES, HOST_GOLDEN, compare_case, thermo_blocks  # noqa: F401

pytestmark = pytest.mark.gpu

EXE = os.path.join(ROOT, "mdff20_b200", "_dropin", "mdff20_dropin.x")


def run_dropin(case, wd, env=None):
    import shutil
    for f in ("control.s", "POSFF"):
        shutil.copy(os.path.join(HOST_GOLDEN, case, f), os.path.join(wd, f))
    e = dict(os.environ)
    e.update(env or {})
    e.setdefault("OMP_NUM_THREADS", "1")
    p = subprocess.run([EXE, "control.s"], cwd=wd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, env=e,
                       timeout=600)
    assert p.returncode == 0, p.stderr.decode()[-2000:] + p.stdout.decode()[-2000:]
    return p.stdout.decode()


@pytest.mark.skipif(not os.access(EXE, os.X_OK), reason="drop-in not built (make -C mdff20_b200 dropin)")
@pytest.mark.parametrize("case", CASES)
def test_reference_program_on_the_engine(case, tmp_path):
    out = run_dropin(case, str(tmp_path))
    compare_case(case, str(tmp_path), out, rtol=1e-7, atol=2e-9)


@pytest.mark.skipif(not os.access(EXE, os.X_OK), reason="drop-in not built (make -C mdff20_b200 dropin)")
def test_reference_program_mixed_fused(tmp_path):
    """The same program on the fast path (environment switches of the shim)."""
    out = run_dropin("pim_nhc", str(tmp_path), {"MDFF20_GPU_PRECISION": "mixed", "MDFF20_GPU_SOLVER": "cg-fused"})
    compare_case("pim_nhc", str(tmp_path), out, rtol=2e-4, atol=2e-5)

"""CPU tests of libmdffhost: the reference's control-file and POSFF parsers, set_autoES,
the initial velocities and the CONTFF/TRAJFF/OSZIFF writers.

The pins are output files of the reference program itself (tests/golden/host/, made by
tests/golden/make_host_golden.py from the compiled reference).
"""
import ctypes as C
import json
import os
import shutil

import numpy as np
import pytest

from mdff20_b200 import cellmath, host
from mdff20_b200.engine import Params, Thermo, params_from_system
from tests.golden import cases
from tests.helpers import GOLDEN

HOST_GOLDEN = os.path.join(GOLDEN, "host")


@pytest.fixture(scope="module")
def lib():
    return host.load_library()


PIM_FIELDS = {"algo_pim", "algo_extrapolate_dipole", "extrapolate_order", "min_scf_pim_iter", "max_scf_pim_iter",
              "conv_tol_ind", "omegakO"}


def _params_equal(a: Params, b: Params):
    """Fields that differ; default_pim runs only for a Coulomb system (src/field.c:329-334),
    so the solver settings of other systems are not compared."""
    bad = []
    for name, _ in Params._fields_:
        if name in PIM_FIELDS and not b.lcoulombic:
            continue
        x, y = getattr(a, name), getattr(b, name)
        if hasattr(x, "__len__"):
            if list(x) != list(y):
                bad.append(name)
        elif x != y:
            bad.append(name)
    return bad


def _parse(tmp_path, s):
    d = str(tmp_path)
    ctl = s.write(d)
    return host.Inputs(ctl, os.path.join(d, "POSFF"))


ALL = {**{f"host:{k}": v for k, v in cases.host_runs().items()}, **{k: f() for k, f in cases.CASES.items()}}


@pytest.mark.parametrize("name", sorted(ALL))
def test_parse_matches_system(lib, tmp_path, name):
    """Control file + POSFF written from a System parse back to the same parameter block
    and the positions wrapped as read_config does."""
    s = ALL[name]
    with _parse(tmp_path, s) as inp:
        bad = _params_equal(inp.run.p, params_from_system(s))
        assert not bad, f"fields differ: {bad}"
        r = inp.run.xyz("r")
        np.testing.assert_array_equal(r, cellmath.wrap_positions(s.cell, s.pos))
        for key in ("npas", "nprint", "fprint", "cprint", "tprint", "tstart"):
            assert getattr(inp.run, key) == getattr(s, key), key
        assert bool(inp.run.lstatic) == s.lstatic and inp.run.Fposff == 2
        s2 = inp.system()
    bad = _params_equal(params_from_system(s2), params_from_system(s))
    assert not bad, f"System round trip differs: {bad}"


def test_auto_es_matches_reference(lib, tmp_path):
    """set_autoES (src/ewald.c:48-71) against the reference's alphaES/kES/cutlongrange."""
    with open(os.path.join(HOST_GOLDEN, "autoes.json")) as fp:
        want = json.load(fp)
    for name, s in cases.autoes_cases().items():
        d = tmp_path / name
        d.mkdir()
        with _parse(d, s) as inp:
            p = inp.run.p
            assert p.alphaES == want[name]["alphaES"], name
            assert list(p.kES) == want[name]["kES"], name
            assert p.cutlongrange == want[name]["cutlongrange"], name
        bad = _params_equal(inp.run.p, params_from_system(s))   # the Python restatement
        assert not bad, f"{name}: {bad}"


def _copy_inputs(case, dst):
    for f in ("control.s", "POSFF"):
        shutil.copy(os.path.join(HOST_GOLDEN, case, f), os.path.join(dst, f))
    return os.path.join(dst, "control.s"), os.path.join(dst, "POSFF")


def _contff_columns(path):
    with open(path) as fp:
        lines = fp.read().splitlines()
    return [ln.split() for ln in lines[9:]]


def test_initial_velocities_and_contff_bytes(lib, tmp_path):
    """init_velocities draws the reference's Maxwell-Boltzmann velocities from rand(), and
    write_config reproduces the reference's CONTFF byte for byte (zero-step run: wrapped
    POSFF positions, initial velocities, forces at t=0 taken from the reference file)."""
    ctl, pos = _copy_inputs("pim_init", str(tmp_path))
    ref_path = os.path.join(HOST_GOLDEN, "pim_init", "CONTFF")
    rows = _contff_columns(ref_path)
    with host.Inputs(ctl, pos) as inp:
        v = inp.init_velocities()
        f = np.array([[float(x) for x in r[7:10]] for r in rows])
        inp.run.set_xyz("f", f)
        out = str(tmp_path / "CONTFF")
        inp.write_config(out, "w")
        for k in range(2):   # TRAJFF appends
            inp.write_config(str(tmp_path / "TRAJFF"), "a")
    vstr = [[f"{x:19.12f}".strip() for x in row] for row in v]
    assert vstr == [r[4:7] for r in rows]
    with open(out, "rb") as a, open(ref_path, "rb") as b:
        assert a.read() == b.read()
    with open(tmp_path / "TRAJFF", "rb") as a, open(ref_path, "rb") as b:
        assert a.read() == 2 * b.read()


def test_oszi_header_and_record_layout(lib, tmp_path):
    """info_thermo key 1: the header every tenth record and the two fixed-width lines."""
    ctl, pos = _copy_inputs("pim_nhc", str(tmp_path))
    with host.Inputs(ctl, pos) as inp:
        t = Thermo()
        t.e_kin, t.u_bhmftd, t.u_coul, t.u_pol, t.e_nvt = 38.1, 197.5, -3828.6, -0.25, 1e-3
        t.pvir_bhmftd, t.pvir_coul = 98.9, -70.4
        text = host.oszi_text(inp.run, [(k, t) for k in range(1, 13)])
    lines = text.splitlines()
    assert len(lines) == 2 * 3 + 2 * 12 and lines[0] == "-" * 105 and lines[23] == "-" * 105
    ref = open(os.path.join(HOST_GOLDEN, "pim_nhc", "OSZIFF")).read().splitlines()
    assert lines[:3] == ref[:3]
    assert [len(x) for x in lines[3:5]] == [len(x) for x in ref[3:5]]
    assert lines[3].split()[1] == "1.00000000e-03"


def test_output_periods(lib):
    """iopnode / iopsnode (src/io.c:62-69); a period <= 0 never fires."""
    L = lib
    assert [s for s in range(1, 11) if L.mdffh_iopnode(s, 10, 4)] == [4, 8, 10]
    assert [s for s in range(1, 11) if L.mdffh_iopsnode(s, 10, 3, 5)] == [6, 9, 10]
    assert not any(L.mdffh_iopnode(s, 10, 0) for s in range(1, 11))


def _write(tmp_path, control: str, posff_from: str = "pim_static"):
    shutil.copy(os.path.join(HOST_GOLDEN, posff_from, "POSFF"), tmp_path / "POSFF")
    (tmp_path / "control.s").write_text(control)
    return str(tmp_path / "control.s"), str(tmp_path / "POSFF")


BASE = """# comment tokens match no keyword
lcoulombic T  qit -1.2 qit 2.4   massit 15.99994 # O
massit 28.084
lbhmft Yes
Abhmftd 1388.773 18003.7572 0.0
Bbhmftd 2.76 4.87318 0.0
Cbhmftd 175.0 133.5381 0.0
cutshortrange 5.0 cutlongrange 6.0 alphaES 0.5 kES 6 6 6
polit 1.0 0 0 0 1.0 0 0 0 1.0
polit 0 0 0 0 0 0 0 0 0
lpoldamping 0 0 1 y
pol_damp_b 0 0 1 2.0 pol_damp_c 0 0 1 1.0 pol_damp_k 0 0 1 4
integrator nvt-nhcn dt 0.001 temp 2500 npas 3 nhc_n 3 timesca_thermo 0.1
"""


def test_control_tokens_and_defaults(lib, tmp_path):
    """Keywords anywhere on a line, comments as inert tokens, the boolean words of
    src/constants.c:20-35, defaults of default_global/default_md/default_pim, and the upper
    pair triangles copied down."""
    ctl, pos = _write(tmp_path, BASE)
    with host.Inputs(ctl, pos) as inp:
        r, p = inp.run, inp.run.p
        assert p.lcoulombic == 1 and p.lbhmft == 1 and p.lbhmftd == 0 and p.lnmlj == 0
        assert list(p.qit[:2]) == [-1.2, 2.4] and list(p.massit[:2]) == [15.99994, 28.084]
        assert p.Abhmftd[0 * 16 + 1] == 18003.7572 and p.Abhmftd[1 * 16 + 0] == 18003.7572
        assert p.lpoldamping[(0 * 16 + 0) * 16 + 1] == 1 and p.pol_damp_k[(0 * 16 + 0) * 16 + 1] == 4
        assert p.skindiff == 0.15 and p.lverletL == 1 and r.Fposff == 2
        assert r.nprint == 1 and r.fprint == 1 and r.cprint == 1000 and r.tprint == 1000 and r.tstart == 0
        assert p.conv_tol_ind == 1e-6 and p.min_scf_pim_iter == 3 and p.max_scf_pim_iter == 100
        assert p.egrator == 2 and list(p.kES) == [6, 6, 6]


def test_control_epsw_reads_twice(lib, tmp_path):
    """read_field tests "epsw" twice (src/field.c:159-164): a second number after it is
    consumed as epsw too."""
    ctl, pos = _write(tmp_path, BASE + "epsw 1e-4 1e-7\nlautoES false\n")
    with host.Inputs(ctl, pos) as inp:
        assert inp.run.epsw == 1e-7


@pytest.mark.parametrize("extra,msg", [
    ("integrator nve-xx\n", "integrator"),
    ("lverletL maybe\n", "lverletL"),
    ("trunc cubic\nlnmlj true\n", "trunc"),
    ("massit 1.0\n", "massit"),
    ("lpoldamping 0 0 16 true\n", "out of range"),
    ("quadit 1 0 0 0 1 0 0 0 1\n", "quadit"),
])
def test_control_errors(lib, tmp_path, extra, msg):
    ctl, pos = _write(tmp_path, BASE + extra)
    with pytest.raises(ValueError, match=msg):
        host.Inputs(ctl, pos)


def test_posff_direct_and_rnn(lib, tmp_path):
    """Direct coordinates are converted with A; Fposff rnn reads positions only."""
    s = cases.crist192(False)
    frac = cellmath.kardir(s.pos, cellmath.lattice(s.cell)[0])
    lines = s.posff_text(with_velocities=False).splitlines()
    out = lines[:8] + ["Direct"]
    names = np.repeat(np.array(s.type_names, dtype=object), s.nionit)
    out += [f"{names[i]} {a:.17e} {b:.17e} {c:.17e}" for i, (a, b, c) in enumerate(frac)]
    (tmp_path / "POSFF").write_text("\n".join(out) + "\n")
    ctl = s.write(str(tmp_path), "ctl.s")
    os.replace(tmp_path / "POSFF", tmp_path / "POSFF.rvf")
    (tmp_path / "POSFF").write_text("\n".join(out) + "\n")
    (tmp_path / "ctl.s").write_text((tmp_path / "ctl.s").read_text().replace("Fposff rvf", "Fposff rnn"))
    with host.Inputs(ctl, str(tmp_path / "POSFF")) as inp:
        r = inp.run.xyz("r")
        want = cellmath.wrap_positions(s.cell, cellmath.dirkar(frac, s.cell))
        np.testing.assert_array_equal(r, want)
        assert not inp.run.xyz("v").any()


def test_host_library_exports_and_layout(lib, tmp_path):
    """libmdffhost exports every function include/mdffhost.h declares, and mdffh_run has
    the same layout in C and in the Python binding."""
    import re
    import subprocess
    from tests.helpers import ROOT

    header = os.path.join(ROOT, "include", "mdffhost.h")
    names = sorted(set(re.findall(r"\b(mdffh_[a-z_0-9]+)\s*\(", open(header).read())))
    assert len(names) >= 14
    assert not [n for n in names if not hasattr(lib, n)]
    src = r"""
#include <stdio.h>
#include <stddef.h>
#include "mdffhost.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu\n", sizeof(mdffh_run), offsetof(mdffh_run, Fposff), offsetof(mdffh_run, B),
         offsetof(mdffh_run, atypia), offsetof(mdffh_run, oszcall), offsetof(mdffh_run, err));
  return 0;
}
"""
    c, x = tmp_path / "t.c", tmp_path / "t.x"
    c.write_text(src)
    subprocess.run(["gcc", "-I", os.path.dirname(header), str(c), "-o", str(x)], check=True)
    got = [int(v) for v in subprocess.run([str(x)], capture_output=True, text=True, check=True).stdout.split()]
    H = host.HostRun
    assert got == [C.sizeof(H), H.Fposff.offset, H.B.offset, H.atypia.offset, H.oszcall.offset, H.err.offset]

"""The C-ABI library builds, loads without a GPU and exports every declared symbol."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ccs_[a-z0-9_]+|mh_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    from massccs_b200 import build, engine
    build.build()
    return engine.load_library()


def test_every_declared_symbol_is_exported(lib):
    from massccs_b200 import engine, host
    names = declared("massccs_gpu.h")
    assert set(names) == set(engine.EXPORTS)
    for n in names:
        assert hasattr(lib, n), n
    hl = host.load_library()
    hnames = declared("massccs_host.h")
    assert set(hnames) == set(host.EXPORTS)
    for n in hnames:
        assert hasattr(hl, n), n


def test_cli_is_built():
    assert os.access(os.path.join(ROOT, "massccs_b200", "bin", "massccs"), os.X_OK)


def test_abi_version_and_strings(lib):
    v = ctypes.c_int32(0)
    assert lib.ccs_version(ctypes.byref(v)) == 0 and v.value == 2
    assert lib.ccs_status_string(0) == b"ok"
    assert lib.ccs_status_string(-4) == b"device watchdog expired"
    assert lib.ccs_last_error(None) == b"no context"


def test_params_default_matches_reference_defaults(lib):
    from massccs_b200 import engine
    p = engine.default_params()
    # Constants.h:69-83 defaults
    assert (p.dt, p.temperature, p.lj_cutoff, p.coul_cutoff, p.skin) == (10.0, 298.0, 12.0, 25.0, 0.01)
    assert p.gas == 1 and p.force_type == 4 and p.precision == 0


def test_create_without_device_fails_cleanly(lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a device is present")
    except ImportError:
        pass
    h = ctypes.c_void_p()
    assert lib.ccs_create(ctypes.byref(h), 0) == -5  # CCS_ERR_NODEVICE
    assert not h.value


def test_ctypes_layouts_match_the_headers(tmp_path):
    """Every C struct of the ABI has the size and field offsets its ctypes
    mirror assumes (compiled with the host C compiler against include/)."""
    import shutil
    import subprocess
    from massccs_b200 import engine, host
    cc = shutil.which("gcc") or "/usr/bin/gcc"
    mirrors = {"ccs_params": engine.CcsParams, "ccs_stats": engine.CcsStats, "ccs_info": engine.CcsInfo,
               "ccs_field_params": engine.CcsFieldParams, "ccs_field_report": engine.CcsFieldReport,
               "mh_info": host.MhInfo}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "massccs_gpu.h"', '#include "massccs_host.h"',
             "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l}
    for cname, py in mirrors.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_field_params_defaults(lib):
    """The learned field's defaults: 16 levels of 2^20 rows (every level up to
    resolution 100 dense), resolutions 8..128 over the domain, 4e6 samples,
    6000 Adam steps, the range-separation switch from 6 to 12 A (the measured
    best of the sweep over table size, resolutions and switch range), exact
    within 2 A of an atom and no error voxels (no exact/learned switching
    where probes go)."""
    from massccs_b200 import engine
    p = engine.field_params()
    assert (p.samples, p.iterations, p.log2_table, p.base_res, p.finest_res) == (4000000, 6000, 20, 8, 128)
    assert (p.fallback_radius, p.voxel, p.err_threshold, p.r_in, p.r_out) == (2.0, 0.5, 0.0, 6.0, 12.0)

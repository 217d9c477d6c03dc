"""The C-ABI library: it loads, exports every entry point declared in
include/gizmo_hydro.h, its ctypes mirror has the C layout, and it fails
cleanly (no trap, an error code) when no GPU is present."""
import ctypes as C
import os
import re
import subprocess

import pytest

from gizmo_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gizmo_hydro.h")


def declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void\s*\*)\s*(gz_\w+)\s*\(", src, re.M)))


def test_header_declares_the_exports():
    assert set(declared_functions()) == set(abi.EXPORTED_SYMBOLS)


def test_library_loads_and_exports_all_symbols():
    lib = abi.load_library()
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_struct_layouts_match_c(tmp_path):
    prog = tmp_path / "layout.c"
    prog.write_text(r'''
#include <stdio.h>
#include <stddef.h>
#include "gizmo_hydro.h"
int main(void) {
  printf("%zu %zu %zu %zu\n", sizeof(gz_params), sizeof(gz_particles), sizeof(gz_outputs), sizeof(gz_status_info));
  printf("%zu %zu %zu %zu\n", offsetof(gz_params, box_size), offsetof(gz_particles, cond), offsetof(gz_outputs, iters),
         offsetof(gz_outputs, flux_abs));
  printf("%zu %zu\n", offsetof(gz_status_info, pairs_density), offsetof(gz_status_info, message));
  printf("%zu %zu %zu %zu\n", sizeof(gz_kick_fields), offsetof(gz_kick_fields, active),
         sizeof(gz_drift_fields), offsetof(gz_drift_fields, status));
  return 0; }
''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.dirname(HEADER), str(prog), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    got = [int(v) for v in out]
    want = [C.sizeof(abi.GzParams), C.sizeof(abi.GzParticles), C.sizeof(abi.GzOutputs), C.sizeof(abi.GzStatusInfo),
            abi.GzParams.box_size.offset, abi.GzParticles.cond.offset, abi.GzOutputs.iters.offset,
            abi.GzOutputs.flux_abs.offset,
            abi.GzStatusInfo.pairs_density.offset, abi.GzStatusInfo.message.offset,
            C.sizeof(abi.GzKickFields), abi.GzKickFields.active.offset,
            C.sizeof(abi.GzDriftFields), abi.GzDriftFields.status.offset]
    assert got == want


@pytest.mark.parametrize("cname,mirror", [("gz_kick_fields", abi.GzKickFields), ("gz_drift_fields", abi.GzDriftFields),
                                          ("gz_params", abi.GzParams), ("gz_particles", abi.GzParticles),
                                          ("gz_outputs", abi.GzOutputs), ("gz_status_info", abi.GzStatusInfo),
                                          ("gz_timestep_params", abi.GzTimestepParams),
                                          ("gz_timestep_fields", abi.GzTimestepFields),
                                          ("gz_tuning", abi.GzTuning), ("gz_graph_info", abi.GzGraphInfo)])
def test_device_field_structs_match_c_field_by_field(tmp_path, cname, mirror):
    """Every field of the ctypes mirror sits at the C offset of the field of the same name: two
    pointer fields in swapped order would keep the size and hand the kernel the wrong arrays."""
    names = [f[0] for f in mirror._fields_]
    prog = tmp_path / "fields.c"
    prog.write_text("#include <stdio.h>\n#include <stddef.h>\n#include \"gizmo_hydro.h\"\nint main(void) {\n"
                    + "".join(f'  printf("%zu\\n", offsetof({cname}, {n}));\n' for n in names)
                    + f'  printf("%zu\\n", sizeof({cname}));\n  return 0; }}\n')
    exe = tmp_path / "fields"
    subprocess.run(["gcc", "-I", os.path.dirname(HEADER), str(prog), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got == [getattr(mirror, n).offset for n in names] + [C.sizeof(mirror)]


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_create_without_device_returns_code():
    lib = abi.load_library()
    from gizmo_b200 import ics
    p = ics.sedov(4).params
    ctx = C.c_void_p()
    assert lib.gz_create(C.byref(p), 0, C.byref(ctx)) == abi.ERR_NO_DEVICE
    assert not ctx


def test_bad_arguments_rejected_before_device_use():
    lib = abi.load_library()
    from gizmo_b200 import ics
    p = ics.sedov(4).params
    p.kernel = 5
    ctx = C.c_void_p()
    assert lib.gz_create(C.byref(p), 0, C.byref(ctx)) == abi.ERR_ARG
    assert lib.gz_create(None, 0, C.byref(ctx)) == abi.ERR_ARG
    assert lib.gz_upload(None, None) == abi.ERR_ARG
    assert lib.gz_hydro_density(None, None, 0) == abi.ERR_ARG


def test_kick_arguments_checked_before_device_use():
    lib = abi.load_library()
    from gizmo_b200 import ics
    p = ics.sedov(4).params
    f = abi.GzKickFields()
    f.n = 0
    assert lib.gz_kick(C.byref(p), C.byref(f), 0, 1e-12, 0.0, None) == abi.OK  # nothing to kick
    assert lib.gz_kick(C.byref(p), C.byref(f), 2, 1e-12, 0.0, None) == abi.ERR_ARG  # no such half kick
    assert lib.gz_kick(None, C.byref(f), 0, 1e-12, 0.0, None) == abi.ERR_ARG
    assert lib.gz_kick(C.byref(p), C.byref(f), 0, -1.0, 0.0, None) == abi.ERR_ARG
    f.n = 10
    assert lib.gz_kick(C.byref(p), C.byref(f), 0, 1e-12, 0.0, None) == abi.ERR_ARG  # required fields missing
    for name in ("vel", "u", "mass", "accel", "dudt", "vel_pred", "u_pred", "dp", "tstart", "tend"):
        setattr(f, name, 16)  # never dereferenced: the MFV fields are still missing
    p.method = abi.METHOD_MFV
    assert lib.gz_kick(C.byref(p), C.byref(f), 0, 1e-12, 0.0, None) == abi.ERR_ARG


def test_drift_arguments_checked_before_device_use():
    lib = abi.load_library()
    from gizmo_b200 import ics
    p = ics.sedov(4).params
    f = abi.GzDriftFields()
    f.n = 0
    assert lib.gz_drift(C.byref(p), C.byref(f), 10, 1e-12, 0.0, None) == abi.OK  # nothing to drift
    assert lib.gz_drift(None, C.byref(f), 10, 1e-12, 0.0, None) == abi.ERR_ARG
    assert lib.gz_drift(C.byref(p), C.byref(f), 10, float("nan"), 0.0, None) == abi.ERR_ARG
    f.n = 10
    assert lib.gz_drift(C.byref(p), C.byref(f), 10, 1e-12, 0.0, None) == abi.ERR_ARG  # required fields missing
    for name in ("pos", "vel", "vel_pred", "accel", "divvel", "mass", "rho", "u_pred", "dudt", "h", "pressure",
                 "ti_current", "status"):
        setattr(f, name, 16)  # never dereferenced: what is missing is caught first
    p.method = abi.METHOD_MFV
    assert lib.gz_drift(C.byref(p), C.byref(f), 10, 1e-12, 0.0, None) == abi.ERR_ARG  # MFV moves with pvel


def test_header_constants_match_the_python_mirror():
    src = open(HEADER).read()
    defines = {m.group(1): int(m.group(2)) for m in re.finditer(r"^#define\s+GZ_(\w+)\s+(-?\d+)", src, re.M)}
    timers = {k[len("TIMER_"):].lower(): v for k, v in defines.items() if k.startswith("TIMER_") and k != "TIMERS"}
    assert timers == abi.TIMERS
    assert defines["TIMERS"] == len(abi.TIMERS)
    for name, value in defines.items():
        if name.startswith("TIMER"):
            continue
        assert hasattr(abi, name), name
        assert getattr(abi, name) == value, name

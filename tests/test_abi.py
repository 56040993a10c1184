"""The C ABI library: it builds, loads and exports every declared entry point,
its struct layouts match the header, and host-side argument checks work
without a GPU (no compute call is made here)."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

from vxsim import native as N

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def lib():
    if not N.LIB_PATH.exists():
        subprocess.run(["make", "-s", "-j8", "-C", str(ROOT / "voxel-sim_b200")], check=True)
    return N.load()


def test_every_declared_symbol_is_exported(lib):
    names = N.header_symbols()
    assert "vx_solve_pcg_f32" in names and "vx_corotational_pass" in names
    for name in names:
        assert hasattr(lib, name), name


def test_abi_version(lib):
    assert lib.vx_abi_version() == 1


def test_struct_layouts_match_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(f'''
#include <stdio.h>
#include <stddef.h>
#include "{ROOT}/include/vxcorot.h"
int main(void) {{
  printf("%zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(vx_material), sizeof(vx_scene_desc), sizeof(vx_pass_params),
         sizeof(vx_pass_stats), offsetof(vx_scene_desc, neighbor), sizeof(vx_step_params),
         offsetof(vx_step_params, pass), sizeof(vx_step_stats));
  printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(vx_server_config), sizeof(vx_request_plan), sizeof(vx_request_result),
         sizeof(vx_server_stats), sizeof(vx_fracture_config), sizeof(vx_dissipation));
  printf("%zu %zu %zu %zu %zu\\n", sizeof(vx_tune_result), sizeof(vx_contact_stats), sizeof(vx_contact_heat),
         offsetof(vx_step_params, contact), offsetof(vx_step_stats, contacts));
  return 0;
}}''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [C.sizeof(N.VxMaterial), C.sizeof(N.VxSceneDesc), C.sizeof(N.VxPassParams), C.sizeof(N.VxPassStats),
            N.VxSceneDesc.neighbor.offset, C.sizeof(N.VxStepParams), N.VxStepParams.pass_.offset,
            C.sizeof(N.VxStepStats), C.sizeof(N.VxServerConfig), C.sizeof(N.VxRequestPlan),
            C.sizeof(N.VxRequestResult), C.sizeof(N.VxServerStats), C.sizeof(N.VxFractureConfig),
            C.sizeof(N.VxDissipation), C.sizeof(N.VxTuneResult), C.sizeof(N.VxContactStats),
            C.sizeof(N.VxContactHeat), N.VxStepParams.contact.offset, N.VxStepStats.contacts.offset]
    assert got == want


def test_footprint_is_positive_and_grows(lib):
    a = lib.vx_scene_footprint_bytes(1000)
    b = lib.vx_scene_footprint_bytes(2000)
    assert 0 < a < b
    # about 1.5 kB per REV for both precision forms and the stress outputs
    assert 1000 < (b - a) / 1000 < 2500


def test_shim_argument_checks_need_no_device(lib):
    z = np.zeros(1, np.float32)
    it = C.c_uint32()
    rel = C.c_float()
    # n = 0 returns an empty correction without touching a device (src/cuda_solver.rs:311-314)
    assert lib.vx_solve_pcg_f32(None, None, None, None, None, 0, 10, 1e-5, None, C.byref(it), C.byref(rel)) == N.VX_OK
    st = lib.vx_solve_pcg_f32(None, None, None, None, None, 3, 10, 1e-5, None, C.byref(it), C.byref(rel))
    assert st == N.VX_BAD_INPUT
    assert "null" in N.last_error()


def test_null_handles_are_rejected(lib):
    assert lib.vx_corotational_pass(None, None, None) == N.VX_BAD_INPUT
    assert lib.vx_scene_set_positions(None, None) == N.VX_BAD_INPUT
    assert lib.vx_scene_set_previous(None, None) == N.VX_BAD_INPUT
    assert lib.vx_ctx_create(0, None) == N.VX_BAD_INPUT
    assert lib.vx_scene_step(None, None, None) == N.VX_BAD_INPUT
    assert lib.vx_scene_update_velocities(None, 0, None, None, 0) == N.VX_BAD_INPUT


def test_persistent_form_codes_match_the_header():
    """The VX_PERSIST_* form codes of the header are the ones the binding names
    (PERSIST_FORMS) and, for the range plan, sizes (RANGE_THREADS)."""
    import re
    text = (ROOT / "include" / "vxcorot.h").read_text()
    codes = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define (VX_PERSIST_\w+) (\d+)", text)}
    assert set(codes.values()) == set(N.PERSIST_FORMS), codes
    assert {codes["VX_PERSIST_RANGE"], codes["VX_PERSIST_RANGE_608"], codes["VX_PERSIST_RANGE_768"],
            codes["VX_PERSIST_RANGE_896"]} == set(N.RANGE_THREADS)
    for name, threads in (("VX_PERSIST_RANGE", 512), ("VX_PERSIST_RANGE_608", 608), ("VX_PERSIST_RANGE_768", 768),
                          ("VX_PERSIST_RANGE_896", 896)):
        assert N.RANGE_THREADS[codes[name]] == threads

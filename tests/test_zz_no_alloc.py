"""vx_solve_pcg_f32_noalloc against vx_solve_pcg_f32, through the C ABI.

The no-allocation entry point serves callers that cannot call cudaMalloc: an
engine that owns all of its GPU memory up front, or a step loop that must not
block on a device allocation. The caller hands it device buffers and it keeps
its own working memory in a fixed array inside the library. These tests give
it device buffers (allocated here by the test, not by the entry point), call
it twice in a row on different systems, and compare each result with the
allocating entry point within the shim tolerance the other tests use. This
file is collected last so a stop-at-first-failure run has run every other
test before it.
"""
import ctypes as C

import numpy as np
import pytest

import pyoracle as O
from vxsim import native as N
from vxsim import scenes as S

pytestmark = pytest.mark.gpu

RTOL = 1e-4  # the shim tolerance of tests/test_gpu_parity.py


def packed_rows(scene):
    o = O.OracleScene(scene)
    o.fit_rotations()
    o.assemble(1e-3)
    return o.pack_rows()


def call_noalloc(rows, max_iterations, tolerance):
    import torch

    dev = torch.device("cuda", 0)
    n = rows["n"]
    buf = {k: torch.from_numpy(np.ascontiguousarray(rows[k], np.float32)).to(dev)
           for k in ("rhs", "diag9", "blocks54", "inv9")}
    nbr = torch.from_numpy(np.ascontiguousarray(rows["nbr6"], np.uint32).view(np.int32)).to(dev)
    out = torch.full((3 * max(n, 1),), float("nan"), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    it = C.c_uint32()
    rel = C.c_float()
    st = N.load().vx_solve_pcg_f32_noalloc(
        C.c_void_p(buf["rhs"].data_ptr()), C.c_void_p(nbr.data_ptr()), C.c_void_p(buf["diag9"].data_ptr()),
        C.c_void_p(buf["blocks54"].data_ptr()), C.c_void_p(buf["inv9"].data_ptr()), n, max_iterations,
        tolerance, C.c_void_p(out.data_ptr()), C.byref(it), C.byref(rel), None)
    torch.cuda.synchronize()
    return st, out[:3 * n].cpu().numpy().reshape(-1, 3), it.value, rel.value


def compare(rows, max_iterations, tolerance):
    st_a, dx_a, it_a, rel_a = N.solve_pcg_f32(rows, max_iterations, tolerance)
    st_b, dx_b, it_b, rel_b = call_noalloc(rows, max_iterations, tolerance)
    assert st_a == N.VX_OK and st_b == N.VX_OK, (st_a, st_b, N.last_error())
    assert it_b == it_a
    err = np.linalg.norm(dx_b - dx_a) / np.linalg.norm(dx_a)
    assert err < RTOL, err
    assert abs(rel_b - rel_a) <= RTOL * max(rel_a, 1e-30) + 1e-12
    return it_b


def test_noalloc_matches_allocating_entry_point_on_two_calls_in_a_row():
    big = packed_rows(S.impose_axis_targets(S.wood_cube()))  # 800 active rows, top layer loaded
    small = packed_rows(S.mixed_block(8, seed=2))  # a different, smaller system after it
    assert small["n"] < big["n"]
    compare(big, 160, 1e-5)
    compare(small, 400, 1e-5)


def test_noalloc_rejects_systems_above_its_fixed_limit():
    n = N.load()  # noqa: F841
    too_big = int(0x10000) + 1  # VX_NOALLOC_MAX_ROWS + 1
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    st = N.load().vx_solve_pcg_f32_noalloc(dummy, dummy, dummy, dummy, dummy, too_big, 10, 1e-5, dummy, None,
                                           None, None)
    assert st == N.VX_BAD_INPUT
    assert "scratch limit" in N.last_error()


def test_noalloc_rejects_out_of_range_neighbours():
    rows = packed_rows(S.wood_cube(4))
    rows["nbr6"] = rows["nbr6"].copy()
    rows["nbr6"][3] = rows["n"] + 5
    st, *_ = call_noalloc(rows, 50, 1e-5)
    assert st == N.VX_BAD_INPUT
    assert "outside" in N.last_error()

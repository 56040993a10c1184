"""The surface capture writer (vxsim_capture, the device counterpart of
src/bin/solver_scale_capture.rs) against the oracle's step.

A 36 x 32 x 32 iron block with its bottom layer kinematic is stepped under
gravity with SceneConfig::default settings (4 substeps, 2 passes, PCG cap
160, tolerance 1e-5, fracture and contact on). The kinematic layer is not
bonded to the block (their kinematic flags differ): the block stands on it
through the contact stage, as in the oracle's step. The CSV's positions are
f32 values in Rust's shortest form: they must read back to the oracle's
positions rounded to f32.
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import pyoracle as O
from vxsim import materials as M
from vxsim import scenes as S

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "voxel-sim_b200"
NX, NY, NZ = 36, 32, 32


def _capture(tmp_path, *args):
    subprocess.run(["make", "-s", "-C", str(PKG), "lib/vxsim_capture"], check=True, capture_output=True)
    csv = tmp_path / "capture.csv"
    out = subprocess.run([str(PKG / "lib" / "vxsim_capture"), str(csv), *map(str, args)], capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    return csv.read_text().splitlines(), out.stderr


def _records(lines):
    head = lines[0].split(",")
    frames, samples = {}, {}
    for line in lines[1:]:
        f = line.split(",")
        if f[0] == "F":
            frames[int(f[1])] = f
            samples[int(f[1])] = []
        else:
            assert f[0] == "V", line
            samples[int(f[1])].append(f)
    return head, frames, samples


def _surface():
    """(sample_id, index, x, y, z) of every boundary REV whose index is not a
    multiple of 3, in index order (src/bin/solver_scale_capture.rs:85-97)."""
    out = []
    for z in range(NZ):
        for y in range(NY):
            for x in range(NX):
                index = (z * NY + y) * NX + x
                boundary = x in (0, NX - 1) or y in (0, NY - 1) or z in (0, NZ - 1)
                if boundary and index % 3 != 0:
                    out.append((len(out), index, x, y, z))
    return out


def _lost(neighbor, x, y, z):
    """Bonds missing around a REV (surface_state, src/bin/solver_scale_capture.rs:20-46)."""
    index = (z * NY + y) * NX + x
    strides, coords, extents = (1, NX, NX * NY), (x, y, z), (NX, NY, NZ)
    lost = 0
    for axis in range(3):
        if coords[axis] + 1 < extents[axis]:
            lost += neighbor[axis, index] == S.EMPTY
        if coords[axis] > 0:
            lost += neighbor[axis, index - strides[axis]] == S.EMPTY
    return int(lost)


def test_capture_records_the_oracle_step(tmp_path):
    lines, log = _capture(tmp_path, 3, 3)
    head, frames, samples = _records(lines)
    assert head == ["H", "0.001", "3", "3"]
    # saved states: 0, the interval boundary 2 (2*2/3 > 1*2/3), and the last
    assert sorted(frames) == [0, 2, 3]
    surface = _surface()
    cells = S.grid_cells(NX, NY, NZ)
    scene = S.from_cells(cells, M.component_id("iron"), M.table(), kinematic=(cells[:, 2] == 0))
    for f in frames.values():
        # no contact, no breaks: one cluster (the kinematic layer has no id)
        assert f[2:11] == ["0", "0", "0", "0", "0", "0", "1", "0", "0"] and f[11:] == ["0", "1", "0"], f
    o = O.OracleStepper(scene, fixed_dt=float(np.float32(1e-3)), substeps=4, iterations=160,
                        solver_tolerance=float(np.float32(1e-5)), corotation_tolerance=float(np.float32(1e-5)),
                        corotation_iterations=2, gravity=(0.0, 0.0, float(np.float32(-9.81))), fracture=True,
                        contact=True, restitution=float(np.float32(0.1)), friction=float(np.float32(0.35)))
    lost = np.array([_lost(scene.neighbor, x, y, z) for _, _, x, y, z in surface])
    for frame in range(4):
        if frame:
            o.step()
        if frame not in frames:
            continue
        rows = samples[frame]
        assert [int(r[2]) for r in rows] == [s[0] for s in surface]
        assert [int(r[8]) for r in rows] == [s[1] for s in surface]
        # Rust's Display for f32: the shortest digits that read back to the
        # same f32, positional, no trailing ".0"
        texts = [v for r in rows for v in r[3:7]]
        assert all(np.format_float_positional(np.float32(v), unique=True, trim="-") == v for v in texts)
        got = np.array([[np.float32(v) for v in r[3:6]] for r in rows], np.float32).astype(np.float64)
        want = o.positions[[s[1] for s in surface]].astype(np.float32).astype(np.float64)
        # the device and the oracle round the FP64 solve differently, far
        # below one f32 ulp
        ulp = float(np.spacing(np.float32(0.4)))
        assert np.max(np.abs(got - want)) <= ulp, (frame, np.max(np.abs(got - want)))
        assert np.all(np.array([float(r[6]) for r in rows]) == 0.0)
        assert np.array_equal(np.array([int(r[7]) for r in rows]), lost)
    # contact holds the layer on the kinematic floor at its rest height (the
    # projection leaves it 1e-6 m above); the layers above settle through the
    # lattice, less than the free fall of 12 substeps of 0.25 ms (78 g h^2 =
    # 4.78e-5 m); the kinematic layer stayed
    idx = np.array([s[1] for s in surface])
    dz = got[:, 2] - scene.position[idx, 2]
    z = cells[idx, 2]
    assert np.all(dz[z == 1] >= -1e-7) and np.all(dz[z == 1] <= 2e-6)
    assert np.all(dz[z > 1] > -4.78e-5)
    assert np.array_equal(got[z == 0], scene.position[idx[z == 0]].astype(np.float32).astype(np.float64))
    assert "complete" in log

"""The C++ host mirror of the solver:: API (voxel-sim_b200/host), tested with
the reference's own API tests restated in tests/host/test_solver_api.cpp."""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "voxel-sim_b200"
EXE = PKG / "lib" / "vxsim_host_tests"
CASES = ["persistent_force_and_acceleration_use_voxel_mass", "velocity_and_impulse_are_mass_consistent",
         "external_actions_reject_fixed_and_missing_voxels",
         "constraint_inputs_are_atomic_and_impulses_respect_fixed_axes", "axis_targets_pull_a_bar"]


def _built():
    subprocess.run(["make", "-s", "-C", str(PKG), "host"], check=True, capture_output=True)
    return EXE


def test_host_library_links_against_the_c_abi():
    exe = _built()
    out = subprocess.run(["ldd", str(exe)], capture_output=True, text=True, check=True).stdout
    assert "libvxsolver.so" in out and "libvxcorot.so" in out and "not found" not in out


@pytest.mark.gpu
def test_solver_api_mirror_on_the_device():
    out = subprocess.run([str(_built())], capture_output=True, text=True, timeout=600)
    for case in CASES:
        assert f"PASS {case}" in out.stdout, out.stdout + out.stderr
    assert out.returncode == 0, out.stdout + out.stderr

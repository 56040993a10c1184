"""Scene configuration files and the capture writer's command line, on the CPU.

The RON loader (voxel-sim_b200/host/vxsim_config.cpp) is tested by the C++
program tests/host/test_scene_config.cpp: every field of SceneConfig
(src/scene.rs:215-307) and FractureConfig (src/fracture.rs:10-60), the two
serde defaults, unknown/missing/duplicate fields, RON syntax and each
validation rule. The example scene files under tests/golden/scenes must load.
"""
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "voxel-sim_b200"
CASES = ["full_file_reads_every_field", "omitted_fields_with_serde_defaults", "unknown_missing_and_duplicate_fields",
         "ron_syntax", "validation_rules", "defaults_match_the_reference", "solver_settings_follow_the_file",
         "material_table_lookup"]


def _make(target):
    subprocess.run(["make", "-s", "-C", str(PKG), target], check=True, capture_output=True)
    return PKG / target


def test_ron_scene_config_loader():
    exe = _make("lib/vxsim_config_tests")
    out = subprocess.run([str(exe), str(ROOT / "tests" / "golden" / "scenes")], capture_output=True, text=True,
                         timeout=120)
    for case in CASES:
        assert f"PASS {case}" in out.stdout, out.stdout + out.stderr
    assert out.stdout.count("PASS load ") >= 2, out.stdout
    assert out.returncode == 0, out.stdout + out.stderr


def test_capture_rejects_bad_arguments(tmp_path):
    """solver_scale_capture's argument rule (src/bin/solver_scale_capture.rs:58-60),
    checked before any device call."""
    exe = _make("lib/vxsim_capture")
    csv = tmp_path / "c.csv"
    for args in (["0"], ["5", "1"], ["5", "7"]):
        out = subprocess.run([str(exe), str(csv), *args], capture_output=True, text=True, timeout=60)
        assert out.returncode == 1
        assert "steps must be positive and saved_frames must be in 2..=steps+1" in out.stderr
    bad = tmp_path / "bad.ron"
    bad.write_text("( dimensions: (1, 1, 1) )")
    out = subprocess.run([str(exe), str(csv), "2", "2", str(bad)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 1 and "missing field `branch_dimensions`" in out.stderr
    assert not csv.exists()

"""The synthetic workloads that bench.py and the GPU tests run, pinned on the CPU.

Each generator stands in for a configuration of the reference's solver-scale
runs with seeded synthetic scenes: the 64^3 mixed block, the 160^3 damaged
lattice, the batched box unions and the served cutting requests
(vxsim/scenes.py, vxsim/batched.py, vxsim/served.py). The bench line's
`config` names them by their sizes; these tests hold those sizes, the fixed
and targeted REVs, the bond counts and the value distributions, so a change
to a generator shows here before it changes what the bench measures.
Topology follows Scene::from_voxels (src/scene.rs:558-570): a bond along
each axis to the next occupied cell.
"""
import math

import numpy as np
import pytest

from vxsim import batched as B
from vxsim import scenes as S
from vxsim import served as V


def test_mixed_block_64():
    s = S.mixed_block(64, seed=1)
    assert s.n == 64 ** 3 == 262_144
    # the bottom layer is fixed: 64^2 REVs without a free axis
    assert s.active_count() == 258_048
    assert int(s.kinematic.sum()) == 64 * 64 and not s.kinematic[s.cells[:, 2] > 0].any()
    assert s.bond_count() == 3 * 64 * 64 * 63
    # wood, iron, stone and aluminium, each drawn per REV with probability 1/4
    counts = np.bincount(s.material, minlength=6)
    assert counts[0] == 0 and counts[4] == 0
    assert np.abs(counts[[1, 2, 3, 5]] / s.n - 0.25).max() < 0.005
    wood = s.material == 1
    assert np.allclose(np.linalg.norm(s.fiber[wood], axis=1), 1.0, atol=1e-6)
    assert (s.anisotropy[wood] == 1.0).all() and (s.anisotropy[~wood] == 0.0).all()
    assert abs(s.materials[5].young - 70e9) < 1.0 and s.meta["passes"] == 5


def test_damaged_lattice_160():
    s = S.damaged_lattice(160, seed=2)
    assert s.n == 160 ** 3 == 4_096_000
    assert s.active_count() == 4_096_000 - 160 * 160
    full = 3 * 160 * 160 * 159
    assert s.bond_count() == full - round(0.10 * full) == 10_990_080
    free = s.kinematic == 0
    assert np.abs(s.loads[~free]).max() == 0.0
    assert abs(s.loads[free].std() - 0.05) < 5e-4 and abs(s.loads[free].mean()) < 5e-4
    assert s.meta["passes"] == 8 and tuple(s.meta["gravity"]) == (0, 0, 0)


@pytest.mark.parametrize("count,revs", [(64, 228_704), (512, 2_643_681)])
def test_batched_box_unions(count, revs):
    scenes = B.batched_scenes(count, seed=2024)
    assert sum(s.n for s in scenes) == revs
    # pool tiles of 256 REVs per scene
    assert B.pool_capacity(scenes) == sum(-(-s.n // 256) * 256 for s in scenes)
    edges = np.array([s.meta["edge"] for s in scenes])
    assert edges.min() >= 8 and edges.max() <= 48
    for s in scenes[:16]:
        e = s.meta["edge"]
        x = s.cells[:, 0]
        # every box spans the clamped axis: the x = 0 face is clamped, the far face targeted
        assert (s.kinematic[x == 0] == 1).all() and (s.kinematic[x > 0] == 0).all()
        far = x == e - 1
        assert (s.target_mask[far] == 7).all() and (s.target_mask[~far] == 0).all()
        assert np.allclose(s.target[far, 0] - s.position[far, 0], 5e-5)
        assert len(np.unique(s.material)) == 1


def test_served_templates():
    """The 16 request templates of the served workload (seed 77): a
    log-spaced grid of sizes over 1k-2M DOF. The raster rounds each block to
    whole cells, so the wood holds 0.38-1.10 of its grid size; the largest
    template's wood is 601,200 REVs (1.80M DOF). Every template carries the
    same 2 x 20 x 40 kinematic blade less its one-REV bevel (1,580 REVs)."""
    rng = np.random.default_rng(77)
    grid = np.exp(np.linspace(math.log(1e3), math.log(2e6), 16))
    wood, total = [], []
    for dof in grid:
        s, moving = V.served_scene(rng, dof=float(dof))
        n_wood = s.meta["wood_revs"]
        assert int(moving.sum()) == 1580 and (s.kinematic[moving] == 1).all()
        assert (s.target_mask[moving] == 7).all() and not moving[:n_wood].any()
        # the wood's bottom layer is clamped, its other REVs are free
        z = s.cells[:n_wood, 2]
        assert (s.kinematic[:n_wood][z == 0] == 1).all() and (s.kinematic[:n_wood][z > 0] == 0).all()
        wood.append(n_wood)
        total.append(s.n)
    assert total[-1] == 602_780 and wood[-1] == 601_200
    ratio = 3 * np.array(wood) / grid
    assert ratio.min() > 0.37 and ratio.max() < 1.11
    assert wood[0] == 256

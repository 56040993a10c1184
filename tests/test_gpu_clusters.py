"""rebuild_clusters on the device (vx_scene_rebuild_clusters) against the
oracle's restatement: the same cluster id for every REV and the same count."""
import numpy as np
import pytest

import pyoracle as O
from vxsim import native as N
from vxsim import scenes as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = N.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("edge,removed", [(8, 0.0), (12, 0.3), (20, 0.6), (33, 0.75)])
def test_clusters_match_the_oracle(ctx, edge, removed):
    rng = np.random.default_rng(edge)
    s = S.wood_cube(edge)
    s.neighbor[rng.random(s.neighbor.shape) < removed] = 0xFFFFFFFF
    d = N.DeviceScene(ctx, s)
    cl, cnt = d.rebuild_clusters()
    want, wcnt = O.rebuild_clusters(s.neighbor, s.kinematic)
    assert cnt == wcnt and np.array_equal(cl, want)
    cl2, cnt2 = d.rebuild_clusters()  # repeatable
    assert cnt2 == cnt and np.array_equal(cl2, cl)
    d.close()


def test_clusters_of_the_damaged_lattice_at_full_size(ctx):
    """The 160^3 damaged lattice (4,096,000 REVs, 10% of bonds removed)."""
    s = S.damaged_lattice(160, seed=1)
    d = N.DeviceScene(ctx, s)
    cl, cnt = d.rebuild_clusters()
    want, wcnt = O.rebuild_clusters(s.neighbor, s.kinematic)
    assert cnt == wcnt and np.array_equal(cl, want)
    d.close()


def test_two_rev_reference_case(ctx):
    cells = np.array([[0, 0, 0], [1, 0, 0]], np.int32)
    for kin, bonded, count in (((1, 0), False, 1), ((0, 0), False, 2), ((0, 0), True, 1)):
        s = S.from_cells(cells, 2, S.M.table(), kinematic=np.array(kin, np.uint8))
        s.neighbor[:] = 0xFFFFFFFF
        if bonded:
            s.neighbor[0, 0] = 1
        d = N.DeviceScene(ctx, s)
        cl, cnt = d.rebuild_clusters()
        want, wcnt = O.rebuild_clusters(s.neighbor, s.kinematic)
        assert cnt == wcnt == count and np.array_equal(cl, want)
        d.close()

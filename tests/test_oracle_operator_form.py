"""The two forms of one operator row, checked on the oracle's FP64 assembly.

The reference's row (src/solver.rs:1576-1699) is D_i p_i - P_i sum_e K_e p_j, with
D_i = P_i (m_i/h^2 I + sum_e K_e) P_i + (I - P_i) assembled. The FP32 kernels build
the same row from the mass term and the bonds they already read:
P_i (m_i/h^2 p_i + sum_e K_e (p_i - p_j)) + (I - P_i) p_i. The two agree on any
direction that vanishes on fixed axes, which every PCG direction does (the
residual is projected, so z = D^-1 r and p are zero there). This test restates
the second form in numpy over the oracle's assembled bonds and compares it with
the oracle's own matvec of the first.
"""
import numpy as np
import pytest

import pyoracle as O
from vxsim import scenes as S

EMPTY = np.uint32(0xFFFFFFFF)


def mass_term_row(sys, scene, h, p):
    n = scene.n
    free = sys["free"]
    k = sys["k"]          # [axis][i] stiffness of the bond i owns along axis
    state = sys["state"]  # [axis][i] 2 = assembled
    m = scene.mass.astype(np.float64) / (h * h)
    s = m[:, None] * p
    for a in range(3):
        j = scene.neighbor[a].astype(np.int64)
        own = (scene.neighbor[a] != EMPTY) & (state[a] == 2)
        i_idx = np.nonzero(own)[0]
        j_idx = j[own]
        d = p[i_idx] - p[j_idx]
        kv = np.einsum("nab,nb->na", k[a, i_idx], d)
        np.add.at(s, i_idx, kv)    # the owner i: K (p_i - p_j)
        np.add.at(s, j_idx, -kv)   # the neighbour j: K (p_j - p_i)
    return free * s + (1.0 - free) * p


@pytest.mark.parametrize("seed", [1, 2])
def test_mass_term_row_is_the_assembled_row(seed):
    scene = S.mixed_block(6, seed=seed)
    h = 1e-3
    o = O.OracleScene(scene)
    o.fit_rotations()
    o.assemble(h)
    sys = o.system_arrays()
    rng = np.random.default_rng(seed)
    p = rng.normal(size=(scene.n, 3)) * sys["free"]  # zero on fixed axes, as PCG directions are
    ref = o.matvec(p)
    alt = mass_term_row(sys, scene, h, p)
    err = np.max(np.abs(alt - ref)) / np.max(np.abs(ref))
    assert err < 1e-12, err


def test_the_forms_differ_off_the_pcg_subspace():
    # on a direction with nonzero fixed components the rows differ (the
    # assembled D is the identity there): the identity above needs the PCG's
    # projected directions, which is why the kernels may use it
    scene = S.mixed_block(6, seed=3)
    h = 1e-3
    o = O.OracleScene(scene)
    o.fit_rotations()
    o.assemble(h)
    sys = o.system_arrays()
    assert np.any(sys["free"] == 0.0)
    p = np.random.default_rng(3).normal(size=(scene.n, 3))
    ref = o.matvec(p)
    alt = mass_term_row(sys, scene, h, p)
    assert np.max(np.abs(alt - ref)) / np.max(np.abs(ref)) > 1e-6

"""The recurrences of the on-chip inner solve, emulated in FP32 on the
oracle's packed rows against the classic recurrence: the one-reduction form
(k_pcg_expanded) and the regrouped product of the one-scene range kernel
(k_pcg_persistent), which forms q = A p as A z + beta q_old so that the
in-range part of A z can be computed inside the r.z reduction.

The classic PCG loop (src/solver.rs:1857-1911) sums p.Ap for alpha, then the
updated r.z for beta: two grid-wide reductions per iteration on the device. The
expanded form (k_pcg_expanded) forms u = D^-1 r and v = D^-1 q for q = A p and
sums r.u, p.q, r.v + q.u, q.v, r.r, r.q and q.q in one reduction; the next
r.z is r.u - alpha (r.v + q.u) + alpha^2 q.v and the next r.r is
r.r - 2 alpha r.q + alpha^2 q.q. Neighbours form the next direction from the
published (u, v, p) as (u - alpha v) + beta' p. Here both loops run in numpy
with FP32 vectors, the FP32 operator of the reference's packed rows
(vxo_pack_rows: diagonal block, six neighbour blocks, inverse diagonal) and
FP64 sums of per-REV FP32 dot products, as on the device. The bar: the same
iteration count to each inner tolerance and the iterates within 2e-6.
"""
import numpy as np
import pytest

import pyoracle as O
from vxsim import scenes as S


def operator(rows):
    n = rows["n"]
    D = rows["diag9"].reshape(n, 3, 3)
    B = rows["blocks54"].reshape(n, 6, 3, 3)
    nb = rows["nbr6"].reshape(n, 6).astype(np.int64)
    ok = nb < n
    nbc = np.where(ok, nb, 0)
    Bz = np.where(ok[:, :, None, None], B, 0).astype(np.float32)
    Minv = rows["inv9"].reshape(n, 3, 3)

    def A(p):
        y = np.einsum("nij,nj->ni", D, p, dtype=np.float32)
        for t in range(6):
            y = y + np.einsum("nij,nj->ni", Bz[:, t], p[nbc[:, t]], dtype=np.float32)
        return y.astype(np.float32)

    def M(r):
        return np.einsum("nij,nj->ni", Minv, r, dtype=np.float32).astype(np.float32)

    return A, M, rows["rhs"].reshape(n, 3).astype(np.float32)


def dot(a, b):  # per-REV FP32 dot, summed in FP64
    return float(np.sum((a * b).sum(axis=1, dtype=np.float32), dtype=np.float64))


def classic(A, M, b, tol, maxit):
    x = np.zeros_like(b)
    r = b.copy()
    z = M(r)
    p = np.zeros_like(b)
    rz, rz_prev = dot(r, z), None
    init = np.sqrt(dot(r, r))
    for k in range(maxit):
        beta = np.float32(0.0) if k == 0 else np.float32(rz / rz_prev)
        p = (z + beta * p).astype(np.float32)
        q = A(p)
        alpha = np.float32(rz / dot(p, q))
        x = (x + alpha * p).astype(np.float32)
        r = (r - alpha * q).astype(np.float32)
        z = M(r)
        rz_prev, rz = rz, dot(r, z)
        if np.sqrt(dot(r, r)) / init < tol:
            return x, k + 1
    return x, maxit


def expanded(A, M, b, tol, maxit):
    x = np.zeros_like(b)
    r = b.copy()
    init = np.sqrt(dot(r, r))
    # the triple published before the first matvec: (u0, 0, 0) with alpha = beta = 0
    u_prev, v_prev, p_prev = M(r), np.zeros_like(b), np.zeros_like(b)
    alpha_prev, beta = np.float32(0.0), np.float32(0.0)
    for k in range(maxit):
        p = ((u_prev - alpha_prev * v_prev).astype(np.float32) + beta * p_prev).astype(np.float32)
        q = A(p)
        u, v = M(r), M(q)
        g, pq = dot(r, u), dot(p, q)
        a2, a3 = dot(r, v) + dot(q, u), dot(q, v)
        rr, rq, qq = dot(r, r), dot(r, q), dot(q, q)
        alpha = np.float32(g / pq)
        al = float(alpha)
        g_next = g - al * a2 + al * al * a3
        rr_next = rr - 2.0 * al * rq + al * al * qq
        x = (x + alpha * p).astype(np.float32)
        r = (r - alpha * q).astype(np.float32)
        u_prev, v_prev, p_prev, alpha_prev = u, v, p, alpha
        beta = np.float32(g_next / g)
        if np.sqrt(max(rr_next, 0.0)) / init < tol:
            return x, k + 1
    return x, maxit


@pytest.mark.parametrize("make", [lambda: S.mixed_block(8, seed=1), lambda: S.mixed_block(12, seed=3),
                                  lambda: S.damaged_lattice(10, seed=2)], ids=["mixed_8", "mixed_12", "damaged_10"])
def test_expanded_recurrence_takes_the_classic_iterations(make):
    s = make()
    o = O.OracleScene(s)
    o.fit_rotations()
    o.assemble(1e-3)
    A, M, b = operator(o.pack_rows())
    for tol in (1e-4, 1e-5, 1e-6):
        xc, kc = classic(A, M, b, tol, 5000)
        xe, ke = expanded(A, M, b, tol, 5000)
        err = np.linalg.norm(xe - xc) / np.linalg.norm(xc)
        assert ke == kc, (tol, kc, ke)
        assert err < 2e-6, (tol, err)


def regrouped(A, M, b, tol, maxit):
    """The classic loop with q = A p formed as A z + beta q_old (A is linear)."""
    x = np.zeros_like(b)
    r = b.copy()
    z = M(r)
    p, q = np.zeros_like(b), np.zeros_like(b)
    rz, rz_prev = dot(r, z), None
    init = np.sqrt(dot(r, r))
    for k in range(maxit):
        beta = np.float32(0.0) if k == 0 else np.float32(rz / rz_prev)
        az = A(z)
        p = (beta * p + z).astype(np.float32)
        q = (beta * q + az).astype(np.float32)
        alpha = np.float32(rz / dot(p, q))
        x = (x + alpha * p).astype(np.float32)
        r = (r - alpha * q).astype(np.float32)
        z = M(r)
        rz_prev, rz = rz, dot(r, z)
        if np.sqrt(dot(r, r)) / init < tol:
            return x, k + 1
    return x, maxit


@pytest.mark.parametrize("make", [lambda: S.mixed_block(8, seed=1), lambda: S.mixed_block(12, seed=3),
                                  lambda: S.damaged_lattice(10, seed=2)], ids=["mixed_8", "mixed_12", "damaged_10"])
def test_regrouped_product_takes_the_classic_iterations(make):
    s = make()
    o = O.OracleScene(s)
    o.fit_rotations()
    o.assemble(1e-3)
    A, M, b = operator(o.pack_rows())
    for tol in (1e-4, 1e-5, 1e-6):
        xc, kc = classic(A, M, b, tol, 5000)
        xg, kg = regrouped(A, M, b, tol, 5000)
        err = np.linalg.norm(xg - xc) / np.linalg.norm(xc)
        assert kg == kc, (tol, kc, kg)
        assert err < 2e-6, (tol, err)

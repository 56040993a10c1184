/*
 * vx_oracle.c — FP64 CPU restatement of the Voxel-sim corotational elastic solve.
 *
 * TEST INFRASTRUCTURE ONLY (the parity checker; never part of the product path).
 * Citations are file:line in TheLastie/Voxel-sim. glam 0.27.0 (Cargo.lock:551-554)
 * supplies the reference's 3x3/quaternion maths; its source is not vendored, so
 * the operations it provides (Mat3::inverse, Quat::from_mat3, Quat::slerp,
 * Quat * Vec3, normalize_or_zero) are restated from their mathematics below.
 */
#include "vx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* f32 constants of the reference: CELL = 0.01, AREA = CELL * CELL (src/scene.rs:10-11). */
static const float CELL_F = 0.01f;
#define AREA_F (CELL_F * CELL_F)
const double VXO_CELL = (double)0.01f;
const double VXO_AREA = (double)(0.01f * 0.01f);
/* 2 * AREA / CELL is an f32 expression in stiffness_matrix (src/solver.rs:72). */
static double k_scale(void) {
    volatile float a = AREA_F;
    volatile float c = CELL_F;
    return (double)(2.0f * a / c);
}

/* ---- small 3-vector / 3x3 / quaternion helpers (row-major m[r*3+c]) ------- */
static inline double dot3(const double* a, const double* b) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
static inline void cross3(const double* a, const double* b, double* o) {
    double x = a[1] * b[2] - a[2] * b[1];
    double y = a[2] * b[0] - a[0] * b[2];
    double z = a[0] * b[1] - a[1] * b[0];
    o[0] = x;
    o[1] = y;
    o[2] = z;
}
/* glam Vec3::normalize_or_zero: v / |v| when 1/|v| is finite and > 0, else zero. */
static inline void normalize_or_zero(const double* v, double* o) {
    double len = sqrt(dot3(v, v));
    double rcp = 1.0 / len;
    if (isfinite(rcp) && rcp > 0.0) {
        o[0] = v[0] * rcp;
        o[1] = v[1] * rcp;
        o[2] = v[2] * rcp;
    } else {
        o[0] = o[1] = o[2] = 0.0;
    }
}
static inline void col(const double* m, int c, double* v) {
    v[0] = m[c];
    v[1] = m[3 + c];
    v[2] = m[6 + c];
}
static inline void set_col(double* m, int c, const double* v) {
    m[c] = v[0];
    m[3 + c] = v[1];
    m[6 + c] = v[2];
}
static void mat_mul(const double* a, const double* b, double* o) {
    double t[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            t[r * 3 + c] = a[r * 3] * b[c] + a[r * 3 + 1] * b[3 + c] + a[r * 3 + 2] * b[6 + c];
    memcpy(o, t, sizeof t);
}
static void mat_transpose(const double* a, double* o) {
    double t[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) t[c * 3 + r] = a[r * 3 + c];
    memcpy(o, t, sizeof t);
}
static inline void mat_vec(const double* m, const double* v, double* o) {
    double x = m[0] * v[0] + m[1] * v[1] + m[2] * v[2];
    double y = m[3] * v[0] + m[4] * v[1] + m[5] * v[2];
    double z = m[6] * v[0] + m[7] * v[1] + m[8] * v[2];
    o[0] = x;
    o[1] = y;
    o[2] = z;
}
static inline void mat_t_vec(const double* m, const double* v, double* o) {
    double x = m[0] * v[0] + m[3] * v[1] + m[6] * v[2];
    double y = m[1] * v[0] + m[4] * v[1] + m[7] * v[2];
    double z = m[2] * v[0] + m[5] * v[1] + m[8] * v[2];
    o[0] = x;
    o[1] = y;
    o[2] = z;
}
/* det = z . (x cross y) over the columns. */
static double mat_det(const double* m) {
    double x[3], y[3], z[3], t[3];
    col(m, 0, x);
    col(m, 1, y);
    col(m, 2, z);
    cross3(x, y, t);
    return dot3(z, t);
}
/* Inverse by the adjugate: rows of the inverse are (y x z, z x x, x x y) / det. */
static void mat_inverse(const double* m, double* o) {
    double x[3], y[3], z[3], t0[3], t1[3], t2[3];
    col(m, 0, x);
    col(m, 1, y);
    col(m, 2, z);
    cross3(y, z, t0);
    cross3(z, x, t1);
    cross3(x, y, t2);
    double inv_det = 1.0 / dot3(z, t2);
    for (int c = 0; c < 3; ++c) {
        o[c] = t0[c] * inv_det;
        o[3 + c] = t1[c] * inv_det;
        o[6 + c] = t2[c] * inv_det;
    }
}
/* Quaternion rotation q * v = v (w^2 - b.b) + b (2 v.b) + (b x v)(2 w), b = (x, y, z). */
static void quat_rotate(const double* q, const double* v, double* o) {
    double b[3] = {q[0], q[1], q[2]};
    double w = q[3];
    double b2 = dot3(b, b);
    double vb2 = 2.0 * dot3(v, b);
    double bxv[3];
    cross3(b, v, bxv);
    double s = w * w - b2;
    for (int k = 0; k < 3; ++k) o[k] = v[k] * s + b[k] * vb2 + bxv[k] * (2.0 * w);
}
static void mat_from_quat(const double* q, double* m) {
    double x = q[0], y = q[1], z = q[2], w = q[3];
    double x2 = x + x, y2 = y + y, z2 = z + z;
    double xx = x * x2, xy = x * y2, xz = x * z2;
    double yy = y * y2, yz = y * z2, zz = z * z2;
    double wx = w * x2, wy = w * y2, wz = w * z2;
    double c0[3] = {1.0 - (yy + zz), xy + wz, xz - wy};
    double c1[3] = {xy - wz, 1.0 - (xx + zz), yz + wx};
    double c2[3] = {xz + wy, yz - wx, 1.0 - (xx + yy)};
    set_col(m, 0, c0);
    set_col(m, 1, c1);
    set_col(m, 2, c2);
}

/* basis(axis, q): columns q*e_axis, q*e_(axis+1), q*e_(axis+2) (src/solver.rs:27-34). */
void vxo_basis(int axis, const double q[4], double frame[9]) {
    for (int c = 0; c < 3; ++c) {
        double e[3] = {0.0, 0.0, 0.0};
        e[(axis + c) % 3] = 1.0;
        double v[3];
        quat_rotate(q, e, v);
        set_col(frame, c, v);
    }
}

/*
 * slerp(a, b, 0.5) (src/solver.rs:1326, glam Quat::slerp): glam flips b when
 * a.b < 0 and interpolates on the short arc; at s = 1/2 both its lerp and its
 * sine branches equal normalize(a + sign(a.b) b) in real arithmetic.
 */
void vxo_slerp_half(const double a[4], const double b[4], double out[4]) {
    double d = a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3];
    double s = d < 0.0 ? -1.0 : 1.0;
    double q[4];
    for (int k = 0; k < 4; ++k) q[k] = a[k] + s * b[k];
    double inv = 1.0 / sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    for (int k = 0; k < 4; ++k) out[k] = q[k] * inv;
}

/*
 * Rotation matrix -> quaternion (Quat::from_mat3, src/solver.rs:398), by the
 * four-branch method of M. Day, "Converting a Rotation Matrix to a Quaternion"
 * (2015): pick the largest of |x|,|y|,|z|,|w| from the diagonal and recover the
 * rest from the off-diagonal sums/differences. The result is not normalised.
 * mAB below is component B of column A.
 */
void vxo_quat_from_mat3(const double m[9], double q[4]) {
    double m00 = m[0], m01 = m[3], m02 = m[6];
    double m10 = m[1], m11 = m[4], m12 = m[7];
    double m20 = m[2], m21 = m[5], m22 = m[8];
    if (m22 <= 0.0) {
        double dif10 = m11 - m00;
        double omm22 = 1.0 - m22;
        if (dif10 <= 0.0) {
            double f = omm22 - dif10;
            double inv = 0.5 / sqrt(f);
            q[0] = f * inv;
            q[1] = (m01 + m10) * inv;
            q[2] = (m02 + m20) * inv;
            q[3] = (m12 - m21) * inv;
        } else {
            double f = omm22 + dif10;
            double inv = 0.5 / sqrt(f);
            q[0] = (m01 + m10) * inv;
            q[1] = f * inv;
            q[2] = (m12 + m21) * inv;
            q[3] = (m20 - m02) * inv;
        }
    } else {
        double sum10 = m11 + m00;
        double opm22 = 1.0 + m22;
        if (sum10 <= 0.0) {
            double f = opm22 - sum10;
            double inv = 0.5 / sqrt(f);
            q[0] = (m02 + m20) * inv;
            q[1] = (m12 + m21) * inv;
            q[2] = f * inv;
            q[3] = (m01 - m10) * inv;
        } else {
            double f = opm22 + sum10;
            double inv = 0.5 / sqrt(f);
            q[0] = (m12 - m21) * inv;
            q[1] = (m20 - m02) * inv;
            q[2] = (m01 - m10) * inv;
            q[3] = f * inv;
        }
    }
}

/*
 * fit_rotations (src/solver.rs:327-417): per-REV deformation columns averaged
 * over intact bonds (both endpoints, unless kinematic), Higham polar iteration
 * F <- (F + F^-T)/2 (<= 5 steps, stop at max change <= 1e-6), Gram-Schmidt,
 * quaternion; returns the largest 2 acos|q_old . q_new|.
 */
double vxo_fit_rotations(vxo_scene* s) {
    uint32_t n = s->n;
    double* grad = (double*)calloc((size_t)9 * n, sizeof(double));
    double* cnt = (double*)calloc((size_t)3 * n, sizeof(double));
    for (int axis = 0; axis < 3; ++axis) {
        for (uint32_t i = 0; i < n; ++i) {
            uint32_t j = s->nbr[(size_t)axis * n + i];
            if (j == VX_EMPTY) continue;
            double d[3];
            for (int k = 0; k < 3; ++k) d[k] = (s->pos[3 * (size_t)j + k] - s->pos[3 * (size_t)i + k]) / VXO_CELL;
            if (!s->kinematic[i]) {
                for (int k = 0; k < 3; ++k) grad[9 * (size_t)i + k * 3 + axis] += d[k];
                cnt[3 * (size_t)i + axis] += 1.0;
            }
            if (!s->kinematic[j]) {
                for (int k = 0; k < 3; ++k) grad[9 * (size_t)j + k * 3 + axis] += d[k];
                cnt[3 * (size_t)j + axis] += 1.0;
            }
        }
    }
    double max_angle = 0.0;
    for (uint32_t i = 0; i < n; ++i) {
        if (s->kinematic[i]) continue;
        double* q = s->rot + 4 * (size_t)i;
        double prev[4] = {q[0], q[1], q[2], q[3]};
        double old[9], f[9];
        mat_from_quat(q, old);
        memcpy(f, grad + 9 * (size_t)i, sizeof f);
        for (int axis = 0; axis < 3; ++axis) {
            double c[3];
            double k = cnt[3 * (size_t)i + axis];
            if (k > 0.0) {
                col(f, axis, c);
                for (int t = 0; t < 3; ++t) c[t] /= k;
            } else {
                col(old, axis, c);
            }
            set_col(f, axis, c);
        }
        if (mat_det(f) <= 1e-6) continue; /* angle 0 */
        for (int it = 0; it < 5; ++it) {
            double inv[9], invt[9], next[9];
            mat_inverse(f, inv);
            mat_transpose(inv, invt);
            double delta = 0.0;
            for (int k = 0; k < 9; ++k) {
                next[k] = (f[k] + invt[k]) * 0.5;
                double e = fabs(next[k] - f[k]);
                if (e > delta) delta = e;
            }
            memcpy(f, next, sizeof f);
            if (delta <= 1e-6) break;
        }
        double fx[3], fy[3], x[3], y[3], t[3];
        col(f, 0, fx);
        col(f, 1, fy);
        normalize_or_zero(fx, x);
        double xy = dot3(x, fy);
        for (int k = 0; k < 3; ++k) t[k] = fy[k] - x[k] * xy;
        normalize_or_zero(t, y);
        if (dot3(x, x) > 0.5 && dot3(y, y) > 0.5) {
            double z[3], m[9], nq[4];
            cross3(x, y, z);
            set_col(m, 0, x);
            set_col(m, 1, y);
            set_col(m, 2, z);
            vxo_quat_from_mat3(m, nq);
            double inv = 1.0 / sqrt(nq[0] * nq[0] + nq[1] * nq[1] + nq[2] * nq[2] + nq[3] * nq[3]);
            for (int k = 0; k < 4; ++k) q[k] = nq[k] * inv;
        }
        double d = fabs(prev[0] * q[0] + prev[1] * q[1] + prev[2] * q[2] + prev[3] * q[3]);
        if (d > 1.0) d = 1.0;
        double angle = 2.0 * acos(d);
        max_angle = fmax(max_angle, angle);
    }
    free(grad);
    free(cnt);
    return max_angle;
}

/* ---- topology (src/scene.rs:558-570, :1668-1681) -------------------------- */
static const int32_t* g_cells;
static int cmp_cell(const void* a, const void* b) {
    const int32_t* ca = g_cells + 3 * (size_t)(*(const uint32_t*)a);
    const int32_t* cb = g_cells + 3 * (size_t)(*(const uint32_t*)b);
    for (int k = 0; k < 3; ++k) {
        if (ca[k] < cb[k]) return -1;
        if (ca[k] > cb[k]) return 1;
    }
    return 0;
}
/*
 * Bond to the +axis cell when it is occupied and both REVs have the same
 * kinematic flag. Returns the number of bonds.
 */
uint32_t vxo_build_topology(const int32_t* cells, const uint8_t* kinematic, uint32_t n,
                            uint32_t* nbr) {
    uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint32_t i = 0; i < n; ++i) order[i] = i;
    g_cells = cells;
    qsort(order, n, sizeof(uint32_t), cmp_cell);
    uint32_t bonds = 0;
    for (int axis = 0; axis < 3; ++axis) {
        for (uint32_t i = 0; i < n; ++i) {
            int32_t key[3] = {cells[3 * (size_t)i], cells[3 * (size_t)i + 1], cells[3 * (size_t)i + 2]};
            key[axis] += 1;
            uint32_t lo = 0, hi = n, found = VX_EMPTY;
            while (lo < hi) {
                uint32_t mid = lo + (hi - lo) / 2;
                const int32_t* c = cells + 3 * (size_t)order[mid];
                int cmp = 0;
                for (int k = 0; k < 3 && !cmp; ++k) cmp = (c[k] < key[k]) ? -1 : (c[k] > key[k]) ? 1 : 0;
                if (cmp == 0) {
                    found = order[mid];
                    break;
                }
                if (cmp < 0) lo = mid + 1;
                else hi = mid;
            }
            uint32_t v = VX_EMPTY;
            if (found != VX_EMPTY && kinematic[i] == kinematic[found]) {
                v = found;
                ++bonds;
            }
            nbr[(size_t)axis * n + i] = v;
        }
    }
    free(order);
    return bonds;
}

/* ---- constitutive --------------------------------------------------------- */
static inline double clampd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline const vx_material* mat_of(const vxo_scene* s, uint32_t n) {
    return &s->materials[s->material[n]];
}
static void world_fiber(const vxo_scene* s, uint32_t n, double* out) {
    quat_rotate(s->rot + 4 * (size_t)n, s->fiber + 3 * (size_t)n, out);
}

/*
 * tensor_compliance (src/solver.rs:37-63): endpoint compliance in the bond
 * frame, diag(E_n, G, G) * solid with E_n = E_t + (E - E_t) f_x^2,
 * E_t = E + a (E_perp - E), minus the Sherman-Morrison rank-one term
 * alpha = G a 0.2. Returns 0 (and a zero matrix) for an invalid endpoint.
 */
int vxo_tensor_compliance(const vxo_scene* s, uint32_t n, const double frame[9], double c[9]) {
    const vx_material* m = mat_of(s, n);
    double solid = clampd(s->solid[n], 1e-4, 1.0);
    double fw[3], fiber[3];
    world_fiber(s, n, fw);
    mat_t_vec(frame, fw, fiber);
    double a = s->anisotropy[n];
    double young = m->young, young_perp = m->young_perp, shear = m->shear;
    double transverse = young + a * (young_perp - young);
    double normal = transverse + (young - transverse) * fiber[0] * fiber[0];
    double d[3] = {normal * solid, shear * solid, shear * solid};
    if (!isfinite(d[0]) || !isfinite(d[1]) || !isfinite(d[2]) || fmin(d[0], fmin(d[1], d[2])) <= 0.0) {
        memset(c, 0, 9 * sizeof(double));
        return 0;
    }
    double inv[3] = {1.0 / d[0], 1.0 / d[1], 1.0 / d[2]};
    double sf[3] = {fiber[0] * inv[0], fiber[1] * inv[1], fiber[2] * inv[2]};
    double alpha = shear * a * 0.2;
    double scale = alpha / (1.0 + alpha * dot3(fiber, sf));
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) c[r * 3 + k] = (r == k ? inv[r] : 0.0) - sf[r] * sf[k] * scale;
    return 1;
}

/* stiffness_matrix (src/solver.rs:65-73): (C_i + C_j)^-1 * 2 AREA / CELL. */
void vxo_stiffness_matrix(const vxo_scene* s, uint32_t i, uint32_t j, const double frame[9],
                          double k[9]) {
    double ci[9], cj[9], sum[9];
    int vi = vxo_tensor_compliance(s, i, frame, ci);
    int vj = vxo_tensor_compliance(s, j, frame, cj);
    if (!vi || !vj) {
        memset(k, 0, 9 * sizeof(double));
        return;
    }
    for (int t = 0; t < 9; ++t) sum[t] = ci[t] + cj[t];
    mat_inverse(sum, k);
    double sc = k_scale();
    for (int t = 0; t < 9; ++t) k[t] *= sc;
}

/*
 * bond_thermal_rest (src/solver.rs:78-95): local rest vector
 * F^T (d CELL + (e_i + e_j) CELL/2), e_n = (d a_perp + f (a_par - a_perp)(f.d)) dT_n.
 */
void vxo_bond_thermal_rest(const vxo_scene* s, uint32_t i, uint32_t j, const double frame[9],
                           double rest[3]) {
    double fx[3], dir[3];
    col(frame, 0, fx);
    normalize_or_zero(fx, dir);
    double e[3] = {0.0, 0.0, 0.0};
    uint32_t ends[2] = {i, j};
    for (int t = 0; t < 2; ++t) {
        uint32_t n = ends[t];
        const vx_material* m = mat_of(s, n);
        double fw[3], f[3];
        world_fiber(s, n, fw);
        normalize_or_zero(fw, f);
        double ap = m->thermal_expansion_parallel, an = m->thermal_expansion_perpendicular;
        double fd = (ap - an) * dot3(f, dir);
        double dT = s->thermal_delta[n];
        for (int k = 0; k < 3; ++k) e[k] += (dir[k] * an + f[k] * fd) * dT;
    }
    double w[3];
    for (int k = 0; k < 3; ++k) w[k] = dir[k] * VXO_CELL + e[k] * (0.5 * VXO_CELL);
    mat_t_vec(frame, w, rest);
}

/* make_constraint (src/solver.rs:1325-1345). */
void vxo_make_constraint(const vxo_scene* s, uint32_t i, int axis, uint32_t j, double frame[9],
                         double material_k[9], double k[9], double rest[3]) {
    double mid[4];
    vxo_slerp_half(s->rot + 4 * (size_t)i, s->rot + 4 * (size_t)j, mid);
    vxo_basis(axis, mid, frame);
    vxo_stiffness_matrix(s, i, j, frame, material_k);
    size_t e = (size_t)axis * s->n + i;
    double scale = fmax(1.0 - s->damage[e], 0.001);
    double local[9], ft[9], tmp[9];
    for (int t = 0; t < 9; ++t) local[t] = material_k[t] * scale;
    mat_transpose(frame, ft);
    mat_mul(frame, local, tmp);
    mat_mul(tmp, ft, k);
    double tr[3], v[3];
    vxo_bond_thermal_rest(s, i, j, frame, tr);
    for (int c = 0; c < 3; ++c) v[c] = tr[c] + s->formation[3 * e + c] + s->plastic[3 * e + c] * VXO_CELL;
    mat_vec(frame, v, rest);
}

/* directional (src/fracture.rs:73-75). */
static double directional(double parallel, double perpendicular, double alignment, double anisotropy) {
    return parallel + anisotropy * (1.0 - clampd(fabs(alignment), 0.0, 1.0)) * (perpendicular - parallel);
}

/* pair_limits (src/fracture.rs:76-133). */
void vxo_pair_limits(const vx_material* a, const vx_material* b, const double alignment[2],
                     const double anisotropy[2], vxo_limits* out) {
    const vx_material* ms[2] = {a, b};
    vxo_limits one[2];
    for (int k = 0; k < 2; ++k) {
        const vx_material* m = ms[k];
        double ductility;
        if (m->fracture_mode == VX_BRITTLE) ductility = 0.0;
        else if (m->fracture_mode == VX_DUCTILE) ductility = 1.0;
        else ductility = (1.0 - anisotropy[k]) * 0.5 + anisotropy[k] * fabs(alignment[k]) * fabs(alignment[k]);
        one[k].tension = directional(m->tensile_strength, m->tensile_strength_perp, alignment[k], anisotropy[k]);
        one[k].compression = directional(m->compressive_strength, m->compressive_strength_perp, alignment[k], anisotropy[k]);
        one[k].shear = directional(m->shear_strength, m->shear_strength_perp, alignment[k], anisotropy[k]);
        one[k].yield_stress = m->yield_strength;
        one[k].hardening = m->hardening_modulus;
        one[k].plastic_failure = m->failure_plastic_strain;
        one[k].ductility = ductility;
        one[k].fracture_energy = directional(m->fracture_energy, m->fracture_energy_perp, alignment[k], anisotropy[k]);
    }
    out->tension = fmin(one[0].tension, one[1].tension);
    out->compression = fmin(one[0].compression, one[1].compression);
    out->shear = fmin(one[0].shear, one[1].shear);
    out->yield_stress = fmin(one[0].yield_stress, one[1].yield_stress);
    out->hardening = fmin(one[0].hardening, one[1].hardening);
    out->plastic_failure = fmin(one[0].plastic_failure, one[1].plastic_failure);
    out->ductility = fmin(one[0].ductility, one[1].ductility);
    out->fracture_energy = fmin(one[0].fracture_energy, one[1].fracture_energy);
}

/* bond_limits (src/solver.rs:124-158): pair limits scaled by solid^2 * thermal strength. */
void vxo_bond_limits(const vxo_scene* s, uint32_t i, uint32_t j, const double direction[3],
                     vxo_limits* out) {
    double fi[3], fj[3];
    world_fiber(s, i, fi);
    world_fiber(s, j, fj);
    double alignment[2] = {dot3(direction, fi), dot3(direction, fj)};
    double aniso[2] = {s->anisotropy[i], s->anisotropy[j]};
    vxo_pair_limits(mat_of(s, i), mat_of(s, j), alignment, aniso, out);
    double solid = 1.0, thermal = 1.0;
    uint32_t ends[2] = {i, j};
    for (int t = 0; t < 2; ++t) {
        solid = fmin(solid, clampd(s->solid[ends[t]], 0.0, 1.0));
        thermal = fmin(thermal, s->thermal_scale[ends[t]]);
    }
    double scale = solid * solid * thermal;
    out->tension *= scale;
    out->compression *= scale;
    out->shear *= scale;
    out->yield_stress *= scale;
    out->hardening *= scale;
    out->fracture_energy *= scale;
}

/* energy (src/fracture.rs:186-188). */
static double energy(const double* u, const double* k, double damage) {
    double ku[3];
    mat_vec(k, u, ku);
    return fmax(0.5 * (1.0 - damage) * dot3(u, ku), 0.0);
}

/* fatigue (src/fracture.rs:190-207). */
void vxo_fatigue(vxo_bond* b, double signed_ratio, const vxo_fracture_config* c) {
    double delta = signed_ratio - b->previous_stress_ratio;
    if (fabs(delta) > 1e-6) {
        if (b->loading_increment * delta < 0.0) {
            double amplitude = fabs(b->previous_stress_ratio - b->reversal_stress_ratio) * 0.5;
            if (amplitude > c->fatigue_threshold) {
                double level = fmin((amplitude - c->fatigue_threshold) / (1.0 - c->fatigue_threshold), 1.0);
                b->fatigue_damage = fmin(b->fatigue_damage + 0.5 * pow(level, c->fatigue_exponent) / c->fatigue_cycles, 1.0);
            }
            b->reversal_stress_ratio = b->previous_stress_ratio;
        }
        b->loading_increment = delta;
    }
    b->previous_stress_ratio = signed_ratio;
}

/*
 * Ductile return map of fracture::update (src/fracture.rs:226-243) as a pure
 * function: returns the plastic increment dp (zero when no yield) and dep.
 */
static int return_map(const double* u_total, const double* plastic, const double* k,
                      const vxo_limits* l, double eq_plastic, double* dp, double* dep_out) {
    dp[0] = dp[1] = dp[2] = 0.0;
    *dep_out = 0.0;
    if (!(l->ductility > 1e-5)) return 0;
    double u[3], trial[3];
    for (int c = 0; c < 3; ++c) u[c] = u_total[c] - plastic[c] * VXO_CELL;
    mat_vec(k, u, trial);
    for (int c = 0; c < 3; ++c) trial[c] /= VXO_AREA;
    double equivalent = sqrt(dot3(trial, trial));
    double yield_now = l->yield_stress + l->hardening * eq_plastic;
    if (!(equivalent > yield_now)) return 0;
    double dir[3], kinv[9], cd[3];
    for (int c = 0; c < 3; ++c) dir[c] = trial[c] / equivalent * VXO_AREA;
    mat_inverse(k, kinv);
    mat_vec(kinv, dir, cd);
    for (int c = 0; c < 3; ++c) cd[c] /= VXO_CELL;
    double elastic_modulus = 1.0 / fmax(sqrt(dot3(cd, cd)), 1e-20);
    double dep = (equivalent - yield_now) / (elastic_modulus + l->hardening) * l->ductility;
    double nd[3];
    normalize_or_zero(cd, nd);
    for (int c = 0; c < 3; ++c) dp[c] = nd[c] * dep;
    *dep_out = dep;
    return 1;
}

static void stress_of(const double* u_total, const double* plastic, const double* k, double* stress) {
    double u[3];
    for (int c = 0; c < 3; ++c) u[c] = u_total[c] - plastic[c] * VXO_CELL;
    mat_vec(k, u, stress);
    for (int c = 0; c < 3; ++c) stress[c] /= VXO_AREA;
}

/* Failure ratio of src/fracture.rs:246-254 from a stress vector. */
static double ratio_of(const double* stress, const vxo_limits* l) {
    double normal_limit = stress[0] >= 0.0 ? l->tension : l->compression;
    double a = stress[0] / fmax(normal_limit, 1.0);
    double sh = fmax(l->shear, 1.0);
    return sqrt(a * a + (stress[1] * stress[1] + stress[2] * stress[2]) / (sh * sh));
}

/* Read-only ratio that fracture::update would evaluate (after its return map). */
double vxo_stress_ratio(const double u_total[3], const double plastic[3], const double k[9],
                        const vxo_limits* l, double eq_plastic) {
    double dp[3], dep, p2[3], stress[3];
    return_map(u_total, plastic, k, l, eq_plastic, dp, &dep);
    for (int c = 0; c < 3; ++c) p2[c] = plastic[c] + dp[c];
    stress_of(u_total, p2, k, stress);
    return ratio_of(stress, l);
}

/* fracture::update (src/fracture.rs:210-292). */
void vxo_fracture_update(vxo_bond* b, const double u_total[3], const double k[9],
                         const vxo_limits* l, double dt, const vxo_fracture_config* c,
                         vxo_dissipation* out) {
    memset(out, 0, sizeof *out);
    if (b->neighbor == VX_EMPTY) return;
    double old_damage = b->damage;
    double u[3];
    for (int t = 0; t < 3; ++t) u[t] = u_total[t] - b->plastic[t] * VXO_CELL;
    double before = energy(u, k, old_damage);
    double dp[3], dep;
    if (return_map(u_total, b->plastic, k, l, b->equivalent_plastic_strain, dp, &dep)) {
        for (int t = 0; t < 3; ++t) b->plastic[t] += dp[t];
        b->equivalent_plastic_strain += dep;
        for (int t = 0; t < 3; ++t) u[t] = u_total[t] - b->plastic[t] * VXO_CELL;
        double lost = fmax(before - energy(u, k, old_damage), 0.0);
        b->plastic_work += lost;
        out->plastic_heat = lost * c->plastic_heat_fraction;
        out->stored_plastic = lost - out->plastic_heat;
    }
    double stress[3];
    double ku[3];
    mat_vec(k, u, ku);
    for (int t = 0; t < 3; ++t) stress[t] = ku[t] / VXO_AREA;
    double ratio = ratio_of(stress, l);
    double principal;
    double ax = fabs(stress[0]), ay = fabs(stress[1]), az = fabs(stress[2]);
    if (ax >= fmax(ay, az)) principal = stress[0];
    else if (ay >= az) principal = stress[1];
    else principal = stress[2];
    vxo_fatigue(b, copysign(ratio, principal), c);
    if (ratio >= 1.0) {
        if (l->ductility <= 1e-5) b->damage = 1.0;
        else b->damage = fmin(b->damage + c->damage_rate * dt * fmin(ratio, 10.0), 1.0);
    }
    if (l->ductility > 1e-5 && b->equivalent_plastic_strain >= fmax(l->plastic_failure, 1e-6))
        b->damage = fmin(b->damage + c->damage_rate * dt, 1.0);
    if (b->fatigue_damage >= 1.0) b->damage = 1.0;
    double lost = fmax(energy(u, k, old_damage) - energy(u, k, b->damage), 0.0);
    double surface_budget = l->fracture_energy * VXO_AREA * (b->damage - old_damage);
    out->surface_work = fmin(lost, surface_budget);
    double available = lost - out->surface_work;
    out->released = available * c->energy_release;
    out->damage_heat = available - out->released;
    if (b->damage >= 1.0) b->neighbor = VX_EMPTY;
}

/* ---- system ---------------------------------------------------------------- */
int vxo_system_alloc(vxo_system* sys, uint32_t n) {
    memset(sys, 0, sizeof *sys);
    sys->n = n;
    size_t m = n ? n : 1;
    sys->free = (double*)calloc(3 * m, sizeof(double));
    sys->diag = (double*)calloc(9 * m, sizeof(double));
    sys->rhs = (double*)calloc(3 * m, sizeof(double));
    sys->k = (double*)calloc(27 * m, sizeof(double));
    sys->material_k = (double*)calloc(27 * m, sizeof(double));
    sys->frame = (double*)calloc(27 * m, sizeof(double));
    sys->rest = (double*)calloc(9 * m, sizeof(double));
    sys->state = (uint8_t*)calloc(3 * m, 1);
    sys->c_i = (uint32_t*)calloc(3 * m, sizeof(uint32_t));
    sys->c_j = (uint32_t*)calloc(3 * m, sizeof(uint32_t));
    sys->c_axis = (uint32_t*)calloc(3 * m, sizeof(uint32_t));
    sys->incidence = (uint32_t*)calloc(6 * m, sizeof(uint32_t));
    sys->incidence_len = (uint8_t*)calloc(m, 1);
    sys->partner = (uint32_t*)calloc(3 * m, sizeof(uint32_t));
    return sys->partner && sys->free && sys->diag && sys->rhs && sys->k && sys->material_k && sys->frame &&
                   sys->rest && sys->state && sys->c_i && sys->c_j && sys->c_axis &&
                   sys->incidence && sys->incidence_len
               ? 0
               : -1;
}

void vxo_system_free(vxo_system* sys) {
    free(sys->free);
    free(sys->diag);
    free(sys->rhs);
    free(sys->k);
    free(sys->material_k);
    free(sys->frame);
    free(sys->rest);
    free(sys->state);
    free(sys->c_i);
    free(sys->c_j);
    free(sys->c_axis);
    free(sys->incidence);
    free(sys->incidence_len);
    free(sys->partner);
    memset(sys, 0, sizeof *sys);
}

static inline int all_zero3(const double* f) { return f[0] == 0.0 && f[1] == 0.0 && f[2] == 0.0; }

/*
 * Assembly of solve_coupled (src/solver.rs:1553-1636): free mask, diagonal
 * m/h^2 I + sum K_e, rhs (pred - x) m/h^2 + load +/- K_e (x_j - x_i - rest_e),
 * projection rhs *= free, D = P D P + (I - P). Bonds with no free DOF at either
 * end are kept for fracture only; those with a kinematic owner are skipped.
 */
void vxo_assemble(const vxo_scene* s, const uint8_t* target_mask, const double* loads,
                  const double* predicted, double h, vxo_system* sys) {
    uint32_t n = s->n;
    for (uint32_t i = 0; i < n; ++i) {
        for (int a = 0; a < 3; ++a) {
            int fixed = s->kinematic[i] || (target_mask && ((target_mask[i] >> a) & 1));
            sys->free[3 * (size_t)i + a] = fixed ? 0.0 : 1.0;
        }
        double m = s->mass[i] / (h * h);
        double* d = sys->diag + 9 * (size_t)i;
        memset(d, 0, 9 * sizeof(double));
        d[0] = d[4] = d[8] = m;
        for (int a = 0; a < 3; ++a) {
            double pred = predicted ? predicted[3 * (size_t)i + a] : s->pos[3 * (size_t)i + a];
            sys->rhs[3 * (size_t)i + a] =
                (pred - s->pos[3 * (size_t)i + a]) * m + (loads ? loads[3 * (size_t)i + a] : 0.0);
        }
        sys->incidence_len[i] = 0;
    }
    memset(sys->state, 0, 3 * (size_t)n);
    memset(sys->k, 0, 27 * (size_t)n * sizeof(double));
    sys->c_count = 0;
    for (int axis = 0; axis < 3; ++axis) {
        for (uint32_t i = 0; i < n; ++i) {
            size_t e = (size_t)axis * n + i;
            uint32_t j = s->nbr[e];
            if (j == VX_EMPTY) continue;
            int fi0 = all_zero3(sys->free + 3 * (size_t)i);
            int fj0 = all_zero3(sys->free + 3 * (size_t)j);
            if (fi0 && fj0 && s->kinematic[i]) continue;
            double* k = sys->k + 9 * e;
            vxo_make_constraint(s, i, axis, j, sys->frame + 9 * e, sys->material_k + 9 * e, k,
                                sys->rest + 3 * e);
            sys->partner[e] = j;
            uint32_t edge = sys->c_count++;
            sys->c_i[edge] = i;
            sys->c_j[edge] = j;
            sys->c_axis[edge] = (uint32_t)axis;
            if (fi0 && fj0) {
                sys->state[e] = 1;
                continue;
            }
            sys->state[e] = 2;
            double dxr[3], force[3];
            for (int c = 0; c < 3; ++c)
                dxr[c] = s->pos[3 * (size_t)j + c] - s->pos[3 * (size_t)i + c] - sys->rest[3 * e + c];
            mat_vec(k, dxr, force);
            for (int c = 0; c < 3; ++c) {
                sys->rhs[3 * (size_t)i + c] += force[c];
                sys->rhs[3 * (size_t)j + c] -= force[c];
            }
            for (int t = 0; t < 9; ++t) {
                sys->diag[9 * (size_t)i + t] += k[t];
                sys->diag[9 * (size_t)j + t] += k[t];
            }
            uint32_t ends[2] = {i, j};
            for (int t = 0; t < 2; ++t) {
                uint32_t v = ends[t];
                sys->incidence[6 * (size_t)v + sys->incidence_len[v]++] = (uint32_t)e;
            }
        }
    }
    for (uint32_t i = 0; i < n; ++i) {
        const double* f = sys->free + 3 * (size_t)i;
        for (int a = 0; a < 3; ++a) sys->rhs[3 * (size_t)i + a] *= f[a];
        double* d = sys->diag + 9 * (size_t)i;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) d[r * 3 + c] = f[r] * d[r * 3 + c] * f[c] + (r == c ? 1.0 - f[r] : 0.0);
    }
}

/*
 * Row apply of src/solver.rs:1674-1699 over all REVs: D_i v_i plus
 * -P_i K_e P_j v_j for every assembled bond in incidence order. Rows of REVs
 * with no free axis are identity rows with zero right-hand side, so they stay
 * zero and leave every dot product unchanged.
 */
/* Rows are independent, so the parallel loop (above the reference's 32,768-REV
 * Rayon threshold, src/solver.rs:1700-1709) gives the same bits as the serial one. */
#define VXO_PAR_REVS 32768u
void vxo_matvec(const vxo_system* sys, const double* p, double* out) {
    uint32_t n = sys->n;
#pragma omp parallel for schedule(static) if (n >= VXO_PAR_REVS)
    for (long li = 0; li < (long)n; ++li) {
        uint32_t i = (uint32_t)li;
        double v[3];
        mat_vec(sys->diag + 9 * (size_t)i, p + 3 * (size_t)i, v);
        const double* fi = sys->free + 3 * (size_t)i;
        for (int t = 0; t < sys->incidence_len[i]; ++t) {
            size_t e = sys->incidence[6 * (size_t)i + t];
            uint32_t owner = (uint32_t)(e % n);
            uint32_t j = (owner == i) ? sys->partner[e] : owner;
            const double* fj = sys->free + 3 * (size_t)j;
            if (all_zero3(fj)) continue; /* slot to an inactive neighbour is zero (:1663-1670) */
            const double* k = sys->k + 9 * e;
            const double* pj = p + 3 * (size_t)j;
            for (int r = 0; r < 3; ++r) {
                double acc = 0.0;
                for (int c = 0; c < 3; ++c) acc += -fi[r] * k[r * 3 + c] * fj[c] * pj[c];
                v[r] += acc;
            }
        }
        memcpy(out + 3 * (size_t)i, v, sizeof v);
    }
}

/* cholesky_lower with the 1e-20 pivot floors (src/solver.rs:1347-1360). */
static void cholesky_lower(const double* m, double* l) {
    double l00 = sqrt(fmax(m[0], 1e-20));
    double l10 = m[3] / l00;
    double l20 = m[6] / l00;
    double l11 = sqrt(fmax(m[4] - l10 * l10, 1e-20));
    double l21 = (m[7] - l20 * l10) / l11;
    double l22 = sqrt(fmax(m[8] - l20 * l20 - l21 * l21, 1e-20));
    double t[9] = {l00, 0.0, 0.0, l10, l11, 0.0, l20, l21, l22};
    memcpy(l, t, sizeof t);
}

/* build_block_jacobi (src/solver.rs:1447-1453): one Cholesky factor per REV. */
void vxo_factor_block_jacobi(const vxo_system* sys, double* factor) {
    for (uint32_t i = 0; i < sys->n; ++i) cholesky_lower(sys->diag + 9 * (size_t)i, factor + 9 * (size_t)i);
}

/* Block-Jacobi apply (src/solver.rs:1525-1535): z = L^-T L^-1 r with the lower solves of :1362-1376. */
static void bj_apply(const double* l, const double* r, double* z) {
    double x = r[0] / l[0];
    double y = (r[1] - l[3] * x) / l[4];
    double w = (r[2] - l[6] * x - l[7] * y) / l[8];
    double zz = w / l[8];
    double yy = (y - l[7] * zz) / l[4];
    double xx = (x - l[3] * yy - l[6] * zz) / l[0];
    z[0] = xx;
    z[1] = yy;
    z[2] = zz;
}

/*
 * Serial in REV order below the threshold (the reference's serial path). Above
 * it the reference sums with Rayon, whose order is not fixed; here each chunk of
 * 4,096 REVs is summed in order and the chunk sums are added in chunk order, so
 * the result does not depend on the thread count.
 */
#define VXO_DOT_CHUNK 4096u
static double vdot(uint32_t n, const double* a, const double* b) {
    if (n < VXO_PAR_REVS) {
        double s = 0.0;
        for (uint32_t i = 0; i < n; ++i) s += dot3(a + 3 * (size_t)i, b + 3 * (size_t)i);
        return s;
    }
    long chunks = (long)((n + VXO_DOT_CHUNK - 1) / VXO_DOT_CHUNK);
    double* part = (double*)malloc((size_t)chunks * sizeof(double));
#pragma omp parallel for schedule(static)
    for (long c = 0; c < chunks; ++c) {
        uint32_t lo = (uint32_t)c * VXO_DOT_CHUNK, hi = lo + VXO_DOT_CHUNK < n ? lo + VXO_DOT_CHUNK : n;
        double s = 0.0;
        for (uint32_t i = lo; i < hi; ++i) s += dot3(a + 3 * (size_t)i, b + 3 * (size_t)i);
        part[c] = s;
    }
    double s = 0.0;
    for (long c = 0; c < chunks; ++c) s += part[c];
    free(part);
    return s;
}

static void bj_apply_all(uint32_t n, const double* factor, const double* r, double* z) {
#pragma omp parallel for schedule(static) if (n >= VXO_PAR_REVS)
    for (long i = 0; i < (long)n; ++i) bj_apply(factor + 9 * (size_t)i, r + 3 * (size_t)i, z + 3 * (size_t)i);
}

/*
 * CPU PCG of solve_coupled (src/solver.rs:1833-1911) in FP64: x0 = 0, z = M^-1 r,
 * p = z; stop when |r|/|r0| < tolerance (strict, checked every iteration), at the
 * cap, or when p.Ap <= 1e-30. fixed_iterations != 0 skips the tolerance test.
 */
int vxo_pcg(const vxo_system* sys, const double* factor, uint32_t max_iterations,
            double tolerance, int fixed_iterations, double* dx, uint32_t* iterations,
            double* residual) {
    uint32_t n = sys->n;
    size_t m = 3 * (size_t)(n ? n : 1);
    double* r = (double*)malloc(m * sizeof(double));
    double* z = (double*)malloc(m * sizeof(double));
    double* p = (double*)malloc(m * sizeof(double));
    double* ap = (double*)malloc(m * sizeof(double));
    memcpy(r, sys->rhs, 3 * (size_t)n * sizeof(double));
    memset(dx, 0, 3 * (size_t)n * sizeof(double));
    bj_apply_all(n, factor, r, z);
    memcpy(p, z, 3 * (size_t)n * sizeof(double));
    double rz = vdot(n, r, z);
    double initial = sqrt(vdot(n, r, r));
    double res = 0.0;
    uint32_t it = 0;
    for (uint32_t k = 0; k < max_iterations; ++k) {
        if (initial <= 1e-12) break;
        vxo_matvec(sys, p, ap);
        ++it;
        double denom = vdot(n, p, ap);
        if (denom <= 1e-30) break;
        double alpha = rz / denom;
#pragma omp parallel for schedule(static) if (n >= VXO_PAR_REVS)
        for (long t = 0; t < 3 * (long)n; ++t) {
            dx[t] += alpha * p[t];
            r[t] -= alpha * ap[t];
        }
        res = sqrt(vdot(n, r, r)) / initial;
        if (!fixed_iterations && res < tolerance) break;
        bj_apply_all(n, factor, r, z);
        double next = vdot(n, r, z);
        double beta = next / rz;
#pragma omp parallel for schedule(static) if (n >= VXO_PAR_REVS)
        for (long t = 0; t < 3 * (long)n; ++t) p[t] = z[t] + beta * p[t];
        rz = next;
    }
    free(r);
    free(z);
    free(p);
    free(ap);
    *iterations = it;
    *residual = res;
    return 0;
}

/* |b - A dx| / |b| with the FP64 operator. */
double vxo_true_residual(const vxo_system* sys, const double* dx) {
    uint32_t n = sys->n;
    double* ax = (double*)malloc(3 * (size_t)(n ? n : 1) * sizeof(double));
    vxo_matvec(sys, dx, ax);
    double num = 0.0, den = 0.0;
    for (size_t t = 0; t < 3 * (size_t)n; ++t) {
        double d = sys->rhs[t] - ax[t];
        num += d * d;
        den += sys->rhs[t] * sys->rhs[t];
    }
    free(ax);
    return den > 0.0 ? sqrt(num / den) : 0.0;
}

/*
 * One corotational pass (solve_coupled, src/solver.rs:1542-1929, CPU branch):
 * assemble, factor unless the previous factor is reused (:1639), PCG, x += dx.
 * factor[9n] holds the block-Jacobi factor across passes.
 */
int vxo_solve_coupled(vxo_scene* s, const uint8_t* target_mask, const double* loads,
                      const double* predicted, double h, uint32_t max_iterations,
                      double tolerance, int reuse_preconditioner, double* factor,
                      vxo_system* sys, uint32_t* iterations, double* residual) {
    vxo_assemble(s, target_mask, loads, predicted, h, sys);
    if (!reuse_preconditioner) vxo_factor_block_jacobi(sys, factor);
    double* dx = (double*)malloc(3 * (size_t)(s->n ? s->n : 1) * sizeof(double));
    vxo_pcg(sys, factor, max_iterations, tolerance, 0, dx, iterations, residual);
    for (size_t t = 0; t < 3 * (size_t)s->n; ++t) s->pos[t] += dx[t];
    free(dx);
    return 0;
}

/*
 * Stress evaluation of the fracture loop (src/solver.rs:627-647): for each
 * constraint of the last assembly whose bond is intact and whose owner is not
 * kinematic, limits from the current rotations, u = F^T (x_j - x_i) - thermal
 * rest - formation offset, last_force = F (K (u - plastic CELL)) (1 - damage),
 * and the ratio fracture::update evaluates after its return map
 * (src/fracture.rs:226-254). Other bonds get ratio -1 and zero force.
 */
void vxo_bond_stress(const vxo_scene* s, const vxo_system* sys, double* ratio, double* force) {
    uint32_t n = s->n;
    for (size_t e = 0; e < 3 * (size_t)n; ++e) {
        if (ratio) ratio[e] = -1.0;
        if (force) force[3 * e] = force[3 * e + 1] = force[3 * e + 2] = 0.0;
    }
    for (uint32_t c = 0; c < sys->c_count; ++c) {
        uint32_t i = sys->c_i[c], j = sys->c_j[c], axis = sys->c_axis[c];
        size_t e = (size_t)axis * n + i;
        if (s->nbr[e] == VX_EMPTY || s->kinematic[i]) continue;
        const double* frame = sys->frame + 9 * e;
        const double* k = sys->material_k + 9 * e;
        double dir[3], lim_dir[3];
        col(frame, 0, dir);
        memcpy(lim_dir, dir, sizeof dir);
        vxo_limits l;
        vxo_bond_limits(s, i, j, lim_dir, &l);
        double d[3], u[3], tr[3];
        for (int t = 0; t < 3; ++t) d[t] = s->pos[3 * (size_t)j + t] - s->pos[3 * (size_t)i + t];
        mat_t_vec(frame, d, u);
        vxo_bond_thermal_rest(s, i, j, frame, tr);
        for (int t = 0; t < 3; ++t) u[t] = u[t] - tr[t] - s->formation[3 * e + t];
        if (force) {
            double ue[3], ku[3], f[3];
            for (int t = 0; t < 3; ++t) ue[t] = u[t] - s->plastic[3 * e + t] * VXO_CELL;
            mat_vec(k, ue, ku);
            mat_vec(frame, ku, f);
            for (int t = 0; t < 3; ++t) force[3 * e + t] = f[t] * (1.0 - s->damage[e]);
        }
        if (ratio)
            ratio[e] = vxo_stress_ratio(u, s->plastic + 3 * e, k, &l, s->eq_plastic ? s->eq_plastic[e] : 0.0);
    }
}

/* ---- packed active-row system (src/solver.rs:1646-1672, :1731-1777) ------- */
uint32_t vxo_pack_rows(const vxo_system* sys, uint32_t* active, float* rhs, uint32_t* nbr6,
                       float* diag9, float* blocks54, float* inv9) {
    uint32_t n = sys->n;
    uint32_t* index = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t count = 0;
    for (uint32_t i = 0; i < n; ++i) {
        index[i] = VX_EMPTY;
        if (!all_zero3(sys->free + 3 * (size_t)i)) {
            index[i] = count;
            if (active) active[count] = i;
            ++count;
        }
    }
    uint32_t slot = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (index[i] == VX_EMPTY) continue;
        const double* fi = sys->free + 3 * (size_t)i;
        for (int t = 0; t < 6; ++t) nbr6[6 * (size_t)slot + t] = VX_EMPTY;
        memset(blocks54 + 54 * (size_t)slot, 0, 54 * sizeof(float));
        for (int t = 0; t < sys->incidence_len[i]; ++t) {
            size_t e = sys->incidence[6 * (size_t)i + t];
            uint32_t owner = (uint32_t)(e % n);
            uint32_t j = (owner == i) ? sys->partner[e] : owner;
            nbr6[6 * (size_t)slot + t] = index[j];
            if (index[j] == VX_EMPTY) continue;
            const double* fj = sys->free + 3 * (size_t)j;
            const double* k = sys->k + 9 * e;
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c)
                    blocks54[54 * (size_t)slot + 9 * t + 3 * r + c] = (float)(-fi[r] * k[3 * r + c] * fj[c]);
        }
        double inv[9];
        mat_inverse(sys->diag + 9 * (size_t)i, inv);
        for (int t = 0; t < 9; ++t) {
            diag9[9 * (size_t)slot + t] = (float)sys->diag[9 * (size_t)i + t];
            inv9[9 * (size_t)slot + t] = (float)inv[t];
        }
        for (int t = 0; t < 3; ++t) rhs[3 * (size_t)slot + t] = (float)sys->rhs[3 * (size_t)i + t];
        ++slot;
    }
    free(index);
    return count;
}

/* ---- the reference's f32 PCG loops --------------------------------------- */
/* glam f32 Mat3 * Vec3: column accumulation with separate multiply and add. */
static inline void m3v_f32(const float* m /* row-major */, const float* v, float* o) {
    float x = m[0] * v[0];
    float y = m[3] * v[0];
    float z = m[6] * v[0];
    x = x + m[1] * v[1];
    y = y + m[4] * v[1];
    z = z + m[7] * v[1];
    x = x + m[2] * v[2];
    y = y + m[5] * v[2];
    z = z + m[8] * v[2];
    o[0] = x;
    o[1] = y;
    o[2] = z;
}
static inline float dot_f32(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

static double vdot_f32(uint32_t n, const float* a, const float* b, int par) {
    double s = 0.0;
    if (par) {
#pragma omp parallel for reduction(+ : s) schedule(static)
        for (long i = 0; i < (long)n; ++i) s += (double)dot_f32(a + 3 * (size_t)i, b + 3 * (size_t)i);
    } else {
        for (uint32_t i = 0; i < n; ++i) s += (double)dot_f32(a + 3 * (size_t)i, b + 3 * (size_t)i);
    }
    return s;
}
static void cholesky_f32(const float* m, float* l) {
    float l00 = sqrtf(fmaxf(m[0], 1e-20f));
    float l10 = m[3] / l00;
    float l20 = m[6] / l00;
    float l11 = sqrtf(fmaxf(m[4] - l10 * l10, 1e-20f));
    float l21 = (m[7] - l20 * l10) / l11;
    float l22 = sqrtf(fmaxf(m[8] - l20 * l20 - l21 * l21, 1e-20f));
    float t[9] = {l00, 0.0f, 0.0f, l10, l11, 0.0f, l20, l21, l22};
    memcpy(l, t, sizeof t);
}
static inline void bj_apply_f32(const float* l, const float* r, float* z) {
    float x = r[0] / l[0];
    float y = (r[1] - l[3] * x) / l[4];
    float w = (r[2] - l[6] * x - l[7] * y) / l[8];
    float zz = w / l[8];
    float yy = (y - l[7] * zz) / l[4];
    float xx = (x - l[3] * yy - l[6] * zz) / l[0];
    z[0] = xx;
    z[1] = yy;
    z[2] = zz;
}
static void apply_rows_f32(uint32_t n, const uint32_t* nbr6, const float* diag9,
                           const float* blocks54, const float* v, float* out, int par) {
#pragma omp parallel for schedule(static) if (par)
    for (long i = 0; i < (long)n; ++i) {
        float value[3];
        m3v_f32(diag9 + 9 * (size_t)i, v + 3 * (size_t)i, value);
        for (int t = 0; t < 6; ++t) {
            uint32_t j = nbr6[6 * (size_t)i + t];
            if (j == VX_EMPTY) continue;
            float add[3];
            m3v_f32(blocks54 + 54 * (size_t)i + 9 * t, v + 3 * (size_t)j, add);
            value[0] = value[0] + add[0];
            value[1] = value[1] + add[1];
            value[2] = value[2] + add[2];
        }
        out[3 * (size_t)i] = value[0];
        out[3 * (size_t)i + 1] = value[1];
        out[3 * (size_t)i + 2] = value[2];
    }
}

/*
 * The reference's CPU block-Jacobi PCG (src/solver.rs:1833-1911) on the packed
 * active-row system, in its precision: f32 vectors and blocks, Vec3 dots in
 * f32 summed in f64 (:1700-1709), alpha/beta rounded to f32 (:1867, :1900),
 * |r|/|r0| < tolerance checked every iteration. The loops run on `threads`
 * OpenMP threads when n >= 32768, the reference's Rayon threshold
 * (src/solver.rs:14-25); below it they are serial, as in the reference.
 */
int vxo_pcg_rows_f32(uint32_t n, const float* rhs, const uint32_t* nbr6, const float* diag9,
                     const float* blocks54, uint32_t max_iterations, float tolerance,
                     int threads, float* dx, uint32_t* iterations, float* residual) {
    int par = n >= 32768 && threads > 1;
#ifdef _OPENMP
    extern void omp_set_num_threads(int);
    if (threads > 0) omp_set_num_threads(threads);
#endif
    size_t m = 3 * (size_t)(n ? n : 1);
    float* r = (float*)malloc(m * sizeof(float));
    float* z = (float*)malloc(m * sizeof(float));
    float* p = (float*)malloc(m * sizeof(float));
    float* ap = (float*)malloc(m * sizeof(float));
    float* l = (float*)malloc(3 * m * sizeof(float));
    memcpy(r, rhs, 3 * (size_t)n * sizeof(float));
    memset(dx, 0, 3 * (size_t)n * sizeof(float));
    for (uint32_t i = 0; i < n; ++i) cholesky_f32(diag9 + 9 * (size_t)i, l + 9 * (size_t)i);
#pragma omp parallel for schedule(static) if (par)
    for (long i = 0; i < (long)n; ++i) bj_apply_f32(l + 9 * (size_t)i, r + 3 * (size_t)i, z + 3 * (size_t)i);
    memcpy(p, z, 3 * (size_t)n * sizeof(float));
    double rz = vdot_f32(n, r, z, par);
    double initial = sqrt(vdot_f32(n, r, r, par));
    float res = 0.0f;
    uint32_t it = 0;
    for (uint32_t k = 0; k < max_iterations; ++k) {
        if (initial <= 1e-12) break;
        apply_rows_f32(n, nbr6, diag9, blocks54, p, ap, par);
        ++it;
        double denom = vdot_f32(n, p, ap, par);
        if (denom <= 1e-30) break;
        float alpha = (float)(rz / denom);
#pragma omp parallel for schedule(static) if (par)
        for (long t = 0; t < 3 * (long)n; ++t) {
            dx[t] = dx[t] + alpha * p[t];
            r[t] = r[t] - alpha * ap[t];
        }
        res = (float)(sqrt(vdot_f32(n, r, r, par)) / initial);
        if (res < tolerance) break;
#pragma omp parallel for schedule(static) if (par)
        for (long i = 0; i < (long)n; ++i) bj_apply_f32(l + 9 * (size_t)i, r + 3 * (size_t)i, z + 3 * (size_t)i);
        double next = vdot_f32(n, r, z, par);
        float beta = (float)(next / rz);
#pragma omp parallel for schedule(static) if (par)
        for (long t = 0; t < 3 * (long)n; ++t) p[t] = z[t] + beta * p[t];
        rz = next;
    }
    free(r);
    free(z);
    free(p);
    free(ap);
    free(l);
    *iterations = it;
    *residual = res;
    return 0;
}

/* dot_product_single (src/cuda/pcg.ptx:563-637): 256 strided f64 lane sums, tree-reduced. */
static double ptx_dot_single(uint32_t n, const float* a, const float* b) {
    double lane[256];
    for (int t = 0; t < 256; ++t) {
        double acc = 0.0;
        for (uint32_t i = (uint32_t)t; i < n; i += 256) {
            const float* x = a + 3 * (size_t)i;
            const float* y = b + 3 * (size_t)i;
            double v = (double)x[0] * (double)y[0];
            v = fma((double)x[1], (double)y[1], v);
            v = fma((double)x[2], (double)y[2], v);
            acc += v;
        }
        lane[t] = acc;
    }
    for (int stride = 128; stride > 0; stride >>= 1)
        for (int t = 0; t < stride; ++t) lane[t] += lane[t + stride];
    return lane[0];
}
/* Row-major 3x3 times vector with the PTX's mul/fma order (pcg.ptx:39-47, :139-147). */
static inline void ptx_m3v(const float* m, const float* v, float* o) {
    for (int r = 0; r < 3; ++r) {
        float acc = m[3 * r] * v[0];
        acc = fmaf(m[3 * r + 1], v[1], acc);
        acc = fmaf(m[3 * r + 2], v[2], acc);
        o[r] = acc;
    }
}

/*
 * The reference's CUDA PCG (src/cuda_solver.rs:301-501 with the kernels of
 * src/cuda/pcg.ptx) restated on the CPU with the same f32 FMA order and f64
 * dot accumulation: z = inverse r, rho = r.z, p = z; per iteration matvec
 * (:4-103), alpha = f32(rho / p.Ap) or 0 when p.Ap <= 1e-30 (:639-724),
 * update + precondition (:468-557), rho' = r.z, beta = f32(rho'/rho) or 0 when
 * rho <= 1e-30 (:437-466), p = beta p + z (:199-230); every 16 iterations and at
 * the cap, relative = f32(sqrt(r.r)/|b|) and stop when <= tolerance.
 * Returns VX_OK, VX_NOT_CONVERGED or VX_NONFINITE like the reference's Err cases.
 */
int vxo_cuda_pcg_emulate(uint32_t n, const float* rhs, const uint32_t* nbr6,
                         const float* diag9, const float* blocks54, const float* inv9,
                         uint32_t max_iterations, float tolerance, float* dx,
                         uint32_t* iterations, float* residual) {
    *iterations = 0;
    *residual = 0.0f;
    if (n == 0) return VX_OK;
    double initial_sq = 0.0;
    for (size_t t = 0; t < 3 * (size_t)n; ++t) initial_sq += (double)rhs[t] * (double)rhs[t];
    double initial = sqrt(initial_sq);
    memset(dx, 0, 3 * (size_t)n * sizeof(float));
    if (initial <= 1e-12) return VX_OK;
    size_t m = 3 * (size_t)n;
    float* r = (float*)malloc(m * sizeof(float));
    float* z = (float*)malloc(m * sizeof(float));
    float* p = (float*)malloc(m * sizeof(float));
    float* ap = (float*)malloc(m * sizeof(float));
    memcpy(r, rhs, m * sizeof(float));
    for (uint32_t i = 0; i < n; ++i) ptx_m3v(inv9 + 9 * (size_t)i, r + 3 * (size_t)i, z + 3 * (size_t)i);
    double rho = ptx_dot_single(n, r, z);
    for (size_t t = 0; t < m; ++t) p[t] = fmaf(0.0f, 0.0f, z[t]);
    double rr = INFINITY;
    uint32_t it = 0;
    for (uint32_t k = 0; k < max_iterations; ++k) {
        for (uint32_t i = 0; i < n; ++i) {
            float acc[3];
            ptx_m3v(diag9 + 9 * (size_t)i, p + 3 * (size_t)i, acc);
            for (int s = 0; s < 6; ++s) {
                uint32_t j = nbr6[6 * (size_t)i + s];
                if (j == VX_EMPTY) continue;
                const float* b = blocks54 + 54 * (size_t)i + 9 * s;
                const float* x = p + 3 * (size_t)j;
                for (int row = 0; row < 3; ++row) {
                    acc[row] = fmaf(b[3 * row], x[0], acc[row]);
                    acc[row] = fmaf(b[3 * row + 1], x[1], acc[row]);
                    acc[row] = fmaf(b[3 * row + 2], x[2], acc[row]);
                }
            }
            memcpy(ap + 3 * (size_t)i, acc, sizeof acc);
        }
        double den = ptx_dot_single(n, p, ap);
        float alpha = den > 1e-30 ? (float)(rho / den) : 0.0f;
        for (size_t t = 0; t < m; ++t) {
            dx[t] = fmaf(alpha, p[t], dx[t]);
            r[t] = fmaf(-alpha, ap[t], r[t]);
        }
        for (uint32_t i = 0; i < n; ++i) ptx_m3v(inv9 + 9 * (size_t)i, r + 3 * (size_t)i, z + 3 * (size_t)i);
        double rho_next = ptx_dot_single(n, r, z);
        float beta = rho > 1e-30 ? (float)(rho_next / rho) : 0.0f;
        for (size_t t = 0; t < m; ++t) p[t] = fmaf(beta, p[t], z[t]);
        rho = rho_next;
        ++it;
        if (it % 16 == 0 || it == max_iterations) {
            rr = ptx_dot_single(n, r, r);
            if (!isfinite(rr) || rr < 0.0) break;
            float relative = (float)(sqrt(rr) / initial);
            if (relative <= tolerance) break;
        }
    }
    free(r);
    free(z);
    free(p);
    free(ap);
    *iterations = it;
    if (!isfinite(rr) || rr < 0.0) return VX_NONFINITE;
    float relative = (float)(sqrt(rr) / initial);
    *residual = relative;
    if (!isfinite(relative) || relative > tolerance) return VX_NOT_CONVERGED;
    for (size_t t = 0; t < m; ++t)
        if (!isfinite(dx[t])) return VX_NONFINITE;
    return VX_OK;
}

/* ---- one fixed step ------------------------------------------------------- */
/*
 * step_with_axis_targets_and_loads (src/solver.rs:440-763) restricted to the
 * elastic path: explicit prediction (:500-523), fit_rotations (:543), the
 * corotation loop (:546-570), the fracture loop (:627-665), velocity recovery
 * (:668-683) and the external-work ledger (:709-725). Tool, contact, bonding,
 * fusion, delayed releases, heat and world bounds are outside this path and
 * are not modelled; REV temperatures stay fixed.
 */
int vxo_step(vxo_scene* s, const vxo_step_config* cfg, vxo_dynamics* d) {
    uint32_t n = s->n;
    size_t m3 = 3 * (size_t)(n ? n : 1);
    double h = cfg->fixed_dt / (double)cfg->substeps;
    double* predicted = (double*)malloc(m3 * sizeof(double));
    double* drift = (double*)malloc(m3 * sizeof(double));
    double* start_pos = (double*)malloc(m3 * sizeof(double));
    double* start_vel = (double*)malloc(m3 * sizeof(double));
    double* solved = (double*)malloc(m3 * sizeof(double));
    double* factor = (double*)calloc(9 * (size_t)(n ? n : 1), sizeof(double));
    double* load_vel = (double*)malloc(m3 * sizeof(double));
    uint8_t* work_mode = (uint8_t*)malloc((size_t)(n ? n : 1));
    vxo_system sys;
    vxo_system_alloc(&sys, n);
    for (uint32_t sub = 0; sub < cfg->substeps; ++sub) {
        memcpy(start_pos, s->pos, 3 * (size_t)n * sizeof(double));
        memcpy(start_vel, d->velocity, 3 * (size_t)n * sizeof(double));
        memcpy(d->previous, s->pos, 3 * (size_t)n * sizeof(double));
        memset(drift, 0, 3 * (size_t)n * sizeof(double));
        for (uint32_t i = 0; i < n; ++i) {
            if (s->kinematic[i]) continue;
            for (int a = 0; a < 3; ++a) {
                double* v = d->velocity + 3 * (size_t)i + a;
                *v += cfg->gravity[a] * h;
                if ((d->target_mask[i] >> a) & 1) *v = 0.0;
                drift[3 * (size_t)i + a] = *v;
                s->pos[3 * (size_t)i + a] += *v * h;
            }
        }
        for (uint32_t i = 0; i < n; ++i)
            for (int a = 0; a < 3; ++a)
                if ((d->target_mask[i] >> a) & 1) s->pos[3 * (size_t)i + a] = d->target[3 * (size_t)i + a];
        memcpy(predicted, s->pos, 3 * (size_t)n * sizeof(double));
        vxo_fit_rotations(s);
        for (uint32_t pass = 0; pass < cfg->corotation_iterations; ++pass) {
            uint32_t it = 0;
            double res = 0.0;
            vxo_solve_coupled(s, d->target_mask, d->applied_loads, predicted, h, cfg->iterations,
                              cfg->solver_tolerance, pass > 0, factor, &sys, &it, &res);
            d->solver_residual = res;
            d->pcg_iterations += it;
            if (pass + 1 == cfg->corotation_iterations) break;
            double change = vxo_fit_rotations(s);
            if (change <= cfg->corotation_tolerance && d->solver_residual <= cfg->solver_tolerance) break;
        }
        memcpy(solved, s->pos, 3 * (size_t)n * sizeof(double));
        /* contacts after the solve, before fracture reads the positions
           (src/solver.rs:575-590) */
        memset(work_mode, 0, (size_t)(n ? n : 1));
        vxo_contact* contacts = NULL;
        uint32_t ncontacts = 0;
        if (cfg->contact_enabled) {
            ncontacts = vxo_contact_project(n, s->pos, d->previous, d->rest, s->kinematic, s->mass, d->target_mask,
                                            s->nbr, &contacts, NULL);
            d->contacts += ncontacts;
            for (uint32_t k = 0; k < ncontacts; ++k) {
                uint8_t mode = contacts[k].new_impact ? 2 : 1;
                if (work_mode[contacts[k].i] < mode) work_mode[contacts[k].i] = mode;
                if (work_mode[contacts[k].j] < mode) work_mode[contacts[k].j] = mode;
            }
        }
        if (cfg->fracture_enabled) {
            for (uint32_t c = 0; c < sys.c_count; ++c) {
                uint32_t i = sys.c_i[c], j = sys.c_j[c], axis = sys.c_axis[c];
                size_t e = (size_t)axis * n + i;
                if (s->nbr[e] == VX_EMPTY || s->kinematic[i]) continue;
                const double* frame = sys.frame + 9 * e;
                const double* k = sys.material_k + 9 * e;
                double dir[3];
                col(frame, 0, dir);
                vxo_limits l;
                vxo_bond_limits(s, i, j, dir, &l);
                double dd[3], u[3], tr[3];
                for (int t = 0; t < 3; ++t) dd[t] = s->pos[3 * (size_t)j + t] - s->pos[3 * (size_t)i + t];
                mat_t_vec(frame, dd, u);
                vxo_bond_thermal_rest(s, i, j, frame, tr);
                vxo_bond* b = &d->bonds[e];
                for (int t = 0; t < 3; ++t) u[t] = u[t] - tr[t] - b->formation[t];
                double ue[3], ku[3], f[3];
                for (int t = 0; t < 3; ++t) ue[t] = u[t] - b->plastic[t] * VXO_CELL;
                mat_vec(k, ue, ku);
                mat_vec(frame, ku, f);
                for (int t = 0; t < 3; ++t) d->last_force[3 * e + t] = f[t] * (1.0 - b->damage);
                vxo_dissipation dis;
                vxo_fracture_update(b, u, k, &l, h, &cfg->fracture, &dis);
                d->plastic_heat += dis.plastic_heat;
                d->stored_plastic += dis.stored_plastic;
                d->surface_work += dis.surface_work;
                d->damage_heat += dis.damage_heat;
                d->pending_release += dis.released;
                /* mirror the bond state the solver reads */
                for (int t = 0; t < 3; ++t) s->plastic[3 * e + t] = b->plastic[t];
                s->damage[e] = b->damage;
                if (s->eq_plastic) s->eq_plastic[e] = b->equivalent_plastic_strain;
                if (b->neighbor == VX_EMPTY) {
                    s->nbr[e] = VX_EMPTY;
                    d->broken += 1;
                }
            }
        }
        for (uint32_t i = 0; i < n; ++i) {
            if (s->kinematic[i]) continue;
            for (int a = 0; a < 3; ++a) {
                size_t t = 3 * (size_t)i + a;
                if ((d->target_mask[i] >> a) & 1)
                    d->velocity[t] = (s->pos[t] - d->previous[t]) / h;
                else
                    d->velocity[t] = drift[t] + (solved[t] - predicted[t]) / h;
            }
        }
        memcpy(load_vel, d->velocity, 3 * (size_t)n * sizeof(double));
        if (cfg->contact_enabled)
            vxo_resolve_velocities(n, d->velocity, drift, s->kinematic, s->mass, d->target_mask, contacts, ncontacts,
                                   cfg->restitution, cfg->friction, &d->restitution_heat, &d->friction_heat);
        free(contacts);
        /* external work (src/solver.rs:744-760): the velocity quadrature, or the
           projected displacement under a persistent contact */
        for (uint32_t i = 0; i < n; ++i) {
            if (s->kinematic[i]) continue;
            double w = 0.0;
            for (int a = 0; a < 3; ++a) {
                size_t t = 3 * (size_t)i + a;
                double force = d->applied_loads[t] + cfg->gravity[a] * s->mass[i];
                if (work_mode[i] == 1)
                    w += force * (s->pos[t] - start_pos[t]);
                else
                    w += force * (start_vel[t] + load_vel[t]) * (0.5 * h);
            }
            d->external_work += w;
        }
    }
    free(work_mode);
    free(load_vel);
    vxo_system_free(&sys);
    free(predicted);
    free(drift);
    free(start_pos);
    free(start_vel);
    free(solved);
    free(factor);
    return 0;
}

/* ---- rebuild_clusters (src/solver.rs:828-858) ---------------------------- */
static uint32_t cluster_root(uint32_t* parent, uint32_t i) {
    while (parent[i] != i) {
        parent[i] = parent[parent[i]];
        i = parent[i];
    }
    return i;
}

uint32_t vxo_rebuild_clusters(uint32_t n, const uint32_t* neighbor, const uint8_t* kinematic, uint32_t* clusters) {
    uint32_t* parent = (uint32_t*)malloc((n ? n : 1) * sizeof(uint32_t));
    uint32_t* ids = (uint32_t*)malloc((n ? n : 1) * sizeof(uint32_t));
    for (uint32_t i = 0; i < n; ++i) {
        parent[i] = i;
        ids[i] = VX_EMPTY;
    }
    for (int a = 0; a < 3; ++a)
        for (uint32_t i = 0; i < n; ++i) {
            uint32_t j = neighbor[(size_t)a * n + i];
            if (j == VX_EMPTY) continue;
            uint32_t ra = cluster_root(parent, i), rc = cluster_root(parent, j);
            parent[rc] = ra;
        }
    /* the HashMap of the reference hands out ids in first-seen order */
    uint32_t count = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (kinematic[i]) {
            clusters[i] = VX_EMPTY;
            continue;
        }
        uint32_t r = cluster_root(parent, i);
        if (ids[r] == VX_EMPTY) ids[r] = count++;
        clusters[i] = ids[r];
    }
    free(parent);
    free(ids);
    return count;
}

/* ---- contact projection (collision::project, src/collision.rs:33-119, :376-505)
 * and velocity resolution (src/collision.rs:133-300), in double precision.
 * The reference's f32 literals are used at their f32 values.                 */
static const double C_BIN_HALF = 0.5001999735832214;     /* 0.5 + 2e-4 in f32 (bin_bounds, :437-444) */
static const double C_START_TOUCH = 0.009998999536037445; /* CELL - 1e-6 (swept_normal, :553) */
static const double C_NEW_IMPACT = 0.010001999326050282;  /* CELL + 2e-6 (project, :75) */
static const double C_1EM6 = 9.999999974752427e-07;
static const double C_SLOP = 1.9999999949504854e-06;     /* CONTACT_SLOP (:447) */
static const double C_1EM8 = 9.99999993922529e-09;
static const double C_1EM12 = 9.999999960041972e-13;
static const double C_1EM3 = 0.0010000000474974513;

typedef struct {
    uint64_t key;
    uint32_t id;
} bin_entry;

static int cmp_bin_entry(const void* a, const void* b) {
    const bin_entry* x = (const bin_entry*)a;
    const bin_entry* y = (const bin_entry*)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->id < y->id ? -1 : (x->id > y->id);
}
static int cmp_u64(const void* a, const void* b) {
    uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : (x > y);
}

static uint64_t bin_key(int32_t x, int32_t y, int32_t z) {
    return ((uint64_t)(uint32_t)(x + (1 << 20)) << 42) | ((uint64_t)(uint32_t)(y + (1 << 20)) << 21) |
           (uint64_t)(uint32_t)(z + (1 << 20));
}

/* bin_bounds (:437-444) over the swept box of REV i, in cell units */
void vxo_contact_box(const double* start, const double* pos, uint32_t i, int32_t lo[3], int32_t hi[3]) {
    for (int t = 0; t < 3; ++t) {
        double s = start[3 * (size_t)i + t], p = pos[3 * (size_t)i + t];
        double a = fmin(s, p) / VXO_CELL, b = fmax(s, p) / VXO_CELL;
        lo[t] = (int32_t)floor(a - C_BIN_HALF);
        hi[t] = (int32_t)floor(b + C_BIN_HALF);
    }
}

/* open-addressing set of pair keys (i << 32 | j) */
typedef struct {
    uint64_t* slot; /* key + 1, 0 = empty */
    size_t cap, count;
} pair_set;

static int pair_set_insert(pair_set* s, uint64_t key);
static void pair_set_grow(pair_set* s) {
    pair_set t = {(uint64_t*)calloc(s->cap * 2, sizeof(uint64_t)), s->cap * 2, 0};
    for (size_t k = 0; k < s->cap; ++k)
        if (s->slot[k]) pair_set_insert(&t, s->slot[k] - 1);
    free(s->slot);
    *s = t;
}
static int pair_set_insert(pair_set* s, uint64_t key) {
    if (2 * (s->count + 1) > s->cap) pair_set_grow(s);
    uint64_t h = (key * 0x9E3779B97F4A7C15ull) >> 17;
    for (size_t k = (size_t)h & (s->cap - 1);; k = (k + 1) & (s->cap - 1)) {
        if (s->slot[k] == key + 1) return 0;
        if (!s->slot[k]) {
            s->slot[k] = key + 1;
            s->count++;
            return 1;
        }
    }
}

/* candidate_pairs (:376-435): every pair whose swept bin boxes share a bin,
   at least one REV non-kinematic; sorted (i < j). */
static uint64_t* candidate_pairs(uint32_t n, const double* start, const double* pos, const uint8_t* kin,
                                 size_t* out_count) {
    size_t cap = 64, cnt = 0, scap = 64, scnt = 0;
    bin_entry* dyn = (bin_entry*)malloc(cap * sizeof(bin_entry));
    bin_entry* sta = (bin_entry*)malloc(scap * sizeof(bin_entry));
    for (uint32_t i = 0; i < n; ++i) {
        int32_t lo[3], hi[3];
        vxo_contact_box(start, pos, i, lo, hi);
        for (int32_t z = lo[2]; z <= hi[2]; ++z)
            for (int32_t y = lo[1]; y <= hi[1]; ++y)
                for (int32_t x = lo[0]; x <= hi[0]; ++x) {
                    bin_entry e = {bin_key(x, y, z), i};
                    if (kin[i]) {
                        if (scnt == scap) sta = (bin_entry*)realloc(sta, (scap *= 2) * sizeof(bin_entry));
                        sta[scnt++] = e;
                    } else {
                        if (cnt == cap) dyn = (bin_entry*)realloc(dyn, (cap *= 2) * sizeof(bin_entry));
                        dyn[cnt++] = e;
                    }
                }
    }
    qsort(dyn, cnt, sizeof(bin_entry), cmp_bin_entry);
    qsort(sta, scnt, sizeof(bin_entry), cmp_bin_entry);
    pair_set set = {(uint64_t*)calloc(1024, sizeof(uint64_t)), 1024, 0};
    size_t s0 = 0;
    for (size_t a = 0; a < cnt;) {
        size_t b = a;
        while (b < cnt && dyn[b].key == dyn[a].key) ++b;
        for (size_t p = a; p < b; ++p)
            for (size_t q = p + 1; q < b; ++q) {
                uint32_t i = dyn[p].id < dyn[q].id ? dyn[p].id : dyn[q].id;
                uint32_t j = dyn[p].id < dyn[q].id ? dyn[q].id : dyn[p].id;
                pair_set_insert(&set, ((uint64_t)i << 32) | j);
            }
        while (s0 < scnt && sta[s0].key < dyn[a].key) ++s0;
        for (size_t q = s0; q < scnt && sta[q].key == dyn[a].key; ++q)
            for (size_t p = a; p < b; ++p) {
                uint32_t i = dyn[p].id < sta[q].id ? dyn[p].id : sta[q].id;
                uint32_t j = dyn[p].id < sta[q].id ? sta[q].id : dyn[p].id;
                pair_set_insert(&set, ((uint64_t)i << 32) | j);
            }
        a = b;
    }
    uint64_t* pairs = (uint64_t*)malloc((set.count ? set.count : 1) * sizeof(uint64_t));
    size_t m = 0;
    for (size_t k = 0; k < set.cap; ++k)
        if (set.slot[k]) pairs[m++] = set.slot[k] - 1;
    qsort(pairs, m, sizeof(uint64_t), cmp_u64);
    free(set.slot);
    free(dyn);
    free(sta);
    *out_count = m;
    return pairs;
}

/* adjacency (:491-503): [6] per REV, slot 2a+1 the +a neighbour, 2a the -a one */
static void contact_adjacency(uint32_t n, const uint32_t* nbr, uint32_t* adj) {
    for (size_t k = 0; k < 6 * (size_t)n; ++k) adj[k] = VX_EMPTY;
    for (int a = 0; a < 3; ++a)
        for (uint32_t i = 0; i < n; ++i) {
            uint32_t j = nbr[(size_t)a * n + i];
            if (j == VX_EMPTY) continue;
            adj[6 * (size_t)i + 2 * a + 1] = j;
            adj[6 * (size_t)j + 2 * a] = i;
        }
}

static int monotone_connected(const uint32_t* adj, uint32_t i, uint32_t j, const double steps[3]) {
    if (steps[0] == 0.0 && steps[1] == 0.0 && steps[2] == 0.0) return i == j;
    for (int a = 0; a < 3; ++a) {
        if (steps[a] == 0.0) continue;
        uint32_t next = adj[6 * (size_t)i + 2 * a + (steps[a] > 0.0 ? 1 : 0)];
        if (next == VX_EMPTY) continue;
        double rem[3] = {steps[0], steps[1], steps[2]};
        rem[a] = 0.0;
        if (monotone_connected(adj, next, j, rem)) return 1;
    }
    return 0;
}

/* local_continuum_pair (:505-540) */
int vxo_local_continuum_pair(const double* rest, const uint32_t* adj, uint32_t i, uint32_t j) {
    double steps[3], dev = 0.0, big = 0.0;
    for (int t = 0; t < 3; ++t) {
        double d = (rest[3 * (size_t)j + t] - rest[3 * (size_t)i + t]) / VXO_CELL;
        steps[t] = round(d);
        dev = fmax(dev, fabs(d - steps[t]));
        big = fmax(big, fabs(steps[t]));
    }
    if (dev > C_1EM3 || big > 1.0) return 0;
    return monotone_connected(adj, i, j, steps);
}

/* swept_normal (:546-590); returns the signed axis code +-(axis + 1), or 0 */
static int swept_normal(const double si[3], const double sj[3], const double ei[3], const double ej[3]) {
    double d0[3], rel[3];
    int inside = 1;
    for (int t = 0; t < 3; ++t) {
        d0[t] = sj[t] - si[t];
        double di = ei[t] - si[t], dj = ej[t] - sj[t];
        rel[t] = dj - di;
        if (!(fabs(d0[t]) <= C_START_TOUCH)) inside = 0;
    }
    if (inside) return 0;
    double enter = 0.0, exit_ = 1.0, sign = 1.0;
    int hit = -1;
    for (int a = 0; a < 3; ++a) {
        if (fabs(rel[a]) < C_1EM12) {
            if (fabs(d0[a]) > VXO_CELL) return 0;
            continue;
        }
        double t0 = (-VXO_CELL - d0[a]) / rel[a];
        double t1 = (VXO_CELL - d0[a]) / rel[a];
        double nearv = fmin(t0, t1), farv = fmax(t0, t1);
        if (nearv > enter || (hit < 0 && nearv >= enter)) {
            enter = nearv;
            hit = a;
            sign = d0[a] + rel[a] * enter >= 0.0 ? 1.0 : -1.0;
        }
        exit_ = fmin(exit_, farv);
        if (enter > exit_) return 0;
    }
    if (exit_ < 0.0 || enter > 1.0 || hit < 0) return 0;
    return sign > 0.0 ? hit + 1 : -(hit + 1);
}

/* overlap_normal (:592-616): axis code, penetration */
static int overlap_normal(const double a[3], const double b[3], const double fallback[3], double* penetration) {
    double d[3], o[3];
    for (int t = 0; t < 3; ++t) {
        d[t] = b[t] - a[t];
        o[t] = VXO_CELL - fabs(d[t]);
    }
    if (fmin(fmin(o[0], o[1]), o[2]) <= 0.0) return 0;
    int axis = (o[0] <= o[1] && o[0] <= o[2]) ? 0 : (o[1] <= o[2] ? 1 : 2);
    double src = fabs(d[axis]) > C_1EM8 ? d[axis] : (fabs(fallback[axis]) > C_1EM8 ? fallback[axis] : 1.0);
    *penetration = o[axis];
    return signbit(src) ? -(axis + 1) : axis + 1;
}

/* touching_normal (:446-468) */
static int touching_normal(const double a[3], const double b[3]) {
    double d[3], g[3];
    for (int t = 0; t < 3; ++t) {
        d[t] = b[t] - a[t];
        g[t] = fabs(d[t]) - VXO_CELL;
    }
    int axis = (g[0] >= g[1] && g[0] >= g[2]) ? 0 : (g[1] >= g[2] ? 1 : 2);
    if (g[axis] > C_SLOP) return 0;
    for (int o = 0; o < 3; ++o)
        if (o != axis && g[o] >= -C_SLOP) return 0;
    return d[axis] >= 0.0 ? axis + 1 : -(axis + 1);
}

static double contact_inverse_mass(const uint8_t* kin, const double* mass, const uint8_t* tmask, uint32_t i, int axis) {
    if (kin[i] || (tmask && ((tmask[i] >> axis) & 1))) return 0.0;
    return 1.0 / mass[i];
}

/* separate (:631-654) */
static int separate(double* pos, double* prev, const uint8_t* kin, const double* mass, const uint8_t* tmask,
                    uint32_t i, uint32_t j, int code, double amount) {
    int axis = (code > 0 ? code : -code) - 1;
    double wi = contact_inverse_mass(kin, mass, tmask, i, axis);
    double wj = contact_inverse_mass(kin, mass, tmask, j, axis);
    double denom = wi + wj;
    if (denom <= 0.0) return 0;
    double nrm[3] = {0.0, 0.0, 0.0};
    nrm[axis] = code > 0 ? 1.0 : -1.0;
    double si = amount * wi / denom, sj = amount * wj / denom;
    for (int t = 0; t < 3; ++t) {
        double di = -nrm[t] * si, dj = nrm[t] * sj;
        pos[3 * (size_t)i + t] += di;
        pos[3 * (size_t)j + t] += dj;
        prev[3 * (size_t)i + t] += di;
        prev[3 * (size_t)j + t] += dj;
    }
    return 1;
}

static double code_dot(int code, const double v[3]) {
    double nrm[3] = {0.0, 0.0, 0.0};
    int axis = (code > 0 ? code : -code) - 1;
    nrm[axis] = code > 0 ? 1.0 : -1.0;
    return v[0] * nrm[0] + v[1] * nrm[1] + v[2] * nrm[2];
}

static int cmp_contact(const void* a, const void* b) {
    const vxo_contact* x = (const vxo_contact*)a;
    const vxo_contact* y = (const vxo_contact*)b;
    if (x->i != y->i) return x->i < y->i ? -1 : 1;
    if (x->j != y->j) return x->j < y->j ? -1 : 1;
    return x->order < y->order ? -1 : (x->order > y->order);
}

uint32_t vxo_contact_project(uint32_t n, double* pos, double* prev, const double* rest, const uint8_t* kin,
                             const double* mass, const uint8_t* tmask, const uint32_t* nbr, vxo_contact** out,
                             vxo_contact_stats* st) {
    double* start = (double*)malloc(3 * (size_t)(n ? n : 1) * sizeof(double));
    memcpy(start, prev, 3 * (size_t)n * sizeof(double));
    uint32_t* adj = (uint32_t*)malloc(6 * (size_t)(n ? n : 1) * sizeof(uint32_t));
    contact_adjacency(n, nbr, adj);
    size_t cand = 0;
    uint64_t* pairs = candidate_pairs(n, start, pos, kin, &cand);
    size_t m = 0;
    for (size_t k = 0; k < cand; ++k) {
        uint32_t i = (uint32_t)(pairs[k] >> 32), j = (uint32_t)pairs[k];
        if (!vxo_local_continuum_pair(rest, adj, i, j)) pairs[m++] = pairs[k];
    }
    size_t ccap = 64, ccnt = 0;
    vxo_contact* c = (vxo_contact*)malloc(ccap * sizeof(vxo_contact));
    uint32_t sweeps = 0;
    for (int sweep = 0; sweep < 6; ++sweep) {
        int changed = 0;
        sweeps++;
        for (size_t k = 0; k < m; ++k) {
            uint32_t i = (uint32_t)(pairs[k] >> 32), j = (uint32_t)pairs[k];
            const double *si = start + 3 * (size_t)i, *sj = start + 3 * (size_t)j;
            double* pi = pos + 3 * (size_t)i;
            double* pj = pos + 3 * (size_t)j;
            double d0[3] = {sj[0] - si[0], sj[1] - si[1], sj[2] - si[2]};
            int code = swept_normal(si, sj, pi, pj);
            int impact = 0;
            if (code) {
                double dd[3] = {pj[0] - pi[0], pj[1] - pi[1], pj[2] - pi[2]};
                double separation = code_dot(code, dd);
                if (separation < VXO_CELL)
                    changed |= separate(pos, prev, kin, mass, tmask, i, j, code, VXO_CELL - separation + C_1EM6);
                impact = code_dot(code, d0) > C_NEW_IMPACT;
            } else {
                double pen = 0.0;
                code = overlap_normal(pi, pj, d0, &pen);
                if (code) {
                    changed |= separate(pos, prev, kin, mass, tmask, i, j, code, pen + C_1EM6);
                    impact = code_dot(code, d0) > C_NEW_IMPACT;
                } else {
                    code = touching_normal(pi, pj);
                }
            }
            if (code) {
                if (ccnt == ccap) c = (vxo_contact*)realloc(c, (ccap *= 2) * sizeof(vxo_contact));
                c[ccnt].i = i;
                c[ccnt].j = j;
                c[ccnt].normal = code;
                c[ccnt].new_impact = impact;
                c[ccnt].order = (uint32_t)ccnt;
                ccnt++;
            }
        }
        if (!changed) break;
    }
    /* sort by (i, j) and keep the first contact of each pair (:105-106) */
    qsort(c, ccnt, sizeof(vxo_contact), cmp_contact);
    size_t u = 0;
    for (size_t k = 0; k < ccnt; ++k)
        if (u == 0 || c[k].i != c[u - 1].i || c[k].j != c[u - 1].j) c[u++] = c[k];
    if (st) {
        st->candidates = cand;
        st->pairs = m;
        st->contacts = u;
        st->sweeps = sweeps;
    }
    free(start);
    free(adj);
    free(pairs);
    *out = c;
    return (uint32_t)u;
}

/* resolve_velocities_with_precontact (:133-300), velocity AoS 3n */
void vxo_resolve_velocities(uint32_t n, double* vel, const double* pre_contact, const uint8_t* kin, const double* mass,
                            const uint8_t* tmask, const vxo_contact* c, uint32_t count, double restitution_cfg,
                            double friction, double* restitution_heat, double* friction_heat) {
    double* phys = (double*)malloc(3 * (size_t)(n ? n : 1) * sizeof(double));
    memcpy(phys, pre_contact, 3 * (size_t)n * sizeof(double));
    for (int iteration = 0; iteration < 4; ++iteration) {
        int changed = 0;
        for (uint32_t k = 0; k < count; ++k) {
            uint32_t i = c[k].i, j = c[k].j;
            int axis = (c[k].normal > 0 ? c[k].normal : -c[k].normal) - 1;
            double nrm[3] = {0.0, 0.0, 0.0};
            nrm[axis] = c[k].normal > 0 ? 1.0 : -1.0;
            double wi = contact_inverse_mass(kin, mass, tmask, i, axis);
            double wj = contact_inverse_mass(kin, mass, tmask, j, axis);
            double denom = wi + wj;
            if (denom <= 0.0) continue;
            double* vi = vel + 3 * (size_t)i;
            double* vj = vel + 3 * (size_t)j;
            double rv[3] = {vj[0] - vi[0], vj[1] - vi[1], vj[2] - vi[2]};
            double closing = rv[0] * nrm[0] + rv[1] * nrm[1] + rv[2] * nrm[2];
            double normal_impulse = 0.0;
            if (closing < -C_1EM6) {
                double rest = (c[k].new_impact && iteration == 0) ? restitution_cfg : 0.0;
                normal_impulse = -(1.0 + rest) * closing / denom;
                double* qi = phys + 3 * (size_t)i;
                double* qj = phys + 3 * (size_t)j;
                double pr[3] = {qj[0] - qi[0], qj[1] - qi[1], qj[2] - qi[2]};
                double physical_closing = pr[0] * nrm[0] + pr[1] * nrm[1] + pr[2] * nrm[2];
                double physical_impulse = c[k].new_impact ? normal_impulse
                                          : (physical_closing < -C_1EM6 ? fmin(-physical_closing / denom, normal_impulse)
                                                                         : 0.0);
                for (int t = 0; t < 3; ++t) {
                    vi[t] -= nrm[t] * (normal_impulse * wi);
                    vj[t] += nrm[t] * (normal_impulse * wj);
                }
                double heat_closing = c[k].new_impact ? closing : physical_closing;
                double rh = 0.0;
                if (heat_closing < -C_1EM6 && physical_impulse > 0.0)
                    rh = fmax(physical_impulse * -heat_closing - 0.5 * (physical_impulse * physical_impulse) * denom, 0.0);
                if (rh > 0.0) *restitution_heat += rh;
                for (int t = 0; t < 3; ++t) {
                    qi[t] -= nrm[t] * (physical_impulse * wi);
                    qj[t] += nrm[t] * (physical_impulse * wj);
                }
                changed = 1;
            }
            if (normal_impulse > 0.0 && friction > 0.0) {
                double rel[3] = {vj[0] - vi[0], vj[1] - vi[1], vj[2] - vi[2]};
                double rn = rel[0] * nrm[0] + rel[1] * nrm[1] + rel[2] * nrm[2];
                double tr[3], rt[3];
                for (int t = 0; t < 3; ++t) {
                    double tangent = rel[t] - nrm[t] * rn;
                    tr[t] = contact_inverse_mass(kin, mass, tmask, i, t) + contact_inverse_mass(kin, mass, tmask, j, t);
                    rt[t] = tr[t] > 0.0 ? tangent : 0.0;
                }
                double speed = sqrt(rt[0] * rt[0] + rt[1] * rt[1] + rt[2] * rt[2]);
                if (speed > C_1EM6) {
                    double dir[3] = {rt[0] / speed, rt[1] / speed, rt[2] / speed};
                    double tw = 0.0;
                    for (int t = 0; t < 3; ++t) tw += dir[t] * dir[t] * tr[t];
                    if (tw > 0.0) {
                        double mag = fmin(speed / tw, friction * normal_impulse);
                        for (int t = 0; t < 3; ++t) {
                            double imp = -dir[t] * mag;
                            vi[t] -= imp * contact_inverse_mass(kin, mass, tmask, i, t);
                            vj[t] += imp * contact_inverse_mass(kin, mass, tmask, j, t);
                        }
                        double fh = fmax(mag * speed - 0.5 * (mag * mag) * tw, 0.0);
                        if (fh > 0.0 && (!kin[i] || !kin[j])) *friction_heat += fh;
                        changed = 1;
                    }
                }
            }
        }
        if (!changed) break;
    }
    free(phys);
}

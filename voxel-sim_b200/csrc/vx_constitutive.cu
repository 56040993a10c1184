// vx_constitutive.cu — bond assembly, REV diagonal/RHS and bond stress.
//
// Per-bond stiffness, frame and rest vector follow make_constraint
// (src/solver.rs:1325-1345) with tensor_compliance / stiffness_matrix
// (:37-73) and bond_thermal_rest (:78-95). The per-REV diagonal and
// right-hand side are the assembly of solve_coupled (:1576-1636), gathered
// per REV instead of scattered per bond. The stress evaluation is the
// read-only part of the fracture loop (src/solver.rs:627-647) with
// bond_limits (:124-158), pair_limits and the failure ratio of
// fracture::update (src/fracture.rs:76-133, :210-262).
#include "vx_device.cuh"
#include "vx_kernels.h"
#include "vx_layout.cuh"
#include "vx_reduce.cuh"

namespace vx {

__device__ __forceinline__ v3 load3(const double* p, size_t stride, size_t i) {
    return mk(p[i], p[stride + i], p[2 * stride + i]);
}
__device__ __forceinline__ quat load_q(const double4* q, uint32_t i) {
    double4 v = q[i];
    return {v.x, v.y, v.z, v.w};
}

// Endpoint compliance in the bond frame (symmetric). False for an invalid endpoint.
__device__ bool compliance(const SceneView& s, uint32_t n, const m3& F, sym6& c) {
    const vx_material& m = s.materials[s.matid[n]];
    float4 p0 = s.param0[n];
    float4 p1 = s.param1[n];
    double solid = fmin(fmax((double)p1.x, 1e-4), 1.0);
    v3 fw = rotate(load_q(s.rot, n), mk(p0.x, p0.y, p0.z));
    v3 f = mul_t(F, fw);
    double a = p0.w;
    double young = m.young, young_perp = m.young_perp, shear = m.shear;
    double transverse = young + a * (young_perp - young);
    double normal = transverse + (young - transverse) * f.x * f.x;
    double d0 = normal * solid, d1 = shear * solid, d2 = shear * solid;
    if (!isfinite(d0) || !isfinite(d1) || !isfinite(d2) || fmin(d0, fmin(d1, d2)) <= 0.0) return false;
    double i0 = 1.0 / d0, i1 = 1.0 / d1, i2 = 1.0 / d2;
    v3 sf = mk(f.x * i0, f.y * i1, f.z * i2);
    double alpha = shear * a * 0.2;
    double scale = alpha / (1.0 + alpha * dot(f, sf));
    c = sym6{{i0 - sf.x * sf.x * scale, i1 - sf.y * sf.y * scale, i2 - sf.z * sf.z * scale,
              -sf.x * sf.y * scale, -sf.x * sf.z * scale, -sf.y * sf.z * scale}};
    return true;
}

// F^T (d CELL + (e_i + e_j) CELL / 2), e_n the endpoint's thermal strain along d.
__device__ v3 thermal_rest(const SceneView& s, uint32_t i, uint32_t j, const m3& F) {
    v3 dir = normalize_or_zero(F.c[0]);
    v3 e = mk(0.0, 0.0, 0.0);
    uint32_t ends[2] = {i, j};
#pragma unroll
    for (int t = 0; t < 2; ++t) {
        uint32_t n = ends[t];
        const vx_material& m = s.materials[s.matid[n]];
        float4 p0 = s.param0[n];
        float dT = s.param1[n].z;
        if (dT == 0.0f) continue;  // adds exactly zero
        v3 f = normalize_or_zero(rotate(load_q(s.rot, n), mk(p0.x, p0.y, p0.z)));
        double ap = m.thermal_expansion_parallel, an = m.thermal_expansion_perpendicular;
        e = e + (dir * an + f * ((ap - an) * dot(f, dir))) * (double)dT;
    }
    return mul_t(F, dir * kCell + e * (0.5 * kCell));
}

// F L F^T for symmetric L, returned as sym6 (upper triangle).
__device__ sym6 rotate_sym(const m3& F, const sym6& L) {
    // rows of F: F[r][a] = F.c[a].r
    double f[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        f[0][a] = F.c[a].x;
        f[1][a] = F.c[a].y;
        f[2][a] = F.c[a].z;
    }
    double l[3][3] = {{L.s[0], L.s[3], L.s[4]}, {L.s[3], L.s[1], L.s[5]}, {L.s[4], L.s[5], L.s[2]}};
    double m[3][3];  // F L
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) m[r][c] = f[r][0] * l[0][c] + f[r][1] * l[1][c] + f[r][2] * l[2][c];
    auto w = [&](int r, int c) { return m[r][0] * f[c][0] + m[r][1] * f[c][1] + m[r][2] * f[c][2]; };
    return sym6{{w(0, 0), w(1, 1), w(2, 2), w(0, 1), w(0, 2), w(1, 2)}};
}

// ---------------------------------------------------------------------------
// One thread per bond e = axis * n + i.
__global__ void k_assemble_bonds(SceneView s, BondArrays b, uint32_t* __restrict__ assembled) {
    const uint32_t n = s.n;
    size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (e >= 3 * (size_t)n) return;
    int a = (int)(e / n);
    uint32_t i = (uint32_t)(e - (size_t)a * n);
    if (!tile_active(s.tile_on, i)) return;
    uint32_t j = s.nbr[e];
    size_t m3n = 3 * (size_t)n;
    uint8_t st = 0;
    sym6 W = sym6{{0, 0, 0, 0, 0, 0}};
    v3 force = mk(0.0, 0.0, 0.0);
    if (j != VX_EMPTY_U32) {
        uint8_t fi = s.flags[i], fj = s.flags[j];
        if (!(fi == 0 && fj == 0 && s.kin[i])) {
            quat mid = slerp_half(load_q(s.rot, i), load_q(s.rot, j));
            m3 F = basis(a, mid);
            sym6 ci, cj, K = sym6{{0, 0, 0, 0, 0, 0}};
            bool vi = compliance(s, i, F, ci);
            bool vj = compliance(s, j, F, cj);
            if (vi && vj) {
                sym6 sum;
#pragma unroll
                for (int t = 0; t < 6; ++t) sum.s[t] = ci.s[t] + cj.s[t];
                K = inverse(sum);
#pragma unroll
                for (int t = 0; t < 6; ++t) K.s[t] *= kStiffScale;
            }
            b.frame_q[e] = make_double4(mid.x, mid.y, mid.z, mid.w);
#pragma unroll
            for (int t = 0; t < 6; ++t) b.mat_k[t * m3n + e] = K.s[t];
            st = 1;
            if (!(fi == 0 && fj == 0)) {
                st = 2;
                float4 ba = s.bond_a[e];
                float4 bb = s.bond_b[e];
                double scale = fmax(1.0 - (double)ba.w, 0.001);
                sym6 L;
#pragma unroll
                for (int t = 0; t < 6; ++t) L.s[t] = K.s[t] * scale;
                W = rotate_sym(F, L);
                v3 tr = thermal_rest(s, i, j, F);
                v3 local = mk(tr.x + (double)ba.x + (double)bb.x * kCell, tr.y + (double)ba.y + (double)bb.y * kCell,
                              tr.z + (double)ba.z + (double)bb.z * kCell);
                v3 rest = mul(F, local);
                v3 xi = load3(s.pos, n, i), xj = load3(s.pos, n, j);
                force = mul(W, xj - xi - rest);
            }
        }
    }
    b.state[e] = st;
    // one mask for the ballot and the leader: two reads could differ under
    // independent thread scheduling and drop or double a group's count
    const unsigned act = __activemask();
    const unsigned ballot = __ballot_sync(act, st == 2);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(act) - 1) && ballot) atomicAdd(assembled, __popc(ballot));
    store_sym(b.k64 + (size_t)a * 6 * n, n, i, W.s[0], W.s[1], W.s[2], W.s[3], W.s[4], W.s[5]);
    const uint32_t kn = kstride32(n);
    store_sym(b.k32 + (size_t)a * 6 * kn, kn, i, W.s[0], W.s[1], W.s[2], W.s[3], W.s[4], W.s[5]);
    b.force[e] = force.x;
    b.force[m3n + e] = force.y;
    b.force[2 * m3n + e] = force.z;
}

struct RevOut {
    double* d64;
    double* dinv64;
    float* d32;
    float* dinv32;
    double* b64;
    float* mh2;
};

// One thread per REV: D = m/h^2 I + sum K_e, b = (pred - x) m/h^2 + load +- f_e,
// then b *= free and D = P D P + (I - P); m/h^2 also in FP32 for the FP32 operator.
__global__ void k_assemble_revs(SceneView s, BondArrays b, RevOut o, double h, int reuse) {
    const uint32_t n = s.n;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !tile_active(s.tile_on, i)) return;
    size_t m3n = 3 * (size_t)n;
    double m = (double)s.param1[i].w / (h * h);
    o.mh2[i] = (float)m;
    double D[6] = {m, m, m, 0.0, 0.0, 0.0};
    v3 x = load3(s.pos, n, i);
    v3 p = load3(s.pred, n, i);
    v3 rhs = (p - x) * m + load3(s.loads, n, i);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        size_t e = (size_t)a * n + i;
        if (b.state[e] == 2) {
            Sym<double> k = load_sym(b.k64 + (size_t)a * 6 * n, n, i);
            D[0] += k.xx, D[1] += k.yy, D[2] += k.zz, D[3] += k.xy, D[4] += k.xz, D[5] += k.yz;
            rhs = rhs + mk(b.force[e], b.force[m3n + e], b.force[2 * m3n + e]);
        }
        uint32_t k = s.rev[e];
        if (k != VX_EMPTY_U32) {
            size_t ek = (size_t)a * n + k;
            if (b.state[ek] == 2) {
                Sym<double> kk = load_sym(b.k64 + (size_t)a * 6 * n, n, k);
                D[0] += kk.xx, D[1] += kk.yy, D[2] += kk.zz, D[3] += kk.xy, D[4] += kk.xz, D[5] += kk.yz;
                rhs = rhs - mk(b.force[ek], b.force[m3n + ek], b.force[2 * m3n + ek]);
            }
        }
    }
    uint8_t fl = s.flags[i];
    double f0 = (fl & 1) ? 1.0 : 0.0, f1 = (fl & 2) ? 1.0 : 0.0, f2 = (fl & 4) ? 1.0 : 0.0;
    rhs = mk(rhs.x * f0, rhs.y * f1, rhs.z * f2);
    sym6 P = sym6{{D[0] * f0 * f0 + (1.0 - f0), D[1] * f1 * f1 + (1.0 - f1), D[2] * f2 * f2 + (1.0 - f2),
                   f0 * D[3] * f1, f0 * D[4] * f2, f1 * D[5] * f2}};
    store_sym(o.d64, n, i, P.s[0], P.s[1], P.s[2], P.s[3], P.s[4], P.s[5]);
    store_sym(o.d32, n, i, P.s[0], P.s[1], P.s[2], P.s[3], P.s[4], P.s[5]);
    o.b64[i] = rhs.x;
    o.b64[n + i] = rhs.y;
    o.b64[2 * (size_t)n + i] = rhs.z;
    if (!reuse) {
        sym6 inv = inverse(P);
        store_sym(o.dinv64, n, i, inv.s[0], inv.s[1], inv.s[2], inv.s[3], inv.s[4], inv.s[5]);
        store_sym(o.dinv32, n, i, inv.s[0], inv.s[1], inv.s[2], inv.s[3], inv.s[4], inv.s[5]);
    }
}

cudaError_t launch_assembly(vx_scene* s, double h, bool reuse_preconditioner) {
    if (s->n == 0) return cudaSuccess;
    SceneView v = view_of(s);
    size_t m = 3 * (size_t)s->n;
    cudaMemsetAsync(s->bond_count, 0, sizeof(uint32_t), s->stream);
    k_assemble_bonds<<<(unsigned)((m + 255) / 256), 256, 0, s->stream>>>(v, s->bonds, s->bond_count);
    RevOut o{s->d64, s->dinv64, s->d32, s->dinv32, s->b64, s->mh2_32};
    k_assemble_revs<<<(s->n + 255) / 256, 256, 0, s->stream>>>(v, s->bonds, o, h, reuse_preconditioner ? 1 : 0);
    return cudaGetLastError();
}

__global__ void k_apply_correction(uint32_t n, double* __restrict__ pos, const double* __restrict__ dx,
                                   const uint8_t* __restrict__ tile_on) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t < 3 * (size_t)n && tile_active(tile_on, t % n)) pos[t] += dx[t];
}

cudaError_t launch_apply_correction(vx_scene* s) {
    size_t m = 3 * (size_t)s->n;
    if (m == 0) return cudaSuccess;
    k_apply_correction<<<(unsigned)((m + 255) / 256), 256, 0, s->stream>>>(s->n, s->pos, s->x64, s->tile_on);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Limits (src/fracture.rs:62-133, src/solver.rs:124-158).
struct Limits {
    double tension, compression, shear, yield_stress, hardening, plastic_failure, ductility, fracture_energy;
};

__device__ __forceinline__ double directional(double par, double perp, double align, double aniso) {
    return par + aniso * (1.0 - fmin(fmax(fabs(align), 0.0), 1.0)) * (perp - par);
}

__device__ Limits endpoint_limits(const vx_material& m, double align, double aniso) {
    Limits l;
    if (m.fracture_mode == VX_BRITTLE) l.ductility = 0.0;
    else if (m.fracture_mode == VX_DUCTILE) l.ductility = 1.0;
    else l.ductility = (1.0 - aniso) * 0.5 + aniso * fabs(align) * fabs(align);
    l.tension = directional(m.tensile_strength, m.tensile_strength_perp, align, aniso);
    l.compression = directional(m.compressive_strength, m.compressive_strength_perp, align, aniso);
    l.shear = directional(m.shear_strength, m.shear_strength_perp, align, aniso);
    l.yield_stress = m.yield_strength;
    l.hardening = m.hardening_modulus;
    l.plastic_failure = m.failure_plastic_strain;
    l.fracture_energy = directional(m.fracture_energy, m.fracture_energy_perp, align, aniso);
    return l;
}

__device__ Limits bond_limits(const SceneView& s, uint32_t i, uint32_t j, v3 dir) {
    float4 pi = s.param0[i], pj = s.param0[j];
    v3 fi = rotate(load_q(s.rot, i), mk(pi.x, pi.y, pi.z));
    v3 fj = rotate(load_q(s.rot, j), mk(pj.x, pj.y, pj.z));
    Limits a = endpoint_limits(s.materials[s.matid[i]], dot(dir, fi), pi.w);
    Limits b = endpoint_limits(s.materials[s.matid[j]], dot(dir, fj), pj.w);
    Limits l;
    l.tension = fmin(a.tension, b.tension);
    l.compression = fmin(a.compression, b.compression);
    l.shear = fmin(a.shear, b.shear);
    l.yield_stress = fmin(a.yield_stress, b.yield_stress);
    l.hardening = fmin(a.hardening, b.hardening);
    l.plastic_failure = fmin(a.plastic_failure, b.plastic_failure);
    l.ductility = fmin(a.ductility, b.ductility);
    l.fracture_energy = fmin(a.fracture_energy, b.fracture_energy);
    float4 qi = s.param1[i], qj = s.param1[j];
    double solid = fmin(1.0, fmin(fmin(fmax((double)qi.x, 0.0), 1.0), fmin(fmax((double)qj.x, 0.0), 1.0)));
    double thermal = fmin(1.0, fmin((double)qi.y, (double)qj.y));
    double scale = solid * solid * thermal;
    l.tension *= scale;
    l.compression *= scale;
    l.shear *= scale;
    l.yield_stress *= scale;
    l.hardening *= scale;
    l.fracture_energy *= scale;
    return l;
}

// Ratio that fracture::update evaluates after its return map (src/fracture.rs:226-254).
__device__ double stress_ratio(v3 u_total, v3 plastic, const sym6& K, const Limits& l, double eq_plastic) {
    v3 u = u_total - plastic * kCell;
    if (l.ductility > 1e-5) {
        v3 ku0 = mul(K, u);
        v3 trial = mk(ku0.x / kArea, ku0.y / kArea, ku0.z / kArea);
        double equivalent = sqrt(dot(trial, trial));
        double yield_now = l.yield_stress + l.hardening * eq_plastic;
        if (equivalent > yield_now) {
            v3 dir = mk(trial.x / equivalent * kArea, trial.y / equivalent * kArea, trial.z / equivalent * kArea);
            v3 cd = mul(inverse(K), dir);
            cd = mk(cd.x / kCell, cd.y / kCell, cd.z / kCell);
            double modulus = 1.0 / fmax(sqrt(dot(cd, cd)), 1e-20);
            double dep = (equivalent - yield_now) / (modulus + l.hardening) * l.ductility;
            v3 dp = normalize_or_zero(cd) * dep;
            u = u_total - (plastic + dp) * kCell;
        }
    }
    v3 ku = mul(K, u);
    v3 stress = mk(ku.x / kArea, ku.y / kArea, ku.z / kArea);
    double normal_limit = stress.x >= 0.0 ? l.tension : l.compression;
    double r0 = stress.x / fmax(normal_limit, 1.0);
    double sh = fmax(l.shear, 1.0);
    return sqrt(r0 * r0 + (stress.y * stress.y + stress.z * stress.z) / (sh * sh));
}

__global__ void k_bond_stress(SceneView s, BondArrays b, float* __restrict__ ratio, float* __restrict__ force,
                              uint32_t* __restrict__ near, uint32_t cap, uint32_t* __restrict__ near_count) {
    const uint32_t n = s.n;
    size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    size_t m3n = 3 * (size_t)n;
    if (e >= m3n) return;
    int a = (int)(e / n);
    uint32_t i = (uint32_t)(e - (size_t)a * n);
    if (!tile_active(s.tile_on, i)) return;
    uint32_t j = s.nbr[e];
    double r = -1.0;
    v3 f = mk(0.0, 0.0, 0.0);
    if (b.state[e] != 0 && j != VX_EMPTY_U32 && !s.kin[i]) {
        double4 q = b.frame_q[e];
        m3 F = basis(a, quat{q.x, q.y, q.z, q.w});
        sym6 K;
#pragma unroll
        for (int t = 0; t < 6; ++t) K.s[t] = b.mat_k[t * m3n + e];
        Limits l = bond_limits(s, i, j, F.c[0]);
        v3 xi = load3(s.pos, n, i), xj = load3(s.pos, n, j);
        float4 ba = s.bond_a[e], bb = s.bond_b[e];
        v3 u = mul_t(F, xj - xi) - thermal_rest(s, i, j, F) - mk(ba.x, ba.y, ba.z);
        v3 plastic = mk(bb.x, bb.y, bb.z);
        f = mul(F, mul(K, u - plastic * kCell)) * (1.0 - (double)ba.w);
        r = stress_ratio(u, plastic, K, l, bb.w);
        if (near && fabs(r - 1.0) <= 1e-6) {
            uint32_t slot = atomicAdd(near_count, 1u);
            if (slot < cap) near[slot] = (uint32_t)e;
        }
    }
    if (ratio) ratio[e] = (float)r;
    if (force) {
        force[3 * e] = (float)f.x;
        force[3 * e + 1] = (float)f.y;
        force[3 * e + 2] = (float)f.z;
    }
}

cudaError_t launch_bond_stress(vx_scene* s, float* d_ratio, float* d_force, uint32_t* d_near, uint32_t cap) {
    cudaMemsetAsync(s->near_count, 0, sizeof(uint32_t), s->stream);
    size_t m = 3 * (size_t)s->n;
    if (m == 0) return cudaGetLastError();
    k_bond_stress<<<(unsigned)((m + 255) / 256), 256, 0, s->stream>>>(view_of(s), s->bonds, d_ratio, d_force,
                                                                       d_near, cap, s->near_count);
    return cudaGetLastError();
}


// ---------------------------------------------------------------------------
// Fracture stage (src/solver.rs:600-665 with fracture::update, src/fracture.rs:
// 186-292), in FP64 on the bond state the reference keeps in f32.
struct FractureCfg {
    double damage_rate, energy_release, fatigue_cycles, fatigue_exponent, fatigue_threshold, plastic_heat_fraction;
};

__device__ __forceinline__ double bond_energy(v3 u, const sym6& K, double damage) {  // energy, :186-188
    return fmax(0.5 * (1.0 - damage) * dot(u, mul(K, u)), 0.0);
}

__global__ void k_fracture_commit(SceneView s, BondArrays b, float4* __restrict__ bond_a, float4* __restrict__ bond_b,
                                  float4* __restrict__ bond_c, float* __restrict__ bond_d, uint32_t* __restrict__ nbr,
                                  float* __restrict__ last_force, double dt, FractureCfg c, double* __restrict__ partials, uint32_t* __restrict__ counter,
                                  double* __restrict__ totals) {
    const uint32_t n = s.n;
    const size_t m3n = 3 * (size_t)n;
    const size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // plastic heat, stored plastic, surface work, damage heat, released
    if (e < m3n) {
        const int a = (int)(e / n);
        const uint32_t i = (uint32_t)(e - (size_t)a * n);
        const uint32_t j = nbr[e];
        if (tile_active(s.tile_on, i) && b.state[e] != 0 && j != VX_EMPTY_U32 && !s.kin[i]) {
            const double4 q = b.frame_q[e];
            const m3 F = basis(a, quat{q.x, q.y, q.z, q.w});
            sym6 K;
#pragma unroll
            for (int t = 0; t < 6; ++t) K.s[t] = b.mat_k[t * m3n + e];
            const Limits l = bond_limits(s, i, j, F.c[0]);
            const v3 xi = load3(s.pos, n, i), xj = load3(s.pos, n, j);
            float4 ba = bond_a[e], bb = bond_b[e], bc = bond_c[e];
            const v3 u_total = mul_t(F, xj - xi) - thermal_rest(s, i, j, F) - mk(ba.x, ba.y, ba.z);
            v3 plastic = mk(bb.x, bb.y, bb.z);
            double eqp = bb.w, damage = ba.w, work = bc.x, fatigue = bc.y, prev = bc.z, reversal = bc.w;
            double increment = bond_d[e];
            const double old_damage = damage;
            v3 u = u_total - plastic * kCell;
            const double before = bond_energy(u, K, old_damage);
            // workspace last_force = F (K (u - plastic CELL)) (1 - damage) before the update (src/solver.rs:638-640)
            const v3 f = mul(F, mul(K, u)) * (1.0 - old_damage);
            last_force[3 * e] = (float)f.x;
            last_force[3 * e + 1] = (float)f.y;
            last_force[3 * e + 2] = (float)f.z;
            if (l.ductility > 1e-5) {  // return map, :226-243
                const v3 ku0 = mul(K, u);
                const v3 trial = mk(ku0.x / kArea, ku0.y / kArea, ku0.z / kArea);
                const double equivalent = sqrt(dot(trial, trial));
                const double yield_now = l.yield_stress + l.hardening * eqp;
                if (equivalent > yield_now) {
                    const v3 dir = mk(trial.x / equivalent * kArea, trial.y / equivalent * kArea,
                                      trial.z / equivalent * kArea);
                    v3 cd = mul(inverse(K), dir);
                    cd = mk(cd.x / kCell, cd.y / kCell, cd.z / kCell);
                    const double modulus = 1.0 / fmax(sqrt(dot(cd, cd)), 1e-20);
                    const double dep = (equivalent - yield_now) / (modulus + l.hardening) * l.ductility;
                    plastic = plastic + normalize_or_zero(cd) * dep;
                    eqp += dep;
                    u = u_total - plastic * kCell;
                    const double lost = fmax(before - bond_energy(u, K, old_damage), 0.0);
                    work += lost;
                    v[0] = lost * c.plastic_heat_fraction;
                    v[1] = lost - v[0];
                }
            }
            const v3 ku = mul(K, u);  // failure after the return map, :244-254
            const v3 stress = mk(ku.x / kArea, ku.y / kArea, ku.z / kArea);
            const double normal_limit = stress.x >= 0.0 ? l.tension : l.compression;
            const double r0 = stress.x / fmax(normal_limit, 1.0);
            const double sh = fmax(l.shear, 1.0);
            const double ratio = sqrt(r0 * r0 + (stress.y * stress.y + stress.z * stress.z) / (sh * sh));
            const double ax = fabs(stress.x), ay = fabs(stress.y), az = fabs(stress.z);
            const double principal = ax >= fmax(ay, az) ? stress.x : (ay >= az ? stress.y : stress.z);
            const double signed_ratio = copysign(ratio, principal);  // fatigue, :190-207
            const double delta = signed_ratio - prev;
            if (fabs(delta) > 1e-6) {
                if (increment * delta < 0.0) {
                    const double amplitude = fabs(prev - reversal) * 0.5;
                    if (amplitude > c.fatigue_threshold) {
                        const double level = fmin((amplitude - c.fatigue_threshold) / (1.0 - c.fatigue_threshold), 1.0);
                        fatigue = fmin(fatigue + 0.5 * pow(level, c.fatigue_exponent) / c.fatigue_cycles, 1.0);
                    }
                    reversal = prev;
                }
                increment = delta;
            }
            prev = signed_ratio;
            if (ratio >= 1.0) {  // damage, :265-277
                if (l.ductility <= 1e-5) damage = 1.0;
                else damage = fmin(damage + c.damage_rate * dt * fmin(ratio, 10.0), 1.0);
            }
            if (l.ductility > 1e-5 && eqp >= fmax(l.plastic_failure, 1e-6)) damage = fmin(damage + c.damage_rate * dt, 1.0);
            if (fatigue >= 1.0) damage = 1.0;
            const double lost = fmax(bond_energy(u, K, old_damage) - bond_energy(u, K, damage), 0.0);  // :280-288
            const double budget = l.fracture_energy * kArea * (damage - old_damage);
            v[2] = fmin(lost, budget);
            const double available = lost - v[2];
            v[4] = available * c.energy_release;
            v[3] = available - v[4];
            bond_a[e] = make_float4(ba.x, ba.y, ba.z, (float)damage);
            bond_b[e] = make_float4((float)plastic.x, (float)plastic.y, (float)plastic.z, (float)eqp);
            bond_c[e] = make_float4((float)work, (float)fatigue, (float)prev, (float)reversal);
            bond_d[e] = (float)increment;
            if (damage >= 1.0) {
                nbr[e] = VX_EMPTY_U32;
                atomicAdd(counter + 1, 1u);
            }
        }
    }
    if (grid_sum<5>(v, partials, counter) && threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 5; ++k) totals[k] = v[k];
    }
}

cudaError_t launch_fracture_commit(vx_scene* s, double dt, const vx_fracture_config* cfg) {
    const size_t m = 3 * (size_t)s->n;
    cudaError_t e = cudaMemsetAsync(s->frac_counter, 0, 2 * sizeof(uint32_t), s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->frac_totals, 0, 8 * sizeof(double), s->stream);
    if (e != cudaSuccess || m == 0) return e;
    FractureCfg c{cfg->damage_rate, cfg->energy_release, cfg->fatigue_cycles, cfg->fatigue_exponent,
                  cfg->fatigue_threshold, cfg->plastic_heat_fraction};
    const unsigned grid = (unsigned)((m + kThreads - 1) / kThreads);
    k_fracture_commit<<<grid, kThreads, 0, s->stream>>>(view_of(s), s->bonds, s->bond_a, s->bond_b, s->bond_c,
                                                        s->bond_d, s->nbr, s->last_force, dt, c, s->frac_partials,
                                                        s->frac_counter,
                                                        s->frac_totals);
    return cudaGetLastError();
}

}  // namespace vx

// vx_lattice.cu — lattice topology, free-axis flags and the rotation fit.
//
// Topology follows Scene::from_voxels / Scene::new (src/scene.rs:558-570,
// :1668-1681); the rotation fit follows fit_rotations (src/solver.rs:327-417).
#include "vx_device.cuh"
#include "vx_kernels.h"

namespace vx {

SceneView view_of(const vx_scene* s) {
    return SceneView{s->n,      s->pos,    s->pred,   s->loads, s->rot,    s->kin,
                     s->flags,  s->param0, s->param1, s->matid, s->materials,
                     s->nbr,    s->rev,    s->bond_a, s->bond_b, s->tile_on, s->tile_scene};
}

// free[i] bit a = axis a is in the system: not kinematic, not targeted
// (src/solver.rs:1554-1565).
__global__ void k_flags(uint32_t n, const uint8_t* __restrict__ kin, const uint8_t* __restrict__ tmask,
                        uint8_t* __restrict__ flags) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flags[i] = kin[i] ? 0 : (uint8_t)(~tmask[i] & 7u);
}

cudaError_t launch_flags(vx_scene* s) {
    if (s->n == 0) return cudaSuccess;
    k_flags<<<(s->n + 255) / 256, 256, 0, s->stream>>>(s->n, s->kin, s->tmask, s->flags);
    return cudaGetLastError();
}

__global__ void k_fill_u32(uint32_t* p, size_t count, uint32_t v) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < count) p[i] = v;
}

// rev[a][j] = i for nbr[a][i] = j. On a lattice each REV has at most one
// -axis neighbour, so the scatter has no conflicts.
__global__ void k_reverse(uint32_t n, const uint32_t* __restrict__ nbr, uint32_t* __restrict__ rev) {
    size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (e >= 3 * (size_t)n) return;
    uint32_t j = nbr[e];
    if (j == VX_EMPTY_U32 || j >= n) return;
    size_t a = e / n;
    uint32_t i = (uint32_t)(e - a * n);
    rev[a * n + j] = i;
}

// Neighbour deltas for the persistent kernel, which keeps them in shared
// memory: entry t of REV i (own x, y, z, then reverse x, y, z) is j - i as an
// int16, 0 for no neighbour, packed two per word. Entries that do not fit
// (|j - i| > 32767, j == i or j >= n) are counted in *bad; the persistent
// kernel is then not used for the scene.
__global__ void k_neighbor_codes(uint32_t n, const uint32_t* __restrict__ nbr, const uint32_t* __restrict__ rev,
                                 uint32_t* __restrict__ code, uint32_t* __restrict__ bad) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t d16[6];
    uint32_t miss = 0;
#pragma unroll
    for (int t = 0; t < 6; ++t) {
        const uint32_t j = t < 3 ? nbr[(size_t)t * n + i] : rev[(size_t)(t - 3) * n + i];
        d16[t] = 0;
        if (j == VX_EMPTY_U32) continue;
        const long long d = (long long)j - (long long)i;
        if (j >= n || d == 0 || d < -32768 || d > 32767) {
            miss += 1;
            continue;
        }
        d16[t] = (uint32_t)(uint16_t)(int16_t)d;
    }
#pragma unroll
    for (int w = 0; w < 3; ++w) code[(size_t)w * n + i] = d16[2 * w] | (d16[2 * w + 1] << 16);
    if (miss) atomicAdd(bad, miss);
}

cudaError_t launch_reverse_neighbors(vx_scene* s) {
    size_t m = 3 * (size_t)s->n;
    s->persist_checked = false;  // the on-chip plan depends on the deltas
    s->nbcode_state = 0;
    if (m == 0) return cudaSuccess;
    unsigned g = (unsigned)((m + 255) / 256);
    k_fill_u32<<<g, 256, 0, s->stream>>>(s->rev, m, VX_EMPTY_U32);
    k_reverse<<<g, 256, 0, s->stream>>>(s->n, s->nbr, s->rev);
    cudaMemsetAsync(s->nbcode_bad, 0, sizeof(uint32_t), s->stream);
    k_neighbor_codes<<<(s->n + 255) / 256, 256, 0, s->stream>>>(s->n, s->nbr, s->rev, s->nbcode, s->nbcode_bad);
    return cudaGetLastError();
}

// Dense occupancy grid over the bounding box: grid[key(cell)] = REV index.
__global__ void k_grid_scatter(uint32_t n, const int32_t* __restrict__ cells, int3 lo, int3 ext,
                               int32_t* __restrict__ grid, uint32_t* __restrict__ dup) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long x = cells[3 * (size_t)i] - lo.x, y = cells[3 * (size_t)i + 1] - lo.y,
              z = cells[3 * (size_t)i + 2] - lo.z;
    long long key = (z * ext.y + y) * ext.x + x;
    int32_t old = atomicExch(&grid[key], (int32_t)i);
    if (old != -1) atomicAdd(dup, 1u);
}

__global__ void k_grid_bonds(uint32_t n, const int32_t* __restrict__ cells, const uint8_t* __restrict__ kin,
                             int3 lo, int3 ext, const int32_t* __restrict__ grid, uint32_t* __restrict__ nbr) {
    size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (e >= 3 * (size_t)n) return;
    int a = (int)(e / n);
    uint32_t i = (uint32_t)(e - (size_t)a * n);
    long long c[3] = {cells[3 * (size_t)i] - lo.x, cells[3 * (size_t)i + 1] - lo.y,
                      cells[3 * (size_t)i + 2] - lo.z};
    c[a] += 1;  // the box has one spare layer on the + side of every axis
    long long key = (c[2] * ext.y + c[1]) * ext.x + c[0];
    int32_t j = grid[key];
    uint32_t v = VX_EMPTY_U32;
    if (j >= 0 && kin[j] == kin[i]) v = (uint32_t)j;
    nbr[e] = v;
}

cudaError_t launch_topology(const int32_t* d_cells, const uint8_t* d_kin, uint32_t n, const int32_t* lo,
                            const int32_t* ext, int32_t* d_grid, uint32_t* d_nbr, uint32_t* dup,
                            cudaStream_t stream) {
    int3 l = make_int3(lo[0], lo[1], lo[2]);
    int3 x = make_int3(ext[0], ext[1], ext[2]);
    cudaMemsetAsync(dup, 0, sizeof(uint32_t), stream);
    k_grid_scatter<<<(n + 255) / 256, 256, 0, stream>>>(n, d_cells, l, x, d_grid, dup);
    size_t m = 3 * (size_t)n;
    k_grid_bonds<<<(unsigned)((m + 255) / 256), 256, 0, stream>>>(n, d_cells, d_kin, l, x, d_grid, d_nbr);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// fit_rotations (src/solver.rs:327-417), one thread per REV, FP64.
// Column a of the deformation gradient is the mean of (x_j - x_i)/CELL over
// the intact bonds along a that touch the REV (as owner or as partner), or the
// old rotation's column when there are none. det <= 1e-6 keeps the rotation.
// Up to five Higham steps F <- (F + F^-T)/2, then Gram-Schmidt and a
// quaternion. The block max of 2 acos|q_old . q_new| is folded into a global
// max via the bit pattern of the non-negative double.
__global__ void k_fit_rotations(SceneView s, double4* __restrict__ rot_out,
                                unsigned long long* __restrict__ max_bits) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double angle = 0.0;
    if (i < s.n && !s.kin[i] && tile_active(s.tile_on, i)) {
        const uint32_t n = s.n;
        v3 xi = mk(s.pos[i], s.pos[n + i], s.pos[2 * (size_t)n + i]);
        m3 f;
        double cnt[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            v3 acc = mk(0.0, 0.0, 0.0);
            double c = 0.0;
            uint32_t k = s.rev[(size_t)a * n + i];
            if (k != VX_EMPTY_U32) {
                v3 xk = mk(s.pos[k], s.pos[n + k], s.pos[2 * (size_t)n + k]);
                acc = acc + mk((xi.x - xk.x) / kCell, (xi.y - xk.y) / kCell, (xi.z - xk.z) / kCell);
                c += 1.0;
            }
            uint32_t j = s.nbr[(size_t)a * n + i];
            if (j != VX_EMPTY_U32) {
                v3 xj = mk(s.pos[j], s.pos[n + j], s.pos[2 * (size_t)n + j]);
                acc = acc + mk((xj.x - xi.x) / kCell, (xj.y - xi.y) / kCell, (xj.z - xi.z) / kCell);
                c += 1.0;
            }
            f.c[a] = acc;
            cnt[a] = c;
        }
        double4 q4 = s.rot[i];
        quat prev = {q4.x, q4.y, q4.z, q4.w};
        m3 old = from_quat(prev);
#pragma unroll
        for (int a = 0; a < 3; ++a)
            f.c[a] = cnt[a] > 0.0 ? mk(f.c[a].x / cnt[a], f.c[a].y / cnt[a], f.c[a].z / cnt[a]) : old.c[a];
        quat q = prev;
        if (det(f) > 1e-6) {
            for (int it = 0; it < 5; ++it) {
                m3 inv_t = transpose(inverse(f));
                m3 next;
                double delta = 0.0;
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    next.c[a] = (f.c[a] + inv_t.c[a]) * 0.5;
                    v3 d = next.c[a] - f.c[a];
                    delta = fmax(delta, fmax(fabs(d.x), fmax(fabs(d.y), fabs(d.z))));
                }
                f = next;
                if (delta <= 1e-6) break;
            }
            v3 x = normalize_or_zero(f.c[0]);
            v3 y = normalize_or_zero(f.c[1] - x * dot(x, f.c[1]));
            if (dot(x, x) > 0.5 && dot(y, y) > 0.5) {
                m3 r;
                r.c[0] = x;
                r.c[1] = y;
                r.c[2] = cross(x, y);
                q = normalize(from_mat3(r));
                rot_out[i] = make_double4(q.x, q.y, q.z, q.w);
            }
            double d = fabs(qdot(prev, q));
            angle = 2.0 * acos(fmin(d, 1.0));
        }
    }
    // block max
    __shared__ double smax[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) angle = fmax(angle, __shfl_xor_sync(0xffffffffu, angle, o));
    if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = angle;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? smax[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        // a 256-thread block is one tile, so its maximum belongs to one pool slot
        unsigned long long* slot = max_bits + (s.tile_scene ? s.tile_scene[blockIdx.x] : 0u);
        if (threadIdx.x == 0 && v > 0.0) atomicMax(slot, (unsigned long long)__double_as_longlong(v));
    }
}

cudaError_t launch_fit_rotations(vx_scene* s) {
    cudaMemsetAsync(s->max_angle_bits, 0, sizeof(unsigned long long) * (s->pool_slots ? s->pool_slots : 1),
                    s->stream);
    if (s->n == 0) return cudaGetLastError();
    // rotations are read (old column, previous quaternion) and written by the
    // same thread only, so in-place update is safe
    k_fit_rotations<<<(s->n + 255) / 256, 256, 0, s->stream>>>(view_of(s), s->rot, s->max_angle_bits);
    return cudaGetLastError();
}

}  // namespace vx

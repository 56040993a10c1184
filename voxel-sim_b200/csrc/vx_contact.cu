// vx_contact.cu — contact projection (collision::project, src/collision.rs:33-119,
// :376-590) and contact velocity resolution (resolve_velocities_with_precontact,
// :133-300) on the device, in FP64 over the scene's FP64 positions and
// velocities. This file is compiled without fused multiply-adds so that every
// value rounds as the FP64 restatement of the same expressions does.
//
// Broadphase. Every REV's swept box (previous and current position, each
// widened by half a cell and 2e-4 cells, floored to bins; bin_bounds :437-444)
// is computed in parallel. Two REVs are a candidate pair when their boxes share
// a bin and at least one of them is not kinematic, which is exactly the set the
// reference's bin maps produce (candidate_pairs :376-435). Small boxes (at most
// 4 bins per axis) are found through a hash of box corners; the rare larger
// boxes of fast REVs through a hash of every bin they cover. Pairs joined
// through the intact lattice inside their elementary cell are dropped
// (local_continuum_pair :505-540) and each pair is written to the segment of
// its smaller REV, so after a per-segment sort the list is the reference's
// sorted pair list.
//
// Projection. The reference sweeps the pairs in order, and each correction is
// seen by the pairs after it (Gauss-Seidel). The device keeps that order
// exactly: with a bound M on how far any REV moves during a sweep, a pair
// whose boxes stay farther apart than the contact tests reach even after both
// REVs move by M cannot act or report a contact in that sweep. Each sweep
// stores only the other pairs, which are grouped into connected components
// over the REVs that can move; one thread replays each component's pairs in
// pair order, so every pair sees the same positions it sees in the reference's
// sweep. After the sweep the largest movement of any REV is checked against M;
// when it is larger the sweep is restored and replayed with the pairs of a
// wider bound (finally with every pair). The contacts of the sweeps are
// merged by pair, the first one of each pair kept. Contact velocity
// resolution runs over components of the contact list; its sweeps stop per
// component when nothing changes, which is what the reference's global stop
// does to that component.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "vx_device.cuh"
#include "vx_kernels.h"

namespace vx {

namespace {

// The reference's f32 literals, at their f32 values.
constexpr double kBinHalf = 0.5001999735832214;      // 0.5 + 2e-4 (bin_bounds)
constexpr double kStartTouch = 0.009998999536037445;  // CELL - 1e-6 (swept_normal)
constexpr double kNewImpact = 0.010001999326050282;   // CELL + 2e-6 (project)
constexpr double k1em6 = 9.999999974752427e-07;
constexpr double kSlop = 1.9999999949504854e-06;  // CONTACT_SLOP (touching_normal)
constexpr double k1em8 = 9.99999993922529e-09;
constexpr double k1em12 = 9.999999960041972e-13;
constexpr double k1em3 = 0.0010000000474974513;

constexpr int kSmallExtent = 4;          // bins per axis of a box found through its corner
constexpr int kSceneBits = 21;  // bin coordinate bits of a single scene's keys
constexpr int kPoolBits = 18;   // ... and of a pool's, whose keys carry the slot
constexpr uint32_t kPoolKeySlots = 1u << (64 - 3 * kPoolBits);
constexpr unsigned kProbeLimit = 1u << 20;
constexpr unsigned kUnionRetries = 1u << 16;
constexpr uint64_t kMaxLargeVolume = 1ull << 24;  // bins one fast REV may sweep in a substep
constexpr uint64_t kMaxLargeEntries = 1ull << 28;  // bins all fast REVs together may sweep (32-bit scan)
constexpr uint64_t kMaxStoredPairs = 1ull << 31;   // pairs one sweep may store (32-bit scan)
constexpr unsigned long long kEmptyKey = ~0ull;
constexpr unsigned kScanBlock = 1024;
constexpr double kSweepBound = 5e-4;  // metres a REV may first move in a sweep before it is replayed with more pairs
constexpr int kMaxAttempts = 8;       // replays of a sweep with wider bounds before every pair is stored

enum : uint32_t {
    E_OK = 0,
    E_RANGE = 1,     // a non-finite position or a bin outside the key range
    E_TABLE = 2,     // a hash probe exceeded its bound
    E_UNION = 4,     // a union exceeded its retry bound
    E_VOLUME = 8,    // a swept box larger than kMaxLargeVolume bins
};

// scalars in ContactState::scal
enum {
    S_ERR = 0, S_EXT = 1, S_LARGE = 4, S_CHANGED = 5, S_CAND_LO = 6, S_CAND_HI = 7, S_PAIRS_LO = 8, S_PAIRS_HI = 9,
    S_MOVED = 10,     // a REV moved farther than its bound in the last sweep
    S_CMIN = 11,      // [3] smallest small-box corner per axis, biased by kCornerBias
    S_CMAX = 14,      // [3] largest small-box corner per axis, biased
    S_STAGE = 17,     // pairs appended to the staging list by one generation
    S_LVOL = 18,      // [2] bins of all large boxes together (u64)
    S_STORED = 20,    // [2] pairs stored by one generation (u64)
    kScalars = 24,    // device words; the host copy holds them and, from kHostCount, counts
    kHostCount = 28
};
constexpr int32_t kCornerBias = 1 << 30;

// Which scene a REV belongs to. A single scene is slot 0 for every REV. In a
// pool, REVs of free tiles, of slots not taking part in the call, and the
// padding after a slot's last REV have no slot (VX_EMPTY_U32).
struct RevFilter {
    const uint8_t* tile_on;      // per 256-REV tile, null = all on
    const uint32_t* tile_scene;  // per tile: slot, null for a single scene
    const uint32_t* slot_first;  // per slot: first tile
    const uint32_t* slot_revs;   // per slot: REV count
};
__device__ __forceinline__ uint32_t rev_slot(const RevFilter& f, uint32_t i) {
    if (!f.tile_scene) return 0;
    const uint32_t tile = i >> 8;
    if (f.tile_on && !f.tile_on[tile]) return VX_EMPTY_U32;
    const uint32_t slot = f.tile_scene[tile];
    if (slot == VX_EMPTY_U32) return VX_EMPTY_U32;
    return i - f.slot_first[slot] * 256u < f.slot_revs[slot] ? slot : VX_EMPTY_U32;
}

// Hash key of a bin of one scene: the slot above three biased bin
// coordinates of `bits` bits each (21 for a single scene, 18 in a pool, which
// leaves 10 bits for up to 1024 slots).
__device__ __forceinline__ unsigned long long bin_key(uint32_t slot, int32_t x, int32_t y, int32_t z, int bits) {
    const int32_t bias = 1 << (bits - 1);
    return ((unsigned long long)slot << (3 * bits)) | ((unsigned long long)(uint32_t)(x + bias) << (2 * bits)) |
           ((unsigned long long)(uint32_t)(y + bias) << bits) | (unsigned long long)(uint32_t)(z + bias);
}
__device__ __forceinline__ uint32_t key_hash(unsigned long long k) {
    k ^= k >> 31;
    k *= 0x9E3779B97F4A7C15ull;
    k ^= k >> 29;
    return (uint32_t)k;
}

// Hash slot holding key, or VX_EMPTY_U32.
__device__ uint32_t table_find(const unsigned long long* keys, uint32_t mask, unsigned long long key) {
    uint32_t slot = key_hash(key) & mask;
    for (unsigned probe = 0; probe <= mask && probe < kProbeLimit; ++probe) {
        const unsigned long long k = keys[slot];
        if (k == key) return slot;
        if (k == kEmptyKey) return VX_EMPTY_U32;
        slot = (slot + 1) & mask;
    }
    return VX_EMPTY_U32;
}
// Slot for key, claiming an empty one; VX_EMPTY_U32 when the probe bound is hit.
__device__ uint32_t table_claim(unsigned long long* keys, uint32_t mask, unsigned long long key) {
    uint32_t slot = key_hash(key) & mask;
    for (unsigned probe = 0; probe <= mask && probe < kProbeLimit; ++probe) {
        const unsigned long long old = atomicCAS(keys + slot, kEmptyKey, key);
        if (old == kEmptyKey || old == key) return slot;
        slot = (slot + 1) & mask;
    }
    return VX_EMPTY_U32;
}

__device__ __forceinline__ v3 load3(const double* f, uint32_t n, uint32_t i) {
    return mk(f[i], f[(size_t)n + i], f[2 * (size_t)n + i]);
}
__device__ __forceinline__ void add3(double* f, uint32_t n, uint32_t i, int axis, double d) {
    f[(size_t)axis * n + i] += d;
}

// ---- narrow-phase tests, as the FP64 restatement --------------------------

// swept_normal (:546-590): signed axis code +-(axis + 1), or 0
__device__ int swept_normal(v3 si, v3 sj, v3 ei, v3 ej) {
    const double d0[3] = {sj.x - si.x, sj.y - si.y, sj.z - si.z};
    const double di[3] = {ei.x - si.x, ei.y - si.y, ei.z - si.z};
    const double dj[3] = {ej.x - sj.x, ej.y - sj.y, ej.z - sj.z};
    double rel[3];
    bool inside = true;
    for (int t = 0; t < 3; ++t) {
        rel[t] = dj[t] - di[t];
        if (!(fabs(d0[t]) <= kStartTouch)) inside = false;
    }
    if (inside) return 0;
    double enter = 0.0, exit_ = 1.0, sign = 1.0;
    int hit = -1;
    for (int a = 0; a < 3; ++a) {
        if (fabs(rel[a]) < k1em12) {
            if (fabs(d0[a]) > kCell) return 0;
            continue;
        }
        const double t0 = (-kCell - d0[a]) / rel[a];
        const double t1 = (kCell - d0[a]) / rel[a];
        const double nearv = fmin(t0, t1), farv = fmax(t0, t1);
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

// overlap_normal (:592-616)
__device__ int overlap_normal(v3 a, v3 b, v3 fallback, double* penetration) {
    const double d[3] = {b.x - a.x, b.y - a.y, b.z - a.z};
    const double f[3] = {fallback.x, fallback.y, fallback.z};
    double o[3];
    for (int t = 0; t < 3; ++t) o[t] = kCell - fabs(d[t]);
    if (fmin(fmin(o[0], o[1]), o[2]) <= 0.0) return 0;
    const int axis = (o[0] <= o[1] && o[0] <= o[2]) ? 0 : (o[1] <= o[2] ? 1 : 2);
    const double src = fabs(d[axis]) > k1em8 ? d[axis] : (fabs(f[axis]) > k1em8 ? f[axis] : 1.0);
    *penetration = o[axis];
    return signbit(src) ? -(axis + 1) : axis + 1;
}

// touching_normal (:446-468)
__device__ int touching_normal(v3 a, v3 b) {
    const double d[3] = {b.x - a.x, b.y - a.y, b.z - a.z};
    double g[3];
    for (int t = 0; t < 3; ++t) g[t] = fabs(d[t]) - kCell;
    const int axis = (g[0] >= g[1] && g[0] >= g[2]) ? 0 : (g[1] >= g[2] ? 1 : 2);
    if (g[axis] > kSlop) return 0;
    for (int o = 0; o < 3; ++o)
        if (o != axis && g[o] >= -kSlop) return 0;
    return d[axis] >= 0.0 ? axis + 1 : -(axis + 1);
}

__device__ __forceinline__ double code_dot(int code, v3 v) {
    const int axis = (code > 0 ? code : -code) - 1;
    const double nx = axis == 0 ? (code > 0 ? 1.0 : -1.0) : 0.0;
    const double ny = axis == 1 ? (code > 0 ? 1.0 : -1.0) : 0.0;
    const double nz = axis == 2 ? (code > 0 ? 1.0 : -1.0) : 0.0;
    return v.x * nx + v.y * ny + v.z * nz;
}

// inverse_mass (:620-627): kinematic REVs and targeted axes are immovable
__device__ __forceinline__ double inverse_mass(const uint8_t* kin, const float4* param1, const uint8_t* tmask, uint32_t i,
                                               int axis) {
    if (kin[i] || ((tmask[i] >> axis) & 1)) return 0.0;
    return 1.0 / (double)param1[i].w;
}

// True when the pair can act or report a contact while its REVs move at most
// m_i and m_j: its end separation within half = CELL + slop + m_i + m_j (+ a
// rounding margin) on every axis, or, unless the starts already overlap (swept_normal
// then answers nothing), its relative path from the start separation to the
// end one meeting the box of that half-width.
__device__ bool may_act(v3 si, v3 sj, v3 ei, v3 ej, double half) {
    const double d0[3] = {sj.x - si.x, sj.y - si.y, sj.z - si.z};
    const double e[3] = {ej.x - ei.x, ej.y - ei.y, ej.z - ei.z};
    bool near_end = true, starts_inside = true;
    for (int t = 0; t < 3; ++t) {
        if (!(fabs(e[t]) <= half)) near_end = false;
        if (!(fabs(d0[t]) <= kStartTouch)) starts_inside = false;
    }
    if (near_end) return true;
    if (starts_inside) return false;
    double t0 = 0.0, t1 = 1.0;
    for (int t = 0; t < 3; ++t) {
        const double r = e[t] - d0[t];
        if (r == 0.0) {
            if (!(fabs(d0[t]) <= half)) return false;
            continue;
        }
        const double a = (-half - d0[t]) / r, b = (half - d0[t]) / r;
        t0 = fmax(t0, fmin(a, b));
        t1 = fmin(t1, fmax(a, b));
        if (!(t0 <= t1)) return false;
    }
    return true;
}

// ---- local continuum test -------------------------------------------------

// adjacency (:491-503): +a neighbour from the bond table, -a from its reverse
__device__ __forceinline__ uint32_t adjacent(const uint32_t* nbr, const uint32_t* rev, uint32_t n, uint32_t i, int a,
                                             bool plus) {
    return plus ? nbr[(size_t)a * n + i] : rev[(size_t)a * n + i];
}

// local_continuum_pair (:505-540). The recursion tries the remaining axes in
// ascending order and backtracks, so it succeeds iff some order of the
// nonzero steps walks from i to j over existing bonds: every order is tried.
__device__ bool local_continuum(const float* rest, const uint32_t* nbr, const uint32_t* rev, uint32_t n, uint32_t i,
                                uint32_t j) {
    double steps[3], dev = 0.0, big = 0.0;
    for (int t = 0; t < 3; ++t) {
        const double d = ((double)rest[(size_t)t * n + j] - (double)rest[(size_t)t * n + i]) / kCell;
        steps[t] = round(d);
        dev = fmax(dev, fabs(d - steps[t]));
        big = fmax(big, fabs(steps[t]));
    }
    if (dev > k1em3 || big > 1.0) return false;
    int axes[3], m = 0;
    for (int t = 0; t < 3; ++t)
        if (steps[t] != 0.0) axes[m++] = t;
    if (m == 0) return i == j;
    // the permutations of m <= 3 axes
    const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    const int count = m == 1 ? 1 : (m == 2 ? 2 : 6);
    for (int p = 0; p < count; ++p) {
        uint32_t at = i;
        bool ok = true;
        for (int s = 0; s < m && ok; ++s) {
            const int slot = m == 2 ? (p == 0 ? s : 1 - s) : perms[p][s];
            const int a = axes[slot];
            at = adjacent(nbr, rev, n, at, a, steps[a] > 0.0);
            ok = at != VX_EMPTY_U32;
        }
        if (ok && at == j) return true;
    }
    return false;
}

// ---- broadphase -------------------------------------------------------------

struct Boxes {
    int32_t* lo;     // [3][n]
    int32_t* hi;     // [3][n]
    uint8_t* large;  // 0 small box, 1 large box, 2 not taking part
    uint32_t* slot;  // [n] the REV's scene (rev_slot)
    int bits;        // key coordinate bits
};

// The extents, corner bounds and counts are reduced per warp first (min, max
// and sums do not depend on order), then one lane updates the scalars.
__global__ void k_boxes(uint32_t n, const double* __restrict__ pos, const double* __restrict__ start, Boxes b,
                        RevFilter f, uint32_t* __restrict__ scal) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool small = false, large = false, bad = false;
    int32_t ext[3] = {0, 0, 0}, lo[3] = {0, 0, 0};
    if (i < n) {  // no early return: the whole warp takes part in the reductions below
        const uint32_t slot = rev_slot(f, i);
        b.slot[i] = slot;
        if (slot == VX_EMPTY_U32) {
            b.large[i] = 2;
            for (int t = 0; t < 3; ++t) b.lo[(size_t)t * n + i] = b.hi[(size_t)t * n + i] = 0;
        } else {
            // |bin| stays 8 below the key range, so corner probes (reach 3) stay inside it
            const double limit = (double)((1 << (b.bits - 1)) - 8);
            for (int t = 0; t < 3; ++t) {
                const double s = start[(size_t)t * n + i], p = pos[(size_t)t * n + i];
                const double a = fmin(s, p) / kCell - kBinHalf, c = fmax(s, p) / kCell + kBinHalf;
                if (!(fabs(a) < limit) || !(fabs(c) < limit)) {
                    bad = true;
                    b.lo[(size_t)t * n + i] = 0;
                    b.hi[(size_t)t * n + i] = 0;
                    ext[t] = 1;
                    continue;
                }
                lo[t] = (int32_t)floor(a);
                const int32_t hi = (int32_t)floor(c);
                b.lo[(size_t)t * n + i] = lo[t];
                b.hi[(size_t)t * n + i] = hi;
                ext[t] = hi - lo[t] + 1;
                if (ext[t] > kSmallExtent) large = true;
            }
            b.large[i] = large ? 1 : 0;
            small = !large;
        }
    }
    const unsigned full = 0xffffffffu, lane = threadIdx.x & 31;
    if (__any_sync(full, bad) && lane == 0) atomicOr(scal + S_ERR, E_RANGE);
    const unsigned large_count = __reduce_add_sync(full, large ? 1u : 0u);
    if (lane == 0 && large_count) atomicAdd(scal + S_LARGE, large_count);
    if (__any_sync(full, small)) {
        for (int t = 0; t < 3; ++t) {
            const uint32_t corner = (uint32_t)(lo[t] + kCornerBias);
            const uint32_t e_max = __reduce_max_sync(full, small ? (uint32_t)ext[t] : 0u);
            const uint32_t c_min = __reduce_min_sync(full, small ? corner : 0xffffffffu);
            const uint32_t c_max = __reduce_max_sync(full, small ? corner : 0u);
            if (lane == 0) {
                atomicMax(scal + S_EXT + t, e_max);
                atomicMin(scal + S_CMIN + t, c_min);
                atomicMax(scal + S_CMAX + t, c_max);
            }
        }
    }
}

// The corner grid of a single scene: when the small boxes' corners fill a
// compact box, chains hang off a dense array indexed by the corner itself.
struct CornerGrid {
    uint32_t* heads;   // [nx * ny * nz], null: the hash is used
    int32_t x0, y0, z0;
    uint32_t nx, ny, nz;
};
__device__ __forceinline__ uint32_t grid_cell(const CornerGrid& g, int32_t x, int32_t y, int32_t z) {
    const uint32_t dx = (uint32_t)(x - g.x0), dy = (uint32_t)(y - g.y0), dz = (uint32_t)(z - g.z0);
    if (dx >= g.nx || dy >= g.ny || dz >= g.nz) return VX_EMPTY_U32;  // also catches x < x0 (wraps)
    return dx + g.nx * (dy + g.ny * dz);
}
__global__ void k_insert_corners_dense(uint32_t n, Boxes b, CornerGrid g, uint32_t* next) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || b.large[i]) return;
    const uint32_t cell = grid_cell(g, b.lo[i], b.lo[(size_t)n + i], b.lo[2 * (size_t)n + i]);
    next[i] = atomicExch(g.heads + cell, i);  // every small corner lies inside the grid
}

// Small boxes: chain REVs by box corner.
__global__ void k_insert_corners(uint32_t n, Boxes b, unsigned long long* keys, uint32_t* heads, uint32_t* next,
                                 uint32_t mask, uint32_t* scal) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || b.large[i]) return;
    const unsigned long long key = bin_key(b.slot[i], b.lo[i], b.lo[(size_t)n + i], b.lo[2 * (size_t)n + i], b.bits);
    const uint32_t slot = table_claim(keys, mask, key);
    if (slot == VX_EMPTY_U32) {
        atomicOr(scal + S_ERR, E_TABLE);
        next[i] = VX_EMPTY_U32;
        return;
    }
    next[i] = atomicExch(heads + slot, i);
}

__global__ void k_large_volume(uint32_t n, Boxes b, uint32_t* vol, uint32_t* scal) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t v = 0;
    if (b.large[i] == 1) {
        v = 1;
        for (int t = 0; t < 3; ++t)
            v *= (uint64_t)(b.hi[(size_t)t * n + i] - b.lo[(size_t)t * n + i] + 1);
        if (v > kMaxLargeVolume) {
            atomicOr(scal + S_ERR, E_VOLUME);
            v = 0;
        }
        if (v) atomicAdd(reinterpret_cast<unsigned long long*>(scal + S_LVOL), (unsigned long long)v);
    }
    vol[i] = (uint32_t)v;
}

// Large boxes: one entry per covered bin, chained by bin.
__global__ void k_insert_large(uint32_t n, Boxes b, const uint32_t* __restrict__ off, unsigned long long* keys,
                               uint32_t* heads, uint32_t* ent_id, uint32_t* ent_next, uint32_t mask, uint32_t* scal) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || b.large[i] != 1) return;
    uint32_t e = off[i];
    const uint32_t end = off[i + 1];
    const int32_t x0 = b.lo[i], y0 = b.lo[(size_t)n + i], z0 = b.lo[2 * (size_t)n + i];
    const int32_t x1 = b.hi[i], y1 = b.hi[(size_t)n + i], z1 = b.hi[2 * (size_t)n + i];
    for (int32_t z = z0; z <= z1; ++z)
        for (int32_t y = y0; y <= y1; ++y)
            for (int32_t x = x0; x <= x1 && e < end; ++x, ++e) {
                const uint32_t slot = table_claim(keys, mask, bin_key(b.slot[i], x, y, z, b.bits));
                ent_id[e] = i;
                if (slot == VX_EMPTY_U32) {
                    atomicOr(scal + S_ERR, E_TABLE);
                    ent_next[e] = VX_EMPTY_U32;
                    continue;
                }
                ent_next[e] = atomicExch(heads + slot, e);
            }
}

struct PairArgs {
    uint32_t n;
    Boxes b;
    const uint8_t* kin;
    const float* rest;
    const uint32_t* nbr;
    const uint32_t* rev;
    const unsigned long long* keys1;  // corner table (when grid.heads is null)
    const uint32_t* heads1;
    const uint32_t* next1;
    uint32_t mask1;
    CornerGrid grid;                  // dense corner grid of a single scene
    const unsigned long long* keys2;  // large-box table (mask2 = 0: none)
    const uint32_t* heads2;
    const uint32_t* ent_id;
    const uint32_t* ent_next;
    uint32_t mask2;
    int32_t wx, wy, wz;  // largest small extent per axis
    const double* pos;    // current positions
    const double* start;  // swept starts
    const double* bound;  // per REV: how far it may move in this sweep
    bool all;             // store every pair (the last resort of a sweep)
    bool count_pairs;     // count candidates and pairs (the call's first generation)
    uint32_t* count;     // per owner: pairs (append pass) / cursor (write pass)
    uint2* stage;         // append pass: (owner, partner) of every stored pair, in no order
    uint32_t stage_cap;
    const uint32_t* off;
    uint32_t* pi;
    uint32_t* pj;
    uint32_t* scal;
};

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// k_pairs passes: count each owner's stored pairs and append them to the
// staging list; or, when that list overflowed, write them into the owners'
// segments in a second pass.
enum { kAppendPass = 0, kWritePass = 1 };

template <int kMode>
__device__ __forceinline__ void emit(const PairArgs& a, uint32_t i, uint32_t j, uint32_t& cand, uint32_t& kept,
                                     uint32_t& stored) {
    const uint32_t lo = i < j ? i : j, hi = i < j ? j : i;
    if (a.kin[lo] && a.kin[hi]) return;
    auto acts = [&] {
        return a.all || may_act(load3(a.start, a.n, lo), load3(a.start, a.n, hi), load3(a.pos, a.n, lo),
                                load3(a.pos, a.n, hi), kCell + kSlop + a.bound[lo] + a.bound[hi] + 1e-9);
    };
    if (a.count_pairs) {  // every candidate through the lattice test, for the counts
        ++cand;
        if (local_continuum(a.rest, a.nbr, a.rev, a.n, lo, hi)) return;
        ++kept;
        if (!acts()) return;
    } else {  // the cheaper test first: most candidates cannot act
        if (!acts() || local_continuum(a.rest, a.nbr, a.rev, a.n, lo, hi)) return;
    }
    ++stored;
    if (kMode == kWritePass) {
        const uint32_t slot = a.off[lo] + atomicAdd(a.count + lo, 1u);
        a.pi[slot] = lo;
        a.pj[slot] = hi;
        return;
    }
    atomicAdd(a.count + lo, 1u);
    {  // append pass: one atomic per group of lanes emitting together
        const unsigned act = __activemask();
        const unsigned lane = threadIdx.x & 31;
        const int leader = __ffs(act) - 1;
        uint32_t base = 0;
        if ((int)lane == leader) base = atomicAdd(a.scal + S_STAGE, (uint32_t)__popc(act));
        base = __shfl_sync(act, base, leader);
        const uint32_t k = base + (uint32_t)__popc(act & ((1u << lane) - 1u));
        if (k < a.stage_cap) a.stage[k] = make_uint2(lo, hi);
    }
}

__device__ __forceinline__ void box_of(const Boxes& b, uint32_t n, uint32_t i, int32_t lo[3], int32_t hi[3]) {
    for (int t = 0; t < 3; ++t) {
        lo[t] = b.lo[(size_t)t * n + i];
        hi[t] = b.hi[(size_t)t * n + i];
    }
}

// kLanes threads per REV share the rows of the REV's probe range, so a small
// scene, which has too few REVs to fill the GPU, examines a REV's candidates in
// parallel. Emission order does not matter: pairs are counted by atomics and
// each segment is sorted afterwards. Measured per projection: the 32^3 block
// 0.712 ms with one thread per REV, 0.645 with 2, 0.630 with 4, 0.693 with 8;
// the 64^3 block 1.132, 1.206, 1.362 and 1.821 ms.
constexpr uint32_t kPairSmallScene = 65536;  // REVs below which four threads share a REV

template <int kMode, int kLanes>
__global__ void __launch_bounds__(256) k_pairs(PairArgs a) {
    const size_t gid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t i = (uint32_t)(gid / kLanes);
    const int32_t t = (int32_t)(gid % kLanes);
    const uint32_t n = a.n;
    uint32_t cand = 0, kept = 0, stored = 0;
    if (i < n && a.b.large[i] != 2) {  // no early return: the whole warp sums the counts below
        const uint32_t slot = a.b.slot[i];
        const int bits = a.b.bits;
        int32_t lo[3], hi[3];
        box_of(a.b, n, i, lo, hi);
        const bool large_i = a.b.large[i] != 0;
        if (!large_i) {
            // small-small: corners within reach of this box; the smaller REV finds the pair
            const int32_t w[3] = {a.wx, a.wy, a.wz};
            const int32_t x0 = lo[0] - (w[0] - 1), y0 = lo[1] - (w[1] - 1), z0 = lo[2] - (w[2] - 1);
            const int32_t ny = hi[1] - y0 + 1, rows = ny * (hi[2] - z0 + 1);
            for (int32_t r = t; r < rows; r += kLanes) {
                const int32_t z = z0 + r / ny, y = y0 + r % ny;
                for (int32_t x = x0; x <= hi[0]; ++x) {
                    uint32_t head;
                    if (a.grid.heads) {
                        const uint32_t cell = grid_cell(a.grid, x, y, z);
                        if (cell == VX_EMPTY_U32) continue;
                        head = a.grid.heads[cell];
                    } else {
                        const uint32_t hs = table_find(a.keys1, a.mask1, bin_key(slot, x, y, z, bits));
                        if (hs == VX_EMPTY_U32) continue;
                        head = a.heads1[hs];
                    }
                    for (uint32_t j = head; j != VX_EMPTY_U32; j = a.next1[j]) {
                        if (j <= i) continue;
                        int32_t lj[3], hj[3];
                        box_of(a.b, n, j, lj, hj);
                        if (lj[0] <= hi[0] && lo[0] <= hj[0] && lj[1] <= hi[1] && lo[1] <= hj[1] &&
                            lj[2] <= hi[2] && lo[2] <= hj[2])
                            emit<kMode>(a, i, j, cand, kept, stored);
                    }
                }
            }
        }
        if (a.mask2) {
            // pairs with large boxes: the bins of this box, each pair counted at the
            // lowest corner of the two boxes' intersection
            const int32_t ny = hi[1] - lo[1] + 1, rows = ny * (hi[2] - lo[2] + 1);
            for (int32_t r = t; r < rows; r += kLanes) {
                const int32_t z = lo[2] + r / ny, y = lo[1] + r % ny;
                for (int32_t x = lo[0]; x <= hi[0]; ++x) {
                    const uint32_t hs = table_find(a.keys2, a.mask2, bin_key(slot, x, y, z, bits));
                    if (hs == VX_EMPTY_U32) continue;
                    for (uint32_t e = a.heads2[hs]; e != VX_EMPTY_U32; e = a.ent_next[e]) {
                        const uint32_t j = a.ent_id[e];
                        if (j == i || (large_i && j < i)) continue;
                        int32_t lj[3], hj[3];
                        box_of(a.b, n, j, lj, hj);
                        if (x == max(lo[0], lj[0]) && y == max(lo[1], lj[1]) && z == max(lo[2], lj[2]))
                            emit<kMode>(a, i, j, cand, kept, stored);
                    }
                }
            }
        }
    }
    if (kMode != kWritePass) {  // 64-bit warp sums, then one lane's atomics
        const unsigned long long c64 = warp_sum_u64(cand), k64 = warp_sum_u64(kept), s64 = warp_sum_u64(stored);
        if ((threadIdx.x & 31) == 0) {
            if (c64) atomicAdd(reinterpret_cast<unsigned long long*>(a.scal + S_CAND_LO), c64);
            if (k64) atomicAdd(reinterpret_cast<unsigned long long*>(a.scal + S_PAIRS_LO), k64);
            if (s64) atomicAdd(reinterpret_cast<unsigned long long*>(a.scal + S_STORED), s64);
        }
    }
}

// Staged pairs into their owners' segments (cursor zeroed; the segment sort
// then fixes the order).
__global__ void k_stage_scatter(uint32_t count, const uint2* __restrict__ stage, const uint32_t* __restrict__ off,
                                uint32_t* cursor, uint32_t* pi, uint32_t* pj) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const uint2 p = stage[k];
    const uint32_t slot = off[p.x] + atomicAdd(cursor + p.x, 1u);
    pi[slot] = p.x;
    pj[slot] = p.y;
}

// Sorts each REV's pair segment by partner (insertion sort; segments are short).
__global__ void k_sort_segments(uint32_t n, const uint32_t* __restrict__ off, uint32_t* pj) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t b = off[i], e = off[i + 1];
    for (uint32_t k = b + 1; k < e; ++k) {
        const uint32_t v = pj[k];
        uint32_t m = k;
        while (m > b && pj[m - 1] > v) {
            pj[m] = pj[m - 1];
            --m;
        }
        pj[m] = v;
    }
}

// ---- projection sweeps -----------------------------------------------------

__global__ void k_iota(uint32_t n, uint32_t* __restrict__ v) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

__device__ __forceinline__ uint32_t uf_find(uint32_t* parent, uint32_t x) {
    uint32_t p = __ldcg(parent + x);
    while (p != x) {
        const uint32_t g = __ldcg(parent + p);
        if (g != p) __stcg(parent + x, g);
        x = p;
        p = g;
    }
    return x;
}

// A REV whose every axis has zero inverse mass (kinematic, or all three axes
// targeted) is never moved by a correction or an impulse: items that share
// only such REVs do not depend on one another.
__device__ __forceinline__ bool movable(const uint8_t* kin, const uint8_t* tmask, uint32_t i) {
    return !kin[i] && (tmask[i] & 7u) != 7u;
}

// Joins the two REVs of each listed item (pairs or contacts) when both can move.
__global__ void k_union(uint32_t count, const uint32_t* __restrict__ items, const uint32_t* __restrict__ ia,
                        const uint32_t* __restrict__ ja, const uint8_t* __restrict__ kin,
                        const uint8_t* __restrict__ tmask, uint32_t* parent, uint32_t* scal) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const uint32_t k = items ? items[t] : t;
    const uint32_t i = ia[k], j = ja[k];
    if (!movable(kin, tmask, i) || !movable(kin, tmask, j)) return;
    for (unsigned tries = 0; tries < kUnionRetries; ++tries) {
        const uint32_t ri = uf_find(parent, i), rj = uf_find(parent, j);
        if (ri == rj) return;
        const uint32_t lo = ri < rj ? ri : rj, hi = ri < rj ? rj : ri;
        if (atomicCAS(parent + hi, hi, lo) == hi) return;
    }
    atomicOr(scal + S_ERR, E_UNION);
}

// After the unions: each item's component root (read-only walk from a REV
// that can move, else from its first REV) and the component sizes.
__global__ void k_roots(uint32_t count, const uint32_t* __restrict__ items, const uint32_t* __restrict__ ia,
                        const uint32_t* __restrict__ ja, const uint8_t* __restrict__ kin,
                        const uint8_t* __restrict__ tmask, const uint32_t* __restrict__ parent,
                        uint32_t* __restrict__ root, uint32_t* comp_count) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const uint32_t k = items ? items[t] : t;
    const uint32_t i = ia[k], j = ja[k];
    uint32_t x = (movable(kin, tmask, i) || !movable(kin, tmask, j)) ? i : j;
    uint32_t p = parent[x];
    while (p != x) {
        x = p;
        p = parent[p];
    }
    root[t] = x;
    atomicAdd(comp_count + x, 1u);
}

__global__ void k_fill(uint32_t count, const uint32_t* __restrict__ items, const uint32_t* __restrict__ root,
                       const uint32_t* __restrict__ comp_off, uint32_t* comp_cursor, uint32_t* __restrict__ out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const uint32_t r = root[t];
    out[comp_off[r] + atomicAdd(comp_cursor + r, 1u)] = items ? items[t] : t;
}

// Ascending sort of v[b, e): insertion sort for short ranges, heapsort for
// long ones (a large component is replayed by one thread).
__device__ void sort_range(uint32_t* v, uint32_t b, uint32_t e) {
    const uint32_t len = e - b;
    if (len <= 32) {
        for (uint32_t k = b + 1; k < e; ++k) {
            const uint32_t x = v[k];
            uint32_t m = k;
            while (m > b && v[m - 1] > x) {
                v[m] = v[m - 1];
                --m;
            }
            v[m] = x;
        }
        return;
    }
    uint32_t* a = v + b;
    auto sift = [a](uint32_t root, uint32_t end) {
        for (;;) {
            uint32_t child = 2 * root + 1;
            if (child >= end) return;
            if (child + 1 < end && a[child] < a[child + 1]) ++child;
            if (!(a[root] < a[child])) return;
            const uint32_t t = a[root];
            a[root] = a[child];
            a[child] = t;
            root = child;
        }
    };
    for (uint32_t k = len / 2; k-- > 0;) sift(k, len);
    for (uint32_t end = len - 1; end > 0; --end) {
        const uint32_t t = a[0];
        a[0] = a[end];
        a[end] = t;
        sift(0, end);
    }
}

struct SweepArgs {
    uint32_t n;
    const uint32_t* comp_off;
    uint32_t* items;
    const uint32_t* pi;
    const uint32_t* pj;
    double* pos;
    double* prev;
    const double* start;
    const uint8_t* kin;
    const float4* param1;
    const uint8_t* tmask;
    double* move;
    int8_t* code;
    uint8_t* impact;
    uint32_t* scal;
};

// separate (:631-654); returns whether the pair could move (denominator > 0)
__device__ bool separate(const SweepArgs& a, uint32_t i, uint32_t j, int code, double amount) {
    const int axis = (code > 0 ? code : -code) - 1;
    const double wi = inverse_mass(a.kin, a.param1, a.tmask, i, axis);
    const double wj = inverse_mass(a.kin, a.param1, a.tmask, j, axis);
    const double denom = wi + wj;
    if (denom <= 0.0) return false;
    const double s = code > 0 ? 1.0 : -1.0;
    const double di = -s * (amount * wi / denom), dj = s * (amount * wj / denom);
    // The other two components of -normal * x and normal * x, and the whole
    // correction of an endpoint with zero inverse mass on this axis, are
    // signed zeros: adding them leaves every coordinate unchanged, so only the
    // moving endpoints are written.
    if (wi > 0.0) {
        add3(a.pos, a.n, i, axis, di);
        add3(a.prev, a.n, i, axis, di);
        a.move[i] += fabs(di);
    }
    if (wj > 0.0) {
        add3(a.pos, a.n, j, axis, dj);
        add3(a.prev, a.n, j, axis, dj);
        a.move[j] += fabs(dj);
    }
    return true;
}

// One thread replays one component's pairs in pair order.
__global__ void k_sweep(SweepArgs a) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.n) return;
    const uint32_t b = a.comp_off[r], e = a.comp_off[r + 1];
    if (b == e) return;
    sort_range(a.items, b, e);
    bool changed = false;
    for (uint32_t t = b; t < e; ++t) {
        const uint32_t k = a.items[t];
        const uint32_t i = a.pi[k], j = a.pj[k];
        const v3 si = load3(a.start, a.n, i), sj = load3(a.start, a.n, j);
        const v3 pi = load3(a.pos, a.n, i), pj = load3(a.pos, a.n, j);
        const v3 d0 = sj - si;
        int code = swept_normal(si, sj, pi, pj);
        bool impact = false;
        if (code) {
            const double separation = code_dot(code, pj - pi);
            if (separation < kCell) changed |= separate(a, i, j, code, kCell - separation + k1em6);
            impact = code_dot(code, d0) > kNewImpact;
        } else {
            double pen = 0.0;
            code = overlap_normal(pi, pj, d0, &pen);
            if (code) {
                changed |= separate(a, i, j, code, pen + k1em6);
                impact = code_dot(code, d0) > kNewImpact;
            } else {
                code = touching_normal(pi, pj);
            }
        }
        a.code[k] = (int8_t)code;
        a.impact[k] = impact ? 1 : 0;
    }
    if (changed) atomicOr(a.scal + S_CHANGED, 1u);
}

// Movement bounds at the start of a sweep: REVs that cannot move keep 0.
__global__ void k_init_bounds(uint32_t n, const uint8_t* __restrict__ kin, const uint8_t* __restrict__ tmask,
                              double base, double* __restrict__ bound) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) bound[i] = movable(kin, tmask, i) ? base : 0.0;
}

// After a sweep: a REV that moved farther than its bound gets a wider one and
// the sweep must be replayed (flag); the others keep theirs.
__global__ void k_check_bounds(uint32_t n, const double* __restrict__ move, double* __restrict__ bound,
                               uint32_t* __restrict__ flag) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double m = move[i];
    if (m > bound[i]) {
        bound[i] = fmax(2.0 * m, 4.0 * bound[i]);
        atomicOr(flag, 1u);
    }
}

// This sweep's contacts, in pair order: key (i << 32 | j), normal code, impact.
__global__ void k_sweep_contact_flags(uint32_t count, const int8_t* __restrict__ code, uint8_t* __restrict__ flag) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) flag[k] = code[k] != 0;
}
__global__ void k_sweep_contact_write(uint32_t count, const uint8_t* __restrict__ flag, const uint32_t* __restrict__ off,
                                      const uint32_t* __restrict__ pi, const uint32_t* __restrict__ pj,
                                      const int8_t* __restrict__ code, const uint8_t* __restrict__ impact,
                                      unsigned long long* key, int8_t* cn, uint8_t* cm) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count || !flag[k]) return;
    const uint32_t o = off[k];
    key[o] = ((unsigned long long)pi[k] << 32) | pj[k];
    cn[o] = code[k];
    cm[o] = impact[k];
}

// First index of v[0, n) not below key (v ascending).
__device__ __forceinline__ uint32_t lower_bound(const unsigned long long* v, uint32_t n, unsigned long long key) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (v[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// The recorded contacts keep each pair's first contact over the sweeps (the
// reference sorts the pushed contacts by pair and keeps one per pair). A
// sweep's list B joins the recorded list A (both ascending): B's pairs already
// in A are dropped, the rest are merged in by rank.
__global__ void k_new_contacts(uint32_t nb, const unsigned long long* __restrict__ bkey, uint32_t na,
                               const unsigned long long* __restrict__ akey, uint8_t* __restrict__ keep) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const uint32_t at = lower_bound(akey, na, bkey[b]);
    keep[b] = !(at < na && akey[at] == bkey[b]);
}
__global__ void k_merge_recorded(uint32_t na, const unsigned long long* __restrict__ akey,
                                 const int8_t* __restrict__ acn, const uint8_t* __restrict__ acm, uint32_t nb,
                                 const unsigned long long* __restrict__ bkey, const int8_t* __restrict__ bcn,
                                 const uint8_t* __restrict__ bcm, const uint8_t* __restrict__ keep,
                                 const uint32_t* __restrict__ boff, unsigned long long* okey, int8_t* ocn,
                                 uint8_t* ocm) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < na) {  // kept B entries before it: B's kept prefix up to its first key not below A's
        const uint32_t o = t + boff[lower_bound(bkey, nb, akey[t])];
        okey[o] = akey[t];
        ocn[o] = acn[t];
        ocm[o] = acm[t];
    } else if (t < na + nb) {
        const uint32_t b = t - na;
        if (!keep[b]) return;
        const uint32_t o = boff[b] + lower_bound(akey, na, bkey[b]);
        okey[o] = bkey[b];
        ocn[o] = bcn[b];
        ocm[o] = bcm[b];
    }
}

__global__ void k_contacts_out(uint32_t count, const unsigned long long* __restrict__ key,
                               const int8_t* __restrict__ rcn, const uint8_t* __restrict__ rcm, uint32_t* ci,
                               uint32_t* cj, int8_t* cn, uint8_t* cm, const uint32_t* __restrict__ rslot,
                               uint32_t* slot_contacts) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const uint32_t i = (uint32_t)(key[k] >> 32);
    ci[k] = i;
    cj[k] = (uint32_t)key[k];
    cn[k] = rcn[k];
    cm[k] = rcm[k];
    if (slot_contacts) atomicAdd(slot_contacts + rslot[i], 1u);
}

// ---- contact velocities -------------------------------------------------

struct ResolveArgs {
    uint32_t n;
    const uint32_t* comp_off;
    uint32_t* items;
    const uint32_t* ci;
    const uint32_t* cj;
    const int8_t* cn;
    const uint8_t* cm;
    double* vel;
    double* phys;  // pre-contact velocities, updated with the physical impulses
    const uint8_t* kin;
    const float4* param1;
    const uint8_t* tmask;
    double restitution;
    double friction;
    double* heat;  // [2][n]: restitution, friction heat per component root
};

// resolve_velocities_with_precontact (:133-300) over one component's contacts
__global__ void k_resolve(ResolveArgs a) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.n) return;
    const uint32_t b = a.comp_off[r], e = a.comp_off[r + 1];
    if (b == e) return;
    sort_range(a.items, b, e);
    const uint32_t n = a.n;
    double rheat = 0.0, fheat = 0.0;
    for (int iteration = 0; iteration < 4; ++iteration) {
        bool changed = false;
        for (uint32_t t = b; t < e; ++t) {
            const uint32_t c = a.items[t];
            const uint32_t i = a.ci[c], j = a.cj[c];
            const int code = a.cn[c];
            const bool new_impact = a.cm[c] != 0;
            const int axis = (code > 0 ? code : -code) - 1;
            double nrm[3] = {0.0, 0.0, 0.0};
            nrm[axis] = code > 0 ? 1.0 : -1.0;
            const double wi = inverse_mass(a.kin, a.param1, a.tmask, i, axis);
            const double wj = inverse_mass(a.kin, a.param1, a.tmask, j, axis);
            const double denom = wi + wj;
            if (denom <= 0.0) continue;
            double vi[3], vj[3];
            for (int q = 0; q < 3; ++q) {
                vi[q] = a.vel[(size_t)q * n + i];
                vj[q] = a.vel[(size_t)q * n + j];
            }
            const double rv[3] = {vj[0] - vi[0], vj[1] - vi[1], vj[2] - vi[2]};
            const double closing = rv[0] * nrm[0] + rv[1] * nrm[1] + rv[2] * nrm[2];
            double normal_impulse = 0.0;
            if (closing < -k1em6) {
                const double rest = (new_impact && iteration == 0) ? a.restitution : 0.0;
                normal_impulse = -(1.0 + rest) * closing / denom;
                double qi[3], qj[3];
                for (int q = 0; q < 3; ++q) {
                    qi[q] = a.phys[(size_t)q * n + i];
                    qj[q] = a.phys[(size_t)q * n + j];
                }
                const double pr[3] = {qj[0] - qi[0], qj[1] - qi[1], qj[2] - qi[2]};
                const double physical_closing = pr[0] * nrm[0] + pr[1] * nrm[1] + pr[2] * nrm[2];
                const double physical_impulse =
                    new_impact ? normal_impulse
                               : (physical_closing < -k1em6 ? fmin(-physical_closing / denom, normal_impulse) : 0.0);
                for (int q = 0; q < 3; ++q) {
                    vi[q] -= nrm[q] * (normal_impulse * wi);
                    vj[q] += nrm[q] * (normal_impulse * wj);
                }
                const double heat_closing = new_impact ? closing : physical_closing;
                double rh = 0.0;
                if (heat_closing < -k1em6 && physical_impulse > 0.0)
                    rh = fmax(physical_impulse * -heat_closing - 0.5 * (physical_impulse * physical_impulse) * denom,
                              0.0);
                if (rh > 0.0) rheat += rh;
                // an endpoint with zero inverse mass on the normal axis keeps
                // its physical velocity (the update is a signed zero)
                for (int q = 0; q < 3; ++q) {
                    if (wi > 0.0) a.phys[(size_t)q * n + i] = qi[q] - nrm[q] * (physical_impulse * wi);
                    if (wj > 0.0) a.phys[(size_t)q * n + j] = qj[q] + nrm[q] * (physical_impulse * wj);
                }
                changed = true;
            }
            if (normal_impulse > 0.0 && a.friction > 0.0) {
                const double rel[3] = {vj[0] - vi[0], vj[1] - vi[1], vj[2] - vi[2]};
                const double rn = rel[0] * nrm[0] + rel[1] * nrm[1] + rel[2] * nrm[2];
                double tr[3], rt[3];
                for (int q = 0; q < 3; ++q) {
                    const double tangent = rel[q] - nrm[q] * rn;
                    tr[q] = inverse_mass(a.kin, a.param1, a.tmask, i, q) + inverse_mass(a.kin, a.param1, a.tmask, j, q);
                    rt[q] = tr[q] > 0.0 ? tangent : 0.0;
                }
                const double speed = sqrt(rt[0] * rt[0] + rt[1] * rt[1] + rt[2] * rt[2]);
                if (speed > k1em6) {
                    const double dir[3] = {rt[0] / speed, rt[1] / speed, rt[2] / speed};
                    double tw = 0.0;
                    for (int q = 0; q < 3; ++q) tw += dir[q] * dir[q] * tr[q];
                    if (tw > 0.0) {
                        const double mag = fmin(speed / tw, a.friction * normal_impulse);
                        for (int q = 0; q < 3; ++q) {
                            const double imp = -dir[q] * mag;
                            vi[q] -= imp * inverse_mass(a.kin, a.param1, a.tmask, i, q);
                            vj[q] += imp * inverse_mass(a.kin, a.param1, a.tmask, j, q);
                        }
                        const double fh = fmax(mag * speed - 0.5 * (mag * mag) * tw, 0.0);
                        if (fh > 0.0 && (!a.kin[i] || !a.kin[j])) fheat += fh;
                        changed = true;
                    }
                }
            }
            // REVs that cannot move keep their velocities (every update to them
            // is a signed zero); they may be shared with other components
            const bool mi = movable(a.kin, a.tmask, i), mj = movable(a.kin, a.tmask, j);
            for (int q = 0; q < 3; ++q) {
                if (mi) a.vel[(size_t)q * n + i] = vi[q];
                if (mj) a.vel[(size_t)q * n + j] = vj[q];
            }
        }
        if (!changed) break;
    }
    a.heat[r] = rheat;
    a.heat[(size_t)n + r] = fheat;
}

// Fixed-order sum of [count] doubles into out (one block).
__global__ void __launch_bounds__(256) k_sum(uint32_t count, const double* __restrict__ v, double* out) {
    __shared__ double part[256];
    double s = 0.0;
    for (uint32_t k = threadIdx.x; k < count; k += blockDim.x) s += v[k];
    part[threadIdx.x] = s;
    __syncthreads();
    for (unsigned w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = part[0];
}

// ---- exclusive scan (u8 or u32 input, u32 output; out[count] = total) -----

template <class T>
__global__ void __launch_bounds__(256) k_scan_blocks(uint32_t count, const T* __restrict__ in, uint32_t* __restrict__ out,
                                                     uint32_t* __restrict__ bsum) {
    __shared__ uint32_t warp_tot[8];
    const uint32_t base = blockIdx.x * kScanBlock + threadIdx.x * 4;
    uint32_t v[4], local = 0;
    for (int k = 0; k < 4; ++k) {
        v[k] = base + k < count ? (uint32_t)in[base + k] : 0u;
        local += v[k];
    }
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = local;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (unsigned)o) incl += t;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    uint32_t before = 0;
    for (unsigned w = 0; w < warp; ++w) before += warp_tot[w];
    uint32_t run = before + incl - local;
    for (int k = 0; k < 4; ++k) {
        if (base + k < count) out[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == blockDim.x - 1) bsum[blockIdx.x] = before + incl;
}

__global__ void __launch_bounds__(1024) k_scan_sums(uint32_t nb, uint32_t* bsum) {
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t lo = 0; lo < nb; lo += blockDim.x) {
        const uint32_t k = lo + threadIdx.x;
        const uint32_t v = k < nb ? bsum[k] : 0u;
        uint32_t incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (unsigned)o) incl += t;
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        uint32_t before = 0;
        for (unsigned w = 0; w < warp; ++w) before += warp_tot[w];
        const uint32_t c0 = carry;
        if (k < nb) bsum[k] = c0 + before + incl - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = c0 + before + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) bsum[nb] = carry;
}

__global__ void k_scan_add(uint32_t count, uint32_t* __restrict__ out, const uint32_t* __restrict__ bsum, uint32_t nb) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) out[k] += bsum[k / kScanBlock];
    if (k == 0) out[count] = bsum[nb];
}

inline unsigned grid(size_t count) { return (unsigned)((count + 255) / 256); }

}  // namespace

// Grow-only device buffers of the contact stage, owned by the scene.
struct ContactState {
    uint32_t n = 0;
    size_t pair_cap = 0;
    size_t large_cap = 0;  // entries of the large-box table
    uint32_t table1 = 0, table2 = 0;
    // per REV
    Boxes box{};
    double* start = nullptr;    // [3][n] previous positions when the call began
    double* snap = nullptr;     // [6][n] positions and previous at the start of a sweep
    double* move = nullptr;     // [n] summed corrections of the sweep
    double* bound = nullptr;    // [n] how far each REV may move in the sweep
    double* heat = nullptr;     // [2][n]
    double* phys = nullptr;     // [3][n]
    uint32_t* next1 = nullptr;  // [n]
    uint32_t* cnt = nullptr;    // [n + 1]
    uint32_t* off = nullptr;    // [n + 1]
    uint32_t* parent = nullptr; // [n]
    uint32_t* comp_cnt = nullptr;  // [n + 1]
    uint32_t* comp_off = nullptr;  // [n + 1]
    uint32_t* bsum = nullptr;      // scan block sums
    uint32_t* grid_heads = nullptr;  // dense corner grid of a single scene
    size_t grid_cap = 0;
    uint2* stage = nullptr;          // stored pairs of the append pass
    size_t stage_cap = 0;
    size_t bsum_cap = 0;
    unsigned long long* keys1 = nullptr;
    uint32_t* heads1 = nullptr;
    // large boxes
    unsigned long long* keys2 = nullptr;
    uint32_t* heads2 = nullptr;
    uint32_t* ent_id = nullptr;
    uint32_t* ent_next = nullptr;
    // per pair
    uint32_t* pi = nullptr;
    uint32_t* pj = nullptr;
    uint32_t* root = nullptr;
    uint32_t* items = nullptr;
    int8_t* code = nullptr;
    uint8_t* impact = nullptr;
    uint8_t* sw_flag = nullptr;     // [cap] this sweep's contact flags
    uint32_t* sw_off = nullptr;     // [cap + 1]
    // contacts: this sweep's list, the recorded list (two buffers), the output
    size_t contact_cap = 0;
    unsigned long long* sw_key = nullptr;
    int8_t* sw_cn = nullptr;
    uint8_t* sw_cm = nullptr;
    uint8_t* sw_keep = nullptr;
    uint32_t* sw_koff = nullptr;   // [contact_cap + 1]
    unsigned long long* rec_key[2] = {nullptr, nullptr};
    int8_t* rec_cn[2] = {nullptr, nullptr};
    uint8_t* rec_cm[2] = {nullptr, nullptr};
    size_t rec_cap[2] = {0, 0};
    uint32_t* ci = nullptr;
    uint32_t* cj = nullptr;
    int8_t* cn = nullptr;
    uint8_t* cm = nullptr;
    uint32_t contacts = 0;
    uint32_t launches = 0;  // kernels launched by the current call
    uint32_t* slot_contacts = nullptr;  // [pool slots] contacts per slot of the last projection
    // scalars: [0] error bits, [1..3] small extents, [4] large count, [5] changed,
    // [6..7] candidate count (u64); max movement (u64 bits of a double); the
    // host copies
    uint32_t* scal = nullptr;
    double* heat_sum = nullptr;  // [2]
    uint32_t* h_scal = nullptr;  // pinned [32]: [0, 16) the scalars, [16, 18) max movement, [18] a count
};

namespace {

int32_t cuda_fail(cudaError_t e, const char* what) {
    set_error("%s: %s", what, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? VX_OOM : VX_CUDA_ERROR;
}

template <class T>
cudaError_t grow(T*& p, size_t& cap, size_t want) {
    if (want <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&p, want * sizeof(T));
    if (e == cudaSuccess) cap = want;
    return e;
}

template <class T>
cudaError_t alloc(T*& p, size_t count) {
    return cudaMalloc(&p, (count ? count : 1) * sizeof(T));
}

uint32_t pow2_at_least(size_t v) {
    uint32_t p = 1024;
    while (p < v && p < (1u << 31)) p <<= 1;
    return p;
}

// out[0..count) = exclusive scan of in, out[count] = total.
template <class T>
cudaError_t scan(ContactState* c, cudaStream_t st, const T* in, uint32_t* out, uint32_t count) {
    const uint32_t nb = (count + kScanBlock - 1) / kScanBlock;
    cudaError_t e = grow(c->bsum, c->bsum_cap, (size_t)nb + 2);
    if (e != cudaSuccess) return e;
    if (count == 0) return cudaMemsetAsync(out, 0, sizeof(uint32_t), st);
    k_scan_blocks<T><<<nb, 256, 0, st>>>(count, in, out, c->bsum);
    k_scan_sums<<<1, 1024, 0, st>>>(nb, c->bsum);
    k_scan_add<<<grid(count), 256, 0, st>>>(count, out, c->bsum, nb);
    c->launches += 3;
    return cudaGetLastError();
}

cudaError_t ensure_state(vx_scene* s) {
    ContactState* c = s->contact;
    if (c && c->n == s->n) return cudaSuccess;
    if (c) {
        contact_release(s);
    }
    c = new (std::nothrow) ContactState();
    if (!c) return cudaErrorMemoryAllocation;
    s->contact = c;
    const size_t n = s->n ? s->n : 1;
    c->n = s->n;
    c->table1 = pow2_at_least(2 * n);
    cudaError_t e = alloc(c->box.lo, 3 * n);
    if (e == cudaSuccess) e = alloc(c->box.hi, 3 * n);
    if (e == cudaSuccess) e = alloc(c->box.large, n);
    if (e == cudaSuccess) e = alloc(c->box.slot, n);
    if (e == cudaSuccess && s->pool_slots) e = alloc(c->slot_contacts, s->pool_slots);
    if (e == cudaSuccess) e = alloc(c->start, 3 * n);
    if (e == cudaSuccess) e = alloc(c->snap, 6 * n);
    if (e == cudaSuccess) e = alloc(c->move, n);
    if (e == cudaSuccess) e = alloc(c->bound, n);
    if (e == cudaSuccess) e = alloc(c->heat, 2 * n);
    if (e == cudaSuccess) e = alloc(c->phys, 3 * n);
    if (e == cudaSuccess) e = alloc(c->next1, n);
    if (e == cudaSuccess) e = alloc(c->cnt, n + 1);
    if (e == cudaSuccess) e = alloc(c->off, n + 1);
    if (e == cudaSuccess) e = alloc(c->parent, n);
    if (e == cudaSuccess) e = alloc(c->comp_cnt, n + 1);
    if (e == cudaSuccess) e = alloc(c->comp_off, n + 1);
    if (e == cudaSuccess) e = alloc(c->keys1, c->table1);
    if (e == cudaSuccess) e = alloc(c->heads1, c->table1);
    if (e == cudaSuccess) e = alloc(c->scal, kScalars);
    if (e == cudaSuccess) e = grow(c->stage, c->stage_cap, n / 4 + 4096);
    if (e == cudaSuccess) e = alloc(c->heat_sum, 2);
    if (e == cudaSuccess) e = cudaMallocHost(&c->h_scal, 32 * sizeof(uint32_t));
    return e;
}

cudaError_t ensure_pairs(ContactState* c, size_t want) {
    if (want <= c->pair_cap && c->pi) return cudaSuccess;
    size_t cap = std::max<size_t>(want + want / 4, 4096);
    void* ptrs[] = {c->pi, c->pj, c->root, c->items, c->code, c->impact, c->sw_flag, c->sw_off};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    c->pi = c->pj = c->root = c->items = c->sw_off = nullptr;
    c->impact = c->sw_flag = nullptr;
    c->code = nullptr;
    c->pair_cap = 0;
    cudaError_t e = alloc(c->pi, cap);
    if (e == cudaSuccess) e = alloc(c->pj, cap);
    if (e == cudaSuccess) e = alloc(c->root, cap);
    if (e == cudaSuccess) e = alloc(c->items, cap);
    if (e == cudaSuccess) e = alloc(c->code, cap);
    if (e == cudaSuccess) e = alloc(c->impact, cap);
    if (e == cudaSuccess) e = alloc(c->sw_flag, cap);
    if (e == cudaSuccess) e = alloc(c->sw_off, cap + 1);
    if (e == cudaSuccess) c->pair_cap = cap;
    return e;
}

// The output contact list and the per-sweep list: want entries.
cudaError_t ensure_contacts(ContactState* c, size_t want) {
    if (want <= c->contact_cap && c->ci) return cudaSuccess;
    size_t cap = std::max<size_t>(want + want / 4, 4096);
    void* own[] = {c->sw_key, c->sw_cn, c->sw_cm, c->sw_keep, c->sw_koff, c->ci, c->cj, c->cn, c->cm};
    for (void* p : own)
        if (p) cudaFree(p);
    c->sw_key = nullptr;
    c->sw_cn = c->cn = nullptr;
    c->sw_cm = c->sw_keep = c->cm = nullptr;
    c->sw_koff = c->ci = c->cj = nullptr;
    c->contact_cap = 0;
    cudaError_t e = alloc(c->sw_key, cap);
    if (e == cudaSuccess) e = alloc(c->sw_cn, cap);
    if (e == cudaSuccess) e = alloc(c->sw_cm, cap);
    if (e == cudaSuccess) e = alloc(c->sw_keep, cap);
    if (e == cudaSuccess) e = alloc(c->sw_koff, cap + 1);
    if (e == cudaSuccess) e = alloc(c->ci, cap);
    if (e == cudaSuccess) e = alloc(c->cj, cap);
    if (e == cudaSuccess) e = alloc(c->cn, cap);
    if (e == cudaSuccess) e = alloc(c->cm, cap);
    if (e == cudaSuccess) c->contact_cap = cap;
    return e;
}

// Recorded-contact buffer b can hold want entries (its contents are not kept).
cudaError_t ensure_recorded(ContactState* c, int b, size_t want) {
    if (want <= c->rec_cap[b] && c->rec_key[b]) return cudaSuccess;
    size_t cap = std::max<size_t>(want + want / 4, 4096);
    if (c->rec_key[b]) cudaFree(c->rec_key[b]);
    if (c->rec_cn[b]) cudaFree(c->rec_cn[b]);
    if (c->rec_cm[b]) cudaFree(c->rec_cm[b]);
    c->rec_key[b] = nullptr;
    c->rec_cn[b] = nullptr;
    c->rec_cm[b] = nullptr;
    c->rec_cap[b] = 0;
    cudaError_t e = alloc(c->rec_key[b], cap);
    if (e == cudaSuccess) e = alloc(c->rec_cn[b], cap);
    if (e == cudaSuccess) e = alloc(c->rec_cm[b], cap);
    if (e == cudaSuccess) c->rec_cap[b] = cap;
    return e;
}

cudaError_t ensure_large(ContactState* c, size_t entries) {
    if (entries <= c->large_cap && c->ent_id) return cudaSuccess;
    if (c->ent_id) cudaFree(c->ent_id);
    if (c->ent_next) cudaFree(c->ent_next);
    if (c->keys2) cudaFree(c->keys2);
    if (c->heads2) cudaFree(c->heads2);
    c->ent_id = c->ent_next = c->heads2 = nullptr;
    c->keys2 = nullptr;
    c->large_cap = 0;
    const size_t cap = std::max<size_t>(entries + entries / 4, 4096);
    c->table2 = pow2_at_least(2 * cap);
    cudaError_t e = alloc(c->ent_id, cap);
    if (e == cudaSuccess) e = alloc(c->ent_next, cap);
    if (e == cudaSuccess) e = alloc(c->keys2, c->table2);
    if (e == cudaSuccess) e = alloc(c->heads2, c->table2);
    if (e == cudaSuccess) c->large_cap = cap;
    return e;
}

int32_t read_scalars(vx_scene* s, ContactState* c, const char* what) {
    cudaError_t e = cudaMemcpyAsync(c->h_scal, c->scal, kScalars * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    const uint32_t err = c->h_scal[S_ERR];
    if (err & E_RANGE) {
        set_error("%s: a position is non-finite or too far from the origin for the bin keys (2^%d cells in a "
                  "scene, 2^%d in a pool)", what, kSceneBits - 1, kPoolBits - 1);
        return VX_NONFINITE;
    }
    if (err & E_VOLUME) {
        set_error("%s: a REV swept more than %llu bins in one substep", what, (unsigned long long)kMaxLargeVolume);
        return VX_BAD_INPUT;
    }
    if (err & (E_TABLE | E_UNION)) {
        set_error("%s: a hash probe or a union exceeded its bound", what);
        return VX_TIMEOUT;
    }
    return VX_OK;
}

// Components of the listed items over shared REVs: comp_off (by root REV) and
// items grouped per component (unsorted inside a component).
cudaError_t components(vx_scene* s, ContactState* c, uint32_t count, const uint32_t* list, const uint32_t* ia,
                       const uint32_t* ja, uint32_t* grouped) {
    const uint32_t n = s->n;
    cudaStream_t st = s->stream;
    k_iota<<<grid(n), 256, 0, st>>>(n, c->parent);
    c->launches += 1;
    cudaError_t e = cudaMemsetAsync(c->comp_cnt, 0, ((size_t)n + 1) * sizeof(uint32_t), st);
    if (e != cudaSuccess || count == 0) {
        if (e == cudaSuccess) e = cudaMemsetAsync(c->comp_off, 0, ((size_t)n + 1) * sizeof(uint32_t), st);
        return e;
    }
    k_union<<<grid(count), 256, 0, st>>>(count, list, ia, ja, s->kin, s->tmask, c->parent, c->scal);
    k_roots<<<grid(count), 256, 0, st>>>(count, list, ia, ja, s->kin, s->tmask, c->parent, c->root, c->comp_cnt);
    c->launches += 3;
    e = scan(c, st, c->comp_cnt, c->comp_off, n);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->comp_cnt, 0, ((size_t)n + 1) * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    k_fill<<<grid(count), 256, 0, st>>>(count, list, c->root, c->comp_off, c->comp_cnt, grouped);
    return cudaGetLastError();
}

}  // namespace

void contact_release(vx_scene* s) {
    ContactState* c = s->contact;
    if (!c) return;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    void* ptrs[] = {c->box.lo, c->box.hi, c->box.large, c->box.slot, c->slot_contacts, c->start, c->snap, c->move, c->bound, c->heat, c->phys, c->next1,
                    c->cnt, c->off, c->parent, c->comp_cnt, c->comp_off, c->bsum, c->keys1, c->heads1, c->keys2,
                    c->heads2, c->ent_id, c->ent_next, c->pi, c->pj, c->root,
                    c->items, c->code, c->impact, c->sw_flag, c->sw_off, c->sw_key, c->sw_cn, c->sw_cm,
                    c->sw_keep, c->sw_koff, c->rec_key[0], c->rec_key[1], c->rec_cn[0], c->rec_cn[1],
                    c->rec_cm[0], c->rec_cm[1], c->ci, c->cj, c->cn, c->cm,
                    c->scal, c->heat_sum, c->grid_heads, c->stage};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (c->h_scal) cudaFreeHost(c->h_scal);
    delete c;
    s->contact = nullptr;
}

// collision::project over the scene's positions, with its previous positions
// as the swept starts; targeted axes have zero inverse mass. In a pool, every
// slot taking part in the call (the tile mask) is projected on its own, and
// slot_contacts (host, [pool slots], or null) receives the contacts per slot.
int32_t contact_project(vx_scene* s, vx_contact_stats* out, uint32_t* slot_contacts) {
    const char* what = "vx_contact_project";
    vx_contact_stats st_out{};
    cudaError_t e = ensure_state(s);
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return VX_OOM;
    }
    ContactState* c = s->contact;
    const uint32_t n = s->n;
    cudaStream_t st = s->stream;
    c->contacts = 0;
    c->launches = 0;
    const bool pooled = s->pool_slots > 0;
    if (pooled && s->pool_slots > kPoolKeySlots) {
        set_error("%s: contact keys hold %u pool slots, the pool has %u", what, kPoolKeySlots, s->pool_slots);
        return VX_BAD_INPUT;
    }
    if (slot_contacts && pooled) std::fill(slot_contacts, slot_contacts + s->pool_slots, 0u);
    if (n < 2) {
        if (out) *out = st_out;
        return VX_OK;
    }
    RevFilter filter{};
    if (pooled) filter = RevFilter{s->tile_on, s->tile_scene, s->pool_slot_first, s->pool_slot_revs};
    c->box.bits = pooled ? kPoolBits : kSceneBits;
    const size_t v3b = 3 * (size_t)n * sizeof(double);
    e = cudaMemcpyAsync(c->start, s->prev, v3b, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->scal, 0, kScalars * sizeof(uint32_t), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->scal + S_CMIN, 0xFF, 3 * sizeof(uint32_t), st);
    if (e != cudaSuccess) return cuda_fail(e, what);
    k_boxes<<<grid(n), 256, 0, st>>>(n, s->pos, c->start, c->box, filter, c->scal);
    c->launches += 1;
    int32_t r = read_scalars(s, c, what);
    if (r != VX_OK) return r;
    // Corners of a single scene that fill a compact box go into a dense grid;
    // the others (pools, sparse scenes) into the hash.
    CornerGrid cgrid{};
    uint64_t cells = 0;
    if (!pooled && c->h_scal[S_CMIN] <= c->h_scal[S_CMAX]) {
        cells = 1;
        for (int t = 0; t < 3; ++t) cells *= (uint64_t)(c->h_scal[S_CMAX + t] - c->h_scal[S_CMIN + t]) + 1;
    }
    if (cells && cells <= 8ull * n + 4096 && cells < (1ull << 31)) {  // 32-bit cell indices
        e = grow(c->grid_heads, c->grid_cap, cells);
        if (e == cudaSuccess) e = cudaMemsetAsync(c->grid_heads, 0xFF, cells * sizeof(uint32_t), st);
        if (e != cudaSuccess) return cuda_fail(e, what);
        cgrid.heads = c->grid_heads;
        cgrid.x0 = (int32_t)(c->h_scal[S_CMIN] - (uint32_t)kCornerBias);
        cgrid.y0 = (int32_t)(c->h_scal[S_CMIN + 1] - (uint32_t)kCornerBias);
        cgrid.z0 = (int32_t)(c->h_scal[S_CMIN + 2] - (uint32_t)kCornerBias);
        cgrid.nx = c->h_scal[S_CMAX] - c->h_scal[S_CMIN] + 1;
        cgrid.ny = c->h_scal[S_CMAX + 1] - c->h_scal[S_CMIN + 1] + 1;
        cgrid.nz = c->h_scal[S_CMAX + 2] - c->h_scal[S_CMIN + 2] + 1;
        k_insert_corners_dense<<<grid(n), 256, 0, st>>>(n, c->box, cgrid, c->next1);
    } else {
        e = cudaMemsetAsync(c->keys1, 0xFF, (size_t)c->table1 * sizeof(unsigned long long), st);
        if (e == cudaSuccess) e = cudaMemsetAsync(c->heads1, 0xFF, (size_t)c->table1 * sizeof(uint32_t), st);
        if (e != cudaSuccess) return cuda_fail(e, what);
        k_insert_corners<<<grid(n), 256, 0, st>>>(n, c->box, c->keys1, c->heads1, c->next1, c->table1 - 1, c->scal);
    }
    c->launches += 1;
    r = read_scalars(s, c, what);
    if (r != VX_OK) return r;
    const uint32_t large = c->h_scal[S_LARGE];
    uint32_t mask2 = 0;
    if (large) {
        k_large_volume<<<grid(n), 256, 0, st>>>(n, c->box, c->cnt, c->scal);
        c->launches += 1;
        e = scan(c, st, c->cnt, c->off, n);
        uint32_t entries = 0;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&c->h_scal[kHostCount], c->off + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, what);
        r = read_scalars(s, c, what);
        if (r != VX_OK) return r;
        const uint64_t total = (uint64_t)c->h_scal[S_LVOL] | ((uint64_t)c->h_scal[S_LVOL + 1] << 32);
        if (total > kMaxLargeEntries) {  // checked before the 32-bit offsets below are used
            set_error("%s: fast REVs swept %llu bins together in one substep, more than %llu", what,
                      (unsigned long long)total, (unsigned long long)kMaxLargeEntries);
            return VX_BAD_INPUT;
        }
        entries = c->h_scal[kHostCount];
        e = ensure_large(c, entries);
        if (e == cudaSuccess) e = cudaMemsetAsync(c->keys2, 0xFF, (size_t)c->table2 * sizeof(unsigned long long), st);
        if (e == cudaSuccess) e = cudaMemsetAsync(c->heads2, 0xFF, (size_t)c->table2 * sizeof(uint32_t), st);
        if (e != cudaSuccess) return cuda_fail(e, what);
        k_insert_large<<<grid(n), 256, 0, st>>>(n, c->box, c->off, c->keys2, c->heads2, c->ent_id, c->ent_next,
                                                 c->table2 - 1, c->scal);
        c->launches += 1;
        mask2 = c->table2 - 1;
    }
    PairArgs pa{};
    pa.n = n;
    pa.b = c->box;
    pa.kin = s->kin;
    pa.rest = s->rest;
    pa.nbr = s->nbr;
    pa.rev = s->rev;
    pa.keys1 = c->keys1;
    pa.heads1 = c->heads1;
    pa.next1 = c->next1;
    pa.mask1 = c->table1 - 1;
    pa.grid = cgrid;
    pa.keys2 = c->keys2;
    pa.heads2 = c->heads2;
    pa.ent_id = c->ent_id;
    pa.ent_next = c->ent_next;
    pa.mask2 = mask2;
    pa.wx = std::max<int32_t>(1, (int32_t)c->h_scal[S_EXT]);
    pa.wy = std::max<int32_t>(1, (int32_t)c->h_scal[S_EXT + 1]);
    pa.wz = std::max<int32_t>(1, (int32_t)c->h_scal[S_EXT + 2]);
    pa.count = c->cnt;
    pa.off = c->off;
    pa.scal = c->scal;
    pa.pos = s->pos;
    pa.start = c->start;
    // Each sweep stores only the pairs that can act in it while every REV
    // moves at most its bound (kSweepBound for REVs that can move, 0 for the
    // others): the lattice's two-cell neighbours never can. When a REV moves
    // farther, its bound is widened and the sweep is restored and replayed;
    // after kMaxAttempts tries every pair is stored. The replay is exact with
    // any bounds.
    bool first_generation = true;
    pa.bound = c->bound;
    auto generate = [&](bool all, uint32_t* out_stored) -> int32_t {
        pa.all = all;
        pa.count_pairs = first_generation;
        pa.pi = nullptr;
        pa.pj = nullptr;
        pa.stage = c->stage;
        pa.stage_cap = (uint32_t)std::min<size_t>(c->stage_cap, 0xffffffffu);
        cudaError_t ge = cudaMemsetAsync(c->cnt, 0, ((size_t)n + 1) * sizeof(uint32_t), st);
        if (ge == cudaSuccess) ge = cudaMemsetAsync(c->scal + S_CAND_LO, 0, 4 * sizeof(uint32_t), st);
        if (ge == cudaSuccess) ge = cudaMemsetAsync(c->scal + S_STAGE, 0, sizeof(uint32_t), st);
        if (ge == cudaSuccess) ge = cudaMemsetAsync(c->scal + S_STORED, 0, 2 * sizeof(uint32_t), st);
        if (ge != cudaSuccess) return cuda_fail(ge, what);
        if (n < kPairSmallScene) k_pairs<kAppendPass, 4><<<grid((size_t)n * 4), 256, 0, st>>>(pa);
        else k_pairs<kAppendPass, 1><<<grid(n), 256, 0, st>>>(pa);
        c->launches += 1;
        ge = scan(c, st, c->cnt, c->off, n);
        if (ge == cudaSuccess)
            ge = cudaMemcpyAsync(&c->h_scal[kHostCount], c->off + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        if (ge != cudaSuccess) return cuda_fail(ge, what);
        int32_t gr = read_scalars(s, c, what);
        if (gr != VX_OK) return gr;
        const uint64_t stored64 = (uint64_t)c->h_scal[S_STORED] | ((uint64_t)c->h_scal[S_STORED + 1] << 32);
        if (stored64 > kMaxStoredPairs) {  // checked before the 32-bit offsets are used
            set_error("%s: %llu pairs can act in one sweep, more than %llu", what, (unsigned long long)stored64,
                      (unsigned long long)kMaxStoredPairs);
            return VX_OOM;
        }
        const uint32_t stored = c->h_scal[kHostCount];
        if (first_generation) {  // the candidate and pair counts do not depend on the bound
            st_out.candidates = (uint64_t)c->h_scal[S_CAND_LO] | ((uint64_t)c->h_scal[S_CAND_HI] << 32);
            st_out.pairs = (uint64_t)c->h_scal[S_PAIRS_LO] | ((uint64_t)c->h_scal[S_PAIRS_HI] << 32);
            first_generation = false;
        }
        st_out.stored = std::max<uint64_t>(st_out.stored, stored);
        ge = ensure_pairs(c, stored);
        if (ge != cudaSuccess) {
            set_error("%s: %u stored pairs: %s", what, stored, cudaGetErrorString(ge));
            return VX_OOM;
        }
        pa.pi = c->pi;
        pa.pj = c->pj;
        if (stored) {
            ge = cudaMemsetAsync(c->cnt, 0, ((size_t)n + 1) * sizeof(uint32_t), st);
            if (ge != cudaSuccess) return cuda_fail(ge, what);
            if (stored <= c->stage_cap) {  // every stored pair was staged
                k_stage_scatter<<<grid(stored), 256, 0, st>>>(stored, c->stage, c->off, c->cnt, c->pi, c->pj);
            } else {  // the staging list overflowed: write the pairs in a second pass
                if (n < kPairSmallScene) k_pairs<kWritePass, 4><<<grid((size_t)n * 4), 256, 0, st>>>(pa);
                else k_pairs<kWritePass, 1><<<grid(n), 256, 0, st>>>(pa);
            }
            k_sort_segments<<<grid(n), 256, 0, st>>>(n, c->off, c->pj);
            c->launches += 2;
        }
        if (stored > c->stage_cap) {  // room for this many next time
            ge = grow(c->stage, c->stage_cap, (size_t)stored + stored / 2 + 4096);
            if (ge != cudaSuccess) {
                set_error("%s: a staging list of %u pairs: %s", what, stored, cudaGetErrorString(ge));
                return VX_OOM;
            }
        }
        *out_stored = stored;
        return VX_OK;
    };
    SweepArgs sa{};  // the pair arrays are bound after each generation, which may reallocate them
    sa.n = n;
    sa.comp_off = c->comp_off;
    sa.pos = s->pos;
    sa.prev = s->prev;
    sa.start = c->start;
    sa.kin = s->kin;
    sa.param1 = s->param1;
    sa.tmask = s->tmask;
    sa.move = c->move;
    sa.scal = c->scal;
    uint32_t recorded = 0;
    int cur = 0;
    for (int sweep = 0; sweep < 6; ++sweep) {  // the sweeps (project :51-103)
        st_out.sweeps += 1;
        e = cudaMemcpyAsync(c->snap, s->pos, v3b, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(c->snap + 3 * (size_t)n, s->prev, v3b, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return cuda_fail(e, what);
        k_init_bounds<<<grid(n), 256, 0, st>>>(n, s->kin, s->tmask, kSweepBound, c->bound);
        c->launches += 1;
        bool changed = false;
        uint32_t stored = 0;
        for (int attempt = 0;; ++attempt) {
            const bool all_pairs = attempt >= kMaxAttempts;
            r = generate(all_pairs, &stored);
            if (r != VX_OK) return r;
            e = cudaMemsetAsync(c->scal + S_CHANGED, 0, sizeof(uint32_t), st);
            if (e == cudaSuccess) e = cudaMemsetAsync(c->scal + S_MOVED, 0, sizeof(uint32_t), st);
            if (e == cudaSuccess) e = cudaMemsetAsync(c->move, 0, (size_t)n * sizeof(double), st);
            if (e != cudaSuccess) return cuda_fail(e, what);
            st_out.live_max = std::max(st_out.live_max, stored);
            sa.pi = c->pi;
            sa.pj = c->pj;
            sa.items = c->items;
            sa.code = c->code;
            sa.impact = c->impact;
            e = components(s, c, stored, nullptr, c->pi, c->pj, c->items);
            if (e != cudaSuccess) return cuda_fail(e, what);
            if (stored) {
                k_sweep<<<grid(n), 256, 0, st>>>(sa);
                c->launches += 1;
            }
            k_check_bounds<<<grid(n), 256, 0, st>>>(n, c->move, c->bound, c->scal + S_MOVED);
            c->launches += 1;
            r = read_scalars(s, c, what);
            if (r != VX_OK) return r;
            changed = c->h_scal[S_CHANGED] != 0;
            if (all_pairs || !c->h_scal[S_MOVED]) break;
            // a REV moved farther than its bound: replay from the sweep's start
            st_out.redone += 1;
            e = cudaMemcpyAsync(s->pos, c->snap, v3b, cudaMemcpyDeviceToDevice, st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(s->prev, c->snap + 3 * (size_t)n, v3b, cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) return cuda_fail(e, what);
        }
        if (stored) {  // this sweep's contacts join the recorded ones
            k_sweep_contact_flags<<<grid(stored), 256, 0, st>>>(stored, c->code, c->sw_flag);
            c->launches += 1;
            e = scan(c, st, c->sw_flag, c->sw_off, stored);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(&c->h_scal[kHostCount], c->sw_off + stored, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return cuda_fail(e, what);
            const uint32_t nb = c->h_scal[kHostCount];
            if (nb) {
                e = ensure_contacts(c, std::max<size_t>(nb, recorded));
                if (e == cudaSuccess) e = ensure_recorded(c, 1 - cur, (size_t)recorded + nb);
                if (e != cudaSuccess) {
                    set_error("%s: %u contacts: %s", what, recorded + nb, cudaGetErrorString(e));
                    return VX_OOM;
                }
                k_sweep_contact_write<<<grid(stored), 256, 0, st>>>(stored, c->sw_flag, c->sw_off, c->pi, c->pj, c->code,
                                                                    c->impact, c->sw_key, c->sw_cn, c->sw_cm);
                k_new_contacts<<<grid(nb), 256, 0, st>>>(nb, c->sw_key, recorded, c->rec_key[cur], c->sw_keep);
                c->launches += 2;
                e = scan(c, st, c->sw_keep, c->sw_koff, nb);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(&c->h_scal[kHostCount + 1], c->sw_koff + nb, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
                if (e != cudaSuccess) return cuda_fail(e, what);
                k_merge_recorded<<<grid((size_t)recorded + nb), 256, 0, st>>>(
                    recorded, c->rec_key[cur], c->rec_cn[cur], c->rec_cm[cur], nb, c->sw_key, c->sw_cn, c->sw_cm,
                    c->sw_keep, c->sw_koff, c->rec_key[1 - cur], c->rec_cn[1 - cur], c->rec_cm[1 - cur]);
                c->launches += 1;
                e = cudaStreamSynchronize(st);
                if (e != cudaSuccess) return cuda_fail(e, what);
                recorded += c->h_scal[kHostCount + 1];
                cur = 1 - cur;
            }
        }
        if (!changed) break;
    }
    // the recorded contacts, sorted by pair
    uint32_t* per_slot = pooled && slot_contacts ? c->slot_contacts : nullptr;
    if (per_slot) {
        e = cudaMemsetAsync(per_slot, 0, s->pool_slots * sizeof(uint32_t), st);
        if (e != cudaSuccess) return cuda_fail(e, what);
    }
    if (recorded) {
        e = ensure_contacts(c, recorded);
        if (e != cudaSuccess) {
            set_error("%s: %u contacts: %s", what, recorded, cudaGetErrorString(e));
            return VX_OOM;
        }
        k_contacts_out<<<grid(recorded), 256, 0, st>>>(recorded, c->rec_key[cur], c->rec_cn[cur], c->rec_cm[cur], c->ci,
                                                       c->cj, c->cn, c->cm, c->box.slot, per_slot);
        c->launches += 1;
    }
    if (per_slot) {
        e = cudaMemcpyAsync(slot_contacts, per_slot, s->pool_slots * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) return cuda_fail(e, what);
    }
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, what);
    c->contacts = recorded;
    st_out.contacts = recorded;
    st_out.launches = c->launches;
    if (out) *out = st_out;
    return VX_OK;
}

// resolve_velocities_with_precontact over the contacts of the last projection
// (or those set by vx_scene_set_contacts); pre_contact = NULL uses the current
// velocities (resolve_velocities, :122-131).
int32_t contact_resolve(vx_scene* s, const double* pre_contact, double restitution, double friction,
                        vx_contact_heat* out) {
    const char* what = "vx_contact_resolve_velocities";
    cudaError_t e = ensure_state(s);
    if (e != cudaSuccess) return cuda_fail(e, what);
    ContactState* c = s->contact;
    const uint32_t n = s->n, count = c->contacts;
    cudaStream_t st = s->stream;
    vx_contact_heat heat{};
    if (count && n) {
        // the component scratch (root, items) is pair-sized: it must hold the contacts
        e = ensure_pairs(c, count);
        if (e != cudaSuccess) return cuda_fail(e, what);
        const size_t v3b = 3 * (size_t)n * sizeof(double);
        e = cudaMemcpyAsync(c->phys, pre_contact ? pre_contact : s->vel, v3b, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(c->scal, 0, kScalars * sizeof(uint32_t), st);
        if (e == cudaSuccess) e = cudaMemsetAsync(c->heat, 0, 2 * (size_t)n * sizeof(double), st);
        if (e == cudaSuccess) e = components(s, c, count, nullptr, c->ci, c->cj, c->items);
        if (e != cudaSuccess) return cuda_fail(e, what);
        ResolveArgs ra{};
        ra.n = n;
        ra.comp_off = c->comp_off;
        ra.items = c->items;
        ra.ci = c->ci;
        ra.cj = c->cj;
        ra.cn = c->cn;
        ra.cm = c->cm;
        ra.vel = s->vel;
        ra.phys = c->phys;
        ra.kin = s->kin;
        ra.param1 = s->param1;
        ra.tmask = s->tmask;
        ra.restitution = restitution;
        ra.friction = friction;
        ra.heat = c->heat;
        k_resolve<<<grid(n), 256, 0, st>>>(ra);
        c->launches += 1;
        k_sum<<<1, 256, 0, st>>>(n, c->heat, c->heat_sum);
        k_sum<<<1, 256, 0, st>>>(n, c->heat + n, c->heat_sum + 1);
        c->launches += 2;
        double h[2] = {0.0, 0.0};
        e = cudaMemcpyAsync(h, c->heat_sum, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, what);
        int32_t r = read_scalars(s, c, what);
        if (r != VX_OK) return r;
        heat.restitution = h[0];
        heat.friction = h[1];
    }
    if (out) *out = heat;
    return VX_OK;
}

uint32_t contact_count(const vx_scene* s) { return s->contact ? s->contact->contacts : 0; }

// Device bytes of the contact buffers that scale with the REV count (the
// pair buffers grow with the stored pairs, usually a small share).
uint64_t contact_state_bytes(uint32_t n) {
    const uint64_t m = n ? n : 1;
    const uint64_t per_rev = 6 * 4 + 1 + 4 + 3 * 8 * 3 + 6 * 8 + 8 + 2 * 8 + 4 * 7;  // boxes .. component offsets
    const uint64_t table = pow2_at_least(2 * m);
    const uint64_t stage = (m / 4 + 4096) * 8;  // the initial staging list
    return per_rev * m + table * (8 + 4) + stage;
}

}  // namespace vx

using namespace vx;

extern "C" int32_t vx_contact_project(vx_scene* s, vx_contact_stats* out) {
    clear_error();
    if (!s) {
        set_error("vx_contact_project: null scene");
        return VX_BAD_INPUT;
    }
    cudaSetDevice(s->device);
    return contact_project(s, out, nullptr);
}

extern "C" int32_t vx_contact_resolve_velocities(vx_scene* s, int32_t pre_contact, double restitution,
                                                 double friction, vx_contact_heat* out) {
    clear_error();
    if (!s || pre_contact < 0 || pre_contact > 1) {
        set_error("vx_contact_resolve_velocities: null scene or unknown pre_contact %d", pre_contact);
        return VX_BAD_INPUT;
    }
    if (!std::isfinite(restitution) || !std::isfinite(friction)) {
        set_error("vx_contact_resolve_velocities: non-finite restitution or friction");
        return VX_BAD_INPUT;
    }
    cudaSetDevice(s->device);
    return contact_resolve(s, pre_contact ? s->drift : nullptr, restitution, friction, out);
}

extern "C" int32_t vx_scene_get_contacts(vx_scene* s, uint32_t capacity, uint32_t* i, uint32_t* j, int32_t* normal,
                                         uint8_t* new_impact, uint32_t* out_count) {
    clear_error();
    if (!s) {
        set_error("vx_scene_get_contacts: null scene");
        return VX_BAD_INPUT;
    }
    cudaSetDevice(s->device);
    const uint32_t count = contact_count(s);
    if (out_count) *out_count = count;
    if (count == 0 || capacity == 0) return VX_OK;
    if (capacity < count) {
        set_error("vx_scene_get_contacts: %u contacts, capacity %u", count, capacity);
        return VX_BAD_INPUT;
    }
    ContactState* c = s->contact;
    std::vector<int8_t> cn(count);
    cudaError_t e = cudaSuccess;
    if (i) e = cudaMemcpyAsync(i, c->ci, count * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess && j) e = cudaMemcpyAsync(j, c->cj, count * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess && normal) e = cudaMemcpyAsync(cn.data(), c->cn, count, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess && new_impact) e = cudaMemcpyAsync(new_impact, c->cm, count, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "vx_scene_get_contacts");
    if (normal)
        for (uint32_t k = 0; k < count; ++k) normal[k] = cn[k];
    return VX_OK;
}

extern "C" int32_t vx_scene_set_contacts(vx_scene* s, uint32_t count, const uint32_t* i, const uint32_t* j,
                                         const int32_t* normal, const uint8_t* new_impact) {
    clear_error();
    if (!s || (count && (!i || !j || !normal || !new_impact))) {
        set_error("vx_scene_set_contacts: null argument");
        return VX_BAD_INPUT;
    }
    for (uint32_t k = 0; k < count; ++k) {
        const int32_t a = normal[k] > 0 ? normal[k] : -normal[k];
        if (i[k] >= s->n || j[k] >= s->n || i[k] == j[k] || a < 1 || a > 3) {
            set_error("vx_scene_set_contacts: contact %u (%u, %u, normal %d) is invalid", k, i[k], j[k], normal[k]);
            return VX_BAD_INPUT;
        }
    }
    cudaSetDevice(s->device);
    cudaError_t e = ensure_state(s);
    if (e == cudaSuccess) e = ensure_contacts(s->contact, count);
    if (e == cudaSuccess) e = ensure_pairs(s->contact, count);
    if (e != cudaSuccess) return cuda_fail(e, "vx_scene_set_contacts");
    ContactState* c = s->contact;
    std::vector<int8_t> cn(count);
    for (uint32_t k = 0; k < count; ++k) cn[k] = (int8_t)normal[k];
    if (count) {
        e = cudaMemcpyAsync(c->ci, i, count * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(c->cj, j, count * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(c->cn, cn.data(), count, cudaMemcpyHostToDevice, s->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(c->cm, new_impact, count, cudaMemcpyHostToDevice, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) return cuda_fail(e, "vx_scene_set_contacts");
    }
    c->contacts = count;
    return VX_OK;
}

// vx_brick.cu — the FP32 inner PCG solve as one persistent kernel over
// spatially compact blocks of REVs, with one grid reduction per iteration.
//
// Ownership. REVs are ordered along a Morton (Z-order) curve of their lattice
// cells and cut into one run of `cap` REVs per block, so a block owns a compact
// brick-like piece of the scene and most of its REVs' six neighbours are its
// own. Shared memory holds, per own REV, the stiffness of its three owned bonds,
// its z, its six neighbour refs (16-bit indices into the block's z table), its
// mass term m/h^2 and free-axis flags; after the own REVs the z table has one
// slot per halo REV (a neighbour owned by another block), and the halo slots
// that stand for an incoming bond (the -axis neighbour's own bond) also hold
// that bond's stiffness, loaded once. x, r, p, s = A p and w = A z live in
// registers of the owning thread.
//
// Recurrence. Preconditioned CG in the Chronopoulos-Gear form: with z = D^-1 r
// and w = A z, the three dot products gamma = r.z, delta = w.z and rho = r.r
// come from one reduction, then beta = gamma / gamma_old,
// p.Ap = delta - beta gamma / alpha_old, alpha = gamma / p.Ap,
// p = z + beta p, s = w + beta s, x += alpha p, r -= alpha s. In exact
// arithmetic these are the iterates of the classic loop of src/solver.rs:1833-1911
// (the same alpha, beta and stopping rule on |r| / |r0|, strict, after every
// update); vectors are FP32, dot products are summed in FP64, and alpha and
// beta are rounded to FP32 where they scale vectors.
//
// One iteration: a release of the block's iteration flag once its z is in
// place; w's terms between the block's own REVs (no wait needed); an acquire
// of the flags of the blocks that own its halo REVs (not a grid barrier),
// overlapped by those terms; the halo z gathered from the global copy and the
// halo terms; one grid reduction of (gamma, delta, rho), which is also what
// keeps a block from overwriting its global z while a neighbour may still be
// reading it; the update, which forms the next z = D^-1 r into the block's
// table and the global copy. Every wait is bounded: a wait that runs out
// records VX_TIMEOUT and every block leaves at its next wait.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "vx_device.cuh"
#include "vx_grid.cuh"
#include "vx_kernels.h"
#include "vx_layout.cuh"

namespace vx {

namespace {

constexpr int kBThreads = 512;
constexpr uint32_t kNoRef = 0xFFFFu;
constexpr int kMaxNeighbourBlocks = 32;
constexpr uint8_t kHaloBit = 0x80;  // in the shared copy of a REV's flags: it has a halo neighbour
// shared memory per own REV: K float4[3] + float2[3], z float4, refs 3 words,
// m/h^2, flags; per halo z slot a float4; per halo K slot float4 + float2
constexpr size_t kOwnBytes = 3 * 16 + 3 * 8 + 16 + 12 + 4 + 1;
constexpr size_t kHaloZBytes = 16;
constexpr size_t kHaloKBytes = 16 + 8;

struct BrickArgs {
    uint32_t n;
    uint32_t cap;     // own REVs per block at most
    uint32_t hz_cap;  // halo z slots per block at most
    uint32_t hk_cap;  // halo K slots per block at most
    uint32_t kn;      // REV stride of the per-axis K arrays
    const uint4* info;
    const uint32_t* own;
    const uint32_t* ref;
    const uint32_t* hzg;
    const uint32_t* hke;
    const uint32_t* nbk;
    uint32_t* pub;
    const uint8_t* flags;
    const float* mh2;
    const float* K;
    const float* Dinv;
    const double* src;         // right-hand side in FP64
    const double* scale_from;  // |src|; r0 = src / |src|
    float* x;                  // correction [3][n]
    float4* zg;                // published z [n]
    double* part;              // [3][G] partials
    unsigned long long* count; // grid reductions' arrivals
    int32_t* err;
    PcgScalars* sc;
    double tolerance;
    uint32_t max_iterations;
    unsigned long long spin_limit;
};

struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 smul(const Sym<float>& s, F3 v) {
    return {s.xx * v.x + s.xy * v.y + s.xz * v.z, s.xy * v.x + s.yy * v.y + s.yz * v.z,
            s.xz * v.x + s.yz * v.y + s.zz * v.z};
}
__device__ __forceinline__ Sym<float> sym_of(float4 a, float2 b) { return {a.x, a.y, a.z, a.w, b.x, b.y}; }
__device__ __forceinline__ float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// R own REVs per thread group; TPR threads (1 or 2) per REV. A group's own
// REV k is local index (threadIdx.x / TPR) + k * (blockDim.x / TPR). With two
// threads per REV, the first takes the mass term and the REV's three own bonds,
// the second its three incoming bonds, and a shuffle adds the halves; both keep
// the REV's vectors, and only the first publishes and writes them.
template <int R, int TPR>
__global__ void __launch_bounds__(kBThreads, 1) k_pcg_brick(BrickArgs a) {
    extern __shared__ float4 smem4[];
    __shared__ double red[3][32];
    __shared__ double tot[3];
    __shared__ int s_ok;
    const uint32_t b = blockIdx.x, T = blockDim.x, n = a.n, cap = a.cap;
    const uint32_t group = threadIdx.x / TPR, half = threadIdx.x % TPR, stride = T / TPR;
    const uint4 info = a.info[b];
    const uint32_t cnt = info.x, nz = info.y, nk = info.z, nnb = info.w;
    float4* sK4 = smem4;                                               // [3][cap] (xx, yy, zz, xy)
    float4* sZ = sK4 + 3 * cap;                                        // [cap + hz_cap] z
    float4* sKh4 = sZ + cap + a.hz_cap;                                // [hk_cap]
    float2* sK2 = reinterpret_cast<float2*>(sKh4 + a.hk_cap);          // [3][cap] (xz, yz)
    float2* sKh2 = sK2 + 3 * cap;                                      // [hk_cap]
    uint32_t* sRef = reinterpret_cast<uint32_t*>(sKh2 + a.hk_cap);     // [3][cap]
    float* sM = reinterpret_cast<float*>(sRef + 3 * cap);              // [cap]
    uint8_t* sFL = reinterpret_cast<uint8_t*>(sM + cap);               // [cap]
    const uint32_t* own = a.own + (size_t)b * cap;

    for (uint32_t l = threadIdx.x; l < cnt; l += T) {
        const uint32_t g = own[l];
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            const float* kb = a.K + (size_t)ax * 6 * a.kn;
            sK4[ax * cap + l] = __ldg(reinterpret_cast<const float4*>(kb) + g);
            sK2[ax * cap + l] = __ldg(reinterpret_cast<const float2*>(kb + 4 * (size_t)a.kn) + g);
            sRef[ax * cap + l] = __ldg(a.ref + ((size_t)b * 3 + ax) * cap + l);
        }
        sM[l] = __ldg(a.mh2 + g);
        // the free-axis flags, plus whether any of the REV's neighbours is a halo REV
        uint8_t fl = __ldg(a.flags + g);
#pragma unroll
        for (int t = 0; t < 6; ++t) {
            const uint32_t ref = (sRef[(t >> 1) * cap + l] >> (16 * (t & 1))) & 0xFFFFu;
            if (ref != kNoRef && ref >= cnt) fl |= kHaloBit;
        }
        sFL[l] = fl;
    }
    for (uint32_t h = threadIdx.x; h < nk; h += T) {
        const uint32_t e = __ldg(a.hke + (size_t)b * a.hk_cap + h);
        const uint32_t ax = e / n, j = e - ax * n;
        const float* kb = a.K + (size_t)ax * 6 * a.kn;
        sKh4[h] = __ldg(reinterpret_cast<const float4*>(kb) + j);
        sKh2[h] = __ldg(reinterpret_cast<const float2*>(kb + 4 * (size_t)a.kn) + j);
    }

    uint32_t gid[R];
    float x[R][3], r[R][3], p[R][3], s[R][3], w[R][3];
    double scale;
    {
        const double rn = *a.scale_from;
        scale = rn > 0.0 ? 1.0 / rn : 1.0;
    }
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const uint32_t l = group + k * stride;
        gid[k] = l < cnt ? own[l] : 0u;
#pragma unroll
        for (int c = 0; c < 3; ++c) x[k][c] = r[k][c] = p[k][c] = s[k][c] = w[k][c] = 0.f;
        if (l < cnt) {
            const size_t g = gid[k];
            r[k][0] = (float)(a.src[g] * scale);
            r[k][1] = (float)(a.src[n + g] * scale);
            r[k][2] = (float)(a.src[2 * (size_t)n + g] * scale);
        }
    }

    const int slots[3] = {0, 1, 2};
    unsigned long long seq = 1;
    uint32_t pub = 0, its = 0;
    double gamma_old = 0.0, alpha_old = 0.0, initial = 0.0, residual = 0.0;
    int32_t status = VX_OK;
    bool first = true;
    const unsigned lane = threadIdx.x & 31;
    // z0 = D^-1 r0; later z's are formed at the end of each update
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const uint32_t l = group + k * stride;
        if (l >= cnt || half != 0) continue;
        const F3 z = smul(load_sym(a.Dinv, n, gid[k]), F3{r[k][0], r[k][1], r[k][2]});
        const float4 z4 = make_float4(z.x, z.y, z.z, 0.f);
        sZ[l] = z4;
        a.zg[gid[k]] = z4;
    }
    // one pass over a REV's bond terms: the ones whose neighbour is the block's
    // own (halo == false) or a halo REV (halo == true), added to acc
    auto terms = [&](uint32_t l, F3 zi, bool halo, float (&acc)[3]) {
        constexpr int kTerms = 6 / TPR;
#pragma unroll
        for (int u = 0; u < kTerms; ++u) {
            const int t = TPR == 1 ? u : (int)half * 3 + u;
            const uint32_t word = sRef[(t >> 1) * cap + l];
            const uint32_t ref = (word >> (16 * (t & 1))) & 0xFFFFu;
            if (ref == kNoRef || (ref >= cnt) != halo) continue;
            const float4 zj = sZ[ref];
            Sym<float> Kb;
            if (t < 3) {
                Kb = sym_of(sK4[t * cap + l], sK2[t * cap + l]);
            } else if (ref < cnt) {
                Kb = sym_of(sK4[(t - 3) * cap + ref], sK2[(t - 3) * cap + ref]);
            } else {
                Kb = sym_of(sKh4[ref - cnt], sKh2[ref - cnt]);
            }
            const F3 kv = smul(Kb, F3{zi.x - zj.x, zi.y - zj.y, zi.z - zj.z});
            acc[0] += kv.x, acc[1] += kv.y, acc[2] += kv.z;
        }
    };
    while (true) {
        // ---- the block's z (from the last update) is in place: publish it ----
        __syncthreads();
        ++pub;
        if (threadIdx.x == 0) st_release_u32(a.pub + b, pub);
        // ---- w = A z, the block's own neighbours first (no wait needed) ----
        // w = P (m/h^2 z + sum K (z - z_nbr)) + (I - P) z; w[k] holds the sum so far
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t l = group + k * stride;
            w[k][0] = w[k][1] = w[k][2] = 0.f;
            if (l >= cnt) continue;
            const float4 zi4 = sZ[l];
            const F3 zi = {zi4.x, zi4.y, zi4.z};
            if (half == 0) {
                const float mh = sM[l];
                w[k][0] = mh * zi.x, w[k][1] = mh * zi.y, w[k][2] = mh * zi.z;
            }
            terms(l, zi, false, w[k]);
        }
        // ---- wait for the blocks that own this block's halo REVs ----
        if (threadIdx.x < 32) {
            int ok = 1;
            for (uint32_t q = lane; q < nnb && ok; q += 32) {
                const uint32_t qb = __ldg(a.nbk + (size_t)b * kMaxNeighbourBlocks + q);
                unsigned long long spins = 0;
                while (ld_acquire_u32(a.pub + qb) < pub) {
                    if (++spins >= a.spin_limit || ((spins & 63) == 0 && *(volatile int32_t*)a.err)) {
                        ok = 0;
                        break;
                    }
                }
            }
            ok = __all_sync(0xffffffffu, ok);
            if (lane == 0) {
                if (!ok) atomicExch(a.err, 1);
                s_ok = ok && !*(volatile int32_t*)a.err;
            }
        }
        __syncthreads();
        if (!s_ok) {
            status = VX_TIMEOUT;
            break;
        }
        // ---- halo z, then the halo terms and the partials ----
        for (uint32_t h = threadIdx.x; h < nz; h += T) sZ[cnt + h] = __ldcg(a.zg + __ldg(a.hzg + (size_t)b * a.hz_cap + h));
        __syncthreads();
        double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t l = group + k * stride;
            const bool valid = l < cnt;
            F3 zi = {0.f, 0.f, 0.f};
            if (valid && (sFL[l] & kHaloBit)) {
                const float4 zi4 = sZ[l];
                zi = {zi4.x, zi4.y, zi4.z};
                terms(l, zi, true, w[k]);
            }
            if constexpr (TPR == 2) {  // every lane takes part: both halves of a REV share a warp
                w[k][0] += __shfl_xor_sync(0xffffffffu, w[k][0], 1);
                w[k][1] += __shfl_xor_sync(0xffffffffu, w[k][1], 1);
                w[k][2] += __shfl_xor_sync(0xffffffffu, w[k][2], 1);
            }
            if (!valid) continue;
            const float4 zi4 = sZ[l];
            zi = {zi4.x, zi4.y, zi4.z};
            const uint8_t fl = sFL[l];
            if (!(fl & 1)) w[k][0] = zi.x;
            if (!(fl & 2)) w[k][1] = zi.y;
            if (!(fl & 4)) w[k][2] = zi.z;
            if (half == 0) {
                const F3 rv = {r[k][0], r[k][1], r[k][2]};
                const F3 wv = {w[k][0], w[k][1], w[k][2]};
                acc[0] += (double)dot3(rv, zi);
                acc[1] += (double)dot3(wv, zi);
                acc[2] += (double)dot3(rv, rv);
            }
        }
        double tt[3];
        if (!grid_reduce<3>(acc, slots, a, seq++, red, tot, &s_ok, tt)) {
            status = VX_TIMEOUT;
            break;
        }
        const double gamma = tt[0], delta = tt[1], rho = tt[2];
        if (!isfinite(gamma) || !isfinite(delta) || !isfinite(rho)) {
            status = VX_NONFINITE;
            break;
        }
        if (first) {
            initial = sqrt(rho);
            if (!(initial > 1e-12)) break;  // zero right-hand side: x = 0
            if (a.max_iterations == 0) {
                status = VX_NOT_CONVERGED;
                break;
            }
        } else {
            residual = sqrt(rho) / initial;
            if (residual < a.tolerance) break;
            if (its >= a.max_iterations) {
                status = VX_NOT_CONVERGED;
                break;
            }
        }
        const double beta = first ? 0.0 : gamma / gamma_old;
        const double pap = first ? delta : delta - beta * gamma / alpha_old;
        if (!isfinite(pap) || pap <= 1e-30) {
            its += 1;  // the matvec happened (src/solver.rs:1861-1866)
            if (!isfinite(pap)) status = VX_NONFINITE;
            break;
        }
        const double alpha = gamma / pap;
        const float af = (float)alpha, bf = (float)beta;
        // ---- update, and the next z = D^-1 r into the block's table and the global copy ----
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t l = group + k * stride;
            if (l >= cnt) continue;
            const Sym<float> Di = load_sym(a.Dinv, n, gid[k]);
            const float4 z4 = sZ[l];
            const float zc[3] = {z4.x, z4.y, z4.z};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                p[k][c] = fmaf(bf, p[k][c], zc[c]);
                s[k][c] = fmaf(bf, s[k][c], w[k][c]);
                x[k][c] = fmaf(af, p[k][c], x[k][c]);
                r[k][c] = fmaf(-af, s[k][c], r[k][c]);
            }
            if (half == 0) {
                const F3 z = smul(Di, F3{r[k][0], r[k][1], r[k][2]});
                const float4 zn = make_float4(z.x, z.y, z.z, 0.f);
                sZ[l] = zn;
                a.zg[gid[k]] = zn;
            }
        }
        its += 1;
        gamma_old = gamma;
        alpha_old = alpha;
        first = false;
    }
    if (*(volatile int32_t*)a.err) status = VX_TIMEOUT;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const uint32_t l = group + k * stride;
        if (l >= cnt || half != 0) continue;
        const size_t g = gid[k];
        a.x[g] = x[k][0], a.x[n + g] = x[k][1], a.x[2 * (size_t)n + g] = x[k][2];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        PcgScalars* sc = a.sc;
        sc->iterations = its;
        sc->residual = residual;
        sc->initial = initial;
        sc->status = status;
        sc->done = 1;
    }
}

template <int R, int TPR>
cudaError_t launch_r(const BrickArgs& a, unsigned G, size_t smem, cudaStream_t st) {
    cudaError_t e =
        cudaFuncSetAttribute(k_pcg_brick<R, TPR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    BrickArgs args = a;
    void* params[] = {&args};
    return cudaLaunchCooperativeKernel((void*)k_pcg_brick<R, TPR>, dim3(G), dim3(kBThreads), params, smem, st);
}

// Morton key of a cell (21 bits per axis, offsets from the scene's lowest cell).
uint64_t spread3(uint64_t v) {
    v &= 0x1FFFFFull;
    v = (v | v << 32) & 0x1F00000000FFFFull;
    v = (v | v << 16) & 0x1F0000FF0000FFull;
    v = (v | v << 8) & 0x100F00F00F00F00Full;
    v = (v | v << 4) & 0x10C30C30C30C30C3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
}

}  // namespace

// The brick plan's tables, built on the host: one byte image holding, at the
// offsets below, info[G], own[G][cap], ref[G][3][cap], hzg[G][hz_cap],
// hke[G][hk_cap], nbk[G][32] and pub[G].
struct BrickTables {
    unsigned G = 0;
    uint32_t cap = 0;
    size_t hz_cap = 0, hk_cap = 0, smem = 0;
    size_t o_info = 0, o_own = 0, o_ref = 0, o_hz = 0, o_hk = 0, o_nb = 0, o_pub = 0;
    std::vector<unsigned char> image;
};

// Builds the tables from the creation positions' lattice cells (f32, [3][n])
// and the bond tables nbr/rev ([3][n], VX_EMPTY for none): at most max_blocks
// blocks of at least min_per_block REVs each (the last one excepted). Returns
// false when a block's tables would not fit `max_smem` bytes of shared memory,
// a block borders more than 32 others, or a block would own more than four
// REVs per group of `tpr` threads.
bool brick_tables(uint32_t n, unsigned max_blocks, unsigned min_per_block, unsigned tpr, size_t max_smem,
                  const float* rest, const uint32_t* nbr, const uint32_t* rev, BrickTables* out) {
    if (n == 0 || min_per_block == 0 || (tpr != 1 && tpr != 2)) return false;
    unsigned G = max_blocks;
    const unsigned min_blocks = (n + min_per_block - 1) / min_per_block;
    if (min_blocks < G) G = min_blocks;
    if (G == 0) G = 1;
    const uint32_t cap = (n + G - 1) / G;
    if (cap > 4u * kBThreads / tpr) return false;
    G = (n + cap - 1) / cap;  // no empty block
    const size_t m = 3 * (size_t)n;

    // lattice cells of the creation positions and their Morton order; a cell
    // estimate that is off only costs locality, never correctness
    std::vector<long long> cell(m);
    long long lo[3] = {0, 0, 0};
    for (int c = 0; c < 3; ++c) {
        for (uint32_t i = 0; i < n; ++i) {
            const double v = (double)rest[(size_t)c * n + i] / kCell;
            cell[(size_t)c * n + i] = std::isfinite(v) && std::fabs(v) < 1e15 ? (long long)std::llround(v) : 0;
        }
        lo[c] = *std::min_element(cell.begin() + (size_t)c * n, cell.begin() + (size_t)(c + 1) * n);
    }
    std::vector<std::pair<uint64_t, uint32_t>> key(n);
    for (uint32_t i = 0; i < n; ++i) {
        uint64_t k = 0;
        for (int c = 0; c < 3; ++c) k |= spread3((uint64_t)(cell[(size_t)c * n + i] - lo[c])) << c;
        key[i] = {k, i};
    }
    std::sort(key.begin(), key.end());
    std::vector<uint32_t> block_of(n), local_of(n);
    for (uint32_t t = 0; t < n; ++t) {
        block_of[key[t].second] = t / cap;
        local_of[key[t].second] = t % cap;
    }

    // per block: refs, halo slots (incoming bonds first, with their K), neighbour blocks
    std::vector<uint32_t> own((size_t)G * cap, 0), ref((size_t)G * 3 * cap, 0xFFFFFFFFu);
    std::vector<std::vector<uint32_t>> hz(G), hk(G), nb(G);
    std::vector<uint32_t> zslot_stamp(n, 0xFFFFFFFFu), zslot(n, 0);
    std::vector<uint32_t> kslot_stamp(m, 0xFFFFFFFFu), kslot(m, 0);
    std::vector<uint32_t> blk_stamp(G, 0xFFFFFFFFu);
    std::vector<uint4> info(G);
    for (unsigned b = 0; b < G; ++b) {
        const uint32_t base = b * cap, cnt = std::min(cap, n - base);
        for (uint32_t l = 0; l < cnt; ++l) own[(size_t)b * cap + l] = key[base + l].second;
        auto note_block = [&](uint32_t j) {
            const uint32_t q = block_of[j];
            if (blk_stamp[q] != b) {
                blk_stamp[q] = b;
                nb[b].push_back(q);
            }
        };
        // incoming bonds of remote -axis neighbours: one halo slot per bond
        for (uint32_t l = 0; l < cnt; ++l) {
            const uint32_t g = own[(size_t)b * cap + l];
            for (int ax = 0; ax < 3; ++ax) {
                const uint32_t j = rev[(size_t)ax * n + g];
                if (j == VX_EMPTY_U32 || j >= n || block_of[j] == b) continue;
                const size_t e = (size_t)ax * n + j;
                if (kslot_stamp[e] == b) continue;
                kslot_stamp[e] = b;
                kslot[e] = (uint32_t)hk[b].size();
                hk[b].push_back((uint32_t)e);
                hz[b].push_back(j);
                if (zslot_stamp[j] != b) {
                    zslot_stamp[j] = b;
                    zslot[j] = kslot[e];
                }
                note_block(j);
            }
        }
        // remote +axis neighbours: one z slot per REV, shared with an incoming slot of it
        for (uint32_t l = 0; l < cnt; ++l) {
            const uint32_t g = own[(size_t)b * cap + l];
            for (int ax = 0; ax < 3; ++ax) {
                const uint32_t j = nbr[(size_t)ax * n + g];
                if (j == VX_EMPTY_U32 || j >= n || block_of[j] == b || zslot_stamp[j] == b) continue;
                zslot_stamp[j] = b;
                zslot[j] = (uint32_t)hz[b].size();
                hz[b].push_back(j);
                note_block(j);
            }
        }
        if (nb[b].size() > (size_t)kMaxNeighbourBlocks || cnt + hz[b].size() >= kNoRef) return false;
        for (uint32_t l = 0; l < cnt; ++l) {
            const uint32_t g = own[(size_t)b * cap + l];
            uint32_t r16[6];
            for (int t = 0; t < 6; ++t) {
                const int ax = t < 3 ? t : t - 3;
                const uint32_t j = t < 3 ? nbr[(size_t)ax * n + g] : rev[(size_t)ax * n + g];
                if (j == VX_EMPTY_U32 || j >= n) r16[t] = kNoRef;
                else if (block_of[j] == b) r16[t] = local_of[j];
                else if (t >= 3) r16[t] = cnt + kslot[(size_t)ax * n + j];
                else r16[t] = cnt + zslot[j];
            }
            for (int wd = 0; wd < 3; ++wd)
                ref[((size_t)b * 3 + wd) * cap + l] = r16[2 * wd] | (r16[2 * wd + 1] << 16);
        }
        info[b] = make_uint4(cnt, (uint32_t)hz[b].size(), (uint32_t)hk[b].size(), (uint32_t)nb[b].size());
    }
    size_t hz_cap = 1, hk_cap = 1;
    for (unsigned b = 0; b < G; ++b) {
        hz_cap = std::max(hz_cap, hz[b].size());
        hk_cap = std::max(hk_cap, hk[b].size());
    }
    const size_t smem = (kOwnBytes * cap + kHaloZBytes * hz_cap + kHaloKBytes * hk_cap + 15) & ~size_t(15);
    if (smem > max_smem) return false;

    BrickTables& T = *out;
    auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
    T.G = G;
    T.cap = cap;
    T.hz_cap = hz_cap;
    T.hk_cap = hk_cap;
    T.smem = smem;
    T.o_info = 0;
    T.o_own = al(T.o_info + G * sizeof(uint4));
    T.o_ref = al(T.o_own + (size_t)G * cap * 4);
    T.o_hz = al(T.o_ref + (size_t)G * 3 * cap * 4);
    T.o_hk = al(T.o_hz + (size_t)G * hz_cap * 4);
    T.o_nb = al(T.o_hk + (size_t)G * hk_cap * 4);
    T.o_pub = al(T.o_nb + (size_t)G * kMaxNeighbourBlocks * 4);
    T.image.assign(al(T.o_pub + (size_t)G * 4), 0);
    unsigned char* img = T.image.data();
    std::memcpy(img + T.o_info, info.data(), G * sizeof(uint4));
    std::memcpy(img + T.o_own, own.data(), own.size() * 4);
    std::memcpy(img + T.o_ref, ref.data(), ref.size() * 4);
    for (unsigned b = 0; b < G; ++b) {
        std::memcpy(img + T.o_hz + (size_t)b * hz_cap * 4, hz[b].data(), hz[b].size() * 4);
        std::memcpy(img + T.o_hk + (size_t)b * hk_cap * 4, hk[b].data(), hk[b].size() * 4);
        std::memcpy(img + T.o_nb + (size_t)b * kMaxNeighbourBlocks * 4, nb[b].data(), nb[b].size() * 4);
    }
    return true;
}

// Builds and uploads the brick plan of a scene in the given form
// (VX_PERSIST_BRICK_*) from its creation positions and current bond tables.
// Returns false (no plan) when brick_tables declines or the device does not
// take cooperative launches.
bool brick_plan(vx_scene* s, int form) {
    s->brick_ok = false;
    if (s->brick_buf) {
        cudaStreamSynchronize(s->stream);
        cudaFree(s->brick_buf);
        s->brick_buf = nullptr;
    }
    const uint32_t n = s->n;
    if (n == 0) return false;
    int dev = s->device, max_smem = 0, coop = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop || max_smem < 4096) return false;
    const size_t m = 3 * (size_t)n;
    std::vector<float> rest(m);
    std::vector<uint32_t> nbr(m), rev(m);
    if (cudaMemcpyAsync(rest.data(), s->rest, m * sizeof(float), cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
        cudaMemcpyAsync(nbr.data(), s->nbr, m * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
        cudaMemcpyAsync(rev.data(), s->rev, m * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
        cudaStreamSynchronize(s->stream) != cudaSuccess)
        return false;
    const unsigned min_per_block = (form == VX_PERSIST_BRICK_T1_128 || form == VX_PERSIST_BRICK_T2_128) ? 128 : 256;
    const unsigned tpr = (form == VX_PERSIST_BRICK_T2_256 || form == VX_PERSIST_BRICK_T2_128) ? 2 : 1;
    BrickTables T;
    // the kernel's static shared memory (reduction slots) takes the last 2 KB
    if (!brick_tables(n, (unsigned)s->sm_count, min_per_block, tpr, (size_t)max_smem - 2048, rest.data(), nbr.data(),
                      rev.data(), &T))
        return false;
    // after the tables, the grid reductions' partials: 3 per block (the scene's
    // own partials array is sized for blocks of at least 256 REVs)
    const size_t part_bytes = ((size_t)3 * T.G * sizeof(double) + 255) & ~size_t(255);
    void* buf = nullptr;
    if (cudaMalloc(&buf, T.image.size() + part_bytes) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    if (cudaMemcpy(buf, T.image.data(), T.image.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(buf);
        return false;
    }
    char* B = static_cast<char*>(buf);
    s->brick_buf = buf;
    s->brick_info = reinterpret_cast<uint4*>(B + T.o_info);
    s->brick_own = reinterpret_cast<uint32_t*>(B + T.o_own);
    s->brick_ref = reinterpret_cast<uint32_t*>(B + T.o_ref);
    s->brick_hzg = reinterpret_cast<uint32_t*>(B + T.o_hz);
    s->brick_hke = reinterpret_cast<uint32_t*>(B + T.o_hk);
    s->brick_nbk = reinterpret_cast<uint32_t*>(B + T.o_nb);
    s->brick_pub = reinterpret_cast<uint32_t*>(B + T.o_pub);
    s->brick_part = reinterpret_cast<double*>(B + T.image.size());
    s->brick_G = T.G;
    s->brick_cap = T.cap;
    s->brick_hz = (unsigned)T.hz_cap;
    s->brick_hk = (unsigned)T.hk_cap;
    const uint32_t groups = kBThreads / tpr;
    s->brick_tpr = tpr;
    s->brick_R = T.cap <= groups ? 1 : (T.cap <= 2u * groups ? 2 : 4);
    s->brick_smem = T.smem;
    s->brick_ok = true;
    return true;
}

// One FP32 inner solve A32 d = r64 / |r64| with the brick plan.
int32_t solve_inner_brick(vx_scene* s, double tolerance, uint32_t max_iterations) {
    BrickArgs a;
    a.n = s->n;
    a.cap = s->brick_cap;
    a.hz_cap = s->brick_hz;
    a.hk_cap = s->brick_hk;
    a.kn = kstride32(s->n);
    a.info = s->brick_info;
    a.own = s->brick_own;
    a.ref = s->brick_ref;
    a.hzg = s->brick_hzg;
    a.hke = s->brick_hke;
    a.nbk = s->brick_nbk;
    a.pub = s->brick_pub;
    a.flags = s->flags;
    a.mh2 = s->mh2_32;
    a.K = s->bonds.k32;
    a.Dinv = s->dinv32;
    a.src = s->r64;
    a.scale_from = &s->sc->r64_norm;
    a.x = s->x32;
    a.zg = reinterpret_cast<float4*>(s->zp32);
    a.part = s->brick_part;
    a.count = reinterpret_cast<unsigned long long*>(s->barrier);
    a.err = reinterpret_cast<int32_t*>(s->barrier + 2);
    a.sc = s->sc32;
    a.tolerance = tolerance;
    a.max_iterations = max_iterations;
    a.spin_limit = 4000000ull;  // ~1-2 s of polling at one wait
    // VXCOROT_BARRIER_SPINS lowers the bound so a test can make a wait run out
    if (const char* v = std::getenv("VXCOROT_BARRIER_SPINS")) {
        unsigned long long lim = std::strtoull(v, nullptr, 10);
        if (lim > 0 && lim < a.spin_limit) a.spin_limit = lim;
    }
    cudaError_t e = cudaMemsetAsync(s->barrier, 0, 4 * sizeof(unsigned), s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->brick_pub, 0, s->brick_G * sizeof(uint32_t), s->stream);
    if (e == cudaSuccess) {
        const unsigned key = s->brick_R * 4 + s->brick_tpr;
        switch (key) {
            case 1 * 4 + 1: e = launch_r<1, 1>(a, s->brick_G, s->brick_smem, s->stream); break;
            case 2 * 4 + 1: e = launch_r<2, 1>(a, s->brick_G, s->brick_smem, s->stream); break;
            case 4 * 4 + 1: e = launch_r<4, 1>(a, s->brick_G, s->brick_smem, s->stream); break;
            case 1 * 4 + 2: e = launch_r<1, 2>(a, s->brick_G, s->brick_smem, s->stream); break;
            case 2 * 4 + 2: e = launch_r<2, 2>(a, s->brick_G, s->brick_smem, s->stream); break;
            default: e = launch_r<4, 2>(a, s->brick_G, s->brick_smem, s->stream); break;
        }
    }
    s->launches += 1;
    if (e != cudaSuccess) {
        set_error("persistent (brick) PCG launch failed: %s", cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    return VX_OK;
}

}  // namespace vx

// vx_expanded.cu — the FP32 inner PCG solve as one persistent kernel with ONE
// grid reduction per iteration (the contiguous-range plan of vx_persistent.cu,
// with the next r.z expanded from the current iteration's vectors).
//
// The classic recurrence (src/solver.rs:1857-1911) needs two grid-wide sums per
// iteration: p.Ap for alpha, then r.z of the updated residual for beta. With
// q = A p, u = D^-1 r and v = D^-1 q, the updated quantities are
//   r' = r - alpha q,   z' = D^-1 r' = u - alpha v,
//   r'.z' = r.u - alpha (r.v + q.u) + alpha^2 q.v,
//   r'.r' = r.r - 2 alpha r.q + alpha^2 q.q,
// so one reduction of (r.u, p.q, r.v + q.u, q.v, r.r, r.q, q.q) gives alpha,
// the next beta and the residual norm together. Each REV's dot products are
// formed in FP32 and summed in FP64, as in the classic loop; r.u is the direct
// value every iteration, so the expansion's rounding does not accumulate
// across iterations. An FP32 CPU emulation of both recurrences takes the same
// iteration counts on mixed blocks of 8^3 to 48^3, a damaged lattice and a
// box union, and the iterates agree to 1e-6
// (tests/test_oracle_expanded_recurrence.py keeps three of those cases).
//
// The next direction p' = z' + beta' p of a neighbour must be formed without a
// second grid barrier, so each block publishes, BEFORE the reduction, the
// triple (u, v, p) of its REVs; the reduction is also the barrier that makes
// the triples visible. Every block, owner or neighbour, then forms
//   z' = fmaf(-alpha, v, u),   p' = fmaf(beta', p, z')
// from the same published bits, so all copies of p' agree bit for bit (a
// block forms its own REVs' p' once, into the p slots of its shared-memory
// triples, where its in-range neighbours read it). The triples are
// double-buffered in global memory by iteration parity: a block writes buffer
// k & 1 only after reduction k - 1, which every block reaches after its matvec
// of iteration k - 1 has read buffer (k - 2) & 1 = k & 1. The partials rows
// are double-buffered by parity for the same reason.
//
// Shared memory per REV of the block's range: the stiffness of its three
// owned bonds (72 B), its triple (36 B: float4 (u, v.x), float4 (v.y, v.z,
// p.x, p.y), float p.z), its six int16 neighbour deltas (12 B), m/h^2 (4 B)
// and the free-axis flags (1 B): 125 B, 1,772 REVs in 221 KB at 64^3.
//
// Compiled with MULTI the same kernel runs a pool's persistent waves
// (solve_inner_slots_expanded): a wave's blocks serve several slots, each slot
// summed over its own blocks, with the grid's count of working blocks as an
// eighth row of the one reduction.
#include <cstdlib>
#include <cstring>

#include "vx_device.cuh"
#include "vx_kernels.h"
#include "vx_grid.cuh"
#include "vx_layout.cuh"

namespace vx {

namespace {

constexpr int kEThreads = 512;
constexpr int kEBytesPerRev = 3 * 16 + 3 * 8 + 16 + 16 + 4 + 12 + 4 + 1;
constexpr int kENV = 7;  // values summed per iteration
constexpr int kEW = 8;   // partials rows per parity: the seven sums and, in pools, the working-block count

struct ExpArgs {
    uint32_t n;
    uint32_t cap;  // REVs per block (contiguous range)
    uint32_t kn;   // REV stride of the per-axis K arrays
    const uint8_t* flags;
    const float* mh2;           // m/h^2 [n]
    const float* K;
    const float* Dinv;
    const uint32_t* code;       // [3][n] neighbour deltas
    const double* src;          // right-hand side in FP64
    const double* scale_from;   // |src|; r0 = src / |src|
    float* x;                   // correction [3][n]
    float4* pa;                 // [2][n] published (u.x, u.y, u.z, v.x)
    float4* pb;                 // [2][n] published (v.y, v.z, p.x, p.y)
    float* pc;                  // [2][n] published p.z
    double* part;               // [2 * kEW][G] partials, two parities
    unsigned long long* count;  // arrivals at the grid reductions so far
    int32_t* err;               // a wait ran out
    PcgScalars* sc;
    double tolerance;
    uint32_t max_iterations;
    unsigned long long spin_limit;
    // pools: one row per block (first REV, REV count, slot, first block of the
    // slot << 16 | blocks of the slot) and the slots' states; null for one scene
    const uint4* blocks;
    SlotState* st;
};

struct E3 {
    float x, y, z;
};
__device__ __forceinline__ E3 emul(const Sym<float>& s, E3 v) {
    return {s.xx * v.x + s.xy * v.y + s.xz * v.z, s.xy * v.x + s.yy * v.y + s.yz * v.z,
            s.xz * v.x + s.yz * v.y + s.zz * v.z};
}
__device__ __forceinline__ Sym<float> esym(float4 a, float2 b) { return {a.x, a.y, a.z, a.w, b.x, b.y}; }
__device__ __forceinline__ float fdot(E3 a, E3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// p' = z' + beta' p with z' = u - alpha v, from a published triple
__device__ __forceinline__ E3 next_dir(float4 A, float4 B, float C, float alpha, float beta) {
    const float zx = fmaf(-alpha, A.w, A.x), zy = fmaf(-alpha, B.x, A.y), zz = fmaf(-alpha, B.y, A.z);
    return {fmaf(beta, B.z, zx), fmaf(beta, B.w, zy), fmaf(beta, C, zz)};
}

// R REVs per thread. With R <= 2 the inverse diagonal block is loaded into
// registers before the matvec, so its L2 latency overlaps the neighbour loads;
// at R = 4 the four loads are issued together after the matvec.
// MULTI: the blocks work for several pool slots (a.blocks, a.st), each slot's
// sums taken over its own blocks in block order, so a slot's bits do not
// depend on the slots beside it; a slot that has stopped leaves its blocks
// idle, and every block leaves at the reduction where no block has work left.
template <int R, bool MULTI>
__global__ void __launch_bounds__(kEThreads, 1) k_pcg_expanded(ExpArgs a) {
    constexpr bool kPrefetch = R <= 2;
    extern __shared__ float4 smem4[];
    __shared__ double red[kENV][32];
    __shared__ double tot[kENV + 1];
    __shared__ int s_ok;
    const uint32_t n = a.n, cap = a.cap, T = blockDim.x;
    float4* sK4 = smem4;                                      // [3][cap] owned bonds (xx, yy, zz, xy)
    float4* sPA = sK4 + 3 * cap;                              // [cap] (u, v.x)
    float4* sPB = sPA + cap;                                  // [cap] (v.y, v.z, p.x, p.y)
    float2* sK2 = reinterpret_cast<float2*>(sPB + cap);       // [3][cap] (xz, yz)
    float* sPC = reinterpret_cast<float*>(sK2 + 3 * cap);     // [cap] p.z
    uint32_t* sNB = reinterpret_cast<uint32_t*>(sPC + cap);   // [3][cap] neighbour deltas
    float* sM = reinterpret_cast<float*>(sNB + 3 * cap);      // [cap] m/h^2
    uint8_t* sFL = reinterpret_cast<uint8_t*>(sM + cap);      // [cap] free-axis flags
    // the (p.x, p.y) halves of the sPB records: record li at [2 li]
    const float2* sPBzw = reinterpret_cast<const float2*>(sPB) + 1;
    // this block's range and problem: the whole grid for one scene, or one
    // slot's blocks in a pool (its own target, iteration cap and outcome)
    uint32_t lo, cnt, slot = 0, fb = 0, nb = gridDim.x;
    double scale_norm, tolerance;
    uint32_t max_iterations;
    bool mine = true;  // this block's problem still iterates
    if constexpr (MULTI) {
        const uint4 bi = a.blocks[blockIdx.x];
        lo = bi.x, cnt = bi.y, slot = bi.z, fb = bi.w >> 16, nb = bi.w & 0xFFFFu;
        const SlotState& S = a.st[slot];
        mine = S.enabled && S.inner_on;
        scale_norm = S.r64_norm, tolerance = S.tol_in, max_iterations = S.max_its;
        if (!mine) cnt = 0;
    } else {
        lo = blockIdx.x * cap;
        cnt = lo < n ? (n - lo < cap ? n - lo : cap) : 0;
        scale_norm = *a.scale_from, tolerance = a.tolerance, max_iterations = a.max_iterations;
    }
    constexpr int W = MULTI ? kEW : kENV;  // partials rows per parity

    for (uint32_t li = threadIdx.x; li < cnt; li += T) {
        const size_t i = lo + li;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            const float* kb = a.K + (size_t)ax * 6 * a.kn;
            sK4[ax * cap + li] = __ldg(reinterpret_cast<const float4*>(kb) + i);
            sK2[ax * cap + li] = __ldg(reinterpret_cast<const float2*>(kb + 4 * (size_t)a.kn) + i);
            sNB[ax * cap + li] = __ldg(a.code + (size_t)ax * n + i);
        }
        sM[li] = __ldg(a.mh2 + i);
        sFL[li] = __ldg(a.flags + i);
    }

    // r0 = src / |src|; the triple of "iteration -1" is (u0, 0, 0) with
    // alpha = beta = 0, so every block's first direction is p0 = u0 = D^-1 r0.
    // It goes to parity 1, which the matvec of iteration 0 reads.
    float x[R][3], r[R][3], q[R][3];
    E3 pown[R];
    Sym<float> ireg[kPrefetch ? R : 1];
    const double scale = scale_norm > 0.0 ? 1.0 / scale_norm : 1.0;
    double acc[2] = {0.0, 0.0};
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const uint32_t li = threadIdx.x + k * T;
#pragma unroll
        for (int c = 0; c < 3; ++c) x[k][c] = r[k][c] = q[k][c] = 0.f;
        pown[k] = {0.f, 0.f, 0.f};
        if (li < cnt) {
            const size_t i = lo + li;
            const E3 rr = {(float)(a.src[i] * scale), (float)(a.src[n + i] * scale),
                           (float)(a.src[2 * (size_t)n + i] * scale)};
            const E3 u = emul(load_sym(a.Dinv, n, i), rr);
            r[k][0] = rr.x, r[k][1] = rr.y, r[k][2] = rr.z;
            const float4 A = make_float4(u.x, u.y, u.z, 0.f);
            const float4 B = make_float4(0.f, 0.f, 0.f, 0.f);
            sPA[li] = A, sPB[li] = B, sPC[li] = 0.f;
            a.pa[n + i] = A, a.pb[n + i] = B, a.pc[n + i] = 0.f;
            acc[0] += (double)fdot(rr, rr);
            acc[1] += (double)fdot(rr, u);
        }
    }
    unsigned long long seq = 1;
    double t[kENV];
    bool alive;
    double act = 0.0;
    {
        const int sl[2] = {W, W + 1};  // parity-1 rows: iteration 0 sums into parity 0
        double t0[2];
        if constexpr (MULTI) alive = grid_reduce_ranged<2>(acc, 0.0, sl, -1, a, seq++, fb, nb, red, tot, &s_ok, t0, &act);
        else alive = grid_reduce<2>(acc, sl, a, seq++, red, tot, &s_ok, t0);
        t[0] = t0[0], t[1] = t0[1];
    }
    const double initial = sqrt(t[0]);
    double residual = 0.0;
    uint32_t its = 0;
    int32_t status = alive ? VX_OK : VX_TIMEOUT;
    if (alive && mine) {
        if (!isfinite(t[0]) || !isfinite(t[1])) {
            mine = false;
            status = VX_NONFINITE;
        } else if (!(initial > 1e-12)) {
            mine = false;
        } else if (max_iterations == 0) {
            mine = false;
            status = VX_NOT_CONVERGED;
        }
    }

    float alpha_prev = 0.f, beta = 0.f;
    uint32_t loop = 0;  // iterations of the loop, the same in every block
    while (alive) {
        if (!MULTI && !mine) break;
        const uint32_t cnt_now = mine ? cnt : 0;
        const uint32_t par = loop & 1u;  // this iteration writes parity par, reads par ^ 1
        const float4* gA = a.pa + (size_t)(par ^ 1u) * n;
        const float4* gB = a.pb + (size_t)(par ^ 1u) * n;
        const float* gC = a.pc + (size_t)(par ^ 1u) * n;
        if constexpr (kPrefetch) {
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const uint32_t li = threadIdx.x + k * T;
                if (li < cnt_now) ireg[k] = load_sym(a.Dinv, n, lo + li);
            }
        }
        // ---- the block's own directions p = z + beta p_old, formed once from
        //      the own triples and kept in the triples' p slots ----
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t li = threadIdx.x + k * T;
            if (li >= cnt_now) continue;
            const float4 B = sPB[li];
            const E3 pi = next_dir(sPA[li], B, sPC[li], alpha_prev, beta);
            sPB[li] = make_float4(B.x, B.y, pi.x, pi.y);
            sPC[li] = pi.z;
        }
        __syncthreads();
        // ---- matvec: q = P (m/h^2 p + sum K (p - p_nbr)) + (I - P) p; a
        //      neighbour in another block forms its p from its published triple ----
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t li = threadIdx.x + k * T;
            if (li >= cnt_now) continue;
            const uint32_t i = lo + li;
            int32_t dl[6];
#pragma unroll
            for (int w = 0; w < 3; ++w) {
                const uint32_t c = sNB[w * cap + li];
                dl[2 * w] = (int32_t)(int16_t)(c & 0xffffu);
                dl[2 * w + 1] = (int32_t)(int16_t)(c >> 16);
            }
            const uint8_t fl = sFL[li];
            const float2 pxy = sPBzw[2 * li];
            const E3 pi = {pxy.x, pxy.y, sPC[li]};
            const float mh = sM[li];
            E3 s = {mh * pi.x, mh * pi.y, mh * pi.z};
#pragma unroll
            for (int tt = 0; tt < 6; ++tt) {
                const uint32_t j = (uint32_t)((int32_t)i + dl[tt]);
                const int ax = tt < 3 ? tt : tt - 3;
                const uint32_t lj = j - lo;
                const bool inb = lj < cnt;
                E3 pn;
                Sym<float> Kb;
                if (inb) {
                    const float2 nxy = sPBzw[2 * lj];
                    pn = {nxy.x, nxy.y, sPC[lj]};
                } else {
                    pn = next_dir(__ldcg(gA + j), __ldcg(gB + j), __ldcg(gC + j), alpha_prev, beta);
                }
                if (tt < 3) Kb = esym(sK4[ax * cap + li], sK2[ax * cap + li]);
                else if (inb) Kb = esym(sK4[ax * cap + lj], sK2[ax * cap + lj]);
                else Kb = load_sym(a.K + (size_t)ax * 6 * a.kn, a.kn, j);
                // a missing neighbour has delta 0: j = i, pn = pi and the term is 0
                const E3 d = {pi.x - pn.x, pi.y - pn.y, pi.z - pn.z};
                const E3 kv = emul(Kb, d);
                s.x += kv.x, s.y += kv.y, s.z += kv.z;
            }
            q[k][0] = (fl & 1) ? s.x : pi.x;
            q[k][1] = (fl & 2) ? s.y : pi.y;
            q[k][2] = (fl & 4) ? s.z : pi.z;
            pown[k] = pi;
        }
        __syncthreads();  // every thread has read the previous triples in shared memory
        // ---- publish (u, v, p) and form the seven partials ----
        double d[kENV];
#pragma unroll
        for (int c = 0; c < kENV; ++c) d[c] = 0.0;
        Sym<float> Dk[kPrefetch ? 1 : R];
        if constexpr (!kPrefetch) {
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const uint32_t li = threadIdx.x + k * T;
                if (li < cnt_now) Dk[k] = load_sym(a.Dinv, n, lo + li);
            }
        }
        float4* wA = a.pa + (size_t)par * n;
        float4* wB = a.pb + (size_t)par * n;
        float* wC = a.pc + (size_t)par * n;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t li = threadIdx.x + k * T;
            if (li >= cnt_now) continue;
            const size_t i = lo + li;
            Sym<float> Di;
            if constexpr (kPrefetch) Di = ireg[k];
            else Di = Dk[k];
            const E3 rr = {r[k][0], r[k][1], r[k][2]};
            const E3 qq = {q[k][0], q[k][1], q[k][2]};
            const E3 pp = pown[k];
            const E3 u = emul(Di, rr);
            const E3 v = emul(Di, qq);
            const float4 A = make_float4(u.x, u.y, u.z, v.x);
            const float4 B = make_float4(v.y, v.z, pp.x, pp.y);
            sPA[li] = A, sPB[li] = B, sPC[li] = pp.z;
            wA[i] = A, wB[i] = B, wC[i] = pp.z;
            d[0] += (double)fdot(rr, u);
            d[1] += (double)fdot(pp, qq);
            d[2] += (double)fdot(rr, v) + (double)fdot(qq, u);
            d[3] += (double)fdot(qq, v);
            d[4] += (double)fdot(rr, rr);
            d[5] += (double)fdot(rr, qq);
            d[6] += (double)fdot(qq, qq);
        }
        int sl[kENV];
#pragma unroll
        for (int c = 0; c < kENV; ++c) sl[c] = c + W * (int)par;
        bool ok;
        if constexpr (MULTI)
            ok = grid_reduce_ranged<kENV>(d, mine ? 1.0 : 0.0, sl, W * (int)par + kENV, a, seq++, fb, nb, red, tot,
                                          &s_ok, t, &act);
        else
            ok = grid_reduce<kENV>(d, sl, a, seq++, red, tot, &s_ok, t);
        if (!ok) {
            status = VX_TIMEOUT;
            break;
        }
        if (MULTI && act == 0.0) break;  // no block of the grid has work left
        ++loop;
        if (!mine) continue;
        const double g = t[0], pq = t[1];
        if (!isfinite(g) || !isfinite(pq) || pq <= 1e-30) {
            its += 1;  // the matvec happened (src/solver.rs:1861-1866)
            if (!isfinite(g) || !isfinite(pq)) status = VX_NONFINITE;
            mine = false;
            continue;
        }
        const float alpha = (float)(g / pq);
        const double al = (double)alpha;  // the vectors move by the FP32 alpha
        const double g_next = g - al * t[2] + al * al * t[3];
        const double rr_next = t[4] - 2.0 * al * t[5] + al * al * t[6];
        // ---- update: x += alpha p, r -= alpha q ----
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t li = threadIdx.x + k * T;
            if (li >= cnt_now) continue;
            x[k][0] = fmaf(alpha, pown[k].x, x[k][0]);
            x[k][1] = fmaf(alpha, pown[k].y, x[k][1]);
            x[k][2] = fmaf(alpha, pown[k].z, x[k][2]);
#pragma unroll
            for (int c = 0; c < 3; ++c) r[k][c] = fmaf(-alpha, q[k][c], r[k][c]);
        }
        its += 1;
        residual = sqrt(fmax(rr_next, 0.0)) / initial;
        if (!isfinite(g_next) || !isfinite(rr_next)) {
            status = VX_NONFINITE;
            mine = false;
        } else if (residual < tolerance) {
            mine = false;
        } else if (its >= max_iterations) {
            status = VX_NOT_CONVERGED;
            mine = false;
        }
        beta = (float)(g_next / g);
        alpha_prev = alpha;
    }
    if (*(volatile int32_t*)a.err) status = VX_TIMEOUT;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const uint32_t li = threadIdx.x + k * T;
        if (li >= cnt) continue;
        const size_t i = lo + li;
        a.x[i] = x[k][0], a.x[n + i] = x[k][1], a.x[2 * (size_t)n + i] = x[k][2];
    }
    if (threadIdx.x == 0 && blockIdx.x == fb) {
        if constexpr (MULTI) {
            SlotState& S = a.st[slot];
            if (S.enabled && S.inner_on) {
                S.its = its;
                S.residual_in = residual;
                S.initial = initial;
                S.status_in = status;
                S.done = 1;
            }
        } else {
            PcgScalars* sc = a.sc;
            sc->iterations = its;
            sc->residual = residual;
            sc->initial = initial;
            sc->status = status;
            sc->done = 1;
        }
    }
}

template <int R, bool MULTI>
cudaError_t launch_e(const ExpArgs& a, unsigned G, size_t smem, cudaStream_t st) {
    cudaError_t e =
        cudaFuncSetAttribute(k_pcg_expanded<R, MULTI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    ExpArgs args = a;
    void* params[] = {&args};
    return cudaLaunchCooperativeKernel((void*)k_pcg_expanded<R, MULTI>, dim3(G), dim3(kEThreads), params, smem, st);
}

}  // namespace

// The published triples (two parities) and the partials (two parities of kEW
// rows for up to one block per SM): one device allocation, kept until the
// scene is released or re-planned.
static bool exp_buffers(vx_scene* s) {
    if (s->exp_buf) return true;
    const size_t n = s->n, G = (size_t)(s->sm_count > 0 ? s->sm_count : 1);
    const size_t o_b = 2 * n * sizeof(float4);
    const size_t o_c = o_b + 2 * n * sizeof(float4);
    const size_t o_p = (o_c + 2 * n * sizeof(float) + 255) & ~size_t(255);
    const size_t bytes = o_p + 2 * (size_t)kEW * G * sizeof(double);
    void* buf = nullptr;
    if (cudaMalloc(&buf, bytes) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    char* B = static_cast<char*>(buf);
    s->exp_buf = buf;
    s->exp_pa = reinterpret_cast<float4*>(B);
    s->exp_pb = reinterpret_cast<float4*>(B + o_b);
    s->exp_pc = reinterpret_cast<float*>(B + o_c);
    s->exp_part = reinterpret_cast<double*>(B + o_p);
    return true;
}

// The plan: block b owns REVs [b cap, (b + 1) cap), as in the range plan, with
// 125 B of shared memory per REV; the published triples (two parities) and
// the partials (two parities) get one device allocation of their own.
bool expanded_plan(vx_scene* s) {
    s->exp_ok = false;
    if (s->exp_buf) {
        cudaStreamSynchronize(s->stream);
        cudaFree(s->exp_buf);
        s->exp_buf = nullptr;
    }
    const uint32_t n = s->n;
    if (n == 0 || !neighbor_deltas_fit(s)) return false;
    int dev = s->device, max_smem = 0, coop = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop) return false;
    unsigned G = (unsigned)s->sm_count;
    const unsigned min_blocks = (n + 255) / 256;  // at least 256 REVs per block
    if (min_blocks < G) G = min_blocks;
    if (G == 0) G = 1;
    const unsigned cap = (n + G - 1) / G;
    const unsigned R = (cap + kEThreads - 1) / kEThreads;
    const size_t smem = ((size_t)kEBytesPerRev * cap + 15) & ~size_t(15);
    // the kernel's static shared memory (reduction slots) takes under 2 KB
    if (R > 4 || smem + 2048 > (size_t)max_smem) return false;
    if (!exp_buffers(s)) return false;
    s->exp_G = G;
    s->exp_cap = cap;
    s->exp_R = R <= 1 ? 1 : (R <= 2 ? 2 : 4);
    s->exp_smem = smem;
    s->exp_ok = true;
    return true;
}

// One FP32 inner solve A32 d = r64 / |r64| with one grid reduction per iteration.
int32_t solve_inner_expanded(vx_scene* s, double tolerance, uint32_t max_iterations) {
    ExpArgs a;
    a.n = s->n;
    a.cap = s->exp_cap;
    a.kn = kstride32(s->n);
    a.flags = s->flags;
    a.mh2 = s->mh2_32;
    a.K = s->bonds.k32;
    a.Dinv = s->dinv32;
    a.code = s->nbcode;
    a.src = s->r64;
    a.scale_from = &s->sc->r64_norm;
    a.x = s->x32;
    a.pa = s->exp_pa;
    a.pb = s->exp_pb;
    a.pc = s->exp_pc;
    a.part = s->exp_part;
    a.count = reinterpret_cast<unsigned long long*>(s->barrier);
    a.err = reinterpret_cast<int32_t*>(s->barrier + 2);
    a.sc = s->sc32;
    a.tolerance = tolerance;
    a.max_iterations = max_iterations;
    a.blocks = nullptr;
    a.st = nullptr;
    a.spin_limit = 4000000ull;  // ~1-2 s of polling at one reduction
    // VXCOROT_BARRIER_SPINS lowers the bound so a test can make the wait run out
    if (const char* v = std::getenv("VXCOROT_BARRIER_SPINS")) {
        unsigned long long lim = std::strtoull(v, nullptr, 10);
        if (lim > 0 && lim < a.spin_limit) a.spin_limit = lim;
    }
    cudaError_t e = cudaMemsetAsync(s->barrier, 0, 4 * sizeof(unsigned), s->stream);
    if (e == cudaSuccess) {
        switch (s->exp_R) {
            case 1: e = launch_e<1, false>(a, s->exp_G, s->exp_smem, s->stream); break;
            case 2: e = launch_e<2, false>(a, s->exp_G, s->exp_smem, s->stream); break;
            default: e = launch_e<4, false>(a, s->exp_G, s->exp_smem, s->stream); break;
        }
    }
    s->launches += 1;
    if (e != cudaSuccess) {
        set_error("persistent PCG launch failed: %s", cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    return VX_OK;
}

// One cooperative launch of the one-reduction inner solve over the pool slots
// of a wave (rows and slot states as solve_inner_slots in vx_persistent.cu).
// One instantiation serves every wave, so a slot's bits do not depend on the
// wave it lands in.
int32_t solve_inner_slots_expanded(vx_scene* s, const uint4* d_blocks, SlotState* st, unsigned G, uint32_t cap) {
    int dev = s->device, max_smem = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t smem = ((size_t)kEBytesPerRev * cap + 15) & ~size_t(15);
    if (cap == 0 || cap > 4u * kEThreads || G > (unsigned)s->sm_count || smem + 2048 > (size_t)max_smem) {
        set_error("persistent pool PCG: a wave of %u blocks of %u REVs does not fit", G, cap);
        return VX_BAD_INPUT;
    }
    if (!exp_buffers(s)) {
        set_error("persistent pool PCG: the published-direction buffers could not be allocated");
        return VX_CUDA_ERROR;
    }
    ExpArgs a;
    a.n = s->n;
    a.cap = cap;
    a.kn = kstride32(s->n);
    a.flags = s->flags;
    a.mh2 = s->mh2_32;
    a.K = s->bonds.k32;
    a.Dinv = s->dinv32;
    a.code = s->nbcode;
    a.src = s->r64;
    a.scale_from = nullptr;
    a.x = s->x32;
    a.pa = s->exp_pa;
    a.pb = s->exp_pb;
    a.pc = s->exp_pc;
    a.part = s->exp_part;
    a.count = reinterpret_cast<unsigned long long*>(s->barrier);
    a.err = reinterpret_cast<int32_t*>(s->barrier + 2);
    a.sc = nullptr;
    a.tolerance = 0.0;
    a.max_iterations = 0;
    a.blocks = d_blocks;
    a.st = st;
    a.spin_limit = 4000000ull;
    if (const char* v = std::getenv("VXCOROT_BARRIER_SPINS")) {
        unsigned long long lim = std::strtoull(v, nullptr, 10);
        if (lim > 0 && lim < a.spin_limit) a.spin_limit = lim;
    }
    cudaError_t e = cudaMemsetAsync(s->barrier, 0, 4 * sizeof(unsigned), s->stream);
    if (e == cudaSuccess) e = launch_e<4, true>(a, G, smem, s->stream);
    s->launches += 1;
    if (e != cudaSuccess) {
        set_error("persistent pool PCG launch failed: %s", cudaGetErrorString(e));
        return VX_CUDA_ERROR;
    }
    return VX_OK;
}

}  // namespace vx

// K3: block direct sum for k >= 16 right-hand sides on the 5th-generation tensor
// cores (tcgen05, sm_100a).
//
//   part[s][i][c0 + c] = sum_{j in split s, j != i} G(i, j) Q(j, c)
//   G(i, j) = n_i . (x_i - y_j) / |x_i - y_j|^3        (generated in FP32 registers)
//   Q(j, c) = w_j p_j X[j][c0 + c]                     (packed per call)
//
// G is the adjoint double-layer kernel of laplace3d_DT (src/kernel/laplace3d.jl:30-40);
// the contraction replaces the batched lfmm3d(nd = K) of
// mul!(Y, ::BatchedDielectricOperator, X) (src/solver/multi_rhs.jl:103-130).
//
// Split-BF16 three-term product: with G = Gh + Gl and Q = Qh + Ql (bf16 hi/lo),
// G Q ~= Gh Qh + Gh Ql + Gl Qh (the dropped Gl Ql term is ~2^-16 relative).
// The tensor cores accumulate FP32 in tensor memory over FP = 4 chunks (256
// sources) into one of two alternating accumulators; the generator threads add
// each finished period into an FP32 running sum also kept in tensor memory. The
// tensor-core accumulation error grows with the number of accumulation steps;
// restarting it every period bounds it by that of 256 sources, and the running
// sum of the periods (round-to-nearest additions) adds a random-walk error of a
// few units in the last place. Each source split writes the sum as an FP32 partial.
//
// CTA = 128 NQ + 64 threads: warps 0 .. 4 NQ - 1 generate the 128 x 64 kernel tile
// of a source chunk (NQ threads per target row, each writing 64 / NQ of the row's
// K-major bf16 values into the 128-byte swizzled layout the UMMA descriptors
// read), fold the accumulators and run the epilogue; the next warp issues the MMAs
// (one thread); the last warp streams the pre-swizzled Q tiles with bulk copies
// into a ring and stages the source coordinates SC - 1 chunks ahead. Up to 64
// columns run two CTAs per SM (NQ = 2), so that one CTA's pipeline bubbles are
// filled by the other; wider tiles run one CTA per SM with NQ = 4. Box faces are
// axis-aligned, so a warp whose 32 rows share a normal axis computes n.(x - y) as
// the signed axis difference and folds the sign into its epilogue.
// Every mbarrier wait is bounded: on expiry the CTA records an error code and
// returns after releasing its tensor memory.
#include <cuda_bf16.h>
#include <algorithm>
#include <cstdlib>
#include <vector>
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "mbar.cuh"
#include "solver.h"

namespace bie {
namespace tc {

constexpr int M = 128;      // targets per tile (MMA M)
constexpr int KC = 64;      // sources per chunk = one 128-byte bf16 row
constexpr int SAMAX = 4;    // A (kernel tile) ring stages at most (Params::sa)
constexpr int SBMAX = 4;    // B (Q tile) ring stages at most (Params::sb)
constexpr int SC = 4;       // source-coordinate ring stages (staged SC - 1 chunks ahead)
// NQ = generator threads per tile row (each 64 / NQ sources of a chunk): 2 for the
// two-CTAs-per-SM shape (320 threads, <= 96 registers), 4 for the one-CTA shape
// (576 threads, <= 112 registers).
template <int NQ> __host__ __device__ constexpr int ngen() { return M * NQ; }
template <int NQ> __host__ __device__ constexpr int nthreads() { return M * NQ + 64; }
// Tensor-memory columns of a CTA: two accumulators and the running sum, npad
// columns each, rounded up to the power-of-two allocation unit.
__host__ __device__ inline uint32_t tmem_cols(int npad) {
    uint32_t c = 32;
    while (c < 3u * (uint32_t)npad) c <<= 1;
    return c;
}
constexpr int FP = 4;          // chunks accumulated in FP32 tensor memory before a compensated fold
constexpr uint32_t kWaitLimit = 1u << 26;  // default wait attempts before a CTA gives up (seconds)
constexpr int kErrTimeout = 1;

struct Params {
    GeomDev g;
    const uint8_t* bpack;  // [nchunks][2][npad][128 B] pre-swizzled bf16 images (hi, lo)
    int npad;              // MMA N (multiple of 16, <= 256)
    int keff;              // columns stored (<= npad)
    int64_t nchunks;
    int64_t cps;           // chunks per split
    int sa, sb;            // A and B ring stages (2 .. SAMAX, 2 .. SBMAX)
    uint32_t wait_limit;   // mbarrier wait attempts before the CTA gives up
    int stall_test;        // nonzero: withhold the first Q tile (exercises the timeout path)
    float* part;           // [nsplit][n][ldp] FP32 split partials
    int ldp, c0;
    int* err;
};

// Shared-memory head holding a CTA's copy of its Params and work item.
constexpr uint32_t kParamHead = ((uint32_t)sizeof(Params) + 2 * sizeof(int) + 15u) & ~15u;

// OR-reduction of a predicate over the NG generator threads (named barrier 1):
// also orders their shared-memory accesses like bar.sync.
template <int NG>
__device__ __forceinline__ bool gen_any(bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.or.pred p, 1, %2, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)v), "n"(NG)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    // K-major, 128-byte swizzle: rows of 128 B, 8-row atoms 1024 B apart (SBO),
    // LBO unused (1), descriptor version 1, layout type 2 (SWIZZLE_128B).
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1u << 16;
    d |= (uint64_t)(1024u >> 4) << 32;
    d |= (uint64_t)1u << 46;
    d |= (uint64_t)2u << 61;
    return d;
}

__device__ __forceinline__ uint32_t idesc_bf16(int n) {
    // c_format F32 (1) @4, a/b format BF16 (1) @7/@10, K-major A/B, N>>3 @17, M>>4 @24
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// Issues a 32-lane x 16-column tensor-memory load; the registers are valid after tmem_wait_ld().
__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// MUFU reciprocal square root (approximate, flush-to-zero): one instruction.
__device__ __forceinline__ float rsqrt_mufu(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float* v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
            taddr),
        "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])),
        "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
        "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])),
        "r"(__float_as_uint(v[11])), "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])),
        "r"(__float_as_uint(v[14])), "r"(__float_as_uint(v[15]))
        : "memory");
}

__device__ __forceinline__ uint32_t pack_bf16(float lo_elem, float hi_elem) {
    __nv_bfloat162 h = __floats2bfloat162_rn(lo_elem, hi_elem);  // .x (low 16 bits) = lo_elem
    return *reinterpret_cast<uint32_t*>(&h);
}

// Split two FP32 values into NP packed bf16 pieces (hi, lo or hi, mid, lo): each
// piece is the bf16 rounding of what the previous pieces leave.
template <int NP>
__device__ __forceinline__ void split_pieces(float a, float b, uint32_t* out) {
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        const uint32_t w = pack_bf16(a, b);
        out[p] = w;
        if (p + 1 < NP) {
            a -= __uint_as_float(w << 16);
            b -= __uint_as_float(w & 0xFFFF0000u);
        }
    }
}

// Packed FP32 pairs (sm_100 f32x2 arithmetic): one instruction applies the same
// round-to-nearest operation to two sources.
__device__ __forceinline__ uint64_t f2(float lo, float hi) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ float2 f2u(uint64_t r) {
    float2 v;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
    return v;
}
__device__ __forceinline__ uint64_t f2sub(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t f2mul(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t f2fma(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// split_pieces on a packed pair (the remainders are formed with one packed subtract).
template <int NP>
__device__ __forceinline__ void split_pieces2(uint64_t x, uint32_t* out) {
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        const float2 xu = f2u(x);
        const uint32_t w = pack_bf16(xu.x, xu.y);
        out[p] = w;
        if (p + 1 < NP) x = f2sub(x, f2(__uint_as_float(w << 16), __uint_as_float(w & 0xFFFF0000u)));
    }
}

// One thread's share of a row of a chunk's kernel tile: 64 / NQ sources (8-source
// groups gq0 .. gq0 + 8 / NQ - 1), processed 16 at a time as 8 packed pairs. AXIS:
// the rows of this warp have normal +-e_a for one axis a (sign applied in the
// epilogue); ca holds the source coordinates along a and cb, cc the other two,
// t2a, t2b, t2c the target's in the same order (duplicated into both halves of a
// pair), so one code path serves the three axes. !AXIS: general normal (n2x, n2y,
// n2z duplicated), with (ca, cb, cc) = (x, y, z).
template <bool AXIS, int NP, int NQ>
__device__ __forceinline__ void gen_row_part(const float* __restrict__ ca, const float* __restrict__ cb,
                                             const float* __restrict__ cc, uint64_t t2a, uint64_t t2b,
                                             uint64_t t2c, uint64_t n2x, uint64_t n2y, uint64_t n2z, int gq0,
                                             bool self, int64_t j0, int64_t i, uint8_t* Astage, uint32_t a_bytes,
                                             uint32_t row_off, uint32_t rsw) {
#pragma unroll 1
    for (int gq = gq0; gq < gq0 + 8 / NQ; gq += 2) {
        uint64_t v[8];  // kernel values of sources gq * 8 + 2 m, + 1
#pragma unroll
        for (int e4 = 0; e4 < 4; ++e4) {
            const int b = gq * 8 + e4 * 4;
            const float4 A4 = *reinterpret_cast<const float4*>(ca + b);
            const float4 B4 = *reinterpret_cast<const float4*>(cb + b);
            const float4 C4 = *reinterpret_cast<const float4*>(cc + b);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint64_t sa = h ? f2(A4.z, A4.w) : f2(A4.x, A4.y);
                const uint64_t sb = h ? f2(B4.z, B4.w) : f2(B4.x, B4.y);
                const uint64_t sc = h ? f2(C4.z, C4.w) : f2(C4.x, C4.y);
                const uint64_t da = f2sub(t2a, sa), db = f2sub(t2b, sb), dc = f2sub(t2c, sc);
                const uint64_t r2 = f2fma(da, da, f2fma(db, db, f2mul(dc, dc)));
                const float2 r2u = f2u(r2);
                const uint64_t ri = f2(rsqrt_mufu(r2u.x), rsqrt_mufu(r2u.y));
                const uint64_t dn = AXIS ? da : f2fma(n2x, da, f2fma(n2y, db, f2mul(n2z, dc)));
                v[e4 * 2 + h] = f2mul(f2mul(dn, ri), f2mul(ri, ri));
            }
        }
        if (self) {
#pragma unroll
            for (int m = 0; m < 8; ++m) {
                float2 u = f2u(v[m]);
                if (j0 + gq * 8 + 2 * m == i) u.x = 0.f;
                if (j0 + gq * 8 + 2 * m + 1 == i) u.y = 0.f;
                v[m] = f2(u.x, u.y);
            }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            uint32_t w[4][NP];
#pragma unroll
            for (int e = 0; e < 4; ++e) split_pieces2<NP>(v[4 * h + e], w[e]);
            const uint32_t off = row_off + ((((uint32_t)(gq + h)) ^ rsw) << 4);
#pragma unroll
            for (int p = 0; p < NP; ++p)
                *reinterpret_cast<uint4*>(Astage + p * a_bytes + off) = make_uint4(w[0][p], w[1][p], w[2][p], w[3][p]);
        }
    }
}

// The CTA body: target tile `tile`, source split `split` of the geometry in P. The plain
// launch (k_dt_tc, grid = tiles x splits) reads P from the kernel parameters; the
// work-list launch (k_dt_tc_list) runs one item of several geometries' tiles per CTA and
// reads its P from a copy at the head of the CTA's shared memory.
template <int NP, int NQ>
__device__ __forceinline__ void tc_body(const Params& P, const int tile, const int split, uint8_t* smem_raw) {
    constexpr int NGEN = ngen<NQ>();
    // carve-up aligned to 1024 bytes in the shared window (128-byte swizzle atoms), after
    // the parameter head
    uint8_t* const head_end = smem_raw + kParamHead;
    uint8_t* base = head_end + ((1024u - (smem_u32(head_end) & 1023u)) & 1023u);
    const int npad = P.npad;
    const uint32_t a_bytes = M * 128;          // one piece of the A tile (16 KB)
    const uint32_t b_bytes = (uint32_t)npad * 128;  // one piece of the B tile
    const int SA = P.sa, SB = P.sb;
    uint8_t* A = base;                               // [SA][NP][a_bytes]
    uint8_t* B = A + SA * NP * a_bytes;              // [SB][NP][b_bytes]
    float* crd = (float*)(B + SB * NP * b_bytes);    // [SC][3][KC] source coordinates (SoA, FP32 relative)
    uint64_t* full_a = (uint64_t*)(crd + SC * 3 * KC);
    uint64_t* empty_a = full_a + SAMAX;  // [SAMAX] A stage consumed (MMA commit)
    uint64_t* full_b = empty_a + SAMAX;  // [SBMAX] Q tile landed (bulk copy)
    uint64_t* empty_b = full_b + SBMAX;  // [SBMAX] Q tile consumed (MMA commit)
    uint64_t* crd_full = empty_b + SBMAX;  // [SC] coordinates staged (producer warp)
    uint64_t* crd_empty = crd_full + SC; // [SC] coordinates consumed (generators)
    uint64_t* acc_full = crd_empty + SC; // [2] accumulation period finished (MMA commit)
    uint64_t* acc_empty = acc_full + 2;  // [2] accumulator folded (generators)
    uint64_t* acc_done = acc_empty + 2;
    uint32_t* tmem_slot = (uint32_t*)(acc_done + 1);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t n = P.g.n;
    const int64_t i0 = (int64_t)tile * M;
    const int64_t ch0 = (int64_t)split * P.cps;
    const int64_t ch1 = min(P.nchunks, ch0 + P.cps);
    const int nch = ch1 > ch0 ? (int)(ch1 - ch0) : 0;
    // tensor memory: two FP32 accumulators (alternating periods) and the running
    // sum, npad columns each
    const uint32_t tcols = tmem_cols(npad);

    if (threadIdx.x == 0) {
        for (int s = 0; s < SAMAX; ++s) {
            mbar_init(&full_a[s], NGEN);
            mbar_init(&empty_a[s], 1);
        }
        for (int s = 0; s < SBMAX; ++s) {
            mbar_init(&full_b[s], 1);
            mbar_init(&empty_b[s], 1);
        }
        for (int s = 0; s < SC; ++s) {
            mbar_init(&crd_full[s], 32);
            mbar_init(&crd_empty[s], NGEN);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], NGEN);
        }
        mbar_init(acc_done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(tcols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const uint32_t t_sum = tmem + 2u * (uint32_t)npad;

    // tile origin: coordinates are rounded to FP32 relative to it
    const int64_t io = P.g.perm[min(i0, n - 1)];
    const double ox = P.g.x[io], oy = P.g.y[io], oz = P.g.z[io];

    if (warp < NGEN / 32) {
        // ------------------------- generators -------------------------------
        const int r = threadIdx.x & (M - 1);  // tile row
        const int qt = threadIdx.x / M;       // which 64 / NQ sources of each chunk (warp-uniform)
        const bool valid = i0 + r < n;
        const int64_t i = valid ? (int64_t)P.g.perm[i0 + r] : n;  // original index of the target
        float xi, yi, zi, n0, n1, n2;
        if (valid) {
            xi = (float)(P.g.x[i] - ox); yi = (float)(P.g.y[i] - oy); zi = (float)(P.g.z[i] - oz);
            n0 = (float)P.g.nx[i]; n1 = (float)P.g.ny[i]; n2 = (float)P.g.nz[i];
        } else {
            xi = yi = zi = -1.0e18f;  // far from every node and every padded source: G underflows to 0
            n0 = n1 = n2 = 0.f;
        }
        // warp-uniform normal axis (code 0/1/2 = +-e_axis, 3 = general)
        int code = 3;
        float sgn = 1.f;
        if (fabsf(n0) == 1.f && n1 == 0.f && n2 == 0.f) { code = 0; sgn = n0; }
        else if (fabsf(n1) == 1.f && n0 == 0.f && n2 == 0.f) { code = 1; sgn = n1; }
        else if (fabsf(n2) == 1.f && n0 == 0.f && n1 == 0.f) { code = 2; sgn = n2; }
        const unsigned full = 0xFFFFFFFFu;
        const int cmin = __reduce_min_sync(full, valid ? code : 4);
        const int cmax = __reduce_max_sync(full, valid ? code : -1);
        const int ax = (cmin == cmax && cmin < 3) ? cmin : 3;
        if (ax == 3) sgn = 1.f;
        // axis path: the normal axis first, then the other two (coordinate-array
        // offsets in the staged chunk and the target's coordinates in that order)
        const int a1 = ax < 3 ? ax : 0, a2 = a1 == 2 ? 0 : a1 + 1, a3 = a2 == 2 ? 0 : a2 + 1;
        const int oa = a1 * KC, ob = a2 * KC, oc = a3 * KC;
        const float tcrd[3] = {xi, yi, zi};
        const float ta = a1 == 0 ? tcrd[0] : (a1 == 1 ? tcrd[1] : tcrd[2]);
        const float tb = a2 == 0 ? tcrd[0] : (a2 == 1 ? tcrd[1] : tcrd[2]);
        const float tc = a3 == 0 ? tcrd[0] : (a3 == 1 ? tcrd[1] : tcrd[2]);
        const uint64_t t2a = f2(ta, ta), t2b = f2(tb, tb), t2c = f2(tc, tc);
        const uint64_t t2x = f2(xi, xi), t2y = f2(yi, yi), t2z = f2(zi, zi);
        const uint64_t n2x = f2(n0, n0), n2y = f2(n1, n1), n2z = f2(n2, n2);
        const uint32_t row_off = (uint32_t)r * 128u;
        const uint32_t rsw = (uint32_t)(r & 7);
        const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;

        // Add the FP32 accumulator of period p into the running sum; the warp
        // decides as a whole.
        auto fold = [&](int p) -> bool {
            const int b = p & 1;
            bool ok = mbar_wait(&acc_full[b], (uint32_t)(p >> 1) & 1u, abort_flag, P.wait_limit);
            if (!__all_sync(full, ok)) return false;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (int c = qt * 16; c < npad; c += 16 * NQ) {
                uint32_t a[16], h[16];
                tmem_ld16_async(tmem + lane_base + (uint32_t)(b * npad + c), a);
                if (p == 0) {
                    tmem_wait_ld();
#pragma unroll
                    for (int q = 0; q < 16; ++q) h[q] = a[q];
                } else {
                    tmem_ld16_async(t_sum + lane_base + (uint32_t)c, h);
                    tmem_wait_ld();
#pragma unroll
                    for (int q = 0; q < 16; ++q) h[q] = __float_as_uint(__uint_as_float(h[q]) + __uint_as_float(a[q]));
                }
                tmem_st16(t_sum + lane_base + (uint32_t)c, reinterpret_cast<const float*>(h));
            }
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            mbar_arrive(&acc_empty[b]);
            return true;
        };

        bool ok = true;
        for (int lc = 0; lc < nch && ok; ++lc) {
            const int s = lc % SA, sc = lc % SC;
            const int64_t j0 = (ch0 + lc) * KC;
            // coordinates staged; A stage s released by the MMAs of chunk lc - S
            if (!mbar_wait(&crd_full[sc], (uint32_t)(lc / SC) & 1u, abort_flag, P.wait_limit)) { ok = false; break; }
            if (lc >= SA && !mbar_wait(&empty_a[s], (uint32_t)(lc / SA - 1) & 1u, abort_flag, P.wait_limit)) { ok = false; break; }
            uint8_t* As = A + s * NP * a_bytes;
            const float* cs = crd + sc * 3 * KC;
            const bool self = (i >= j0) && (i < j0 + KC);  // this chunk holds the target's own node
            const int gq0 = qt * (8 / NQ);
            if (ax < 3)
                gen_row_part<true, NP, NQ>(cs + oa, cs + ob, cs + oc, t2a, t2b, t2c, n2x, n2y, n2z, gq0, self, j0, i,
                                           As, a_bytes, row_off, rsw);
            else
                gen_row_part<false, NP, NQ>(cs, cs + KC, cs + 2 * KC, t2x, t2y, t2z, n2x, n2y, n2z, gq0, self, j0, i,
                                            As, a_bytes, row_off, rsw);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive(&full_a[s]);
            mbar_arrive(&crd_empty[sc]);
            // end of period p: fold period p - 1 (its MMAs finished while p was generated)
            if (lc % FP == FP - 1 || lc == nch - 1) {
                const int p = lc / FP;
                if (p >= 1) ok = fold(p - 1);
            }
        }
        // ------------------------- epilogue ---------------------------------
        ok = ok && !*abort_flag;
        if (nch > 0 && ok) ok = fold((nch - 1) / FP);
        ok = !gen_any<NGEN>(!ok);  // every generator warp takes the same branch
        if (ok) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            float* out = P.part + ((int64_t)split * n + i) * P.ldp + P.c0;
            for (int c = qt * 16; c < npad; c += 16 * NQ) {
                float h[16];
                if (nch > 0) {
                    tmem_ld16(t_sum + lane_base + (uint32_t)c, h);
                } else {
#pragma unroll
                    for (int q = 0; q < 16; ++q) h[q] = 0.f;
                }
                if (valid) {
#pragma unroll
                    for (int q = 0; q < 16; ++q)
                        if (c + q < P.keff) out[c + q] = sgn * h[q];
                }
            }
        }
    } else if (warp == NGEN / 32) {
        // ------------------------- MMA issuer --------------------------------
        if (lane == 0) {
            const uint32_t idesc = idesc_bf16(npad);
            for (int lc = 0; lc < nch; ++lc) {
                const int s = lc % SA, sb = lc % SB;
                const int p = lc / FP, b = p & 1;
                const bool pfirst = (lc % FP) == 0;
                if (!mbar_wait(&full_a[s], (uint32_t)(lc / SA) & 1u, abort_flag, P.wait_limit)) break;
                if (!mbar_wait(&full_b[sb], (uint32_t)(lc / SB) & 1u, abort_flag, P.wait_limit)) break;
                // accumulator b is reused from period p - 2 once the generators folded it
                if (pfirst && p >= 2 && !mbar_wait(&acc_empty[b], (uint32_t)((p - 2) >> 1) & 1u, abort_flag, P.wait_limit)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                // descriptors of the stage; the start-address field (bits 0-13, address >> 4)
                // is advanced in place: every address stays below 256 KB
                const uint64_t da = sw128_desc(smem_u32(A + s * NP * a_bytes));
                const uint64_t db = sw128_desc(smem_u32(B + sb * NP * b_bytes));
                const uint32_t dacc = tmem + (uint32_t)(b * npad);
                // products of pieces whose orders sum to at most NP - 1
#pragma unroll
                for (int kk = 0; kk < KC / 16; ++kk) {
                    bool first = pfirst && kk == 0;
#pragma unroll
                    for (int pa = 0; pa < NP; ++pa)
#pragma unroll
                        for (int pb = 0; pb + pa < NP; ++pb) {
                            mma_bf16(dacc, da + (uint64_t)((pa * a_bytes + kk * 32) >> 4),
                                     db + (uint64_t)((pb * b_bytes + kk * 32) >> 4), idesc, first ? 0u : 1u);
                            first = false;
                        }
                }
                mma_commit(&empty_a[s]);
                mma_commit(&empty_b[sb]);
                if (lc % FP == FP - 1 || lc == nch - 1) mma_commit(&acc_full[b]);
            }
            mma_commit(acc_done);
            // on abort, drain this thread's MMAs before the CTA releases tensor memory
            if (*abort_flag) mbar_wait_raw(acc_done, 0, P.wait_limit);
        }
        __syncwarp();
    } else {
        // ------------- Q-tile and source-coordinate producer -----------------
        // Runs SB - 1 chunks ahead on the Q tiles and SC - 1 chunks ahead on the
        // coordinates; each slot is refilled once its consumer of SB (SC) chunks
        // earlier has finished.
        const uint32_t bytes = NP * b_bytes;
        int issued = 0;
        auto stage_b = [&](int c) -> bool {
            const int sb = c % SB;
            if (c >= SB && !mbar_wait(&empty_b[sb], (uint32_t)(c / SB - 1) & 1u, abort_flag, P.wait_limit)) return false;
            if (lane == 0) {
                mbar_arrive_tx(&full_b[sb], bytes);
                // test of the timeout path: the first Q tile is announced but never copied
                if (!(P.stall_test && c == 0))
                    bulk_g2s(B + sb * NP * b_bytes, P.bpack + (size_t)(ch0 + c) * bytes, bytes, &full_b[sb]);
                issued = c + 1;
            }
            return true;
        };
        // coordinates of chunk c, FP32 relative to the tile origin; the global
        // loads are issued before the wait for the slot
        auto stage_crd = [&](int c) -> bool {
            const int64_t j0 = (ch0 + c) * KC;
            float x[KC / 32], y[KC / 32], z[KC / 32];
#pragma unroll
            for (int h = 0; h < KC / 32; ++h) {
                const int64_t j = j0 + lane + 32 * h;
                x[h] = y[h] = z[h] = 1.0e18f;  // padded source: G underflows to 0
                if (j < n) {
                    x[h] = (float)(P.g.x[j] - ox); y[h] = (float)(P.g.y[j] - oy); z[h] = (float)(P.g.z[j] - oz);
                }
            }
            const int sc = c % SC;
            if (c >= SC && !mbar_wait(&crd_empty[sc], (uint32_t)(c / SC - 1) & 1u, abort_flag, P.wait_limit)) return false;
            float* cs = crd + sc * 3 * KC;
#pragma unroll
            for (int h = 0; h < KC / 32; ++h) {
                const int t = lane + 32 * h;
                cs[t] = x[h]; cs[KC + t] = y[h]; cs[2 * KC + t] = z[h];
            }
            mbar_arrive(&crd_full[sc]);
            return true;
        };
        bool ok = true;
        for (int c = 0; c < SC - 1 && c < nch && ok; ++c) ok = stage_crd(c);
        for (int c = 0; c < SB - 1 && c < nch && ok; ++c) ok = stage_b(c);
        for (int lc = 0; lc < nch && ok; ++lc) {
            if (lc + SB - 1 < nch) ok = stage_b(lc + SB - 1);
            if (ok && lc + SC - 1 < nch) ok = stage_crd(lc + SC - 1);
        }
        // on abort, wait for the copies still in flight (at most one per slot)
        if (lane == 0 && *abort_flag)
            for (int c = issued > SB ? issued - SB : 0; c < issued; ++c)
                if (!(P.stall_test && c == 0)) mbar_wait_raw(&full_b[c % SB], (c / SB) & 1, P.wait_limit);
        __syncwarp();
    }

    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (*abort_flag && threadIdx.x == 0) atomicOr(P.err, kErrTimeout);
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tcols) : "memory");
    }
}

template <int NP, int NQ>
__global__ void __launch_bounds__(nthreads<NQ>(), 4 / NQ) k_dt_tc(Params P) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    tc_body<NP, NQ>(P, (int)blockIdx.x, (int)blockIdx.y, smem_raw);
}

// Work-list launch: CTA b runs items[b] = (member, target tile, source split, unused) with
// the member's parameters plist[member]; one launch covers the tiles of several geometries,
// each with its own nodes, right-hand-side block, width and partials.
template <int NP, int NQ>
__global__ void __launch_bounds__(nthreads<NQ>(), 4 / NQ)
    k_dt_tc_list(const Params* __restrict__ plist, const int4* __restrict__ items) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    Params* sP = reinterpret_cast<Params*>(smem_raw);
    int* s_item = reinterpret_cast<int*>(smem_raw + sizeof(Params));
    if (threadIdx.x == 0) {
        const int4 it = items[blockIdx.x];
        *sP = plist[it.x];
        s_item[0] = it.y;
        s_item[1] = it.z;
    }
    __syncthreads();
    tc_body<NP, NQ>(*sP, s_item[0], s_item[1], smem_raw);
}

// Packs Q(j, c) = w_j p_j X[j][c0 + c] as NP bf16 pieces, in the swizzled K-major
// smem image of each 64-source chunk: [chunk][piece][row c][128 B]. Rows c >= keff
// and sources j >= n are zero.
template <int NP>
__global__ void k_pack_q(GeomDev g, const double* __restrict__ X, int ldx, int c0, int keff,
                         const double* __restrict__ pre, int npad, int64_t nchunks, uint8_t* __restrict__ out) {
    // one thread per (chunk, row c, 8-source group)
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = nchunks * npad * 8;
    if (e >= total) return;
    const int gq = (int)(e & 7);
    const int c = (int)((e >> 3) % npad);
    const int64_t ch = (e >> 3) / npad;
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int64_t j = ch * KC + gq * 8 + q;
        double val = 0.0;
        if (j < g.n && c < keff) val = g.w[j] * (pre ? pre[j] : 1.0) * X[j * ldx + c0 + c];
        v[q] = (float)val;
    }
    uint32_t w[4][NP];
#pragma unroll
    for (int q = 0; q < 4; ++q) split_pieces<NP>(v[2 * q], v[2 * q + 1], w[q]);
    const size_t tile = (size_t)npad * 128;
    uint8_t* base = out + (size_t)ch * NP * tile;
    const uint32_t off = (uint32_t)c * 128u + ((((uint32_t)gq) ^ (uint32_t)(c & 7)) << 4);
#pragma unroll
    for (int p = 0; p < NP; ++p)
        *reinterpret_cast<uint4*>(base + p * tile + off) = make_uint4(w[0][p], w[1][p], w[2][p], w[3][p]);
}

size_t smem_bytes(int npad, int np, int sa, int sb) {
    size_t a = (size_t)sa * np * M * 128, b = (size_t)sb * np * npad * 128;
    size_t c = (size_t)SC * 3 * KC * sizeof(float);
    size_t bars = (2 * SAMAX + 2 * SBMAX + 2 * SC + 5) * sizeof(uint64_t) + 16;
    return kParamHead + 1024 + a + b + c + bars;
}

// Ring depths for one CTA per SM: the deepest A ring (<= SAMAX) that fits with a
// 2-slot B ring (the kernel-tile generators run SA - 1 chunks ahead of the MMAs),
// then the deepest B ring that still fits.
void ring_stages(int npad, int np, int* sa, int* sb) {
    const size_t cap = 227 * 1024;
    int a = SAMAX;
    while (a > 2 && smem_bytes(npad, np, a, 2) > cap) --a;
    int b = SBMAX;
    while (b > 2 && smem_bytes(npad, np, a, b) > cap) --b;
    *sa = a;
    *sb = b;
}

// Launch shape for npad columns and np pieces: two CTAs per SM (NQ = 2, A ring of
// two) when their tensor memory (3 npad columns each, allocated as a power of two)
// and shared memory fit, else
// one CTA per SM (NQ = 4) with the deepest rings that fit.
struct Shape {
    int ctas, nq, sa, sb;
    size_t smem;
};

// force_ctas = 1 or 2 selects that shape when it fits (0 = the default choice).
Shape shape(int npad, int np, int force_ctas = 0) {
    const size_t half_sm = 113 * 1024;  // 228 KB per SM, 1 KB reserved per CTA
    Shape sh;
    const bool two = tmem_cols(npad) <= 256 && smem_bytes(npad, np, 2, 2) <= half_sm;
    if (two && force_ctas != 1) {
        sh.ctas = 2;
        sh.nq = 2;
        sh.sa = 2;
        sh.sb = 2;
        while (sh.sb < SBMAX && smem_bytes(npad, np, 2, sh.sb + 1) <= half_sm) ++sh.sb;
    } else {
        sh.ctas = 1;
        sh.nq = 4;
        ring_stages(npad, np, &sh.sa, &sh.sb);
    }
    sh.smem = smem_bytes(npad, np, sh.sa, sh.sb);
    return sh;
}

template <int NP, int NQ>
void launch_k(const Params& P, dim3 grid, size_t sm, cudaStream_t s) {
    ensure_smem_limit((const void*)k_dt_tc<NP, NQ>, sm);
    k_dt_tc<NP, NQ><<<grid, nthreads<NQ>(), sm, s>>>(P);
    BIE_CK(cudaGetLastError());
}

template <int NP>
void pack_q(const GeomDev& g, const double* X, int ldx, int c0, int kc, const double* pre, uint8_t* bpack,
            cudaStream_t s) {
    const int npad = ((kc + 15) / 16) * 16;
    const int64_t nchunks = (g.n + KC - 1) / KC;
    const int64_t pk = nchunks * npad * 8;
    k_pack_q<NP><<<(unsigned)((pk + 255) / 256), 256, 0, s>>>(g, X, ldx, c0, kc, pre, npad, nchunks, bpack);
    BIE_CK(cudaGetLastError());
}

template <int NP>
void launch_tc(const GeomDev& g, const double* X, int ldx, int c0, int kc, const double* pre, int nsplit, int64_t cps,
               float* part, int ldp, uint8_t* bpack, int* err, int force_ctas, cudaStream_t s) {
    const int npad = ((kc + 15) / 16) * 16;
    const int64_t nchunks = (g.n + KC - 1) / KC;
    pack_q<NP>(g, X, ldx, c0, kc, pre, bpack, s);
    Params P;
    P.g = g;
    P.bpack = bpack;
    P.npad = npad;
    P.keff = kc;
    P.nchunks = nchunks;
    P.cps = cps;
    const Shape sh = shape(npad, NP, force_ctas);
    // BIE_TEST_TC_STALL (tests only): every CTA's first Q tile never arrives, so the
    // bounded waits expire quickly and the launch reports a timeout
    P.stall_test = std::getenv("BIE_TEST_TC_STALL") != nullptr;
    P.wait_limit = P.stall_test ? (1u << 14) : kWaitLimit;
    P.sa = sh.sa;
    P.sb = sh.sb;
    P.part = part;
    P.ldp = ldp;
    P.c0 = c0;
    P.err = err;
    dim3 grid((unsigned)((g.n + M - 1) / M), (unsigned)nsplit);
    if (sh.nq == 2)
        launch_k<NP, 2>(P, grid, sh.smem, s);
    else
        launch_k<NP, 4>(P, grid, sh.smem, s);
}

// Work-list launch over the members' (tile, split) items; the shape (CTAs per SM, rings)
// is that of the widest member, the others run inside it.
template <int NP>
void launch_tc_list(const std::vector<TcMember>& ms, int* err, void* dscratch, size_t scratch_bytes, cudaStream_t s) {
    int npad_max = 16;
    for (const auto& m : ms) npad_max = std::max(npad_max, ((m.kc + 15) / 16) * 16);
    const Shape sh = shape(npad_max, NP);
    std::vector<Params> ps(ms.size());
    std::vector<int4> items;
    // members in the caller's order (largest first), each member's tiles x splits
    for (size_t m = 0; m < ms.size(); ++m) {
        const TcMember& t = ms[m];
        pack_q<NP>(t.g, t.X, t.ldx, t.c0, t.kc, t.pre, t.bpack, s);
        Params& P = ps[m];
        P.g = t.g;
        P.bpack = t.bpack;
        P.npad = ((t.kc + 15) / 16) * 16;
        P.keff = t.kc;
        P.nchunks = (t.g.n + KC - 1) / KC;
        P.cps = t.cps;
        P.stall_test = 0;
        P.wait_limit = kWaitLimit;
        P.sa = sh.sa;
        P.sb = sh.sb;
        P.part = t.part;
        P.ldp = t.ldp;
        P.c0 = t.c0;
        P.err = err;
        const int tiles = (int)((t.g.n + M - 1) / M);
        for (int sp = 0; sp < t.nsplit; ++sp)
            for (int ti = 0; ti < tiles; ++ti) items.push_back(make_int4((int)m, ti, sp, 0));
    }
    const size_t need = block_tc_list_bytes((int)ms.size(), (int64_t)items.size());
    if (need > scratch_bytes) throw Error(BIE_EINVAL, "launch_block_tc_list: work-list buffer too small");
    uint8_t* d = static_cast<uint8_t*>(dscratch);
    const size_t poff = 0, ioff = ((sizeof(Params) * ms.size() + 255) / 256) * 256;
    BIE_CK(cudaMemcpyAsync(d + poff, ps.data(), sizeof(Params) * ps.size(), cudaMemcpyHostToDevice, s));
    BIE_CK(cudaMemcpyAsync(d + ioff, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice, s));
    // the host vectors are pageable: the copies are staged before cudaMemcpyAsync returns
    const Params* dp = reinterpret_cast<const Params*>(d + poff);
    const int4* di = reinterpret_cast<const int4*>(d + ioff);
    const dim3 grid((unsigned)items.size());
    if (sh.nq == 2) {
        ensure_smem_limit((const void*)k_dt_tc_list<NP, 2>, sh.smem);
        k_dt_tc_list<NP, 2><<<grid, nthreads<2>(), sh.smem, s>>>(dp, di);
    } else {
        ensure_smem_limit((const void*)k_dt_tc_list<NP, 4>, sh.smem);
        k_dt_tc_list<NP, 4><<<grid, nthreads<4>(), sh.smem, s>>>(dp, di);
    }
    BIE_CK(cudaGetLastError());
}

}  // namespace tc

size_t block_tc_list_bytes(int nmembers, int64_t nitems) {
    return ((sizeof(tc::Params) * (size_t)nmembers + 255) / 256) * 256 + sizeof(int4) * (size_t)nitems;
}

void launch_block_tc_list(const std::vector<TcMember>& ms, int pieces, int* err, void* dscratch, size_t scratch_bytes,
                          cudaStream_t s) {
    if (ms.empty()) return;
    if (pieces == 3)
        tc::launch_tc_list<3>(ms, err, dscratch, scratch_bytes, s);
    else
        tc::launch_tc_list<2>(ms, err, dscratch, scratch_bytes, s);
}

int tc_npad(int kc) { return ((kc + 15) / 16) * 16; }

// Runs K3 for columns [c0, c0 + kc) (kc <= 128) of X into part[s][i][c0 + c],
// with the kernel and right-hand sides split into `pieces` (2: three products,
// 3: six products) bf16 pieces.
void launch_block_tc(const GeomDev& g, const double* X, int ldx, int c0, int kc, const double* pre, int nsplit,
                     int64_t cps, float* part, int ldp, uint8_t* bpack, int* err, int pieces, int force_ctas,
                     cudaStream_t s) {
    if (pieces == 3)
        tc::launch_tc<3>(g, X, ldx, c0, kc, pre, nsplit, cps, part, ldp, bpack, err, force_ctas, s);
    else
        tc::launch_tc<2>(g, X, ldx, c0, kc, pre, nsplit, cps, part, ldp, bpack, err, force_ctas, s);
}

size_t block_tc_pack_bytes(int64_t n, int kc, int pieces) {
    const int64_t nchunks = (n + tc::KC - 1) / tc::KC;
    return (size_t)nchunks * pieces * tc_npad(kc) * 128;
}

int block_tc_ctas_per_sm(int kc, int pieces, int force_ctas) {
    return tc::shape(tc_npad(kc), pieces, force_ctas).ctas;
}

}  // namespace bie

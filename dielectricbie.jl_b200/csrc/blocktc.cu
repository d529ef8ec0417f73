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
// G Q ~= Gh Qh + Gh Ql + Gl Qh (the dropped Gl Ql term is ~2^-16 relative),
// accumulated in FP32 in tensor memory; each source split writes an FP64 partial.
//
// CTA = 320 threads: warps 0-7 generate the 128 x 64 kernel tile of a source
// chunk (two threads per target row, each writing 32 of the row's 64 K-major
// bf16 values into the 128-byte swizzled layout the UMMA descriptors read) and
// run the epilogue; warp 8 issues the MMAs (one thread); warp 9 streams the
// pre-swizzled Q tiles with bulk copies. Box faces are axis-aligned, so a warp
// whose 32 rows share a normal axis computes n.(x - y) as the signed axis
// difference and folds the sign into its epilogue.
// Every mbarrier wait is bounded: on expiry the CTA records an error code and
// returns after releasing its tensor memory.
#include <cuda_bf16.h>
#include <algorithm>
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "solver.h"

namespace bie {
namespace tc {

constexpr int M = 128;      // targets per tile (MMA M)
constexpr int KC = 64;      // sources per chunk = one 128-byte bf16 row
constexpr int S = 2;        // pipeline stages
constexpr int NGEN = 256;      // generator threads: 2 per tile row (two halves of a chunk)
constexpr int NTHREADS = NGEN + 64;
constexpr uint32_t kWaitLimit = 1u << 26;
constexpr int kErrTimeout = 1;

struct Params {
    GeomDev g;
    const uint8_t* bpack;  // [nchunks][2][npad][128 B] pre-swizzled bf16 images (hi, lo)
    int npad;              // MMA N (multiple of 16, <= 256)
    int keff;              // columns stored (<= npad)
    int64_t nchunks;
    int64_t cps;           // chunks per split
    double* part;          // [nsplit][n][ldp]
    int ldp, c0;
    int* err;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait; returns false (and flags the CTA) when the limit expires.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort_flag) {
    for (uint32_t it = 0; it < kWaitLimit; ++it) {
        if (mbar_try(b, parity)) return true;
        if (*abort_flag) return false;
    }
    *abort_flag = 1;
    return false;
}

// Wait bounded by an iteration limit only (used to drain in-flight work on the abort path).
__device__ __forceinline__ bool mbar_wait_raw(uint64_t* b, uint32_t parity) {
    for (uint32_t it = 0; it < kWaitLimit; ++it)
        if (mbar_try(b, parity)) return true;
    return false;
}

// OR-reduction of a predicate over the 256 generator threads (named barrier 1):
// also orders their shared-memory accesses like bar.sync.
__device__ __forceinline__ bool gen_any(bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.or.pred p, 1, 256, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)v)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
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

// One thread's half row of a chunk's kernel tile: 32 sources (groups gq0..gq0+3),
// processed 16 at a time. AX = 0/1/2: the rows of this warp have normal +-e_AX
// (sign applied in the epilogue); AX = 3: general normal.
template <int AX, int NP>
__device__ __forceinline__ void gen_half_row(const float* __restrict__ cs, float xi, float yi, float zi, float n0,
                                             float n1, float n2, int gq0, bool self, int64_t j0, int64_t i,
                                             uint8_t* Astage, uint32_t a_bytes, uint32_t row_off, uint32_t rsw) {
#pragma unroll 1
    for (int gq = gq0; gq < gq0 + 4; gq += 2) {
        float v[16];
#pragma unroll
        for (int e4 = 0; e4 < 4; ++e4) {
            const int b = gq * 8 + e4 * 4;
            const float4 X4 = *reinterpret_cast<const float4*>(cs + b);
            const float4 Y4 = *reinterpret_cast<const float4*>(cs + KC + b);
            const float4 Z4 = *reinterpret_cast<const float4*>(cs + 2 * KC + b);
            const float sx[4] = {X4.x, X4.y, X4.z, X4.w}, sy[4] = {Y4.x, Y4.y, Y4.z, Y4.w},
                        sz[4] = {Z4.x, Z4.y, Z4.z, Z4.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const float dx = xi - sx[e], dy = yi - sy[e], dz = zi - sz[e];
                const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                const float ri = rsqrt_mufu(r2);
                float dn;
                if (AX == 0) dn = dx;
                else if (AX == 1) dn = dy;
                else if (AX == 2) dn = dz;
                else dn = fmaf(n0, dx, fmaf(n1, dy, n2 * dz));
                v[e4 * 4 + e] = (dn * ri) * (ri * ri);
            }
        }
        if (self) {
#pragma unroll
            for (int e = 0; e < 16; ++e)
                if (j0 + gq * 8 + e == i) v[e] = 0.f;
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            uint32_t w[4][NP];
#pragma unroll
            for (int e = 0; e < 4; ++e) split_pieces<NP>(v[8 * h + 2 * e], v[8 * h + 2 * e + 1], w[e]);
            const uint32_t off = row_off + ((((uint32_t)(gq + h)) ^ rsw) << 4);
#pragma unroll
            for (int p = 0; p < NP; ++p)
                *reinterpret_cast<uint4*>(Astage + p * a_bytes + off) = make_uint4(w[0][p], w[1][p], w[2][p], w[3][p]);
        }
    }
}

template <int NP>
__global__ void __launch_bounds__(NTHREADS, 1) k_dt_tc(Params P) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // carve-up aligned to 1024 bytes in the shared window (128-byte swizzle atoms)
    uint8_t* base = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    const int npad = P.npad;
    const uint32_t a_bytes = M * 128;          // one term of the A tile (16 KB)
    const uint32_t b_bytes = (uint32_t)npad * 128;  // one term of the B tile
    uint8_t* A = base;                               // [S][NP][a_bytes]
    uint8_t* B = A + S * NP * a_bytes;               // [S][NP][b_bytes]
    float* crd = (float*)(B + S * NP * b_bytes);     // [S][3][KC] source coordinates (SoA, FP32 relative)
    uint64_t* full_a = (uint64_t*)(crd + S * 3 * KC);
    uint64_t* full_b = full_a + S;
    uint64_t* empty = full_b + S;
    uint64_t* crd_full = empty + S;
    uint64_t* acc_done = crd_full + S;
    uint32_t* tmem_slot = (uint32_t*)(acc_done + 1);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t n = P.g.n;
    const int64_t i0 = (int64_t)blockIdx.x * M;
    const int64_t ch0 = (int64_t)blockIdx.y * P.cps;
    const int64_t ch1 = min(P.nchunks, ch0 + P.cps);
    const int nch = ch1 > ch0 ? (int)(ch1 - ch0) : 0;
    const uint32_t tcols = npad <= 32 ? 32 : (npad <= 64 ? 64 : (npad <= 128 ? 128 : 256));

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full_a[s], NGEN);
            mbar_init(&full_b[s], 1);
            mbar_init(&empty[s], 1);
            mbar_init(&crd_full[s], 32);
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

    // tile origin: coordinates are rounded to FP32 relative to it
    const int64_t io = P.g.perm[min(i0, n - 1)];
    const double ox = P.g.x[io], oy = P.g.y[io], oz = P.g.z[io];

    if (warp < NGEN / 32) {
        // ------------------------- generators -------------------------------
        const int r = threadIdx.x & (M - 1);  // tile row
        const int half = threadIdx.x / M;     // which 32 sources of each chunk
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
        const uint32_t row_off = (uint32_t)r * 128u;
        const uint32_t rsw = (uint32_t)(r & 7);
        for (int lc = 0; lc < nch; ++lc) {
            const int s = lc % S;
            const uint32_t u = (uint32_t)(lc / S);
            const int64_t j0 = (ch0 + lc) * KC;
            // coordinates staged (and stage s released by the MMAs of chunk lc - S)
            if (!mbar_wait(&crd_full[s], u & 1, abort_flag)) break;
            uint8_t* As = A + s * NP * a_bytes;
            const float* cs = crd + s * 3 * KC;
            const bool self = (i >= j0) && (i < j0 + KC);  // this chunk holds the target's own node
            const int gq0 = half * 4;
            switch (ax) {
                case 0: gen_half_row<0, NP>(cs, xi, yi, zi, n0, n1, n2, gq0, self, j0, i, As, a_bytes, row_off, rsw); break;
                case 1: gen_half_row<1, NP>(cs, xi, yi, zi, n0, n1, n2, gq0, self, j0, i, As, a_bytes, row_off, rsw); break;
                case 2: gen_half_row<2, NP>(cs, xi, yi, zi, n0, n1, n2, gq0, self, j0, i, As, a_bytes, row_off, rsw); break;
                default: gen_half_row<3, NP>(cs, xi, yi, zi, n0, n1, n2, gq0, self, j0, i, As, a_bytes, row_off, rsw); break;
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive(&full_a[s]);
        }
        // ------------------------- epilogue ---------------------------------
        bool ok = !*abort_flag;
        if (nch > 0 && ok) ok = mbar_wait(acc_done, 0, abort_flag);
        ok = !gen_any(!ok);  // every generator warp takes the same branch
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (ok) {
            const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
            double* out = P.part + ((int64_t)blockIdx.y * n + i) * P.ldp + P.c0;
            for (int c = half * 16; c < npad; c += 32) {
                float v[16];
                if (nch > 0) {
                    tmem_ld16(tmem + lane_base + (uint32_t)c, v);
                } else {
#pragma unroll
                    for (int q = 0; q < 16; ++q) v[q] = 0.f;
                }
                if (valid) {
#pragma unroll
                    for (int q = 0; q < 16; ++q)
                        if (c + q < P.keff) out[c + q] = (double)(sgn * v[q]);
                }
            }
        }
    } else if (warp == NGEN / 32) {
        // ------------------------- MMA issuer --------------------------------
        if (lane == 0) {
            const uint32_t idesc = idesc_bf16(npad);
            for (int lc = 0; lc < nch; ++lc) {
                const int s = lc % S;
                const uint32_t u = (uint32_t)(lc / S);
                if (!mbar_wait(&full_a[s], u & 1, abort_flag)) break;
                if (!mbar_wait(&full_b[s], u & 1, abort_flag)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t a0 = smem_u32(A + s * NP * a_bytes), b0 = smem_u32(B + s * NP * b_bytes);
                // products of pieces whose orders sum to at most NP - 1
#pragma unroll
                for (int kk = 0; kk < KC / 16; ++kk) {
                    const uint32_t ko = (uint32_t)kk * 32u;
                    bool first = (lc == 0 && kk == 0);
#pragma unroll
                    for (int pa = 0; pa < NP; ++pa)
#pragma unroll
                        for (int pb = 0; pb + pa < NP; ++pb) {
                            mma_bf16(tmem, sw128_desc(a0 + pa * a_bytes + ko), sw128_desc(b0 + pb * b_bytes + ko), idesc,
                                     first ? 0u : 1u);
                            first = false;
                        }
                }
                mma_commit(&empty[s]);
            }
            mma_commit(acc_done);
            // on abort, drain this thread's MMAs before the CTA releases tensor memory
            if (*abort_flag) mbar_wait_raw(acc_done, 0);
        }
        __syncwarp();
    } else {
        // ------------- Q-tile and source-coordinate producer -----------------
        const uint32_t bytes = NP * b_bytes;
        int issued = 0;
        for (int lc = 0; lc < nch; ++lc) {
            const int s = lc % S;
            const uint32_t u = (uint32_t)(lc / S);
            if (lc >= S && !mbar_wait(&empty[s], (u - 1) & 1, abort_flag)) break;
            if (lane == 0) {
                mbar_arrive_tx(&full_b[s], bytes);
                bulk_g2s(B + s * NP * b_bytes, P.bpack + (size_t)(ch0 + lc) * bytes, bytes, &full_b[s]);
                issued = lc + 1;
            }
            // source coordinates of the chunk, FP32 relative to the tile origin
            float* cs = crd + s * 3 * KC;
            const int64_t j0 = (ch0 + lc) * KC;
#pragma unroll
            for (int h = 0; h < KC / 32; ++h) {
                const int t = lane + 32 * h;
                const int64_t j = j0 + t;
                float x = 1.0e18f, y = 1.0e18f, z = 1.0e18f;  // padded source: G underflows to 0
                if (j < n) {
                    x = (float)(P.g.x[j] - ox); y = (float)(P.g.y[j] - oy); z = (float)(P.g.z[j] - oz);
                }
                cs[t] = x; cs[KC + t] = y; cs[2 * KC + t] = z;
            }
            mbar_arrive(&crd_full[s]);
        }
        // on abort, wait for the copies still in flight (at most one per stage)
        if (lane == 0 && *abort_flag)
            for (int lc = issued > S ? issued - S : 0; lc < issued; ++lc) mbar_wait_raw(&full_b[lc % S], (lc / S) & 1);
        __syncwarp();
    }

    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (*abort_flag && threadIdx.x == 0) atomicOr(P.err, kErrTimeout);
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tcols) : "memory");
    }
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

size_t smem_bytes(int npad, int np) {
    size_t a = (size_t)S * np * M * 128, b = (size_t)S * np * npad * 128;
    size_t c = (size_t)S * 3 * KC * sizeof(float);
    size_t bars = (4 * S + 1) * sizeof(uint64_t) + 16;
    return 1024 + a + b + c + bars;
}

template <int NP>
void launch_tc(const GeomDev& g, const double* X, int ldx, int c0, int kc, const double* pre, int nsplit, int64_t cps,
               double* part, int ldp, uint8_t* bpack, int* err, cudaStream_t s) {
    const int npad = ((kc + 15) / 16) * 16;
    const int64_t nchunks = (g.n + KC - 1) / KC;
    const int64_t pk = nchunks * npad * 8;
    k_pack_q<NP><<<(unsigned)((pk + 255) / 256), 256, 0, s>>>(g, X, ldx, c0, kc, pre, npad, nchunks, bpack);
    BIE_CK(cudaGetLastError());
    Params P;
    P.g = g;
    P.bpack = bpack;
    P.npad = npad;
    P.keff = kc;
    P.nchunks = nchunks;
    P.cps = cps;
    P.part = part;
    P.ldp = ldp;
    P.c0 = c0;
    P.err = err;
    const size_t sm = smem_bytes(npad, NP);
    static size_t configured = 0;
    if (sm > configured) {
        BIE_CK(cudaFuncSetAttribute(k_dt_tc<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        configured = sm;
    }
    dim3 grid((unsigned)((g.n + M - 1) / M), (unsigned)nsplit);
    k_dt_tc<NP><<<grid, NTHREADS, sm, s>>>(P);
    BIE_CK(cudaGetLastError());
}

}  // namespace tc

int tc_npad(int kc) { return ((kc + 15) / 16) * 16; }

// Runs K3 for columns [c0, c0 + kc) (kc <= 256) of X into part[s][i][c0 + c],
// with the kernel and right-hand sides split into `pieces` (2: three products,
// 3: six products) bf16 pieces.
void launch_block_tc(const GeomDev& g, const double* X, int ldx, int c0, int kc, const double* pre, int nsplit,
                     int64_t cps, double* part, int ldp, uint8_t* bpack, int* err, int pieces, cudaStream_t s) {
    if (pieces == 3)
        tc::launch_tc<3>(g, X, ldx, c0, kc, pre, nsplit, cps, part, ldp, bpack, err, s);
    else
        tc::launch_tc<2>(g, X, ldx, c0, kc, pre, nsplit, cps, part, ldp, bpack, err, s);
}

size_t block_tc_pack_bytes(int64_t n, int kc, int pieces) {
    const int64_t nchunks = (n + tc::KC - 1) / tc::KC;
    return (size_t)nchunks * pieces * tc_npad(kc) * 128;
}

int block_tc_ctas_per_sm(int kc, int pieces) {
    const size_t sm = tc::smem_bytes(tc_npad(kc), pieces);
    return std::max(1, (int)((227 * 1024) / (sm + 1024)));
}

}  // namespace bie

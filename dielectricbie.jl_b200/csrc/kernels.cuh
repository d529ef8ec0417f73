// CUDA kernels of the layer-potential hot path (sm_100a).
//
// Device layout: node coordinates, normals and weights as SoA FP64 arrays of
// length N; multi-column vectors node-major (X[i * ldx + c], the k values of
// node i contiguous). Direct sums are split over source chunks; every chunk
// writes an FP64 partial that the combine kernel reduces in a fixed order
// (deterministic, no atomics).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "common.cuh"

namespace bie {

// ---------------------------------------------------------------------------
// K1: FP64 direct D^T sum ("plain").  part[s][i][c0 + c] =
//   sum_{j in chunk s, j != i} n_i.(x_i - y_j) / |x_i - y_j|^3 * w_j * p_j * X[j][c0 + c]
// (the 1/(4 pi) is applied by the combine kernel). p = optional right
// preconditioner (nullptr = 1). Replaces laplace3d_DT (src/kernel/laplace3d.jl:30-40)
// and the lfmm3d pg=2 far field (src/kernel/laplace3d.jl:100-107).
// ---------------------------------------------------------------------------
template <int C>
__global__ void __launch_bounds__(kTB) k_dt_f64(GeomDev g, const double* __restrict__ X, int ldx, int c0,
                                                  const double* __restrict__ pre, int64_t chunk,
                                                  double* __restrict__ part, int ldp) {
    extern __shared__ double sm[];
    double* sx = sm;
    double* sy = sx + kTS;
    double* sz = sy + kTS;
    double* sq = sz + kTS;  // [kTS][C]
    const int64_t i0 = (int64_t)blockIdx.x * kTB;
    const int64_t i = i0 + threadIdx.x;
    const bool valid = i < g.n;
    double xi = 0, yi = 0, zi = 0, n0 = 0, n1 = 0, n2 = 0;
    if (valid) {
        xi = g.x[i]; yi = g.y[i]; zi = g.z[i];
        n0 = g.nx[i]; n1 = g.ny[i]; n2 = g.nz[i];
    }
    double acc[C];
#pragma unroll
    for (int c = 0; c < C; ++c) acc[c] = 0.0;
    const int64_t j0 = (int64_t)blockIdx.y * chunk;
    const int64_t j1 = min(g.n, j0 + chunk);
    for (int64_t jt = j0; jt < j1; jt += kTS) {
        const int cnt = (int)min((int64_t)kTS, j1 - jt);
        __syncthreads();
        for (int t = threadIdx.x; t < cnt; t += kTB) {
            const int64_t j = jt + t;
            sx[t] = g.x[j]; sy[t] = g.y[j]; sz[t] = g.z[j];
            double wj = g.w[j] * (pre ? pre[j] : 1.0);
            const double* xr = X + j * ldx + c0;
#pragma unroll
            for (int c = 0; c < C; ++c) sq[t * C + c] = wj * xr[c];
        }
        __syncthreads();
        const bool self_tile = (jt < i0 + kTB) && (jt + cnt > i0);
        if (!self_tile) {
#pragma unroll 2
            for (int t = 0; t < cnt; ++t) {
                double dx = xi - sx[t], dy = yi - sy[t], dz = zi - sz[t];
                double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
                double ri = rsqrt(r2);
                double nd = fma(n0, dx, fma(n1, dy, n2 * dz));
                double gk = nd * (ri * ri * ri);
#pragma unroll
                for (int c = 0; c < C; ++c) acc[c] = fma(gk, sq[t * C + c], acc[c]);
            }
        } else {
            for (int t = 0; t < cnt; ++t) {
                if (jt + t == i) continue;
                double dx = xi - sx[t], dy = yi - sy[t], dz = zi - sz[t];
                double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
                double ri = rsqrt(r2);
                double nd = fma(n0, dx, fma(n1, dy, n2 * dz));
                double gk = nd * (ri * ri * ri);
#pragma unroll
                for (int c = 0; c < C; ++c) acc[c] = fma(gk, sq[t * C + c], acc[c]);
            }
        }
    }
    if (valid) {
        double* o = part + ((int64_t)blockIdx.y * g.n + i) * ldp + c0;
#pragma unroll
        for (int c = 0; c < C; ++c) o[c] = acc[c];
    }
}

// ---------------------------------------------------------------------------
// K2: FP32 direct D^T sum with FP64 tile partials ("refined" inner operator).
// Targets are taken in the Morton order g.perm (compact tiles); coordinates are
// shifted to the CTA's first target in FP64 before rounding to FP32 (keeps
// near-pair differences accurate), rsqrt runs on the MUFU pipe, each
// shared-memory tile accumulates in FP32 and is folded into FP64.
// ---------------------------------------------------------------------------
template <int C>
__global__ void __launch_bounds__(kTB) k_dt_f32(GeomDev g, const double* __restrict__ X, int ldx, int c0,
                                                  const double* __restrict__ pre, int64_t chunk,
                                                  double* __restrict__ part, int ldp) {
    // Source pairs (t, t + 1) run as packed f32x2 operations. Staged tiles are padded to
    // kTS sources with far-away coordinates and zero values, so pairs never straddle
    // the tile end.
    extern __shared__ __align__(16) float smf[];
    float* sx = smf;
    float* sy = sx + kTS;
    float* sz = sy + kTS;
    float* sq = sz + kTS;  // [C][kTS]: column c of the tile's sources, contiguous
    const int64_t i0 = (int64_t)blockIdx.x * kTB;
    const bool valid = i0 + threadIdx.x < g.n;
    const int64_t i = valid ? (int64_t)g.perm[i0 + threadIdx.x] : g.n;  // original index of the target
    const int64_t io = g.perm[min(i0, g.n - 1)];
    const double ox = g.x[io], oy = g.y[io], oz = g.z[io];
    float xi = -1.0e18f, yi = -1.0e18f, zi = -1.0e18f, n0 = 0.f, n1 = 0.f, n2 = 0.f;
    if (valid) {
        xi = (float)(g.x[i] - ox); yi = (float)(g.y[i] - oy); zi = (float)(g.z[i] - oz);
        n0 = (float)g.nx[i]; n1 = (float)g.ny[i]; n2 = (float)g.nz[i];
    }
    // warp-uniform normal axis: n.(x - y) is then the signed axis difference, the sign
    // applied to the output
    int code = 3;
    float sgn = 1.f;
    if (fabsf(n0) == 1.f && n1 == 0.f && n2 == 0.f) { code = 0; sgn = n0; }
    else if (fabsf(n1) == 1.f && n0 == 0.f && n2 == 0.f) { code = 1; sgn = n1; }
    else if (fabsf(n2) == 1.f && n0 == 0.f && n1 == 0.f) { code = 2; sgn = n2; }
    const int cmin = __reduce_min_sync(0xFFFFFFFFu, valid ? code : 4);
    const int cmax = __reduce_max_sync(0xFFFFFFFFu, valid ? code : -1);
    const int ax = (cmin == cmax && cmin < 3) ? cmin : 3;
    if (ax == 3) sgn = 1.f;
    const float tc[3] = {xi, yi, zi};
    const int a1 = ax < 3 ? ax : 0, a2 = a1 == 2 ? 0 : a1 + 1, a3 = a2 == 2 ? 0 : a2 + 1;
    const float* sA = a1 == 0 ? sx : (a1 == 1 ? sy : sz);
    const float* sB = a2 == 0 ? sx : (a2 == 1 ? sy : sz);
    const float* sC = a3 == 0 ? sx : (a3 == 1 ? sy : sz);
    const uint64_t tA = pk2(tc[a1], tc[a1]), tB = pk2(tc[a2], tc[a2]), tCc = pk2(tc[a3], tc[a3]);
    const uint64_t nA = pk2(n0, n0), nB = pk2(n1, n1), nC = pk2(n2, n2);
    const uint64_t tiny = pk2(1e-24f, 1e-24f);  // keeps the self pair's r^-3 finite: it contributes 0
    double acc[C];
#pragma unroll
    for (int c = 0; c < C; ++c) acc[c] = 0.0;
    const int64_t j0 = (int64_t)blockIdx.y * chunk;
    const int64_t j1 = min(g.n, j0 + chunk);
    for (int64_t jt = j0; jt < j1; jt += kTS) {
        const int cnt = (int)min((int64_t)kTS, j1 - jt);
        __syncthreads();
        for (int t = threadIdx.x; t < kTS; t += kTB) {
            if (t < cnt) {
                const int64_t j = jt + t;
                sx[t] = (float)(g.x[j] - ox); sy[t] = (float)(g.y[j] - oy); sz[t] = (float)(g.z[j] - oz);
                const double wj = g.w[j] * (pre ? pre[j] : 1.0);
                const double* xr = X + j * ldx + c0;
#pragma unroll
                for (int c = 0; c < C; ++c) sq[c * kTS + t] = (float)(wj * xr[c]);
            } else {
                sx[t] = sy[t] = sz[t] = 1.0e18f;
#pragma unroll
                for (int c = 0; c < C; ++c) sq[c * kTS + t] = 0.f;
            }
        }
        __syncthreads();
        uint64_t a2c[C];
#pragma unroll
        for (int c = 0; c < C; ++c) a2c[c] = 0ull;
        const int cnt2 = (cnt + 1) & ~1;
        if (ax < 3) {
#pragma unroll 4
            for (int t = 0; t < cnt2; t += 2) {
                const uint64_t da = sub2(tA, *reinterpret_cast<const uint64_t*>(sA + t));
                const uint64_t db = sub2(tB, *reinterpret_cast<const uint64_t*>(sB + t));
                const uint64_t dc = sub2(tCc, *reinterpret_cast<const uint64_t*>(sC + t));
                const float2 r2 = upk2(fma2(da, da, fma2(db, db, fma2(dc, dc, tiny))));
                const uint64_t ri = pk2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
                const uint64_t gk = mul2(mul2(da, ri), mul2(ri, ri));
#pragma unroll
                for (int c = 0; c < C; ++c)
                    a2c[c] = fma2(gk, *reinterpret_cast<const uint64_t*>(sq + c * kTS + t), a2c[c]);
            }
        } else {
#pragma unroll 4
            for (int t = 0; t < cnt2; t += 2) {
                const uint64_t dx = sub2(tA, *reinterpret_cast<const uint64_t*>(sx + t));
                const uint64_t dy = sub2(tB, *reinterpret_cast<const uint64_t*>(sy + t));
                const uint64_t dz = sub2(tCc, *reinterpret_cast<const uint64_t*>(sz + t));
                const float2 r2 = upk2(fma2(dx, dx, fma2(dy, dy, fma2(dz, dz, tiny))));
                const uint64_t ri = pk2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
                const uint64_t nd = fma2(nA, dx, fma2(nB, dy, mul2(nC, dz)));
                const uint64_t gk = mul2(mul2(nd, ri), mul2(ri, ri));
#pragma unroll
                for (int c = 0; c < C; ++c)
                    a2c[c] = fma2(gk, *reinterpret_cast<const uint64_t*>(sq + c * kTS + t), a2c[c]);
            }
        }
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const float2 s2 = upk2(a2c[c]);
            acc[c] += (double)s2.x + (double)s2.y;
        }
    }
    if (valid) {
        double* o = part + ((int64_t)blockIdx.y * g.n + i) * ldp + c0;
#pragma unroll
        for (int c = 0; c < C; ++c) o[c] = (double)sgn * acc[c];
    }
}

// ---------------------------------------------------------------------------
// K6: single-layer potential at targets (FP64):
//   phi[m][c] = (1/4pi) sum_j w_j S[j][c] / |x_m - y_j|   (laplace3d_pottrg,
//   src/kernel/laplace3d.jl:69-82). One chunk of sources per blockIdx.y.
// ---------------------------------------------------------------------------
template <int C>
__global__ void __launch_bounds__(kTB) k_pot_f64(GeomDev g, const double* __restrict__ S, int lds, int c0,
                                                   const double* __restrict__ T /*3 x M*/, int64_t M,
                                                   int64_t chunk, double* __restrict__ part, int ldp) {
    extern __shared__ double sm[];
    double* sx = sm;
    double* sy = sx + kTS;
    double* sz = sy + kTS;
    double* sq = sz + kTS;
    const int64_t m = (int64_t)blockIdx.x * kTB + threadIdx.x;
    const bool valid = m < M;
    double xm = 0, ym = 0, zm = 0;
    if (valid) { xm = T[3 * m]; ym = T[3 * m + 1]; zm = T[3 * m + 2]; }
    double acc[C];
#pragma unroll
    for (int c = 0; c < C; ++c) acc[c] = 0.0;
    const int64_t j0 = (int64_t)blockIdx.y * chunk;
    const int64_t j1 = min(g.n, j0 + chunk);
    for (int64_t jt = j0; jt < j1; jt += kTS) {
        const int cnt = (int)min((int64_t)kTS, j1 - jt);
        __syncthreads();
        for (int t = threadIdx.x; t < cnt; t += kTB) {
            const int64_t j = jt + t;
            sx[t] = g.x[j]; sy[t] = g.y[j]; sz[t] = g.z[j];
            const double* sr = S + j * lds + c0;
#pragma unroll
            for (int c = 0; c < C; ++c) sq[t * C + c] = g.w[j] * sr[c];
        }
        __syncthreads();
        for (int t = 0; t < cnt; ++t) {
            double dx = xm - sx[t], dy = ym - sy[t], dz = zm - sz[t];
            double ri = rsqrt(fma(dx, dx, fma(dy, dy, dz * dz)));
#pragma unroll
            for (int c = 0; c < C; ++c) acc[c] = fma(ri, sq[t * C + c], acc[c]);
        }
    }
    if (valid) {
        double* o = part + ((int64_t)blockIdx.y * M + m) * ldp + c0;
#pragma unroll
        for (int c = 0; c < C; ++c) o[c] = acc[c];
    }
}

// out[m][c] = scale * sum_s part[s][m][c]
__global__ void k_reduce_parts(const double* __restrict__ part, int nsplit, int64_t rows, int k, double scale,
                               double* __restrict__ out) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t tot = rows * k;
    if (e >= tot) return;
    double s = 0.0;
    for (int p = 0; p < nsplit; ++p) s += part[(int64_t)p * tot + e];
    out[e] = s * scale;
}

// ---------------------------------------------------------------------------
// K4 + K5: combine. Y[i][c] = (1/4pi) sum_s part[s][i][c]       (far field)
//                          + sum_{blocks (P, Q)} B[r, :] . (p X)[Q rows][c]   (near corrections)
//                          + t_i p_i X[i][c]                      (diagonal contrast)
// i = P * nb + r. BSR blocks column-major (val[b*nb*nb + s*nb + r]).
// Replaces corrections * x (src/kernel/laplace3d_near.jl:417) and the glue loop
// of mul!(Y, ::BatchedDielectricOperator, X) (src/solver/multi_rhs.jl:120-128).
// One thread per output; threads of a warp cover consecutive (i, c).
// ---------------------------------------------------------------------------
template <typename TP>
__global__ void k_combine(int64_t n, int k, const TP* __restrict__ part, int nsplit,
                          const double* __restrict__ X, int ldx, const double* __restrict__ pre,
                          const double* __restrict__ diag, const int32_t* __restrict__ rowptr,
                          const int32_t* __restrict__ col, const double* __restrict__ val, int nb,
                          double* __restrict__ Y, int ldy) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * k) return;
    int64_t i = e / k;
    int c = (int)(e - i * k);
    double s = 0.0;
    const int64_t tot = n * (int64_t)k;
    for (int p = 0; p < nsplit; ++p) s += (double)part[(int64_t)p * tot + e];
    s *= kInv4Pi;
    if (val) {
        int64_t P = i / nb;
        int r = (int)(i - P * nb);
        double a = 0.0;
        for (int b = rowptr[P]; b < rowptr[P + 1]; ++b) {
            const double* vb = val + (int64_t)b * nb * nb + r;
            int64_t base = (int64_t)col[b] * nb;
            if (pre) {
                for (int q = 0; q < nb; ++q) a = fma(vb[(int64_t)q * nb], pre[base + q] * X[(base + q) * ldx + c], a);
            } else {
                for (int q = 0; q < nb; ++q) a = fma(vb[(int64_t)q * nb], X[(base + q) * ldx + c], a);
            }
        }
        s += a;
    }
    if (diag) s += diag[i] * (pre ? pre[i] : 1.0) * X[i * ldx + c];
    Y[i * ldy + c] = s;
}

// K4 + K5, block-row form: one CTA per target panel P (nb consecutive rows).
// Each block (P, Q) of the row is staged once in shared memory together with the
// nb x kt slab of (p X)[Q rows] it multiplies, so block values and source slabs
// are read once per panel instead of once per output. Thread t owns column
// c = t % kt and the rows [g R, g R + R) of group g = t / kt: every slab value it
// loads feeds R FMAs, and the R block values are warp-wide broadcasts. Then
//   Y[i][c] = (1/4pi) sum_s part[s][i][c] + sum_b B . (p X) + t_i p_i X[i][c].
// ---------------------------------------------------------------------------
// K4 (block-row form): one CTA per (target panel P, 32-column tile). The BSR
// blocks of the panel's row, C_b (nb x nb, column-major), multiply the slabs
// p .* X[source panel of b] on the FP64 tensor path (mma.sync m8n8k4 f64; a
// warp owns one 8-column n-tile and the panel's MT 8-row m-tiles); blocks and
// slabs are double-buffered in shared memory by cp.async. The epilogue adds the
// split partials (times 1/(4 pi)) and the diagonal term:
//   Y[i][c] = (1/4pi) sum_s part[s][i][c] + sum_b (C_b (p X)[col_b])[i][c] + t_i p_i X[i][c]
// Replaces the CSC SpMV / sparse mat-mat of laplace3d_DT_fmm3d_corrected and
// BatchedDielectricOperator (src/kernel/laplace3d_near.jl:395-419,
// src/solver/multi_rhs.jl:103-136).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

constexpr int kCombTile = 32;  // columns per CTA

// Slab row stride for a kt-column tile: kt rounded up to 8, plus 4 (stride = 4 or 12
// mod 16 doubles, so a half-warp's fragment loads hit distinct banks).
__host__ __device__ inline int comb_ldx(int kt) { return ((kt + 7) / 8) * 8 + 4; }

// Shared memory of the block-row combine for nb-row panels, kt-column tiles and
// `stages` pipeline stages (reused for the warps' final reduction).
inline size_t combine_smem_bytes(int nb, int kt, int stages) {
    const int mt = (nb + 7) / 8, kp = ((nb + 3) / 4) * 4;
    const int ldc = mt * 8 + 4;
    const size_t pipe = (size_t)stages * kp * (ldc + comb_ldx(kt) + 1);
    const size_t red = (size_t)4 * mt * 2 * 32;  // cross-warp reduction of the accumulators
    return sizeof(double) * std::max(pipe, red);
}

// With gsum != nullptr the panel's block list is split into groups of bpg blocks
// (blockIdx.z = group) and each group writes its block sum to gsum[z][i][c]; the
// reduction over groups, split partials and diagonal is then k_combine_groups.
template <int MT, int NST, typename TP>
__global__ void __launch_bounds__(128) k_combine_dmma(int64_t n, int k, const TP* __restrict__ part, int nsplit,
                                                      const double* __restrict__ X, const double* __restrict__ pre,
                                                      const double* __restrict__ diag,
                                                      const int32_t* __restrict__ rowptr,
                                                      const int32_t* __restrict__ col,
                                                      const double* __restrict__ val, int nb,
                                                      double* __restrict__ Y, int bpg, double* __restrict__ gsum) {
    // column stride of a staged block: MT * 8 rows + 4 (= 4 or 12 mod 16 doubles)
    constexpr int LDC = MT * 8 + 4;
    const int c0 = blockIdx.y * kCombTile;
    const int kt = min(kCombTile, k - c0);
    const int LDX = comb_ldx(kt);
    const int KS = (nb + 3) / 4, KP = KS * 4;
    const int SSTR = KP * (LDC + LDX + 1);  // doubles per pipeline stage
    extern __shared__ __align__(16) double smd[];
    // stage t: sC = smd + t SSTR ([KP][LDC], sC[q LDC + r] = C_b[r][q]),
    //          sX = sC + KP LDC ([KP][LDX], sX[q LDX + cc] = X[col_b nb + q][c0 + cc]),
    //          sP = sX + KP LDX ([KP] preconditioner of the slab rows)
    const int P = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t row0 = (int64_t)P * nb;
    int b0 = val ? rowptr[P] : 0, b1 = val ? rowptr[P + 1] : 0;
    if (gsum) {
        b0 += (int)blockIdx.z * bpg;
        b1 = min(b1, b0 + bpg);
    }
    // padding rows/columns stay zero: the copies below write only the live part
    for (int e = threadIdx.x; e < NST * SSTR; e += blockDim.x) smd[e] = 0.0;
    __syncthreads();

    const bool v16 = (nb & 1) == 0;  // 16-byte copies of block columns (the blocks are 16-byte aligned)
    const bool x16 = (k & 1) == 0 && (kt & 1) == 0 &&  // and of slab rows (c0 is even)
                     (reinterpret_cast<uintptr_t>(X) & 15) == 0;
    auto issue = [&](int b, int st) {
        const double* vb = val + (int64_t)b * nb * nb;
        double* dC = smd + st * SSTR;
        if (v16) {
            const int h = nb >> 1;
            for (int e = threadIdx.x; e < nb * h; e += blockDim.x) {
                const int q = e / h, r = (e - q * h) * 2;
                cp_async16(dC + q * LDC + r, vb + q * nb + r);
            }
        } else {
            for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
                const int q = e / nb, r = e - q * nb;
                cp_async8(dC + q * LDC + r, vb + q * nb + r);
            }
        }
        const int64_t base = (int64_t)col[b] * nb;
        double* dX = dC + KP * LDC;
        if (x16) {
            const int h = kt >> 1;
            for (int e = threadIdx.x; e < nb * h; e += blockDim.x) {
                const int q = e / h, cc = (e - q * h) * 2;
                cp_async16(dX + q * LDX + cc, X + (base + q) * k + c0 + cc);
            }
        } else {
            for (int e = threadIdx.x; e < nb * kt; e += blockDim.x) {
                const int q = e / kt, cc = e - q * kt;
                cp_async8(dX + q * LDX + cc, X + (base + q) * k + c0 + cc);
            }
        }
        if (pre)
            for (int q = threadIdx.x; q < nb; q += blockDim.x) cp_async8(dX + KP * LDX + q, pre + base + q);
    };

    // warps to (n-tile, k-step subset): with fewer than four n-tiles the warps sharing an
    // n-tile split the block's k-steps (each keeps all MT accumulator chains busy) and
    // their partial sums are added through shared memory at the end
    const int ntiles = (kt + 7) / 8;
    const int nw = ntiles >= 4 ? 4 : ntiles;  // distinct n-tiles in use
    const int ksplit = 4 / nw;                // 1, 2 or 4 (nw = 3: one warp idle)
    const int nt = warp % nw, kq = warp / nw;
    const bool wact = kq < ksplit;
    double acc[MT][2];
#pragma unroll
    for (int m = 0; m < MT; ++m) acc[m][0] = acc[m][1] = 0.0;

    // NST-stage pipeline: blocks b .. b + NST - 2 are in flight while block b is used;
    // one (possibly empty) copy group is committed per step so the group count is uniform
#pragma unroll
    for (int t = 0; t < NST - 1; ++t) {
        if (b0 + t < b1) issue(b0 + t, t);
        cp_async_commit();
    }
    for (int b = b0; b < b1; ++b) {
        const int st = (b - b0) % NST;
        cp_async_wait<NST - 2>();
        __syncthreads();  // block b landed for all threads; stage (b - 1) % NST is free
        if (b + NST - 1 < b1) issue(b + NST - 1, (b - b0 + NST - 1) % NST);
        cp_async_commit();
        if (wact) {
            const double* cC = smd + st * SSTR + (lane >> 2);
            const double* cX = smd + st * SSTR + KP * LDC + 8 * nt + (lane >> 2);
            const double* cP = smd + st * SSTR + KP * LDC + KP * LDX;
            for (int ks = kq; ks < KS; ks += ksplit) {
                const int q = 4 * ks + (lane & 3);
                double bv = cX[q * LDX];
                if (pre) bv *= cP[q];
#pragma unroll
                for (int m = 0; m < MT; ++m) dmma884(acc[m][0], acc[m][1], cC[q * LDC + 8 * m], bv);
            }
        }
    }
    cp_async_wait<0>();
    if (ksplit > 1) {
        // add the k-step partial sums of the warps sharing an n-tile (stage memory reused)
        __syncthreads();
        double* red = smd;  // [warp][MT][2][32]
        if (wact && kq > 0)
#pragma unroll
            for (int m = 0; m < MT; ++m) {
                red[((warp * MT + m) * 2 + 0) * 32 + lane] = acc[m][0];
                red[((warp * MT + m) * 2 + 1) * 32 + lane] = acc[m][1];
            }
        __syncthreads();
        if (wact && kq == 0)
            for (int o = 1; o < ksplit; ++o) {
                const int w2 = nt + o * nw;
#pragma unroll
                for (int m = 0; m < MT; ++m) {
                    acc[m][0] += red[((w2 * MT + m) * 2 + 0) * 32 + lane];
                    acc[m][1] += red[((w2 * MT + m) * 2 + 1) * 32 + lane];
                }
            }
    }

    if (!wact || kq > 0) return;
    const int64_t tot = n * (int64_t)k;
#pragma unroll
    for (int m = 0; m < MT; ++m) {
        const int r = 8 * m + (lane >> 2);
        if (r >= nb) continue;
        const int64_t i = row0 + r;
        const double dgi = diag ? diag[i] * (pre ? pre[i] : 1.0) : 0.0;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int c = c0 + 8 * nt + 2 * (lane & 3) + h;
            if (c >= c0 + kt) continue;
            const int64_t e = i * k + c;
            if (gsum) {
                gsum[(int64_t)blockIdx.z * tot + e] = acc[m][h];
                continue;
            }
            double sp = 0.0;
            for (int p = 0; p < nsplit; ++p) sp += (double)part[(int64_t)p * tot + e];
            double y = sp * kInv4Pi + acc[m][h];
            if (diag) y += dgi * X[e];
            Y[e] = y;
        }
    }
}

// Y[e] = sum_z gsum[z][e] + (1/4pi) sum_s part[s][e] + t_i p_i X[e], e = i k + c.
template <typename TP>
__global__ void k_combine_groups(int64_t n, int k, const double* __restrict__ gsum, int ngroups,
                                 const TP* __restrict__ part, int nsplit, const double* __restrict__ X,
                                 const double* __restrict__ pre, const double* __restrict__ diag,
                                 double* __restrict__ Y) {
    const int64_t tot = n * (int64_t)k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        double a = 0.0;
        for (int z = 0; z < ngroups; ++z) a += gsum[(int64_t)z * tot + e];
        double sp = 0.0;
        for (int p = 0; p < nsplit; ++p) sp += (double)part[(int64_t)p * tot + e];
        double y = sp * kInv4Pi + a;
        if (diag) {
            const int64_t i = e / k;
            y += diag[i] * (pre ? pre[i] : 1.0) * X[e];
        }
        Y[e] = y;
    }
}

// ---------------------------------------------------------------------------
// K8: point-source right-hand sides (src/solver/dielectric_box3d.jl:95-104):
//   F[i][c] = -q_c n_i.(x_i - s_c) / (4 pi |x_i - s_c|^3) / eps_c
// ---------------------------------------------------------------------------
__global__ void k_rhs_point(GeomDev g, const double* __restrict__ src /*3 x k*/, const double* __restrict__ q,
                            const double* __restrict__ eps, int k, double* __restrict__ F) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= g.n * k) return;
    int64_t i = e / k;
    int c = (int)(e - i * k);
    double dx = g.x[i] - src[3 * c], dy = g.y[i] - src[3 * c + 1], dz = g.z[i] - src[3 * c + 2];
    double r2 = dx * dx + dy * dy + dz * dz;
    double ri = 1.0 / sqrt(r2);
    double nd = g.nx[i] * dx + g.ny[i] * dy + g.nz[i] * dz;
    F[e] = -q[c] * (nd * ri * ri * ri * kInv4Pi) / eps[c];
}

// ---------------------------------------------------------------------------
// Layout conversion between Julia's column-major N x k and node-major.
// ---------------------------------------------------------------------------
__global__ void k_colmajor_to_nodemajor(const double* __restrict__ A, int64_t n, int k, double* __restrict__ B) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * k) return;
    int64_t i = e / k;
    int c = (int)(e - i * k);
    B[e] = A[(int64_t)c * n + i];
}
__global__ void k_nodemajor_to_colmajor(const double* __restrict__ B, int64_t n, int k, double* __restrict__ A) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * k) return;
    int c = (int)(e / n);
    int64_t i = e - (int64_t)c * n;
    A[e] = B[i * k + c];
}

// ---------------------------------------------------------------------------
// K7: device GMRES building blocks (FP64). Multi-column vectors node-major
// (n x k); each of the k columns runs its own Arnoldi process.
// ---------------------------------------------------------------------------
// Column dot products, one CTA per (row block, vector v): partial[blk][v][c] = sum over
// the block's rows of A_v[i][c] B[i][c], A_v = A + v * strideA. blockDim.x = k * groups
// (groups a power of two): thread t owns column t % k and every groups-th row.
__global__ void k_dots_blk(const double* __restrict__ A, int64_t strideA, int nv, const double* __restrict__ B,
                           int64_t n, int k, int64_t rows_per_blk, double* __restrict__ partial) {
    extern __shared__ double red[];
    const int groups = blockDim.x / k;
    const int c = threadIdx.x % k, grp = threadIdx.x / k;
    const int v = blockIdx.y;
    const double* Av = A + (int64_t)v * strideA;
    const int64_t r0 = (int64_t)blockIdx.x * rows_per_blk;
    const int64_t r1 = min(n, r0 + rows_per_blk);
    double sacc = 0.0;
    for (int64_t r = r0 + grp; r < r1; r += groups) sacc = fma(Av[r * k + c], B[r * k + c], sacc);
    red[threadIdx.x] = sacc;
    __syncthreads();
    for (int h = groups / 2; h > 0; h >>= 1) {
        if (threadIdx.x < (unsigned)(h * k)) red[threadIdx.x] += red[threadIdx.x + h * k];
        __syncthreads();
    }
    if (threadIdx.x < (unsigned)k)
        partial[(int64_t)blockIdx.x * nv * k + (int64_t)v * k + threadIdx.x] = red[threadIdx.x];
}

// W[i][c] -= sum_{v < nv} V_v[i][c] h[v][c], then partial[blk][c] = sum over the block's
// rows of W[i][c]^2 (the second Gram-Schmidt pass fused with the column norm).
__global__ void k_gs_update_norm(double* __restrict__ W, const double* __restrict__ V, int64_t strideV, int nv,
                                 const double* __restrict__ h, int64_t n, int k, int64_t rows_per_blk,
                                 double* __restrict__ partial) {
    extern __shared__ double red[];
    const int groups = blockDim.x / k;
    const int c = threadIdx.x % k, grp = threadIdx.x / k;
    const int64_t r0 = (int64_t)blockIdx.x * rows_per_blk;
    const int64_t r1 = min(n, r0 + rows_per_blk);
    double sacc = 0.0;
    if (grp < groups)
        for (int64_t r = r0 + grp; r < r1; r += groups) {
            const int64_t e = r * k + c;
            double w = W[e];
            for (int v = 0; v < nv; ++v) w = fma(-V[(int64_t)v * strideV + e], h[v * k + c], w);
            W[e] = w;
            sacc = fma(w, w, sacc);
        }
    red[threadIdx.x] = sacc;
    __syncthreads();
    for (int hh = groups / 2; hh > 0; hh >>= 1) {
        if (threadIdx.x < (unsigned)(hh * k)) red[threadIdx.x] += red[threadIdx.x + hh * k];
        __syncthreads();
    }
    if (threadIdx.x < (unsigned)k) partial[(int64_t)blockIdx.x * k + threadIdx.x] = red[threadIdx.x];
}

// out[e] = sum_blk partial[blk][e] for e < nout, in a fixed order (8 outputs x 32 block
// subsets per CTA); mode 0: assign, 1: accumulate, 2: assign the square root.
__global__ void __launch_bounds__(256) k_dots_finish(const double* __restrict__ partial, int nblk, int64_t nout,
                                                     double* __restrict__ out, int mode) {
    __shared__ double red[32][8];
    const int o = threadIdx.x & 7, sub = threadIdx.x >> 3;
    const int64_t e = (int64_t)blockIdx.x * 8 + o;
    double sacc = 0.0;
    if (e < nout)
        for (int b = sub; b < nblk; b += 32) sacc += partial[(int64_t)b * nout + e];
    red[sub][o] = sacc;
    __syncthreads();
    if (threadIdx.x < 8 && e < nout) {
        double t = 0.0;
        for (int q = 0; q < 32; ++q) t += red[q][o];
        out[e] = mode == 1 ? out[e] + t : (mode == 2 ? sqrt(t) : t);
    }
}

// W[i][c] -= sum_{v < nv} V_v[i][c] h[v][c]
__global__ void k_gs_update(double* __restrict__ W, const double* __restrict__ V, int64_t strideV, int nv,
                            const double* __restrict__ h, int64_t n, int k) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * k) return;
    int c = (int)(e % k);
    double s = W[e];
    for (int v = 0; v < nv; ++v) s = fma(-V[(int64_t)v * strideV + e], h[v * k + c], s);
    W[e] = s;
}

// Y[i][c] = X[i][c] * f[c]; f[c] = 0 where den[c] == 0 (breakdown guard), else num[c] / den[c]
__global__ void k_scale_cols(const double* __restrict__ X, const double* __restrict__ den, int64_t n, int k,
                             double* __restrict__ Y) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * k) return;
    int c = (int)(e % k);
    double d = den[c];
    Y[e] = d > 0.0 ? X[e] / d : 0.0;
}

// Y[i][c] = a * X[i][c] + b * Y[i][c] (column mask: only where mask[c] != 0 when mask given)
__global__ void k_axpby(double a, const double* __restrict__ X, double b, double* __restrict__ Y, int64_t n, int k,
                        const int* __restrict__ mask) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * k) return;
    if (mask && !mask[e % k]) return;
    Y[e] = a * X[e] + b * Y[e];
}

// Givens step of iteration j for every active column (one thread per column).
// R: [(m+1) x (m+1) x k] column j holds h[0..j+1]; cs/sn: [m x k]; gv: [(m+1) x k].
__global__ void k_givens(double* __restrict__ R, const double* __restrict__ h /*[(j+1) x k]*/,
                         const double* __restrict__ h2 /*[(j+1) x k], second Gram-Schmidt pass, or null*/,
                         const double* __restrict__ hnorm /*[k]*/, double* __restrict__ cs, double* __restrict__ sn,
                         double* __restrict__ gv, int* __restrict__ active, int* __restrict__ jlast,
                         const double* __restrict__ eps, double* __restrict__ resid, int j, int m1, int k) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= k) return;
    if (!active[c]) return;
    double* Rj = R + ((int64_t)j * m1) * k;  // column j: Rj[i * k + c]
    for (int i = 0; i <= j; ++i) Rj[i * k + c] = h[i * k + c] + (h2 ? h2[i * k + c] : 0.0);
    Rj[(j + 1) * k + c] = hnorm[c];
    for (int i = 0; i < j; ++i) {
        double a = Rj[i * k + c], b = Rj[(i + 1) * k + c];
        double ci = cs[i * k + c], si = sn[i * k + c];
        Rj[i * k + c] = ci * a + si * b;
        Rj[(i + 1) * k + c] = -si * a + ci * b;
    }
    double a = Rj[j * k + c], b = Rj[(j + 1) * k + c];
    double r = hypot(a, b);
    double cj = r > 0 ? a / r : 1.0, sj = r > 0 ? b / r : 0.0;
    cs[j * k + c] = cj; sn[j * k + c] = sj;
    Rj[j * k + c] = r; Rj[(j + 1) * k + c] = 0.0;
    double gj = gv[j * k + c];
    gv[(j + 1) * k + c] = -sj * gj;
    gv[j * k + c] = cj * gj;
    double res = fabs(gv[(j + 1) * k + c]);
    resid[c] = res;
    jlast[c] = j + 1;
    if (res <= eps[c] || hnorm[c] == 0.0) active[c] = 0;
}

// y = R^{-1} g for each column over its own jlast[c] (one thread per column).
__global__ void k_backsolve(const double* __restrict__ R, const double* __restrict__ gv, const int* __restrict__ jlast,
                            int m1, int k, double* __restrict__ y) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= k) return;
    int n = jlast[c];
    for (int i = n - 1; i >= 0; --i) {
        double s = gv[i * k + c];
        for (int l = i + 1; l < n; ++l) s -= R[((int64_t)l * m1 + i) * k + c] * y[l * k + c];
        double d = R[((int64_t)i * m1 + i) * k + c];
        y[i * k + c] = d != 0.0 ? s / d : 0.0;
    }
    for (int i = n; i < m1; ++i) y[i * k + c] = 0.0;
}

// Coefficients of each column's GMRES residual in its basis: with n = jlast[c] and the
// rotations G_i of k_givens, r - A u = V (beta e_1 - H y) = V G_0^T .. G_{n-1}^T (gv[n] e_n),
// formed by undoing the rotations in reverse; z (m1 x k) receives them (zero above n).
__global__ void k_givens_resid(const double* __restrict__ gv, const double* __restrict__ cs,
                               const double* __restrict__ sn, const int* __restrict__ jlast, int m1, int k,
                               double* __restrict__ z) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= k) return;
    const int n = jlast[c];
    for (int i = 0; i < m1; ++i) z[i * k + c] = 0.0;
    z[n * k + c] = gv[n * k + c];
    for (int i = n - 1; i >= 0; --i) {
        const double a = z[i * k + c], b = z[(i + 1) * k + c], ci = cs[i * k + c], si = sn[i * k + c];
        z[i * k + c] = ci * a - si * b;
        z[(i + 1) * k + c] = si * a + ci * b;
    }
}

// out[i][c] = sum over v <= jlast[c] of z[v][c] V_v[i][c] (terms with z = 0 skipped, so a
// direction left undefined by a breakdown does not enter)
__global__ void k_basis_combine(double* __restrict__ out, const double* __restrict__ V, int64_t strideV,
                                const double* __restrict__ z, const int* __restrict__ jlast, int64_t n, int k) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * k) return;
    const int c = (int)(e % k);
    const int nv = jlast[c] + 1;
    double s = 0.0;
    for (int v = 0; v < nv; ++v) {
        const double zv = z[v * k + c];
        if (zv != 0.0) s = fma(zv, V[(int64_t)v * strideV + e], s);
    }
    out[e] = s;
}

// X[i][c] += p_i * sum_{v < jlast[c]} y[v][c] V_v[i][c]
__global__ void k_update_solution(double* __restrict__ X, const double* __restrict__ V, int64_t strideV,
                                  const double* __restrict__ y, const int* __restrict__ jlast, int jmax,
                                  const double* __restrict__ pre, int64_t n, int k) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * k) return;
    int c = (int)(e % k);
    int nv = min(jlast[c], jmax);
    double s = 0.0;
    for (int v = 0; v < nv; ++v) s = fma(y[v * k + c], V[(int64_t)v * strideV + e], s);
    if (pre) s *= pre[e / k];
    X[e] += s;
}

}  // namespace bie

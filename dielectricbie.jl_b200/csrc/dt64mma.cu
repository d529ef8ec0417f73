// K1 for k >= 8 right-hand sides: FP64 direct D^T sum whose RHS contraction runs
// on the FP64 tensor-core path (mma.sync m8n8k4 f64), the plain path of the
// solver (FP64 end to end).
//
//   part[s][i][c0 + c] = sum_{j in split s, j != i} n_i.(x_i - y_j)/|x_i - y_j|^3 Q(j, c)
//   Q(j, c) = w_j p_j X[j][c0 + c]
//
// Same operator as laplace3d_DT (src/kernel/laplace3d.jl:30-40) / lfmm3d pg=2
// (src/kernel/laplace3d.jl:100-107); the 1/(4 pi) is applied by the combine.
//
// CTA = 4 warps = 64 targets; a warp owns 16 targets (MTW = 2 8-row m-tiles) and NC
// columns (NC/8 n-tiles). Two m-tiles per warp keep the accumulators at 2 x NC
// doubles, so three CTAs fit per SM (measured 10 % faster at NC = 64 than four m-tiles
// per warp at two CTAs per SM; FP64 MMA and FP64 FMA share one throughput budget, and
// more resident warps overlap the kernel-value generation with the MMAs). Per k-step of 4 sources each thread generates the four
// FP64 kernel values of its A fragments (target = m-tile row l/4, source = l%4)
// and loads its B fragments (source l%4, column l/4 of each n-tile) from shared
// memory; 4 x NC/8 DMMAs follow. Box faces are axis-aligned, so a warp whose 32
// targets share a normal axis forms n.(x - y) as the signed axis difference and
// folds the sign into its output.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "common.cuh"
#include "solver.h"

namespace bie {
namespace d64 {

constexpr int MTW = 2;  // m-tiles per warp
constexpr int NTHR = 128;  // threads per CTA
constexpr int TB = 32 * MTW;   // targets per CTA
constexpr int TSRC = 32;  // sources per shared-memory tile

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <int AX>
__device__ __forceinline__ double kernel_val(double tx, double ty, double tz, double n0, double n1, double n2,
                                             double sx, double sy, double sz) {
    const double dx = tx - sx, dy = ty - sy, dz = tz - sz;
    const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
    const double ri = rsqrt(r2);
    double dn;
    if (AX == 0) dn = dx;
    else if (AX == 1) dn = dy;
    else if (AX == 2) dn = dz;
    else dn = fma(n0, dx, fma(n1, dy, n2 * dz));
    return (dn * ri) * (ri * ri);
}

template <int NC, int AX>
__device__ __forceinline__ void tile_step(const double* __restrict__ ssx, const double* __restrict__ ssy,
                                          const double* __restrict__ ssz, const double* __restrict__ sq, int cnt,
                                          const double (&tx)[MTW], const double (&ty)[MTW], const double (&tz)[MTW],
                                          const double (&tn)[MTW][3], double (&acc)[MTW][NC / 8][2], int lane,
                                          bool self, int64_t jt, const int64_t (&ti)[MTW]) {
    constexpr int LDQ = NC + 4;
    const int kq = lane & 3, grp = lane >> 2;
#pragma unroll 2
    for (int k0 = 0; k0 < cnt; k0 += 4) {
        const int j = k0 + kq;
        const double sx = ssx[j], sy = ssy[j], sz = ssz[j];
        double a[MTW];
#pragma unroll
        for (int mt = 0; mt < MTW; ++mt) {
            a[mt] = kernel_val<AX>(tx[mt], ty[mt], tz[mt], tn[mt][0], tn[mt][1], tn[mt][2], sx, sy, sz);
            if (self && jt + j == ti[mt]) a[mt] = 0.0;
        }
        if (j >= cnt) {
#pragma unroll
            for (int mt = 0; mt < MTW; ++mt) a[mt] = 0.0;
        }
        double b[NC / 8];
#pragma unroll
        for (int nt = 0; nt < NC / 8; ++nt) b[nt] = sq[j * LDQ + nt * 8 + grp];
#pragma unroll
        for (int mt = 0; mt < MTW; ++mt)
#pragma unroll
            for (int nt = 0; nt < NC / 8; ++nt) dmma(acc[mt][nt][0], acc[mt][nt][1], a[mt], b[nt]);
    }
}

template <int NC>
__global__ void __launch_bounds__(NTHR, 3) k_dt_f64_mma(GeomDev g, const double* __restrict__ X, int ldx, int c0,
                                                     int kc, const double* __restrict__ pre, int64_t chunk,
                                                     double* __restrict__ part, int ldp) {
    // padded row of NC + 4 doubles (4 mod 16): the four k-rows a half-warp's B-fragment
    // load touches fall on distinct banks
    constexpr int LDQ = NC + 4;
    __shared__ double ssx[TSRC + 4], ssy[TSRC + 4], ssz[TSRC + 4];
    __shared__ double sq[(TSRC + 4) * LDQ];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane >> 2, kq = lane & 3;
    const int64_t i0 = (int64_t)blockIdx.x * TB;
    const int64_t wbase = i0 + warp * 8 * MTW;
    // the warp's 8 MTW targets: m-tile mt, row grp -> target wbase + 8 mt + grp
    double tx[MTW], ty[MTW], tz[MTW], tn[MTW][3];
    int64_t ti[MTW];
    int code_min = 4, code_max = -1;
#pragma unroll
    for (int mt = 0; mt < MTW; ++mt) {
        const int64_t i = wbase + mt * 8 + grp;
        ti[mt] = i;
        if (i < g.n) {
            tx[mt] = g.x[i]; ty[mt] = g.y[i]; tz[mt] = g.z[i];
            tn[mt][0] = g.nx[i]; tn[mt][1] = g.ny[i]; tn[mt][2] = g.nz[i];
            int code = 3;
            if (fabs(tn[mt][0]) == 1.0 && tn[mt][1] == 0.0 && tn[mt][2] == 0.0) code = 0;
            else if (fabs(tn[mt][1]) == 1.0 && tn[mt][0] == 0.0 && tn[mt][2] == 0.0) code = 1;
            else if (fabs(tn[mt][2]) == 1.0 && tn[mt][0] == 0.0 && tn[mt][1] == 0.0) code = 2;
            code_min = min(code_min, code);
            code_max = max(code_max, code);
        } else {
            tx[mt] = ty[mt] = tz[mt] = -1.0e150;  // far away: the kernel underflows to 0
            tn[mt][0] = tn[mt][1] = tn[mt][2] = 0.0;
        }
    }
    const unsigned full = 0xFFFFFFFFu;
    code_min = __reduce_min_sync(full, code_min);
    code_max = __reduce_max_sync(full, code_max);
    const int ax = (code_min == code_max && code_min < 3) ? code_min : 3;
    double acc[MTW][NC / 8][2];
#pragma unroll
    for (int mt = 0; mt < MTW; ++mt)
#pragma unroll
        for (int nt = 0; nt < NC / 8; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = 0.0;

    const int64_t j0 = (int64_t)blockIdx.y * chunk;
    const int64_t j1 = min(g.n, j0 + chunk);
    for (int64_t jt = j0; jt < j1; jt += TSRC) {
        const int cnt = (int)min((int64_t)TSRC, j1 - jt);
        __syncthreads();
        for (int t = threadIdx.x; t < TSRC + 4; t += NTHR) {
            const int64_t j = jt + t;
            const bool v = t < cnt;
            ssx[t] = v ? g.x[j] : 1.0e150;
            ssy[t] = v ? g.y[j] : 1.0e150;
            ssz[t] = v ? g.z[j] : 1.0e150;
        }
        for (int e = threadIdx.x; e < TSRC * NC; e += NTHR) {
            const int t = e / NC, c = e - t * NC;
            const int64_t j = jt + t;
            double q = 0.0;
            if (t < cnt && c < kc) q = g.w[j] * (pre ? pre[j] : 1.0) * X[j * ldx + c0 + c];
            sq[t * LDQ + c] = q;
        }
        __syncthreads();
        const bool self = (jt < i0 + TB) && (jt + cnt > i0);
        switch (ax) {
            case 0: tile_step<NC, 0>(ssx, ssy, ssz, sq, cnt, tx, ty, tz, tn, acc, lane, self, jt, ti); break;
            case 1: tile_step<NC, 1>(ssx, ssy, ssz, sq, cnt, tx, ty, tz, tn, acc, lane, self, jt, ti); break;
            case 2: tile_step<NC, 2>(ssx, ssy, ssz, sq, cnt, tx, ty, tz, tn, acc, lane, self, jt, ti); break;
            default: tile_step<NC, 3>(ssx, ssy, ssz, sq, cnt, tx, ty, tz, tn, acc, lane, self, jt, ti); break;
        }
    }
    // D fragment: (row grp, columns 2 kq, 2 kq + 1) of each (m-tile, n-tile)
#pragma unroll
    for (int mt = 0; mt < MTW; ++mt) {
        const int64_t i = ti[mt];
        if (i >= g.n) continue;
        const double sgn = ax == 0 ? tn[mt][0] : ax == 1 ? tn[mt][1] : ax == 2 ? tn[mt][2] : 1.0;
        double* o = part + ((int64_t)blockIdx.y * g.n + i) * ldp + c0;
#pragma unroll
        for (int nt = 0; nt < NC / 8; ++nt) {
            const int c = nt * 8 + 2 * kq;
            if (c < kc) o[c] = sgn * acc[mt][nt][0];
            if (c + 1 < kc) o[c + 1] = sgn * acc[mt][nt][1];
        }
    }
}

}  // namespace d64

// Columns [c0, c0 + kc) with kc <= 64 (NC = 8, 16, 32 or 64 columns per launch).
void launch_dt_f64_mma(const GeomDev& g, const double* X, int ldx, int c0, int kc, const double* pre, int nsplit,
                       int64_t chunk, double* part, int ldp, cudaStream_t s) {
    dim3 grid((unsigned)((g.n + d64::TB - 1) / d64::TB), (unsigned)nsplit);
    if (kc > 32)
        d64::k_dt_f64_mma<64><<<grid, d64::NTHR, 0, s>>>(g, X, ldx, c0, kc, pre, chunk, part, ldp);
    else if (kc > 16)
        d64::k_dt_f64_mma<32><<<grid, d64::NTHR, 0, s>>>(g, X, ldx, c0, kc, pre, chunk, part, ldp);
    else if (kc > 8)
        d64::k_dt_f64_mma<16><<<grid, d64::NTHR, 0, s>>>(g, X, ldx, c0, kc, pre, chunk, part, ldp);
    else
        d64::k_dt_f64_mma<8><<<grid, d64::NTHR, 0, s>>>(g, X, ldx, c0, kc, pre, chunk, part, ldp);
    BIE_CK(cudaGetLastError());
}

}  // namespace bie

// K4, streaming form: the block-row correction apply for narrow right-hand-side
// blocks (k <= 16), where the apply is bound by HBM reads of the FP64 correction
// blocks (nb x nb per near pair, about 10 KB at n_quad = 6) and not by arithmetic.
//
//   Y[i][c] = (1/4pi) sum_s part[s][i][c] + sum_b (C_b (p X)[col_b])[i][c] + t_i p_i X[i][c]
//
// (the CSC SpMV / sparse mat-mat of laplace3d_DT_fmm3d_corrected and
// BatchedDielectricOperator, src/kernel/laplace3d_near.jl:395-419,
// src/solver/multi_rhs.jl:103-136, fused with the reduction of the direct-sum split
// partials and the diagonal term).
//
// Persistent CTAs of 4 consumer warps + 1 producer warp walk the block rows
// blockIdx.x, blockIdx.x + gridDim.x, ... The producer streams every block of those
// rows, with the nb x k slab of X (and of the preconditioner p) it multiplies, into a
// ring of shared-memory stages by cp.async.bulk, one mbarrier per stage, running
// ahead across row boundaries; a block and its slab are contiguous in global memory
// (column-major blocks; node-major X), so a stage is two or three bulk copies. The
// consumer warps contract each staged block with mma.sync.m8n8k4.f64 (k-steps split
// across the warps sharing an 8-column n-tile) and release the stage; at the end of
// a row they add their partial products through shared memory and write the row's
// outputs together with the split partials and the diagonal term. Where a row's split
// partials, X rows, diagonal and preconditioner fit one row slot, the producer
// prefetches them by bulk copies too: once the previous row's epilogue has released the
// slot, right after the row's first S blocks, so they land while the rest of the row's
// blocks are consumed and the epilogue reads shared memory only.
//
// Stage layout, column stride nb for the block (nb = 4 or 12 mod 16 doubles keeps a
// half-warp's A-fragment loads on distinct banks) and row stride k for the slab. The
// fragments of padded rows (8 MT > nb) and padded columns (8 n-tiles > k) read the
// next region of shared memory: they only feed outputs that are discarded. The
// k-steps cover exactly nb sources (nb % 4 == 0), so no padding enters a kept sum.
// Every mbarrier wait is bounded; on expiry the CTA flags the error, drains its
// copies in flight and returns.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "common.cuh"
#include "mbar.cuh"
#include "solver.h"

namespace bie {
namespace {

constexpr int kConsumers = 4;                        // consumer warps
constexpr int kThreadsCB = 32 * (kConsumers + 1);    // + the producer warp
constexpr int kStages = 4;                           // ring stages
constexpr uint32_t kWaitLimitCB = 1u << 26;          // wait attempts before a CTA gives up (seconds)

__device__ __forceinline__ void dmma_cb(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <typename TP>
struct CombBulk {
    int64_t n;
    int k, nb, npanels, nsplit;
    const TP* part;
    const double* X;
    const double* pre;
    const double* diag;
    const int32_t* rowptr;
    const int32_t* col;
    const double* val;
    double* Y;
    uint32_t vbytes, xbytes, pbytes, stage_bytes;
    uint32_t row_bytes;  // bytes of the row slot ([nsplit][nb k] partials, [nb k] X, [nb] diag, [nb] pre), 0: none
    int* err;
};

template <int MT, typename TP>
__global__ void __launch_bounds__(kThreadsCB) k_combine_bulk(CombBulk<TP> P) {
    extern __shared__ __align__(16) uint8_t smc[];
    constexpr int S = kStages;
    uint8_t* ring = smc;                                                 // [S][stage_bytes]
    uint8_t* rs = ring + (size_t)S * P.stage_bytes;                      // [row_bytes] row slot
    double* red = reinterpret_cast<double*>(rs + (size_t)P.row_bytes);   // [4][MT][2][32]
    uint64_t* full = reinterpret_cast<uint64_t*>(red + kConsumers * MT * 2 * 32);
    uint64_t* empty = full + S;
    uint64_t* rfull = empty + S;   // row slot landed
    uint64_t* rempty = rfull + 1;  // row slot read by the epilogue
    volatile int* abort_flag = reinterpret_cast<volatile int*>(rempty + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nb = P.nb, k = P.k;
    const int64_t tot = P.n * (int64_t)k;
    // row slot regions
    const uint32_t rpart = (uint32_t)(nb * k * sizeof(TP));  // one split's partials of a row
    const uint32_t rx = (uint32_t)P.nsplit * rpart, rdg = rx + (uint32_t)nb * k * 8, rpre = rdg + (uint32_t)nb * 8;
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kConsumers);
        }
        mbar_init(rfull, 1);
        mbar_init(rempty, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == kConsumers) {
        // ------------------------------ producer ------------------------------
        if (lane != 0) return;
        int64_t it = 0, rw = 0;  // blocks and rows whose copies were issued
        int ps = 0;              // stage of the next block
        uint32_t pph = 0;        // parity of the empty-barrier phase awaited for stage ps (from the second use)
        bool ok = true;
        // the row's epilogue operands into the row slot, once the previous row released it
        auto issue_row = [&](int p) -> bool {
            if (rw >= 1 && !mbar_wait(rempty, (uint32_t)((rw - 1) & 1), abort_flag, kWaitLimitCB)) return false;
            uint64_t* bar = rfull;
            const int64_t row0 = (int64_t)p * nb;
            mbar_arrive_tx(bar, P.row_bytes);
            for (int q = 0; q < P.nsplit; ++q) bulk_g2s(rs + (size_t)q * rpart, P.part + q * tot + row0 * k, rpart, bar);
            if (P.diag) {
                bulk_g2s(rs + rx, P.X + row0 * k, (uint32_t)nb * k * 8, bar);
                bulk_g2s(rs + rdg, P.diag + row0, (uint32_t)nb * 8, bar);
                if (P.pre) bulk_g2s(rs + rpre, P.pre + row0, (uint32_t)nb * 8, bar);
            }
            ++rw;
            return true;
        };
        for (int p = blockIdx.x; p < P.npanels && ok; p += gridDim.x) {
            const int b0 = P.rowptr[p], b1 = P.rowptr[p + 1];
            // the row data goes out after the row's first S blocks: by then the previous row's
            // epilogue has (nearly) released the slot, and the copies still precede this
            // row's epilogue by the row's remaining blocks (issuing them at the row's start,
            // with a second slot, delays the row's first blocks and measured slower)
            const int row_at = b0 + min(S, b1 - b0);
            for (int b = b0; b <= b1; ++b) {
                if (P.row_bytes && b == row_at && !(ok = issue_row(p))) break;
                if (b == b1) break;
                // stage s of block it, and the parity of that stage's previous use
                if (it >= S && !mbar_wait(&empty[ps], pph, abort_flag, kWaitLimitCB)) {
                    ok = false;
                    break;
                }
                const int s = ps;
                uint8_t* st = ring + (size_t)s * P.stage_bytes;
                const int64_t src = (int64_t)P.col[b] * nb;
                mbar_arrive_tx(&full[s], P.vbytes + P.xbytes + P.pbytes);
                bulk_g2s(st, P.val + (int64_t)b * nb * nb, P.vbytes, &full[s]);
                bulk_g2s(st + P.vbytes, P.X + src * k, P.xbytes, &full[s]);
                if (P.pbytes) bulk_g2s(st + P.vbytes + P.xbytes, P.pre + src, P.pbytes, &full[s]);
                ++it;
                if (++ps == S) {
                    ps = 0;
                    if (it > S) pph ^= 1u;
                }
            }
        }
        if (!ok || *abort_flag) {
            // the CTA gives up: wait for the copies still in flight (the latest of each stage)
            for (int64_t j = it > S ? it - S : 0; j < it; ++j)
                mbar_wait_raw(&full[j % S], (uint32_t)((j / S) & 1), kWaitLimitCB);
            if (P.row_bytes && rw >= 1) mbar_wait_raw(rfull, (uint32_t)((rw - 1) & 1), kWaitLimitCB);
        }
        return;
    }

    // ------------------------------ consumers ------------------------------
    const int ntiles = (k + 7) / 8;         // 1 or 2
    const int nw = ntiles;                  // distinct n-tiles
    const int ksplit = kConsumers / nw;     // warps sharing an n-tile split its k-steps
    const int nt = warp % nw, kq = warp / nw;
    const int KS = nb / 4;
    double acc[MT][2];
#pragma unroll
    for (int m = 0; m < MT; ++m) acc[m][0] = acc[m][1] = 0.0;
    bool ok = true;  // false once this warp gave up: it still takes every barrier below
    int64_t it = 0, rw = 0;
    int cs = 0;        // stage of the next block
    uint32_t cph = 0;  // parity of its full-barrier phase
    for (int p = blockIdx.x; p < P.npanels; p += gridDim.x, ++rw) {
        const int b1 = P.rowptr[p + 1];
        for (int b = P.rowptr[p]; b < b1; ++b, ++it) {
            const int s = cs;
            const uint32_t ph = cph;
            if (++cs == S) {
                cs = 0;
                cph ^= 1u;
            }
            if (ok) ok = mbar_wait(&full[s], ph, abort_flag, kWaitLimitCB);
            if (ok) {
                const double* st = reinterpret_cast<const double*>(ring + (size_t)s * P.stage_bytes);
                const double* cC = st + (lane >> 2);
                const double* cX = st + nb * nb + 8 * nt + (lane >> 2);
                const double* cP = st + nb * nb + nb * k;
                for (int ks = kq; ks < KS; ks += ksplit) {
                    const int q = 4 * ks + (lane & 3);
                    double bv = cX[q * k];
                    if (P.pbytes) bv *= cP[q];
#pragma unroll
                    for (int m = 0; m < MT; ++m) dmma_cb(acc[m][0], acc[m][1], cC[q * nb + 8 * m], bv);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
        }
        // row epilogue: partial products of the warps, split partials, diagonal
#pragma unroll
        for (int m = 0; m < MT; ++m) {
            red[((warp * MT + m) * 2 + 0) * 32 + lane] = acc[m][0];
            red[((warp * MT + m) * 2 + 1) * 32 + lane] = acc[m][1];
            acc[m][0] = acc[m][1] = 0.0;
        }
        asm volatile("bar.sync 1, %0;" ::"n"(32 * kConsumers) : "memory");
        const int64_t row0 = (int64_t)p * nb;
        if (P.row_bytes && ok) ok = mbar_wait(rfull, (uint32_t)(rw & 1), abort_flag, kWaitLimitCB);
        for (int e = threadIdx.x; e < nb * k; e += 32 * kConsumers) {
            const int r = e / k, c = e - r * k;
            const int m = r >> 3, t = c >> 3, cc = c & 7;
            const int ln = (r & 7) * 4 + (cc >> 1), h = cc & 1;
            double sb = 0.0;
            for (int q = 0; q < ksplit; ++q) sb += red[(((t + q * nw) * MT + m) * 2 + h) * 32 + ln];
            const int64_t i = row0 + r;
            const int64_t idx = i * k + c;
            double sp = 0.0, y;
            if (P.row_bytes) {
                if (!ok) continue;
                const TP* rp = reinterpret_cast<const TP*>(rs);
                for (int sidx = 0; sidx < P.nsplit; ++sidx) sp += (double)rp[sidx * nb * k + e];
                y = sp * kInv4Pi + sb;
                if (P.diag) {
                    const double* rxv = reinterpret_cast<const double*>(rs + rx);
                    const double* rdv = reinterpret_cast<const double*>(rs + rdg);
                    const double* rpv = reinterpret_cast<const double*>(rs + rpre);
                    y += rdv[r] * (P.pre ? rpv[r] : 1.0) * rxv[e];
                }
            } else {
                // eight loads in flight at a time, added in split order
                int sidx = 0;
                for (; sidx + 8 <= P.nsplit; sidx += 8) {
                    double v[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) v[u] = (double)P.part[(int64_t)(sidx + u) * tot + idx];
#pragma unroll
                    for (int u = 0; u < 8; ++u) sp += v[u];
                }
                for (; sidx < P.nsplit; ++sidx) sp += (double)P.part[(int64_t)sidx * tot + idx];
                y = sp * kInv4Pi + sb;
                if (P.diag) y += P.diag[i] * (P.pre ? P.pre[i] : 1.0) * P.X[idx];
            }
            if (ok && !*abort_flag) P.Y[idx] = y;
        }
        asm volatile("bar.sync 1, %0;" ::"n"(32 * kConsumers) : "memory");  // red and the row slot are reused
        if (P.row_bytes && threadIdx.x == 0) mbar_arrive(rempty);
    }
    if (threadIdx.x == 0 && *abort_flag) {
        atomicOr(P.err, 1);
        // the producer may have finished issuing before the CTA gave up: wait for the
        // latest copy of each stage so none is in flight when the CTA exits
        for (int64_t j = it > S ? it - S : 0; j < it; ++j)
            mbar_wait_raw(&full[j % S], (uint32_t)((j / S) & 1), kWaitLimitCB);
        if (P.row_bytes && rw >= 1) mbar_wait_raw(rfull, (uint32_t)((rw - 1) & 1), kWaitLimitCB);
    }
}

}  // namespace

// Stage bytes of one block + slabs, or 0 when the streaming form does not apply.
static uint32_t comb_bulk_stage(int nb, int k, bool pre) {
    if (k < 1 || k > 16 || nb % 4 != 0 || (nb % 16 != 4 && nb % 16 != 12) || (nb + 7) / 8 > 8) return 0;
    const uint32_t v = (uint32_t)nb * nb * 8, x = (uint32_t)nb * k * 8, p = pre ? (uint32_t)nb * 8 : 0;
    if (v % 16 || x % 16 || p % 16) return 0;
    return v + x + p;
}

template <typename TP>
bool launch_combine_bulk(int64_t n, int k, int nb, int npanels, const TP* part, int nsplit, const double* X,
                         const double* pre, const double* diag, const int32_t* rowptr, const int32_t* col,
                         const double* val, double* Y, int* err, int sms, cudaStream_t s) {
    const uint32_t stage = comb_bulk_stage(nb, k, pre != nullptr);
    if (!stage || !val || !rowptr || npanels <= 0) return false;
    auto al16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
    if (!al16(X) || !al16(val) || (pre && !al16(pre))) return false;
    const int mt = (nb + 7) / 8;
    // row slot: every split's partials of the row, and with the diagonal term the row's X,
    // diag and preconditioner; kept when it fits 48 KB and every copy is aligned
    size_t row = (size_t)nsplit * nb * k * sizeof(TP) + (diag ? (size_t)nb * k * 8 + nb * 8 * (pre ? 2 : 1) : 0);
    if (row > 48 * 1024 || (nb * k * sizeof(TP)) % 16 || !al16(part) || (diag && !al16(diag))) row = 0;
    const void* f = nullptr;
    switch (mt) {
        case 1: f = (const void*)k_combine_bulk<1, TP>; break;
        case 2: f = (const void*)k_combine_bulk<2, TP>; break;
        case 3: f = (const void*)k_combine_bulk<3, TP>; break;
        case 4: f = (const void*)k_combine_bulk<4, TP>; break;
        case 5: f = (const void*)k_combine_bulk<5, TP>; break;
        case 6: f = (const void*)k_combine_bulk<6, TP>; break;
        case 7: f = (const void*)k_combine_bulk<7, TP>; break;
        default: f = (const void*)k_combine_bulk<8, TP>; break;
    }
    // ring depth 4: the row slot goes out after a row's first 4 blocks, so deeper rings
    // would leave its copies less time before the epilogue (measured slower)
    const size_t smem = (size_t)kStages * stage + row + sizeof(double) * kConsumers * mt * 2 * 32 +
                        sizeof(uint64_t) * (2 * kStages + 2) + 16;
    const int occ = occupancy(f, kThreadsCB, smem);
    CombBulk<TP> P{n, k, nb, npanels, nsplit, part, X, pre, diag, rowptr, col, val, Y,
                   (uint32_t)nb * nb * 8, (uint32_t)nb * k * 8, pre ? (uint32_t)nb * 8 : 0u, stage,
                   (uint32_t)row, err};
    const int grid = (int)std::min<int64_t>(npanels, (int64_t)sms * occ);
    void* args[] = {&P};
    BIE_CK(cudaLaunchKernel(f, dim3(grid), dim3(kThreadsCB), args, smem, s));
    return true;
}

template bool launch_combine_bulk<float>(int64_t, int, int, int, const float*, int, const double*, const double*,
                                         const double*, const int32_t*, const int32_t*, const double*, double*, int*,
                                         int, cudaStream_t);
template bool launch_combine_bulk<double>(int64_t, int, int, int, const double*, int, const double*, const double*,
                                          const double*, const int32_t*, const int32_t*, const double*, double*,
                                          int*, int, cudaStream_t);

}  // namespace bie

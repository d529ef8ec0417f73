// Small dense kernels of the block GMRES solver (solver.cu, bgmres): Cholesky factors of
// the k x k Gram matrices (CholQR of each new block of basis vectors) and their inverses,
// their products, the incremental Householder QR of the block upper-Hessenberg matrix with
// its right-hand sides, partial-sum reduction and column gathers. One CTA runs each
// factorisation step (a Cholesky, a new block's reflectors); for blocks of up to 64 columns
// each block column's reflectors are also kept in compact-WY form, which several CTAs apply
// as small matrix products (the earlier blocks to a new block column, and all blocks in
// reverse to form the Krylov residual).
//
// Storage is column-major: A[i + j * lda].
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.cuh"

namespace bie {

constexpr int kCholThreads = 1024;  // block size of k_chol_inv_smem in the solver

// Cholesky factor R of the k x k Gram matrix G (ld k, upper triangle read) and its inverse,
// in shared memory (2 k (k + 1) doubles, k <= 64): R into Rout (ld ldr, lower triangle zeroed),
// R^-1 into Rinv (ld k). A pivot below 1e-30 max(diag G) (a direction the block cannot
// extend: its columns are linearly dependent to working precision) is replaced by that floor
// and counted in *nclamp, so the basis stays orthonormal and the corresponding coupling in the
// Hessenberg matrix is tiny. The factorisation is
// right-looking with one barrier per pivot (row p of the factor goes to its own array while
// the trailing matrix is updated from the unscaled row; thread (q, rg) updates row q = tid
// mod 64 in the columns r = rg mod (blockDim.x / 64)). The inverse is formed by back
// substitution, warp w taking columns w + m nwarp with the columns in registers and each
// column of R read once for all of them. NT (the block size): 256, 512 or 1024.
template <int NT>
__global__ void __launch_bounds__(NT) k_chol_inv_smem(const double* __restrict__ G, int k, double* __restrict__ Rout,
                                                      int ldr, double* __restrict__ Rinv, int* __restrict__ nclamp) {
    extern __shared__ double sm[];
    const int ld = k + 1;     // padded: a row of the matrix spreads over the shared-memory banks
    double* A = sm;           // k x k, ld: the trailing matrix
    double* R = sm + ld * k;  // k x k, ld: the factor
    __shared__ double s_floor;
    __shared__ double s_rinv[64];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
    for (int e = tid; e < k * k; e += blockDim.x) {
        const int i = e % k, jj = e / k;
        A[i + jj * ld] = i <= jj ? G[i + jj * k] : 0.0;
        R[i + jj * ld] = 0.0;
    }
    __syncthreads();
    if (warp == 0) {
        double mx = 0.0;
        for (int i = lane; i < k; i += 32) mx = fmax(mx, A[i + i * ld]);
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
        if (lane == 0) s_floor = mx > 0.0 ? 1e-30 * mx : 1e-300;
    }
    __syncthreads();
    const double fl = s_floor;
    const int qq = tid & 63, rg = tid >> 6, ng = blockDim.x >> 6;  // ng: a power of two
    for (int p = 0; p < k; ++p) {
        double d = A[p + p * ld];
        const bool clamp = !(d > fl);
        if (clamp) d = fl;
        const double inv = rsqrt(d);  // one reciprocal square root on the pivot chain
        const double piv = d * inv;
        // step p reads row p and writes rows > p of A and row p of R: one barrier per pivot
        if (qq > p && qq < k) {
            const double apq = A[p + qq * ld] * inv;
            const int r0 = p + 1 + ((rg - (p + 1)) & (ng - 1));  // first r >= p + 1 with r = rg mod ng
            for (int r = r0; r < k; r += ng)
                if (r >= qq) A[qq + r * ld] -= apq * (A[p + r * ld] * inv);
        }
        if (tid >= p && tid < k) R[p + tid * ld] = tid == p ? piv : A[p + tid * ld] * inv;
        if (tid == 0 && clamp && nclamp) atomicAdd(nclamp, 1);
        __syncthreads();
    }
    for (int i = tid; i < k; i += blockDim.x) s_rinv[i] = 1.0 / R[i + i * ld];
    __syncthreads();
    // column jj of R^-1: x = e_jj; for l = jj .. 0: x_l /= R_ll, x_i -= R_il x_l (i < l);
    // lane holds rows lane and lane + 32 of up to 8 columns jj = warp + m nwarp
    constexpr int MC = 2048 / NT;  // columns per warp: 64 / (NT / 32)
    double x0[MC], x1[MC];
    int top = -1;
#pragma unroll
    for (int m = 0; m < MC; ++m) {
        const int jj = warp + m * nwarp;
        x0[m] = lane == jj ? 1.0 : 0.0;
        x1[m] = lane + 32 == jj ? 1.0 : 0.0;
        if (jj < k) top = jj;
    }
    for (int l = top; l >= 0; --l) {
        const double rl = s_rinv[l];
        const double u0 = lane < l ? R[lane + l * ld] : 0.0;
        const double u1 = lane + 32 < l ? R[lane + 32 + l * ld] : 0.0;
#pragma unroll
        for (int m = 0; m < MC; ++m) {
            if (warp + m * nwarp >= k) continue;  // uniform per warp
            const double xl = __shfl_sync(0xFFFFFFFFu, l < 32 ? x0[m] : x1[m], l & 31) * rl;
            if (lane == (l & 31)) {
                if (l < 32) x0[m] = xl;
                else x1[m] = xl;
            }
            x0[m] = fma(-u0, xl, x0[m]);
            x1[m] = fma(-u1, xl, x1[m]);
        }
    }
#pragma unroll
    for (int m = 0; m < MC; ++m) {
        const int jj = warp + m * nwarp;
        if (jj >= k) continue;
        if (lane < k) Rinv[lane + jj * k] = lane <= jj ? x0[m] : 0.0;
        if (lane + 32 < k) Rinv[lane + 32 + jj * k] = lane + 32 <= jj ? x1[m] : 0.0;
    }
    for (int e = tid; e < k * k; e += blockDim.x) {
        const int i = e % k, jj = e / k;
        Rout[i + (int64_t)jj * ldr] = R[i + jj * ld];
    }
}

// C = A B for upper-triangular k x k A and B (C upper triangular), C may not alias A or B.
__global__ void k_trmm_upper(const double* __restrict__ A, int lda, const double* __restrict__ B, int ldb,
                             double* __restrict__ C, int ldc, int k) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)k * k;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(e % k), j = (int)(e / k);
        double s = 0.0;
        for (int l = i; l <= j; ++l) s += A[i + (int64_t)l * lda] * B[l + (int64_t)j * ldb];
        C[i + (int64_t)j * ldc] = i <= j ? s : 0.0;
    }
}

// G = sum_b P[b] of nb partial matrices of kk entries each, in a fixed order: CTAs of 256
// threads take 32 consecutive entries, thread (e, sp) sums the partials b = sp mod 8 and the
// eight split sums are added in order.
__global__ void __launch_bounds__(256) k_sum_partials(const double* __restrict__ P, int nb, int kk,
                                                      double* __restrict__ G) {
    __shared__ double part[8][32];
    const int c = threadIdx.x & 31, sp = threadIdx.x >> 5;
    const int e = blockIdx.x * 32 + c;
    double s = 0.0;
    if (e < kk) {
#pragma unroll 4
        for (int b = sp; b < nb; b += 8) s += P[(int64_t)b * kk + e];
    }
    part[sp][c] = s;
    __syncthreads();
    if (sp == 0 && e < kk) {
        double t = part[0][c];
        for (int q = 1; q < 8; ++q) t += part[q][c];
        G[e] = t;
    }
}

// Xa[i][a] = X[i][idx[a]] (node-major, X n x k, Xa n x ka)
__global__ void k_gather_cols(const double* __restrict__ X, int k, const int* __restrict__ idx, int ka, int64_t n,
                              double* __restrict__ Xa) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * ka) return;
    const int64_t i = e / ka;
    const int a = (int)(e - i * ka);
    Xa[e] = X[i * k + idx[a]];
}

// X[i][idx[a]] = Xa[i][a]
__global__ void k_scatter_cols(const double* __restrict__ Xa, int ka, const int* __restrict__ idx, int k, int64_t n,
                               double* __restrict__ X) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * ka) return;
    const int64_t i = e / ka;
    const int a = (int)(e - i * ka);
    X[i * k + idx[a]] = Xa[e];
}

// X[i][a] += p_i U[i][a] (p = null: 1)
__global__ void k_add_rows_scaled(double* __restrict__ X, const double* __restrict__ U, const double* __restrict__ p,
                                  int64_t n, int ka) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * ka) return;
    X[e] += p ? p[e / ka] * U[e] : U[e];
}

}  // namespace bie

namespace bie {

// Sum over the 8 lanes of a column group (lanes 8 c .. 8 c + 7 of a warp).
__device__ __forceinline__ double group8_sum(double v) {
    v += __shfl_xor_sync(0xFFFFFFFFu, v, 1);
    v += __shfl_xor_sync(0xFFFFFFFFu, v, 2);
    v += __shfl_xor_sync(0xFFFFFFFFu, v, 4);
    return v;
}

// Doubles per block column in the compact-WY buffer: V (2k x k, ld 2k; unit diagonal and zeros
// in place) followed by T^T (k x k, ld k), the total rounded up to an even count so that every
// block starts on a 16-byte boundary.
__host__ __device__ inline int wy_stride(int k) { return (2 * k * k + k * k + 1) & ~1; }

// One reflector t of k_bhess_qr_tile, for t in 8 P .. 8 P + 7: reflector t spans rows
// t .. t + k <= 8 P + 7 + 64, so only the row slots P .. P + 8 take part (compile-time range).
template <int P>
__device__ __forceinline__ void tile_reflector(double (&x)[2][16], int t, int k, int g, int cg, int warp, int G,
                                               bool live, double* vbuf, double* tbuf, double* stau, double* U,
                                               double* tau_out) {
    constexpr int R0 = P, R1 = P + 8 < 15 ? P + 8 : 15;
    double* vb = vbuf + (t & 1) * 128;
    if (warp == (t >> 2)) {
        // every group of the warp reduces its own column; only the group of column t keeps it.
        // Rows below t + k of column t are zero (the lower block is triangular and the earlier
        // reflectors end above row t + k), so the tail sum runs over all rows below t.
        const bool og = cg == (t & 3);
        double s0 = 0.0, s1 = 0.0, al = 0.0;
#pragma unroll
        for (int r = R0; r <= R1; ++r) {
            const int i = g + 8 * r;
            const double a = i > t ? x[0][r] : 0.0;
            if (r & 1) s1 = fma(a, a, s1);
            else s0 = fma(a, a, s0);
            al = i == t ? x[0][r] : al;
        }
        const double sg = group8_sum(s0 + s1);
        al = group8_sum(al);
        double tc = 0.0, scale = 0.0, beta = al;
        if (sg != 0.0) {
            const double q = fma(al, al, sg);
            const double rq = rsqrt(q);  // 1 / mu
            const double mu = q * rq;
            beta = al <= 0.0 ? mu : -mu;
            const double d = al - beta;
            tc = al <= 0.0 ? -d * rq : d * rq;  // (beta - al) / beta
            scale = __drcp_rn(d);
        }
        if (og) {
#pragma unroll
            for (int r = R0; r <= R1; ++r) {
                const int i = g + 8 * r;
                const bool tail = i > t && i <= t + k && tc != 0.0;
                const double xs = tail ? x[0][r] * scale : x[0][r];
                x[0][r] = i == t ? beta : xs;
                vb[i] = i == t ? 1.0 : (tail ? xs : 0.0);
            }
            if (g == 0) {
                tbuf[t & 1] = tc;
                stau[t] = tc;
                tau_out[t] = tc;
            }
        }
    }
    __syncthreads();
    const double tc = tbuf[t & 1];
    if (tc != 0.0) {  // uniform: every lane takes part in the shuffles (idle groups hold zeros)
        double v[R1 - R0 + 1];
#pragma unroll
        for (int r = R0; r <= R1; ++r) v[r - R0] = vb[g + 8 * r];
        double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0;
#pragma unroll
        for (int r = R0; r <= R1; ++r) {
            if (r & 1) {
                a1 = fma(v[r - R0], x[0][r], a1);
                b1 = fma(v[r - R0], x[1][r], b1);
            } else {
                a0 = fma(v[r - R0], x[0][r], a0);
                b0 = fma(v[r - R0], x[1][r], b0);
            }
        }
        const double p0 = group8_sum(a0 + a1), p1 = group8_sum(b0 + b1);
        if (live && G < t && g == 0) U[G + t * 65] = p0;
        const double f0 = live && G > t ? p0 * tc : 0.0, f1 = live ? p1 * tc : 0.0;
#pragma unroll
        for (int r = R0; r <= R1; ++r) {
            x[0][r] = fma(-f0, v[r - R0], x[0][r]);
            x[1][r] = fma(-f1, v[r - R0], x[1][r]);
        }
    }
}

// k_bhess_qr_tile: the new block's reflectors on its 2k x k tile (rows c0 .. c0 + 2k - 1 of
// block column j, after k_bhess_apply_prev) together with the same rows of the k right-hand
// sides Gv, and every right-hand side's residual. One CTA of 512 threads: column group
// G = 4 warp + lane / 8 (8 lanes) holds tile column G and right-hand side G in registers,
// lane g = lane mod 8 the local rows g + 8 r (r < 16). For reflector t the group of column t
// forms it (LAPACK dlarfg convention: mu = |column t from row t on|, beta = mu for alpha <= 0
// and -mu otherwise, tau = (beta - alpha) / beta, tail scaled by 1 / (alpha - beta)) and
// publishes v through shared memory; after one barrier every group applies it to its columns
// right of t, over the row slots the reflector meets (tile_reflector; no data-dependent
// branches).
//
// The block's compact-WY form comes out as well: Q_j = H_0 .. H_{k-1} = I - V T V^T with
// T = (strictly-upper(V^T V) + diag(1 / tau))^-1 (a zero tau gives a zero row and column of
// T). The dot product group G < t forms for reflector t is (V^T V)[G][t], since its column
// is final (v_G, with beta at row G where v_t is zero). V (unit diagonal and zeros in place)
// and T^T (Tt[a + l k] = T[l][a]) are written to wy (wy_stride(k) doubles).
__global__ void __launch_bounds__(512) k_bhess_qr_tile(double* __restrict__ H, int ldh, double* __restrict__ tau,
                                                       double* __restrict__ Gv, int ldg, int k, int j,
                                                       double* __restrict__ resid, double* __restrict__ wy) {
    constexpr int NR = 16, LDU = 65;
    __shared__ double vbuf[2 * 128];
    __shared__ double tbuf[2];
    __shared__ double stau[64];
    __shared__ double U[64 * LDU];  // strictly upper part of V^T V, column-major
    for (int e = threadIdx.x; e < 64 * LDU; e += blockDim.x) U[e] = 0.0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane & 7, cg = lane >> 3;
    const int G = 4 * warp + cg;
    const bool live = G < k;
    const int c0 = j * k, k2 = 2 * k;
    double x[2][NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        const int i = g + 8 * r;
        const bool in = live && i < k2;
        x[0][r] = in ? H[(c0 + i) + (int64_t)(c0 + G) * ldh] : 0.0;
        x[1][r] = in ? Gv[(c0 + i) + (int64_t)G * ldg] : 0.0;
    }
    __syncthreads();  // U cleared
    for (int t = 0; t < k; ++t) {
#define BIE_TILE_PHASE(P)                                                                                  \
    case P:                                                                                                \
        tile_reflector<P>(x, t, k, g, cg, warp, G, live, vbuf, tbuf, stau, U, tau + c0);                  \
        break;
        switch (t >> 3) {
            BIE_TILE_PHASE(0)
            BIE_TILE_PHASE(1)
            BIE_TILE_PHASE(2)
            BIE_TILE_PHASE(3)
            BIE_TILE_PHASE(4)
            BIE_TILE_PHASE(5)
            BIE_TILE_PHASE(6)
            BIE_TILE_PHASE(7)
        }
#undef BIE_TILE_PHASE
    }
    // the store addresses are formed afresh (opaque copies of the bases and strides), so the
    // load addresses are not kept live through the reflector loop
    double* Hs = H;
    double* Gs = Gv;
    double* Ws = wy;
    int ldhs = ldh, ldgs = ldg;
    asm volatile("" : "+l"(Hs), "+l"(Gs), "+l"(Ws), "+r"(ldhs), "+r"(ldgs));
    double rs = 0.0;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        const int i = g + 8 * r;
        if (!live || i >= k2) continue;
        Hs[(c0 + i) + (int64_t)(c0 + G) * ldhs] = x[0][r];
        Gs[(c0 + i) + (int64_t)G * ldgs] = x[1][r];
        Ws[i + G * k2] = i < G || i > G + k ? 0.0 : (i == G ? 1.0 : x[0][r]);
        if (i >= k) rs += x[1][r] * x[1][r];
    }
    rs = group8_sum(rs);
    if (live && g == 0) resid[G] = sqrt(rs);
    __syncthreads();
    // T = U^-1 (U with diagonal 1 / tau): column a by back substitution, x = e_a, for
    // l = a .. 0: x_l *= tau_l, x_i -= U[i][l] x_l (i < l); warp w takes columns w + 16 m,
    // interleaved; lane holds rows lane and lane + 32
    double y0[4], y1[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const int a = warp + 16 * m;
        y0[m] = lane == a ? 1.0 : 0.0;
        y1[m] = lane + 32 == a ? 1.0 : 0.0;
    }
    for (int l = k - 1; l >= 0; --l) {
        const double tl = stau[l];
        const double u0 = lane < l ? U[lane + l * LDU] : 0.0;
        const double u1 = lane + 32 < l ? U[lane + 32 + l * LDU] : 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const double xl = __shfl_sync(0xFFFFFFFFu, l < 32 ? y0[m] : y1[m], l & 31) * tl;
            if (lane == (l & 31)) {
                if (l < 32) y0[m] = xl;
                else y1[m] = xl;
            }
            y0[m] = fma(-u0, xl, y0[m]);
            y1[m] = fma(-u1, xl, y1[m]);
        }
    }
    double* Tt = Ws + k2 * k;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const int a = warp + 16 * m;
        if (a >= k) continue;
        if (lane < k) Tt[a + lane * k] = lane <= a ? y0[m] : 0.0;
        if (lane + 32 < k) Tt[a + (lane + 32) * k] = lane + 32 <= a ? y1[m] : 0.0;
    }
}

// k_bhess_apply_prev: the reflectors of block columns 0 .. j - 1 applied to block column j as
// compact-WY block reflectors, in order: on rows b k .. b k + 2k - 1,
//   C <- Q_b^T C = C - V_b T_b^T (V_b^T C)
// with V_b the block's unit lower-trapezoidal reflectors (column t nonzero on rows t .. t + k)
// and T_b^T, both from k_bhess_qr_tile (wy + b wy_stride(k)). Each CTA (256 threads) takes
// kApplyCols columns of the block column and keeps their 2k-row window in shared memory; the
// next block's V and T^T are copied by cp.async (16-byte pieces) while the current one is
// applied. Three barrier-separated products per block: W = V^T C (k x NC), W2 = T^T W,
// C -= V W2, each sum over the rows where V is nonzero. After block b the window's top k rows
// are final and written back and the window moves down by k rows. Launched only for j > 0;
// k <= 64.
constexpr int kApplyCols = 4;
inline size_t apply_prev_smem(int k) {
    return sizeof(double) * (2 * (size_t)wy_stride(k) + 4 * (size_t)k * kApplyCols);
}
__global__ void __launch_bounds__(256) k_bhess_apply_prev(double* __restrict__ H, int ldh,
                                                          const double* __restrict__ wy, int k, int j) {
    constexpr int NC = kApplyCols;
    extern __shared__ double sm[];
    const int k2 = 2 * k, bs = wy_stride(k), tid = threadIdx.x;
    double* C = sm + 2 * bs;  // 2k x NC (ld 2k)
    double* W = C + k2 * NC;  // k x NC (ld k)
    double* W2 = W + k * NC;  // k x NC (ld k)
    const int q0 = blockIdx.x * NC, nc = min(NC, k - q0);
    const int c0 = j * k;
    auto colp = [&](int c) { return H + (int64_t)(c0 + q0 + c) * ldh; };
    auto prefetch = [&](int b, int buf) {
        const double* src = wy + (int64_t)b * bs;
        double* dst = sm + buf * bs;
        for (int e = 2 * tid; e < bs; e += 2 * blockDim.x) cp_async16(dst + e, src + e);
        cp_async_commit();
    };
    for (int c = 0; c < NC; ++c)
        for (int i = tid; i < k2; i += blockDim.x) C[i + c * k2] = c < nc ? colp(c)[i] : 0.0;
    prefetch(0, 0);
    for (int b = 0; b < j; ++b) {
        const int r0 = b * k, buf = b & 1;
        if (b + 1 < j) {
            prefetch(b + 1, buf ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const double* V = sm + buf * bs;
        const double* T = V + k2 * k;
        // W = V^T C: W[t][c] = sum over i = t .. t + k of V[i][t] C[i][c]
        for (int o = tid; o < k * NC; o += blockDim.x) {
            const int c = o / k, t = o - c * k;
            const double* v = V + t * k2 + t;
            const double* x = C + c * k2 + t;
            double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
            int i = 0;
            for (; i + 3 <= k; i += 4) {
                a0 = fma(v[i], x[i], a0);
                a1 = fma(v[i + 1], x[i + 1], a1);
                a2 = fma(v[i + 2], x[i + 2], a2);
                a3 = fma(v[i + 3], x[i + 3], a3);
            }
            for (; i <= k; ++i) a0 = fma(v[i], x[i], a0);
            W[t + c * k] = (a0 + a1) + (a2 + a3);
        }
        __syncthreads();
        // W2 = T^T W: W2[a][c] = sum over l <= a of T[l][a] W[l][c]  (T^T stored: T[a + l k] = T[l][a])
        for (int o = tid; o < k * NC; o += blockDim.x) {
            const int c = o / k, a = o - c * k;
            const double* w = W + c * k;
            double a0 = 0.0, a1 = 0.0;
            int l = 0;
            for (; l + 1 <= a; l += 2) {
                a0 = fma(T[a + l * k], w[l], a0);
                a1 = fma(T[a + (l + 1) * k], w[l + 1], a1);
            }
            if (l == a) a0 = fma(T[a + l * k], w[l], a0);
            W2[a + c * k] = a0 + a1;
        }
        __syncthreads();
        // C -= V W2: C[i][c] -= sum over t = max(0, i - k) .. min(i, k - 1) of V[i][t] W2[t][c]
        for (int o = tid; o < k2 * NC; o += blockDim.x) {
            const int c = o / k2, i = o - c * k2;
            const int t0 = max(0, i - k), t1 = min(i, k - 1);
            const double* w = W2 + c * k;
            double a0 = 0.0, a1 = 0.0;
            int t = t0;
            for (; t + 1 <= t1; t += 2) {
                a0 = fma(V[i + t * k2], w[t], a0);
                a1 = fma(V[i + (t + 1) * k2], w[t + 1], a1);
            }
            if (t == t1) a0 = fma(V[i + t * k2], w[t], a0);
            C[o] -= a0 + a1;
        }
        __syncthreads();
        if (b + 1 == j) {
            for (int c = 0; c < nc; ++c)
                for (int i = tid; i < k2; i += blockDim.x) colp(c)[r0 + i] = C[i + c * k2];
        } else {
            // rows r0 .. r0 + k - 1 are final; the window moves down by k rows
            for (int c = 0; c < nc; ++c)
                for (int i = tid; i < k; i += blockDim.x) {
                    double* x = C + c * k2;
                    colp(c)[r0 + i] = x[i];
                    x[i] = x[i + k];
                    x[i + k] = colp(c)[r0 + 2 * k + i];
                }
        }
        __syncthreads();  // the window is complete and buffer buf is free for block b + 2
    }
}

// k_bhess_apply_q: Z <- Q Z with Q = Q_0 Q_1 .. Q_{jend-1} the product of the block columns'
// compact-WY reflectors (wy, as written by k_bhess_qr_tile), applied from the last block to the
// first: on rows b k .. b k + 2k - 1, C <- C - V_b T_b (V_b^T C). Z has (jend + 1) k rows and
// k columns (ld ldz). With Z = [0; g] (g the last k rows of the transformed right-hand sides)
// the result is the least-squares residual in the basis, G - H Y, so that the Krylov residual
// is the basis times Z. Each CTA (256 threads) takes kApplyCols columns and keeps their 2k-row
// window in shared memory, moving it up by k rows per block; V_b and T_b are read from global
// memory (one call per Krylov cycle). k <= 64, jend >= 1.
inline size_t apply_q_smem(int k) {
    return sizeof(double) * (2 * (size_t)k * k + (size_t)k * (k + 1) + 4 * (size_t)k * kApplyCols);
}
__global__ void __launch_bounds__(256) k_bhess_apply_q(const double* __restrict__ wy, int k, int jend,
                                                       double* __restrict__ Z, int ldz) {
    constexpr int NC = kApplyCols;
    extern __shared__ double sm[];
    const int k2 = 2 * k, bs = wy_stride(k), tid = threadIdx.x, ldt = k + 1;
    double* V = sm;                 // 2k x k (ld 2k)
    double* Ts = V + k2 * k;        // k x k (ld k + 1): Ts[a + l ldt] = T[a][l]
    double* C = Ts + k * ldt;       // 2k x NC (ld 2k)
    double* W = C + k2 * NC;        // k x NC (ld k)
    double* W2 = W + k * NC;        // k x NC (ld k)
    const int q0 = blockIdx.x * NC, nc = min(NC, k - q0);
    auto colp = [&](int c) { return Z + (int64_t)(q0 + c) * ldz; };
    {
        const int r0 = (jend - 1) * k;
        for (int c = 0; c < NC; ++c)
            for (int i = tid; i < k2; i += blockDim.x) C[i + c * k2] = c < nc ? colp(c)[r0 + i] : 0.0;
    }
    for (int b = jend - 1; b >= 0; --b) {
        const int r0 = b * k;
        const double* src = wy + (int64_t)b * bs;
        for (int e = tid; e < k2 * k; e += blockDim.x) V[e] = src[e];
        const double* Tt = src + k2 * k;  // Tt[a + l k] = T[l][a]
        for (int e = tid; e < k * k; e += blockDim.x) {
            const int a = e / k, l = e - a * k;  // e = l + a k: T[a][l]
            Ts[a + l * ldt] = Tt[e];
        }
        __syncthreads();
        // W = V^T C: W[t][c] = sum over i = t .. t + k of V[i][t] C[i][c]
        for (int o = tid; o < k * NC; o += blockDim.x) {
            const int c = o / k, t = o - c * k;
            const double* v = V + t * k2 + t;
            const double* x = C + c * k2 + t;
            double a0 = 0.0, a1 = 0.0;
            int i = 0;
            for (; i + 1 <= k; i += 2) {
                a0 = fma(v[i], x[i], a0);
                a1 = fma(v[i + 1], x[i + 1], a1);
            }
            if (i == k) a0 = fma(v[i], x[i], a0);
            W[t + c * k] = a0 + a1;
        }
        __syncthreads();
        // W2 = T W: W2[a][c] = sum over l >= a of T[a][l] W[l][c]
        for (int o = tid; o < k * NC; o += blockDim.x) {
            const int c = o / k, a = o - c * k;
            const double* w = W + c * k;
            double a0 = 0.0;
            for (int l = a; l < k; ++l) a0 = fma(Ts[a + l * ldt], w[l], a0);
            W2[a + c * k] = a0;
        }
        __syncthreads();
        // C -= V W2
        for (int o = tid; o < k2 * NC; o += blockDim.x) {
            const int c = o / k2, i = o - c * k2;
            const int t0 = max(0, i - k), t1 = min(i, k - 1);
            const double* w = W2 + c * k;
            double a0 = 0.0;
            for (int t = t0; t <= t1; ++t) a0 = fma(V[i + t * k2], w[t], a0);
            C[o] -= a0;
        }
        __syncthreads();
        if (b == 0) {
            for (int c = 0; c < nc; ++c)
                for (int i = tid; i < k2; i += blockDim.x) colp(c)[i] = C[i + c * k2];
        } else {
            // rows r0 + k .. r0 + 2k - 1 are final; the window moves up by k rows
            for (int c = 0; c < nc; ++c)
                for (int i = tid; i < k; i += blockDim.x) {
                    double* x = C + c * k2;
                    colp(c)[r0 + k + i] = x[i + k];
                    x[i + k] = x[i];
                    x[i] = colp(c)[r0 - k + i];
                }
        }
        __syncthreads();
    }
}

}  // namespace bie

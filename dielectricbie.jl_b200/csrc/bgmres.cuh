// Small dense kernels of the block GMRES solver (solver.cu, bgmres): Cholesky factors of
// the k x k Gram matrices (CholQR of each new block of basis vectors) and their inverses,
// their products, the incremental Householder QR of the block upper-Hessenberg matrix with
// its right-hand sides, partial-sum reduction and column gathers. One CTA runs each
// factorisation step; blocks of up to 64 columns keep their tiles in shared memory.
//
// Storage is column-major: A[i + j * lda].
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace bie {

// In-place Cholesky factor of the symmetric positive (semi)definite k x k matrix G
// (upper triangle read): G = R^T R with R upper triangular written to the upper triangle,
// the strict lower triangle zeroed. A pivot below 1e-30 max(diag G) (a direction the block
// cannot extend: its columns are linearly dependent to working precision) is replaced by
// that floor and counted in *nclamp, so the basis stays orthonormal and the corresponding
// coupling in the Hessenberg matrix is tiny. Used for blocks wider than 64 columns.
__global__ void k_chol_upper(double* __restrict__ G, int k, int ldg, int* __restrict__ nclamp) {
    __shared__ double s_piv, s_floor;
    const int tid = threadIdx.x;
    if (tid == 0) {
        double mx = 0.0;
        for (int i = 0; i < k; ++i) mx = fmax(mx, G[i + (int64_t)i * ldg]);
        s_floor = mx > 0.0 ? 1e-30 * mx : 1e-300;
    }
    __syncthreads();
    for (int p = 0; p < k; ++p) {
        if (tid == 0) {
            double d = G[p + (int64_t)p * ldg];
            if (!(d > s_floor)) {
                d = s_floor;
                if (nclamp) atomicAdd(nclamp, 1);
            }
            s_piv = sqrt(d);
            G[p + (int64_t)p * ldg] = s_piv;
        }
        __syncthreads();
        const double piv = s_piv;
        for (int q = p + 1 + tid; q < k; q += blockDim.x) G[p + (int64_t)q * ldg] /= piv;
        __syncthreads();
        const int w = k - p - 1;
        const int64_t cnt = (int64_t)w * w;
        for (int64_t e = tid; e < cnt; e += blockDim.x) {
            const int q = p + 1 + (int)(e / w), r = p + 1 + (int)(e % w);
            if (q <= r) G[q + (int64_t)r * ldg] -= G[p + (int64_t)q * ldg] * G[p + (int64_t)r * ldg];
        }
        __syncthreads();
    }
    for (int64_t e = tid; e < (int64_t)k * k; e += blockDim.x) {
        const int i = (int)(e % k), j = (int)(e / k);
        if (i > j) G[i + (int64_t)j * ldg] = 0.0;
    }
}

// Cholesky factor R of the k x k Gram matrix G (ld k, upper triangle read) and its inverse,
// in shared memory (2 k^2 doubles, k <= 64): R into Rout (ld ldr, lower triangle zeroed),
// R^-1 into Rinv (ld k). Pivots are clamped as in k_chol_upper.
__global__ void k_chol_inv_smem(const double* __restrict__ G, int k, double* __restrict__ Rout, int ldr,
                                double* __restrict__ Rinv, int* __restrict__ nclamp) {
    extern __shared__ double sm[];
    double* A = sm;          // k x k
    double* B = sm + k * k;  // k x k, the inverse
    __shared__ double s_floor;
    const int tid = threadIdx.x;
    for (int e = tid; e < k * k; e += blockDim.x) {
        const int i = e % k, jj = e / k;
        A[e] = i <= jj ? G[i + jj * k] : 0.0;
    }
    __syncthreads();
    if (tid == 0) {
        double mx = 0.0;
        for (int i = 0; i < k; ++i) mx = fmax(mx, A[i + i * k]);
        s_floor = mx > 0.0 ? 1e-30 * mx : 1e-300;
    }
    __syncthreads();
    for (int p = 0; p < k; ++p) {
        // every thread derives the pivot itself
        double d = A[p + p * k];
        const bool clamp = !(d > s_floor);
        if (clamp) d = s_floor;
        const double piv = sqrt(d);
        __syncthreads();  // all have read A[p][p] before it is overwritten
        if (tid == 0) {
            A[p + p * k] = piv;
            if (clamp && nclamp) atomicAdd(nclamp, 1);
        }
        const double inv = 1.0 / piv;
        // trailing update of the upper triangle with the scaled row p, then the row itself
        const int w = k - p - 1;
        for (int e = tid; e < w * w; e += blockDim.x) {
            const int q = p + 1 + e / w, r = p + 1 + e % w;
            if (q <= r) A[q + r * k] -= (A[p + q * k] * inv) * (A[p + r * k] * inv);
        }
        __syncthreads();  // the trailing update has read row p
        for (int q = p + 1 + tid; q < k; q += blockDim.x) A[p + q * k] *= inv;
        __syncthreads();
    }
    // inverse of the upper-triangular R, one column per thread (back substitution)
    for (int jj = tid; jj < k; jj += blockDim.x) {
        for (int i = k - 1; i >= 0; --i) {
            double x = 0.0;
            if (i <= jj) {
                double acc = i == jj ? 1.0 : 0.0;
                for (int l = i + 1; l <= jj; ++l) acc -= A[i + l * k] * B[l + jj * k];
                x = acc / A[i + i * k];
            }
            B[i + jj * k] = x;
        }
    }
    __syncthreads();
    for (int e = tid; e < k * k; e += blockDim.x) {
        const int i = e % k, jj = e / k;
        Rout[i + (int64_t)jj * ldr] = A[e];
        Rinv[e] = B[e];
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

// G = sum_b P[b] of nb partial matrices of kk entries each (a fixed summation order)
__global__ void k_sum_partials(const double* __restrict__ P, int nb, int kk, double* __restrict__ G) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= kk) return;
    double s = 0.0;
    for (int b = 0; b < nb; ++b) s += P[(int64_t)b * kk + e];
    G[e] = s;
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

// Applies the reflector (1, v[c + 1 .. c + k]) with scalar tc to column x over rows c .. c + k,
// the G threads of a group (G consecutive lanes of a warp, sub = lane in the group) sharing the
// dot product. Every lane of the warp calls it (lanes of an idle group with x = null).
__device__ __forceinline__ void apply_reflector(const double* __restrict__ v, double tc, double* x, int c, int k,
                                                int G, int sub) {
    double part = 0.0;
    if (x)
        for (int i = sub; i <= k; i += G) part += (i == 0 ? 1.0 : v[c + i]) * x[c + i];
    for (int o = G / 2; o > 0; o >>= 1) part += __shfl_xor_sync(0xFFFFFFFFu, part, o);
    const double s = part * tc;
    if (x)
        for (int i = sub; i <= k; i += G) x[c + i] -= s * (i == 0 ? 1.0 : v[c + i]);
}

// Threads per column group: the largest power of two G <= 32 with 2 G k <= blockDim.x (k columns
// updated at once by blockDim.x / G groups).
__device__ __forceinline__ int group_width(int k) {
    int G = 1;
    while (G < 32 && 2 * G * k <= (int)blockDim.x) G *= 2;
    return G;
}

// Forms the Householder reflector of column t0 of the tile (local rows t0 .. t0 + k; LAPACK
// dlarfg convention: the column becomes (beta, v tail), tau returned) and applies it to the
// tile's later columns and to the k right-hand-side columns Gt (same rows). Tiles in shared or
// global memory, ld ldt; red: blockDim.x doubles of shared memory.
__device__ __forceinline__ double reflect_column(double* T, int ldt, double* Gt, int ldgt, int t0, int k, double* red,
                                                 double* s_tau, double* s_scale, int G, int sub, int grp, int ngrp) {
    const int tid = threadIdx.x;
    double* col = T + (int64_t)t0 * ldt;
    double part = 0.0;
    for (int i = 1 + tid; i <= k; i += blockDim.x) part += col[t0 + i] * col[t0 + i];
    red[tid] = part;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (tid < w) red[tid] += red[tid + w];
        __syncthreads();
    }
    if (tid == 0) {
        const double sigma = red[0], alpha = col[t0];
        if (sigma == 0.0) {
            *s_tau = 0.0;
            *s_scale = 0.0;
        } else {
            const double mu = sqrt(alpha * alpha + sigma);
            const double beta = alpha <= 0.0 ? mu : -mu;
            *s_tau = (beta - alpha) / beta;
            *s_scale = 1.0 / (alpha - beta);
            col[t0] = beta;
        }
    }
    __syncthreads();
    const double tc = *s_tau;
    if (tc != 0.0) {
        for (int i = 1 + tid; i <= k; i += blockDim.x) col[t0 + i] *= *s_scale;
        __syncthreads();
        const int nrest = k - 1 - t0;
        for (int q0 = 0; q0 < nrest + k; q0 += ngrp) {
            const int q = q0 + grp;
            double* x = q < nrest ? T + (int64_t)(t0 + 1 + q) * ldt
                                  : (q < nrest + k ? Gt + (int64_t)(q - nrest) * ldgt : nullptr);
            apply_reflector(col, tc, x, t0, k, G, sub);
        }
    }
    __syncthreads();
    return tc;
}

// One block column of the incremental Householder QR of the block upper-Hessenberg matrix H
// ((m + 1) k x m k, ldh = (m + 1) k) with the right-hand sides Gv ((m + 1) k x k, ldg). Block
// column j (columns jk .. jk + k - 1) holds the new Gram-Schmidt coefficients in rows
// 0 .. (j + 2) k - 1; its lower k x k block is upper triangular (the CholQR factor), so column
// c has nonzeros down to row c + k and every reflector spans k + 1 rows. The earlier columns'
// reflectors (tails below the diagonal, tau) are applied to the block column in order; then
// each of its columns gets its own reflector, applied to the block's later columns and to Gv.
// resid[a] = || Gv[(j + 1) k .. (j + 2) k - 1, a] ||, the least-squares residual of
// right-hand side a. One CTA of 256 threads, everything in global memory (any k).
__global__ void k_bhess_qr_step(double* __restrict__ H, int ldh, double* __restrict__ tau, double* __restrict__ Gv,
                                int ldg, int k, int j, double* __restrict__ resid) {
    __shared__ double red[256];
    __shared__ double s_tau, s_scale;
    const int tid = threadIdx.x;
    const int c0 = j * k;
    const int G = group_width(k), sub = tid % G, grp = tid / G, ngrp = blockDim.x / G;
    for (int c = 0; c < c0; ++c) {
        const double tc = tau[c];
        if (tc == 0.0) continue;
        const double* v = H + (int64_t)c * ldh;
        for (int t0 = 0; t0 < k; t0 += ngrp) {
            const int t = t0 + grp;
            apply_reflector(v, tc, t < k ? H + (int64_t)(c0 + t) * ldh : nullptr, c, k, G, sub);
        }
    }
    __syncthreads();
    // the new block's tile starts at row c0 of column c0: local row t0 == global row c0 + t0
    double* T = H + (int64_t)c0 * ldh + c0;
    double* Gt = Gv + c0;
    for (int t0 = 0; t0 < k; ++t0) {
        const double tc = reflect_column(T, ldh, Gt, ldg, t0, k, red, &s_tau, &s_scale, G, sub, grp, ngrp);
        if (tid == 0) tau[c0 + t0] = tc;
    }
    for (int a = tid; a < k; a += blockDim.x) {
        const double* g = Gv + (int64_t)a * ldg;
        double s = 0.0;
        for (int i = (j + 1) * k; i < (j + 2) * k; ++i) s += g[i] * g[i];
        resid[a] = sqrt(s);
    }
}

// k_bhess_qr_step with its tiles in shared memory, for k <= 64 (dynamic shared memory
// 4 k^2 + k doubles): the earlier reflectors are applied block by block to the 2k x k tile of
// the new block column that each block touches, then the new block's reflectors are formed on
// its own 2k x k tile together with the matching rows of the right-hand sides.
__global__ void k_bhess_qr_step_smem(double* __restrict__ H, int ldh, double* __restrict__ tau,
                                     double* __restrict__ Gv, int ldg, int k, int j, double* __restrict__ resid) {
    extern __shared__ double sm[];
    const int k2 = 2 * k;
    double* T = sm;           // 2k x k, ld 2k
    double* V = T + k2 * k;   // 2k x k, ld 2k: reflectors of block b, then the right-hand-side rows
    double* tb = V + k2 * k;  // k taus
    __shared__ double red[256];
    __shared__ double s_tau, s_scale;
    const int tid = threadIdx.x;
    const int c0 = j * k;
    const int G = group_width(k), sub = tid % G, grp = tid / G, ngrp = blockDim.x / G;
    for (int b = 0; b < j; ++b) {
        const int r0 = b * k;
        for (int e = tid; e < k2 * k; e += blockDim.x) {
            const int i = e % k2, t = e / k2;
            T[e] = H[(r0 + i) + (int64_t)(c0 + t) * ldh];
            V[e] = H[(r0 + i) + (int64_t)(r0 + t) * ldh];
        }
        for (int t = tid; t < k; t += blockDim.x) tb[t] = tau[r0 + t];
        __syncthreads();
        // each group owns one column of T and applies the block's reflectors to it in order
        for (int t = 0; t < k; ++t) {
            const double tc = tb[t];
            if (tc == 0.0) continue;
            for (int q0 = 0; q0 < k; q0 += ngrp) {
                const int q = q0 + grp;
                apply_reflector(V + t * k2, tc, q < k ? T + q * k2 : nullptr, t, k, G, sub);
            }
        }
        __syncthreads();
        for (int e = tid; e < k2 * k; e += blockDim.x) {
            const int i = e % k2, t = e / k2;
            H[(r0 + i) + (int64_t)(c0 + t) * ldh] = T[e];
        }
        __syncthreads();
    }
    for (int e = tid; e < k2 * k; e += blockDim.x) {
        const int i = e % k2, t = e / k2;
        T[e] = H[(c0 + i) + (int64_t)(c0 + t) * ldh];
        V[e] = Gv[(c0 + i) + (int64_t)t * ldg];
    }
    __syncthreads();
    for (int t0 = 0; t0 < k; ++t0) {
        const double tc = reflect_column(T, k2, V, k2, t0, k, red, &s_tau, &s_scale, G, sub, grp, ngrp);
        if (tid == 0) tau[c0 + t0] = tc;
    }
    for (int e = tid; e < k2 * k; e += blockDim.x) {
        const int i = e % k2, t = e / k2;
        H[(c0 + i) + (int64_t)(c0 + t) * ldh] = T[e];
        Gv[(c0 + i) + (int64_t)t * ldg] = V[e];
    }
    for (int a = tid; a < k; a += blockDim.x) {
        const double* g = V + a * k2;
        double s = 0.0;
        for (int i = k; i < k2; ++i) s += g[i] * g[i];
        resid[a] = sqrt(s);
    }
}

}  // namespace bie

// Adaptive near-field blocks on the GPU: the moment sums of touching panel pairs
// (adaptive_block_moments_inplace!, src/kernel/laplace3d_near_adaptive.jl:308-387)
// over the quadtree leaves the host's walk produced.
//
//   Kb[t][a nq + b] = sum_{leaf} sum_{gi, gj} (w_gi w_gj s_leaf) r_a(u) r_b(v) G_n(y(u, v), x_t, n_trg)
//
// One CTA per pair. Per leaf the CTA stages the barycentric rows r(u), r(v), the
// quadrature weights and the kernel values at every (quadrature point, target) in
// shared memory; each thread then accumulates its (target, basis) outputs over the
// leaf's quadrature points in the host's order with explicitly rounded operations,
// so the blocks are bitwise those of the host code (which has no fused multiply-add).
//
// Upsampled near-field blocks on the GPU (laplace3d_DT_corrections,
// src/kernel/laplace3d_near_upsampling.jl:127-270): for source panel i at its upsampling
// order n_up (the maximum over its neighbours) and each of its target panels j,
//
//   block[s][t] = sum_alpha Mt[s][alpha] G_n(p_up[alpha], x_t, n_j) - G_n(y_s, x_t, n_j) w_s
//
// with Mt the barycentric-interpolated upsampled quadrature (build_source_cache). One CTA
// per source panel stages p_up and Mt once, then the kernel values of each target panel;
// every sum runs in the host's order with explicitly rounded operations, so the blocks are
// bitwise those of the host code.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include "host_setup.h"

namespace bie {
namespace {

constexpr int kMaxNq = 16;
constexpr int kMaxGL = 16;
constexpr double kFourPiD = 4.0 * 3.14159265358979323846;  // the host's 4.0 * M_PI

struct V3d {
    double x, y, z;
};

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// G_n(src -> trg) with normal n, in the host's operation order (lap_grad).
__device__ double lap_grad_d(V3d s, V3d t, V3d n) {
    const double dx = sub(s.x, t.x), dy = sub(s.y, t.y), dz = sub(s.z, t.z);
    const double r2 = add(add(mul(dx, dx), mul(dy, dy)), mul(dz, dz));
    const double ir = __ddiv_rn(1.0, __dsqrt_rn(r2));
    const double i3 = mul(mul(ir, ir), ir);
    const double ex = sub(t.x, s.x), ey = sub(t.y, s.y), ez = sub(t.z, s.z);
    return __ddiv_rn(add(add(mul(n.x, mul(i3, ex)), mul(n.y, mul(i3, ey))), mul(n.z, mul(i3, ez))), kFourPiD);
}

// Barycentric Lagrange row at xq (bary_row): unit row at a node (isapprox rtol sqrt(eps)).
__device__ void bary_row_d(int n, const double* x, const double* lam, double xq, double* r) {
    const double rt = 1.4901161193847656e-08;
    for (int i = 0; i < n; ++i)
        if (xq == x[i] || fabs(sub(xq, x[i])) <= mul(rt, fmax(fabs(xq), fabs(x[i])))) {
            for (int k = 0; k < n; ++k) r[k] = 0.0;
            r[i] = 1.0;
            return;
        }
    double den = 0.0;
    for (int i = 0; i < n; ++i) {
        r[i] = __ddiv_rn(lam[i], sub(xq, x[i]));
        den = add(den, r[i]);
    }
    const double inv = __ddiv_rn(1.0, den);
    for (int i = 0; i < n; ++i) r[i] = mul(r[i], inv);
}

struct Tables {
    int nq, ngl;
    double glx[kMaxNq], bary[kMaxNq], xg[kMaxGL], wg[kMaxGL];
};

// frame[p] = cc (3), bma (3), dma (3), scale; trg[p] = target panel; leaves[l] = ulo, uhi, vlo, vhi.
__global__ void __launch_bounds__(256) k_adaptive_blocks(Tables tb, const double* __restrict__ pts,
                                                         const double* __restrict__ normals,
                                                         const double* __restrict__ frames,
                                                         const int* __restrict__ trg,
                                                         const int64_t* __restrict__ leaf_off,
                                                         const double* __restrict__ leaves, double* __restrict__ Kb) {
    extern __shared__ double sm[];
    const int nq = tb.nq, ng = tb.ngl, np = nq * nq, nqp = ng * ng;
    double* kv = sm;                   // [nqp][np] kernel values
    double* rx = kv + (size_t)nqp * np;  // [ng][nq] rows at u_gi
    double* ry = rx + ng * nq;         // [ng][nq] rows at v_gj
    double* wq = ry + ng * nq;         // [nqp] w_gi w_gj s_leaf
    const int pr = blockIdx.x;
    const double* fr = frames + (size_t)pr * 10;
    const V3d cc{fr[0], fr[1], fr[2]}, bma{fr[3], fr[4], fr[5]}, dma{fr[6], fr[7], fr[8]};
    const double scale = fr[9];
    const int j = trg[pr];
    const V3d nt{normals[3 * j], normals[3 * j + 1], normals[3 * j + 2]};
    const int nout = np * np;
    double acc[6];  // outputs o = threadIdx.x + 256 u (np^2 <= 1296 for nq <= 6)
    const int nu = (nout + 255) / 256;
    for (int u = 0; u < 6; ++u) acc[u] = 0.0;
    for (int64_t l = leaf_off[pr]; l < leaf_off[pr + 1]; ++l) {
        const double* L = leaves + 4 * l;
        const double hu = __ddiv_rn(sub(L[1], L[0]), 2.0), hv = __ddiv_rn(sub(L[3], L[2]), 2.0);
        const double mu = __ddiv_rn(add(L[1], L[0]), 2.0), mv = __ddiv_rn(add(L[3], L[2]), 2.0);
        const double sc = mul(mul(hu, hv), scale);
        __syncthreads();  // previous leaf's staging consumed
        for (int e = threadIdx.x; e < ng; e += blockDim.x) {
            bary_row_d(nq, tb.glx, tb.bary, add(mu, mul(hu, tb.xg[e])), rx + e * nq);
            bary_row_d(nq, tb.glx, tb.bary, add(mv, mul(hv, tb.xg[e])), ry + e * nq);
        }
        for (int e = threadIdx.x; e < nqp; e += blockDim.x) {
            const int gi = e / ng, gj = e - gi * ng;
            wq[e] = mul(mul(tb.wg[gi], tb.wg[gj]), sc);
        }
        for (int e = threadIdx.x; e < nqp * np; e += blockDim.x) {
            const int q = e / np, t = e - q * np;
            const int gi = q / ng, gj = q - gi * ng;
            const double uu = add(mu, mul(hu, tb.xg[gi])), vv = add(mv, mul(hv, tb.xg[gj]));
            const double hu2 = __ddiv_rn(uu, 2.0), hv2 = __ddiv_rn(vv, 2.0);
            const V3d y{add(add(cc.x, mul(bma.x, hu2)), mul(dma.x, hv2)),
                        add(add(cc.y, mul(bma.y, hu2)), mul(dma.y, hv2)),
                        add(add(cc.z, mul(bma.z, hu2)), mul(dma.z, hv2))};
            const double* xt = pts + 3 * ((size_t)j * np + t);
            kv[e] = lap_grad_d(y, V3d{xt[0], xt[1], xt[2]}, nt);
        }
        __syncthreads();
        for (int u = 0; u < nu && u < 6; ++u) {
            const int o = threadIdx.x + 256 * u;
            if (o >= nout) break;
            const int t = o / np, ab = o - t * np, a = ab / nq, b = ab - a * nq;
            double s = acc[u];
            for (int q = 0; q < nqp; ++q) {
                const int gi = q / ng, gj = q - gi * ng;
                const double wm = mul(mul(wq[q], rx[gi * nq + a]), ry[gj * nq + b]);
                s = add(s, mul(wm, kv[q * np + t]));
            }
            acc[u] = s;
        }
    }
    double* out = Kb + (size_t)pr * nout;
    for (int u = 0; u < nu && u < 6; ++u) {
        const int o = threadIdx.x + 256 * u;
        if (o < nout) out[o] = acc[u];
    }
}

constexpr int kMaxUp = 8;  // upsampling orders handled on the GPU (n_up^2 <= 64 staged points)

// One CTA per job (source panel). job_frame[10 q ..] = (cc, b - a, d - a, scale) of the
// source; tables per order n (stride kMaxUp + 1): xu[n][i], wu[n][i], ex[n][i][m] (the
// barycentric rows of the upsampled nodes on the panel's n_quad Gauss nodes). Output:
// block of pair p = tgt_off[q] + e at out[p * np^2], column-major (s * np + t).
__global__ void __launch_bounds__(256) k_upsampled_blocks(int nq, const double* __restrict__ pts,
                                                          const double* __restrict__ w,
                                                          const double* __restrict__ normals,
                                                          const int* __restrict__ job_src,
                                                          const int* __restrict__ job_nup,
                                                          const double* __restrict__ job_frame,
                                                          const int64_t* __restrict__ tgt_off,
                                                          const int* __restrict__ tgt, const double* __restrict__ xu,
                                                          const double* __restrict__ wu, const double* __restrict__ ex,
                                                          double* __restrict__ out) {
    extern __shared__ double sm[];
    const int q = blockIdx.x;
    const int np = nq * nq;
    const int n_up = job_nup[q], nu2 = n_up * n_up;
    const int src = job_src[q];
    double* pu = sm;                  // [nu2][3] upsampled source points
    double* Mt = pu + 3 * nu2;        // [np][nu2]
    double* km = Mt + (size_t)np * nu2;  // [np][nu2] kernel values at one target panel
    const double* fr = job_frame + (size_t)q * 10;
    const double* xn = xu + (size_t)n_up * (kMaxUp + 1);
    const double* wn = wu + (size_t)n_up * (kMaxUp + 1);
    const double* en = ex + (size_t)n_up * (kMaxUp + 1) * nq;
    for (int a = threadIdx.x; a < nu2; a += blockDim.x) {
        const int i = a / n_up, j = a - i * n_up;
        const double hi = __ddiv_rn(xn[i], 2.0), hj = __ddiv_rn(xn[j], 2.0);
        pu[3 * a + 0] = add(add(fr[0], mul(fr[3], hi)), mul(fr[6], hj));
        pu[3 * a + 1] = add(add(fr[1], mul(fr[4], hi)), mul(fr[7], hj));
        pu[3 * a + 2] = add(add(fr[2], mul(fr[5], hi)), mul(fr[8], hj));
    }
    for (int e = threadIdx.x; e < np * nu2; e += blockDim.x) {
        const int mm = e / nu2, a = e - mm * nu2;
        const int mx = mm / nq, my = mm - mx * nq, i = a / n_up, j = a - i * n_up;
        Mt[e] = mul(mul(mul(mul(fr[9], wn[i]), wn[j]), en[i * nq + mx]), en[j * nq + my]);
    }
    for (int64_t p = tgt_off[q]; p < tgt_off[q + 1]; ++p) {
        const int trg = tgt[p];
        const V3d nt{normals[3 * trg], normals[3 * trg + 1], normals[3 * trg + 2]};
        __syncthreads();  // staging done / previous target's values consumed
        for (int e = threadIdx.x; e < np * nu2; e += blockDim.x) {
            const int t = e / nu2, a = e - t * nu2;
            const double* xt = pts + 3 * ((size_t)trg * np + t);
            km[e] = lap_grad_d(V3d{pu[3 * a], pu[3 * a + 1], pu[3 * a + 2]}, V3d{xt[0], xt[1], xt[2]}, nt);
        }
        __syncthreads();
        double* o = out + (size_t)p * np * np;
        for (int e = threadIdx.x; e < np * np; e += blockDim.x) {
            const int t = e / np, mm = e - t * np;
            const double* mt = Mt + (size_t)mm * nu2;
            const double* kv = km + (size_t)t * nu2;
            double acc = 0.0;
            for (int a = 0; a < nu2; ++a) acc = add(acc, mul(mt[a], kv[a]));
            const size_t js = (size_t)src * np + mm;
            const double* xt = pts + 3 * ((size_t)trg * np + t);
            const double kd = mul(lap_grad_d(V3d{pts[3 * js], pts[3 * js + 1], pts[3 * js + 2]},
                                             V3d{xt[0], xt[1], xt[2]}, nt),
                                  w[js]);
            o[(size_t)mm * np + t] = sub(acc, kd);
        }
    }
}

}  // namespace

int upsampled_blocks_gpu(int device, int nq, const double* pts, int64_t npts, const double* w, const double* normals,
                         int npanels, int njobs, const int* job_src, const int* job_nup, const double* job_frame,
                         const int64_t* tgt_off, const int* tgt, const double* xu, const double* wu, const double* ex,
                         double* out, std::string& err) {
    if (njobs == 0) return 0;
    if (nq > 6) {
        err = "upsampled blocks on the GPU support n_quad <= 6";
        return -1;
    }
    int max_up = 0;
    for (int q = 0; q < njobs; ++q) max_up = std::max(max_up, job_nup[q]);
    if (max_up > kMaxUp) {
        err = "upsampled blocks on the GPU support n_up <= 8";
        return -1;
    }
    const int np = nq * nq;
    const int64_t npairs = tgt_off[njobs];
    int prev = 0;
    cudaGetDevice(&prev);
    std::vector<void*> bufs;
    // set-up work runs on its own non-blocking stream with stream-ordered allocations, so it
    // neither waits for nor stalls the solves running on other streams (a cudaFree would
    // synchronise the whole device)
    cudaStream_t st = nullptr;
    auto fail = [&](cudaError_t e, const char* what) {
        for (void* p : bufs) cudaFreeAsync(p, st);
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        cudaSetDevice(prev);
        err = std::string(what) + ": " + cudaGetErrorString(e);
        cudaGetLastError();
        return -1;
    };
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(e, "cudaSetDevice");
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "cudaStreamCreate");
    auto upload = [&](const void* src, size_t bytes, void** dst) -> cudaError_t {
        cudaError_t r = cudaMallocAsync(dst, bytes > 0 ? bytes : 8, st);
        if (r != cudaSuccess) return r;
        bufs.push_back(*dst);
        return bytes ? cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, st) : cudaSuccess;
    };
    auto finish = [&]() {
        for (void* p : bufs) cudaFreeAsync(p, st);
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
        cudaSetDevice(prev);
    };
    const size_t tab = (size_t)(kMaxUp + 1) * (kMaxUp + 1);
    void *d_pts, *d_w, *d_nrm, *d_js, *d_jn, *d_fr, *d_off, *d_tgt, *d_xu, *d_wu, *d_ex, *d_out;
    if ((e = upload(pts, sizeof(double) * 3 * npts, &d_pts)) != cudaSuccess) return fail(e, "upload");
    if ((e = upload(w, sizeof(double) * npts, &d_w)) != cudaSuccess) return fail(e, "upload");
    if ((e = upload(normals, sizeof(double) * 3 * npanels, &d_nrm)) != cudaSuccess) return fail(e, "upload");
    if ((e = upload(job_src, sizeof(int) * njobs, &d_js)) != cudaSuccess) return fail(e, "upload");
    if ((e = upload(job_nup, sizeof(int) * njobs, &d_jn)) != cudaSuccess) return fail(e, "upload");
    if ((e = upload(job_frame, sizeof(double) * 10 * njobs, &d_fr)) != cudaSuccess) return fail(e, "upload");
    if ((e = upload(tgt_off, sizeof(int64_t) * (njobs + 1), &d_off)) != cudaSuccess) return fail(e, "upload");
    if ((e = upload(tgt, sizeof(int) * npairs, &d_tgt)) != cudaSuccess) return fail(e, "upload");
    if ((e = upload(xu, sizeof(double) * tab, &d_xu)) != cudaSuccess) return fail(e, "upload");
    if ((e = upload(wu, sizeof(double) * tab, &d_wu)) != cudaSuccess) return fail(e, "upload");
    if ((e = upload(ex, sizeof(double) * tab * nq, &d_ex)) != cudaSuccess) return fail(e, "upload");
    if ((e = cudaMallocAsync(&d_out, sizeof(double) * (size_t)npairs * np * np, st)) != cudaSuccess)
        return fail(e, "cudaMallocAsync");
    bufs.push_back(d_out);
    const int nu2 = max_up * max_up;
    const size_t smem = sizeof(double) * (3 * (size_t)nu2 + 2 * (size_t)np * nu2);
    if (smem > 48 * 1024 &&
        (e = cudaFuncSetAttribute(k_upsampled_blocks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
            cudaSuccess)
        return fail(e, "cudaFuncSetAttribute");
    k_upsampled_blocks<<<njobs, 256, smem, st>>>(nq, (const double*)d_pts, (const double*)d_w, (const double*)d_nrm,
                                             (const int*)d_js, (const int*)d_jn, (const double*)d_fr,
                                             (const int64_t*)d_off, (const int*)d_tgt, (const double*)d_xu,
                                             (const double*)d_wu, (const double*)d_ex, (double*)d_out);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "k_upsampled_blocks launch");
    if ((e = cudaMemcpyAsync(out, d_out, sizeof(double) * (size_t)npairs * np * np, cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return fail(e, "k_upsampled_blocks");
    finish();
    return 0;
}

int adaptive_blocks_gpu(int device, int nq, int ngl, const double* glx, const double* bary, const double* xg,
                        const double* wg, const double* pts, int64_t npts, const double* normals, int npanels,
                        int npairs, const int* trg, const double* frames, const int64_t* leaf_off,
                        const double* leaves, double* Kb, std::string& err) {
    if (npairs == 0) return 0;
    if (nq > 6 || ngl > kMaxGL) {
        err = "adaptive blocks on the GPU support n_quad <= 6 and n_GL <= 16";
        return -1;
    }
    Tables tb{};
    tb.nq = nq;
    tb.ngl = ngl;
    for (int i = 0; i < nq; ++i) {
        tb.glx[i] = glx[i];
        tb.bary[i] = bary[i];
    }
    for (int i = 0; i < ngl; ++i) {
        tb.xg[i] = xg[i];
        tb.wg[i] = wg[i];
    }
    const int np = nq * nq;
    const int64_t nleaves = leaf_off[npairs];
    int prev = 0;
    cudaGetDevice(&prev);
    std::vector<void*> bufs;
    // set-up work runs on its own non-blocking stream with stream-ordered allocations, so it
    // neither waits for nor stalls the solves running on other streams (a cudaFree would
    // synchronise the whole device)
    cudaStream_t st = nullptr;
    auto fail = [&](cudaError_t e, const char* what) {
        for (void* p : bufs) cudaFreeAsync(p, st);
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        cudaSetDevice(prev);
        err = std::string(what) + ": " + cudaGetErrorString(e);
        cudaGetLastError();
        return -1;
    };
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(e, "cudaSetDevice");
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "cudaStreamCreate");
    auto upload = [&](const void* src, size_t bytes, void** dst) -> cudaError_t {
        cudaError_t r = cudaMallocAsync(dst, bytes > 0 ? bytes : 8, st);
        if (r != cudaSuccess) return r;
        bufs.push_back(*dst);
        return bytes ? cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, st) : cudaSuccess;
    };
    auto finish = [&]() {
        for (void* p : bufs) cudaFreeAsync(p, st);
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
        cudaSetDevice(prev);
    };
    void *d_pts, *d_nrm, *d_fr, *d_trg, *d_off, *d_leaves, *d_kb;
    if ((e = upload(pts, sizeof(double) * 3 * npts, &d_pts)) != cudaSuccess) return fail(e, "upload");
    if ((e = upload(normals, sizeof(double) * 3 * npanels, &d_nrm)) != cudaSuccess) return fail(e, "upload");
    if ((e = upload(frames, sizeof(double) * 10 * npairs, &d_fr)) != cudaSuccess) return fail(e, "upload");
    if ((e = upload(trg, sizeof(int) * npairs, &d_trg)) != cudaSuccess) return fail(e, "upload");
    if ((e = upload(leaf_off, sizeof(int64_t) * (npairs + 1), &d_off)) != cudaSuccess) return fail(e, "upload");
    if ((e = upload(leaves, sizeof(double) * 4 * nleaves, &d_leaves)) != cudaSuccess) return fail(e, "upload");
    if ((e = cudaMallocAsync(&d_kb, sizeof(double) * (size_t)npairs * np * np, st)) != cudaSuccess)
        return fail(e, "cudaMallocAsync");
    bufs.push_back(d_kb);
    const size_t smem = sizeof(double) * ((size_t)ngl * ngl * np + 2 * ngl * nq + ngl * ngl);
    if (smem > 48 * 1024 &&
        (e = cudaFuncSetAttribute(k_adaptive_blocks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
            cudaSuccess)
        return fail(e, "cudaFuncSetAttribute");
    k_adaptive_blocks<<<npairs, 256, smem, st>>>(tb, (const double*)d_pts, (const double*)d_nrm, (const double*)d_fr,
                                             (const int*)d_trg, (const int64_t*)d_off, (const double*)d_leaves,
                                             (double*)d_kb);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "k_adaptive_blocks launch");
    if ((e = cudaMemcpyAsync(Kb, d_kb, sizeof(double) * (size_t)npairs * np * np, cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return fail(e, "k_adaptive_blocks");
    finish();
    return 0;
}

}  // namespace bie

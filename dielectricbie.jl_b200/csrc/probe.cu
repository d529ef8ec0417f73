// Device side of near-accurate probe potentials (laplace3d_pottrg_fmm3d_corrected_hcubature,
// src/kernel/laplace3d_near_hcubature.jl:278-316):
//
//   sigma_ref = P sigma                 (prolongation onto the refined interface, CSR)
//   phi       = S_refined sigma_ref     (FP64 direct sum of the refined nodes at the probes)
//             + C sigma_ref             (adaptive-quadrature corrections, CSR)
//
// P and C come from the host set-up (probe_setup.cpp); the direct sum is the library's
// potential kernel on a geometry of the refined nodes.
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "common.cuh"
#include "host_setup.h"
#include "solver.h"

namespace bie {
namespace {

// sref[r][c] = sum_j P[r, j] S[j + c N]  (S column-major N x k, sref node-major nref x k)
__global__ void k_prolong(const int64_t* __restrict__ prow, const int32_t* __restrict__ pcol,
                          const double* __restrict__ pval, const double* __restrict__ S, int64_t N, int64_t nref,
                          int k, double* __restrict__ sref) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nref * k) return;
    const int64_t r = e / k;
    const int c = (int)(e - r * k);
    double s = 0.0;
    for (int64_t j = prow[r]; j < prow[r + 1]; ++j) s += pval[j] * S[pcol[j] + c * N];
    sref[e] = s;
}

// out[m + c M] = phi[m k + c] + sum_j C[m, j] sref[j k + c]
__global__ void k_probe_correct(const int64_t* __restrict__ crow, const int32_t* __restrict__ ccol,
                                const double* __restrict__ cval, const double* __restrict__ sref,
                                const double* __restrict__ phi, int64_t M, int k, double* __restrict__ out) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M * k) return;
    const int64_t m = e / k;
    const int c = (int)(e - m * k);
    double s = phi[e];
    for (int64_t j = crow[m]; j < crow[m + 1]; ++j) s += cval[j] * sref[(int64_t)ccol[j] * k + c];
    out[m + c * M] = s;
}

template <class T>
void put(Buf& b, const std::vector<T>& v, cudaStream_t s) {
    b.ensure(sizeof(T) * std::max<size_t>(v.size(), 1));
    if (!v.empty()) BIE_CK(cudaMemcpyAsync(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s));
}

unsigned blocks_for(int64_t n) { return (unsigned)std::max<int64_t>(1, (n + 255) / 256); }

}  // namespace

struct ProbeDev {
    int device = 0;
    bie_geom* gref = nullptr;
    int64_t M = 0, N = 0, nref = 0;
    Buf prow, pcol, pval, crow, ccol, cval, tgt, sig, sref, phi, out;
};

ProbeDev* probe_upload(const ProbeSetup& ps, const double* targets, int64_t M, int64_t ncoarse, int device) {
    ProbeDev* d = new ProbeDev();
    d->device = device;
    d->M = M;
    d->N = ncoarse;
    const Mesh& r = ps.refined;
    d->nref = r.npoints();
    const int np = r.nq * r.nq;
    std::vector<double> nrm((size_t)3 * d->nref), zeros((size_t)d->nref, 0.0);
    for (int p = 0; p < r.npanels; ++p)
        for (int t = 0; t < np; ++t)
            for (int c = 0; c < 3; ++c) nrm[3 * ((size_t)p * np + t) + c] = r.normals[3 * p + c];
    try {
        d->gref = geom_create(r.pts.data(), nrm.data(), r.w.data(), zeros.data(), d->nref, r.npanels, 0, nullptr,
                              nullptr, nullptr, 0, device);
        int prev = 0;
        BIE_CK(cudaGetDevice(&prev));
        BIE_CK(cudaSetDevice(device));
        cudaStream_t s = (cudaStream_t)geom_stream(d->gref);
        put(d->prow, ps.prow, s);
        put(d->pcol, ps.pcol, s);
        put(d->pval, ps.pval, s);
        put(d->crow, ps.crow, s);
        put(d->ccol, ps.ccol, s);
        put(d->cval, ps.cval, s);
        d->tgt.ensure(sizeof(double) * std::max<int64_t>(3 * M, 1));
        if (M) BIE_CK(cudaMemcpyAsync(d->tgt.p, targets, sizeof(double) * 3 * M, cudaMemcpyHostToDevice, s));
        BIE_CK(cudaStreamSynchronize(s));
        cudaSetDevice(prev);
    } catch (...) {
        probe_free(d);
        throw;
    }
    return d;
}

void probe_apply(ProbeDev* d, const double* Sigma, int k, double* phi_out) {
    int prev = 0;
    BIE_CK(cudaGetDevice(&prev));
    BIE_CK(cudaSetDevice(d->device));
    cudaStream_t s = (cudaStream_t)geom_stream(d->gref);
    const int64_t M = d->M, N = d->N, nref = d->nref;
    d->sig.ensure(sizeof(double) * std::max<int64_t>(N * k, 1));
    d->sref.ensure(sizeof(double) * std::max<int64_t>(nref * k, 1));
    d->phi.ensure(sizeof(double) * std::max<int64_t>(M * k, 1));
    d->out.ensure(sizeof(double) * std::max<int64_t>(M * k, 1));
    BIE_CK(cudaMemcpyAsync(d->sig.p, Sigma, sizeof(double) * N * k, cudaMemcpyHostToDevice, s));
    k_prolong<<<blocks_for(nref * k), 256, 0, s>>>(d->prow.as<int64_t>(), d->pcol.as<int32_t>(), d->pval.as<double>(),
                                                  d->sig.as<double>(), N, nref, k, d->sref.as<double>());
    BIE_CK(cudaGetLastError());
    if (M > 0) {
        potential_device(d->gref, d->sref.as<double>(), k, d->tgt.as<double>(), M, d->phi.as<double>(), s);
        k_probe_correct<<<blocks_for(M * k), 256, 0, s>>>(d->crow.as<int64_t>(), d->ccol.as<int32_t>(),
                                                         d->cval.as<double>(), d->sref.as<double>(),
                                                         d->phi.as<double>(), M, k, d->out.as<double>());
        BIE_CK(cudaGetLastError());
        BIE_CK(cudaMemcpyAsync(phi_out, d->out.p, sizeof(double) * M * k, cudaMemcpyDeviceToHost, s));
    }
    BIE_CK(cudaStreamSynchronize(s));
    cudaSetDevice(prev);
}

void probe_free(ProbeDev* d) {
    if (!d) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(d->device);
    Buf* bufs[] = {&d->prow, &d->pcol, &d->pval, &d->crow, &d->ccol, &d->cval, &d->tgt, &d->sig, &d->sref, &d->phi, &d->out};
    for (Buf* b : bufs) b->release();
    if (d->gref) geom_destroy(d->gref);
    cudaSetDevice(prev);
    delete d;
}

}  // namespace bie

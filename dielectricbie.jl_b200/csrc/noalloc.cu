// FP64 direct sum of the adjoint double layer that allocates no device memory.
//
//   Y[i][c] = 1/(4 pi) sum_{j != i} n_i.(x_i - y_j)/|x_i - y_j|^3 w_j X[j][c]
//
// The regular entry points keep their split partials in device buffers that a
// geometry handle grows with cudaMalloc. Some callers cannot have the library
// allocate: a host runtime whose pool allocator already owns the device memory
// (Julia's CUDA.jl, PyTorch's caching allocator), where a foreign cudaMalloc can
// fail although the pool holds free memory, and latency-bound services that
// reserve their memory at start-up, because cudaMalloc and cudaFree synchronise
// the device and stall the other streams. For them the partials live in one
// file-scope device array of a fixed size, and the caller passes every input and
// output buffer.
//
// The split partials come from the FP64 tensor-core direct-sum kernel of the
// regular path (K1, dt64mma.cu); the reduction over splits below writes Y.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "common.cuh"
#include "solver.h"

namespace bie {
namespace {

// 4,194,304 doubles (32 MiB): split partials of the column group being summed.
constexpr int64_t kScratchDoubles = int64_t(1) << 22;
static __device__ __align__(256) double g_dt_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
double* g_scratch_ptr[kMaxDevices] = {};
int g_sms[kMaxDevices] = {};

// Device address of the scratch array and the SM count of the current device,
// looked up on the first call on that device. In host code g_dt_scratch names a
// host-side stand-in, so the address comes from cudaGetSymbolAddress. The array is
// part of the library's device module: with lazy module loading (the CUDA 12 default)
// the module, and with it the 32 MiB, is committed on the device at this lookup, so
// the first call must come before a pool allocator reserves the device's memory; with
// CUDA_MODULE_LOADING=EAGER every context that loads the library holds the 32 MiB from
// the start, whether or not this entry point is used.
void scratch_for_current_device(double** ptr, int* sms) {
    int dev = -1;
    BIE_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw Error(BIE_EUNSUPPORTED, "dt_apply_static: device index out of range");
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_dt_scratch);
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            throw Error(BIE_ENOMEM,
                        "dt_apply_static: the device had no room to load the library's 32 MiB scratch array; make "
                        "the first call on each device before a pool allocator reserves its memory");
        }
        BIE_CK(e);
        int n_sm = 0;
        BIE_CK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
        g_sms[dev] = n_sm;
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    *ptr = g_scratch_ptr[dev];
    *sms = g_sms[dev];
}

// Y[i * ldy + c0 + c] = 1/(4 pi) sum_s part[(s n + i) kc + c], for i < n, c < kc.
__global__ void k_sum_splits(const double* __restrict__ part, int nsplit, int64_t n, int kc, double* __restrict__ Y,
                             int ldy, int c0) {
    const int64_t total = n * kc;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / kc;
        const int c = (int)(e - i * kc);
        double acc = 0.0;
        for (int s = 0; s < nsplit; ++s) acc += part[((int64_t)s * n + i) * kc + c];
        Y[i * ldy + c0 + c] = kInv4Pi * acc;
    }
}

}  // namespace

int64_t dt_apply_static_max_nodes() { return kScratchDoubles; }

// Sizes are checked before any CUDA call, so a rejected request touches no device.
void dt_apply_static(const double* x, const double* y, const double* z, const double* nx, const double* ny,
                     const double* nz, const double* w, int64_t n, const double* X, int k, double* Y,
                     cudaStream_t s) {
    if (!x || !y || !z || !nx || !ny || !nz || !w || !X || !Y || n < 1 || k < 1)
        throw Error(BIE_EINVAL, "dt_apply_static: bad argument");
    if (n > kScratchDoubles)
        throw Error(BIE_EINVAL, "dt_apply_static: n = " + std::to_string(n) + " nodes exceeds the maximum of " +
                                    std::to_string(kScratchDoubles) +
                                    " (its fixed 32 MiB scratch holds one partial column per node at least)");
    double* scratch = nullptr;
    int sms = 0;
    scratch_for_current_device(&scratch, &sms);

    GeomDev g;
    g.x = x; g.y = y; g.z = z;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.w = w;
    g.n = n;
    g.perm = nullptr;  // the FP64 kernel reads targets in node order

    // columns per group and source splits, so that nsplit * n * kc fits the scratch. The
    // split count follows the regular FP64 path's base rule (about four waves of 128-target
    // tiles at two per SM); the kernel's CTAs hold 64 targets at three per SM, so this gives
    // them about twice the splits of a matched wave model, which measured faster there
    const int kc = (int)std::min<int64_t>({64, (int64_t)k, kScratchDoubles / n});
    const int64_t tiles = (n + 127) / 128;
    const int64_t want = (int64_t)sms * 2 * 4;
    int64_t ns = std::max<int64_t>(1, (want + tiles - 1) / tiles);
    ns = std::min<int64_t>(ns, std::max<int64_t>(1, (n + 127) / 128));
    ns = std::min<int64_t>(ns, kScratchDoubles / (n * kc));
    int64_t chunk = (n + ns - 1) / ns;
    chunk = (chunk + 127) / 128 * 128;
    ns = (n + chunk - 1) / chunk;

    for (int c0 = 0; c0 < k; c0 += kc) {
        const int kg = std::min(kc, k - c0);
        launch_dt_f64_mma(g, X + c0, k, 0, kg, nullptr, (int)ns, chunk, scratch, kg, s);
        const int64_t total = n * kg;
        const unsigned blocks = (unsigned)std::min<int64_t>((total + 255) / 256, (int64_t)sms * 8);
        k_sum_splits<<<blocks, 256, 0, s>>>(scratch, (int)ns, n, kg, Y, k, c0);
        BIE_CK(cudaGetLastError());
    }
}

}  // namespace bie

// Device-side types shared by the kernel translation units.
#pragma once
#include <vector>
#include <cuda_runtime.h>
#include <stdint.h>

namespace bie {

// Packed FP32 pairs (sm_100 f32x2 arithmetic): one instruction applies the same
// round-to-nearest operation to two lanes of data.
__device__ __forceinline__ uint64_t pk2(float lo, float hi) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ float2 upk2(uint64_t r) {
    float2 v;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
    return v;
}
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t mul2(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}


constexpr double kInv4Pi = 0.079577471545947667884;  // 1 / (4 pi)
constexpr int kTB = 128;  // targets per CTA of the direct-sum kernels (one per thread)
constexpr int kTS = 128;  // sources per shared-memory tile

// MUFU reciprocal square root (approximate, flush-to-zero): a single instruction.
__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Device-resident geometry: SoA FP64 arrays of length n.
struct GeomDev {
    const double *x, *y, *z;     // node positions
    const double *nx, *ny, *nz;  // node normals
    const double* w;             // quadrature weights
    int64_t n;
    // Target order of the reduced-precision kernels: nodes sorted along a Morton
    // curve, so that a 128-target tile is spatially compact and coordinates rounded
    // to FP32 relative to the tile's first target stay accurate for near pairs.
    const int32_t* perm;
};

// K3 (blocktc.cu): tensor-core block direct sum for columns [c0, c0 + kc), kc <= 128,
// kernel and right-hand sides split into `pieces` bf16 pieces (2 or 3).
void launch_block_tc(const GeomDev& g, const double* X, int ldx, int c0, int kc, const double* pre, int nsplit,
                     int64_t cps, float* part, int ldp, uint8_t* bpack, int* err, int pieces, int force_ctas,
                     cudaStream_t s);
size_t block_tc_pack_bytes(int64_t n, int kc, int pieces);
// One geometry's share of a K3 work-list launch: columns [c0, c0 + kc) (kc <= 128) of X,
// nsplit source splits of cps chunks, partials into part (ldp), Q images into bpack.
struct TcMember {
    GeomDev g;
    const double* X;
    int ldx, c0, kc;
    const double* pre;
    int nsplit;
    int64_t cps;
    float* part;
    int ldp;
    uint8_t* bpack;
};
// K3 over the (target tile, source split) work items of several geometries in one launch
// (members in the given order, each member's Q packed first); the work list and the
// members' parameters go to dscratch (block_tc_list_bytes of it).
void launch_block_tc_list(const std::vector<TcMember>& ms, int pieces, int* err, void* dscratch, size_t scratch_bytes,
                          cudaStream_t s);
size_t block_tc_list_bytes(int nmembers, int64_t nitems);
int block_tc_ctas_per_sm(int kc, int pieces, int force_ctas = 0);
int tc_npad(int kc);
// K1 with the FP64 tensor-core contraction (dt64mma.cu), columns [c0, c0 + kc), kc <= 64.
void launch_dt_f64_mma(const GeomDev& g, const double* X, int ldx, int c0, int kc, const double* pre, int nsplit,
                       int64_t chunk, double* part, int ldp, cudaStream_t s);
constexpr int kTcTileM = 128;   // targets per tensor-core tile
constexpr int kTcChunk = 64;    // sources per tensor-core chunk

}  // namespace bie

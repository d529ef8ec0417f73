// Internal declarations shared by the ABI layer and the device orchestration.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "../../include/bie_b200.h"

namespace bie {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void cuda_check(cudaError_t e, const char* what);
#define BIE_CK(call) ::bie::cuda_check((call), #call)

// Raises the dynamic shared-memory limit of kernel f on the current device to at
// least `bytes` (never lowers it). Thread-safe; the limit is kept per device.
void ensure_smem_limit(const void* f, size_t bytes);
// CTAs per SM of kernel f with `threads` threads and `smem` bytes, cached per device.
int occupancy(const void* f, int threads, size_t smem);

// Count of the library's device allocations and releases so far (all Buf objects).
uint64_t alloc_epoch();

// Grow-only device buffer owned by a geometry handle.
struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
    void ensure(size_t need);
    void release();
    template <class T>
    T* as() const { return (T*)p; }
};

bie_geom* geom_create(const double* pts, const double* nrm, const double* w, const double* diag, int64_t n,
                      int32_t npanels, int32_t nb, const int32_t* rowptr, const int32_t* col, const double* val,
                      int64_t nblocks, int device);
void geom_destroy(bie_geom* g);
// Releases the geometry's operator/solver workspace and graphs (see solver.cu); the
// _if_short form does so only when less than a quarter of device memory is free.
void geom_trim(bie_geom* g);
void geom_trim_if_short(bie_geom* g);
// geom_trim when the device has less than max(total / 4, free_floor) bytes free (or with
// BIE_TRIM_WORKSPACE); returns whether it trimmed.
bool geom_trim_if_below(bie_geom* g, size_t free_floor);
void geom_info(const bie_geom* g, int64_t* n, int64_t* nblocks, size_t* bytes);
void* geom_stream(bie_geom* g);
// Device correction blocks to host (nblocks*nb*nb doubles); false when len differs.
bool geom_near_values(bie_geom* g, double* val, int64_t len);
void profile_enable(bie_geom* g, int on);
void profile_read(bie_geom* g, int kind, bie_kernel_time* out);
bool tuning_read(bie_geom* g, int family, int columns, int pieces, int* nsplit, int* ctas, double* ms);
// K4 streaming form (combine_bulk.cu) for k <= 16; returns false (nothing launched)
// where its layout or alignment conditions do not hold.
template <typename TP>
bool launch_combine_bulk(int64_t n, int k, int nb, int npanels, const TP* part, int nsplit, const double* X,
                         const double* pre, const double* diag, const int32_t* rowptr, const int32_t* col,
                         const double* val, double* Y, int* err, int sms, cudaStream_t s);
// Near-accurate probe potentials on a device (probe.cu).
struct ProbeSetup;
struct ProbeDev;
ProbeDev* probe_upload(const ProbeSetup& ps, const double* targets, int64_t M, int64_t ncoarse, int device);
// Sigma: N x k column-major (host); phi: M x k column-major (host)
void probe_apply(ProbeDev* d, const double* Sigma, int k, double* phi);
void probe_free(ProbeDev* d);
// Arithmetic-throughput probe `which` on `device` (peaks.cu).
void peak_probe(int device, int which, double* per_second, double* ms);

void matvec_host(bie_geom* g, const double* X, double* Y, int k, int precision, uint32_t flags);
void matvec_device(bie_geom* g, const double* dX, double* dY, int k, int precision, uint32_t flags, cudaStream_t s);
void rhs_point_host(bie_geom* g, const double* src, const double* q, const double* eps, int k, double* F);
void rhs_point_device(bie_geom* g, const double* src, const double* q, const double* eps, int k, double* F,
                      cudaStream_t s);
void potential_host(bie_geom* g, const double* S, int k, const double* T, int64_t M, double* phi);
void potential_device(bie_geom* g, const double* S, int k, const double* T, int64_t M, double* phi, cudaStream_t s);
void energy_host(bie_geom* g, const double* S, int k, const double* src, const double* q, double* W);
int solve_host(bie_geom* g, const double* F, double* Sigma, int k, const bie_solve_opts& o, bie_stats* st);
int solve_point_host(bie_geom* g, const double* src, const double* q, const double* eps, int k, double* Sigma,
                     const bie_solve_opts& o, bie_stats* st);
int solve_device(bie_geom* g, const double* dF, double* dSigma, int k, const bie_solve_opts& o, bie_stats* st,
                 cudaStream_t s);
// Block solves of G geometries in lockstep (split-BF16 precisions): each reduced-precision
// operator application is one work-list launch of the tensor-core direct sum over all
// members. Device arrays node-major; st (if not null) has G entries.
int solve_group(bie_geom* const* gs, int G, const double* const* dF, double* const* dX, const int* ks,
                const bie_solve_opts& o, bie_stats* st, cudaStream_t s);
// Point-source right-hand sides built on the device per member, solved as a group, Sigma
// copied back per member (host, column-major); the members' k source values in src/q/eps.
int solve_group_point_host(bie_geom* const* gs, int G, const double* const* src, const double* const* q,
                           const double* const* eps, const int* ks, double* const* Sigma, const bie_solve_opts& o,
                           bie_stats* st);
// Y_m = A_low X_m for every member in one work-list launch of the tensor-core direct sum.
void matvec_group_device(bie_geom* const* gs, int G, const double* const* dX, double* const* dY, const int* ks,
                         int prec, uint32_t flags, cudaStream_t s);

// server.cu: request server with continuous batching of block solves.
bie_server* server_create(const bie_server_opts& o);
void server_destroy(bie_server* s);
uint64_t server_submit(bie_server* s, bie_geom* g, const double* F, int k, const bie_solve_opts& o);
uint64_t server_submit_point(bie_server* s, bie_geom* g, const double* src, const double* q, const double* eps,
                             int k, const bie_solve_opts& o);
int server_poll(bie_server* s, uint64_t ticket, int timeout_ms, double* Sigma, bie_stats* st, double* latency_ms,
                int* done, std::string* err);
void server_counters(bie_server* s, bie_server_counters* out);

// noalloc.cu: direct sum with the split partials in a fixed device array.
int64_t dt_apply_static_max_nodes();
void dt_apply_static(const double* x, const double* y, const double* z, const double* nx, const double* ny,
                     const double* nz, const double* w, int64_t n, const double* X, int k, double* Y,
                     cudaStream_t s);

}  // namespace bie

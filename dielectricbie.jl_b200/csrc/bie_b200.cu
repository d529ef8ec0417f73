// libbie_b200: C ABI, device-resident geometry, operator and solver
// orchestration for the B200 layer-potential library. See include/bie_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <atomic>
#include <mutex>
#include <tuple>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/bie_b200.h"
#include "host_setup.h"
#include "solver.h"

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
namespace bie {
thread_local std::string g_last_error;

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(BIE_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {
std::mutex g_attr_mu;
std::map<std::pair<int, const void*>, size_t> g_smem_limit;
std::map<std::tuple<int, const void*, int, size_t>, int> g_occ;
int current_device() {
    int d = 0;
    cuda_check(cudaGetDevice(&d), "cudaGetDevice");
    return d;
}
}  // namespace

void ensure_smem_limit(const void* f, size_t bytes) {
    if (bytes <= 48 * 1024) return;
    const int dev = current_device();
    std::lock_guard<std::mutex> lock(g_attr_mu);
    size_t& cur = g_smem_limit[{dev, f}];
    if (bytes <= cur) return;
    cuda_check(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes),
               "cudaFuncSetAttribute");
    cur = bytes;
}

int occupancy(const void* f, int threads, size_t smem) {
    const int dev = current_device();
    {
        std::lock_guard<std::mutex> lock(g_attr_mu);
        auto it = g_occ.find({dev, f, threads, smem});
        if (it != g_occ.end()) return it->second;
    }
    ensure_smem_limit(f, smem);
    int occ = 0;
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, f, threads, smem),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    occ = std::max(occ, 1);
    std::lock_guard<std::mutex> lock(g_attr_mu);
    g_occ[{dev, f, threads, smem}] = occ;
    return occ;
}

std::atomic<uint64_t> g_alloc_epoch{0};

void Buf::ensure(size_t need) {
    if (need <= bytes) return;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    size_t want = need + need / 4 + 256;
    g_alloc_epoch.fetch_add(1);
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        p = nullptr;
        throw Error(BIE_ENOMEM, "device allocation of " + std::to_string(want) + " bytes failed");
    }
    bytes = want;
}
void Buf::release() {
    if (p) {
        cudaFree(p);
        g_alloc_epoch.fetch_add(1);
    }
    p = nullptr;
    bytes = 0;
}
uint64_t alloc_epoch() { return g_alloc_epoch.load(); }
}  // namespace bie

using bie::Error;

template <class F>
static int guarded(F&& f) {
    try {
        f();
        return BIE_OK;
    } catch (const Error& e) {
        bie::g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        bie::g_last_error = "host allocation failed";
        return BIE_ENOMEM;
    } catch (const std::exception& e) {
        bie::g_last_error = e.what();
        return BIE_EINVAL;
    } catch (...) {
        bie::g_last_error = "unknown error";
        return BIE_EINVAL;
    }
}

#define REQUIRE(cond, msg) \
    do {                   \
        if (!(cond)) throw Error(BIE_EINVAL, msg); \
    } while (0)

struct bie_mesh {
    bie::Mesh m;
};
struct bie_near {
    bie::Near n;
    bool values_released = false;
};
struct bie_probe {
    bie::ProbeSetup ps;
    bie::ProbeDev* dev = nullptr;
    int64_t M = 0, N = 0;
};

extern "C" {

int bie_last_error(char* buf, size_t len) {
    const std::string& s = bie::g_last_error;
    if (buf && len) {
        size_t c = std::min(len - 1, s.size());
        std::memcpy(buf, s.data(), c);
        buf[c] = 0;
    }
    return (int)s.size();
}

const char* bie_version(void) { return "bie_b200 0.1 sm_100a"; }

int bie_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

// ----------------------------- host setup ---------------------------------
int bie_gausslegendre(int n, double* x, double* w) {
    return guarded([&] {
        REQUIRE(n >= 1 && n <= 128 && x && w, "gausslegendre: n must be in [1, 128]");
        bie::gauss_legendre(n, x, w);
    });
}

int bie_best_grid(double W, double H, double alpha, int* m, int* n) {
    return guarded([&] {
        REQUIRE(m && n, "best_grid: null output");
        int rc = bie::best_grid(W, H, alpha, m, n);
        if (rc == -1) throw Error(BIE_EINVAL, "best_grid: W and H must be positive and alpha >= 1");
        if (rc != 0) throw Error(BIE_EINVAL, "best_grid: no (m, n) found within search limits");
    });
}

int bie_mesh_single_box(double Lx, double Ly, double Lz, int n_quad, double l_ec, double eps_in, double eps_out,
                        double alpha, bie_mesh** out) {
    return guarded([&] {
        REQUIRE(out, "null output");
        auto h = std::make_unique<bie_mesh>();
        std::string err;
        if (bie::mesh_single_box(Lx, Ly, Lz, n_quad, l_ec, eps_in, eps_out, alpha, h->m, err))
            throw Error(BIE_EINVAL, err);
        *out = h.release();
    });
}

int bie_mesh_multi_box(int n_quad, double l_ec, int nbox, const double* centers, const double* dims,
                       const double* epses, double eps_out, double alpha, bie_mesh** out) {
    return guarded([&] {
        REQUIRE(out && centers && dims && epses, "null argument");
        auto h = std::make_unique<bie_mesh>();
        std::string err;
        if (bie::mesh_multi_box(n_quad, l_ec, nbox, centers, dims, epses, eps_out, alpha, h->m, err))
            throw Error(BIE_EINVAL, err);
        *out = h.release();
    });
}

int bie_mesh_from_panels(int npanels, int n_quad, const double* corners, const double* normals, const int* is_edge,
                         const double* eps_in, const double* eps_out, bie_mesh** out) {
    return guarded([&] {
        REQUIRE(out && (npanels == 0 || (corners && normals && is_edge && eps_in && eps_out)), "null argument");
        auto h = std::make_unique<bie_mesh>();
        std::string err;
        if (bie::mesh_from_panels(npanels, n_quad, corners, normals, is_edge, eps_in, eps_out, h->m, err))
            throw Error(BIE_EINVAL, err);
        *out = h.release();
    });
}

int bie_mesh_info(const bie_mesh* m, int64_t* npoints, int* npanels, int* n_quad) {
    return guarded([&] {
        REQUIRE(m, "null mesh");
        if (npoints) *npoints = m->m.npoints();
        if (npanels) *npanels = m->m.npanels;
        if (n_quad) *n_quad = m->m.nq;
    });
}

int bie_mesh_copy(const bie_mesh* mh, double* corners, double* normals, int* is_edge, double* eps_in, double* eps_out,
                  double* pts, double* nrm, double* w, double* diag) {
    return guarded([&] {
        REQUIRE(mh, "null mesh");
        const bie::Mesh& m = mh->m;
        if (corners) std::copy(m.corners.begin(), m.corners.end(), corners);
        if (normals) std::copy(m.normals.begin(), m.normals.end(), normals);
        if (is_edge) std::copy(m.is_edge.begin(), m.is_edge.end(), is_edge);
        if (eps_in) std::copy(m.eps_in.begin(), m.eps_in.end(), eps_in);
        if (eps_out) std::copy(m.eps_out.begin(), m.eps_out.end(), eps_out);
        if (pts) std::copy(m.pts.begin(), m.pts.end(), pts);
        if (w) std::copy(m.w.begin(), m.w.end(), w);
        const int np = m.nq * m.nq;
        if (nrm)
            for (int p = 0; p < m.npanels; ++p)
                for (int t = 0; t < np; ++t)
                    for (int c = 0; c < 3; ++c) nrm[3 * ((size_t)p * np + t) + c] = m.normals[3 * p + c];
        if (diag) m.diag(diag);
    });
}

void bie_mesh_destroy(bie_mesh* m) { delete m; }

void bie_near_opts_default(bie_near_opts* o) {
    if (!o) return;
    bie::NearOpts d;
    o->max_order = d.max_order;
    o->up_tol = d.up_tol;
    o->correct_edges = d.correct_edges;
    o->adaptive_atol = d.adaptive_atol;
    o->adaptive_rtol = d.adaptive_rtol;
    o->adaptive_n_GL = d.adaptive_n_GL;
    o->adaptive_max_depth = d.adaptive_max_depth;
    o->nthreads = d.nthreads;
    o->device = d.device;
}

int bie_near_build(const bie_mesh* m, const bie_near_opts* o, bie_near** out) {
    return guarded([&] {
        REQUIRE(m && out, "null argument");
        bie::NearOpts no;
        if (o) {
            no.max_order = o->max_order;
            no.up_tol = o->up_tol;
            no.correct_edges = o->correct_edges;
            no.adaptive_atol = o->adaptive_atol;
            no.adaptive_rtol = o->adaptive_rtol;
            no.adaptive_n_GL = o->adaptive_n_GL;
            no.adaptive_max_depth = o->adaptive_max_depth;
            no.nthreads = o->nthreads;
            no.device = o->device;
        }
        auto h = std::make_unique<bie_near>();
        std::string err;
        if (bie::near_build(m->m, no, h->n, err)) throw Error(BIE_EINVAL, err);
        *out = h.release();
    });
}

int bie_near_info(const bie_near* n, int64_t* nblocks, int* nb, int* n_ups, int* n_adp, int* hit_max) {
    return guarded([&] {
        REQUIRE(n, "null near");
        if (nblocks) *nblocks = n->n.nblocks();
        if (nb) *nb = n->n.nb;
        if (n_ups) *n_ups = (int)n->n.ups_i.size();
        if (n_adp) *n_adp = (int)n->n.adp_i.size();
        if (hit_max) *hit_max = n->n.hit_max;
    });
}

int bie_near_copy(const bie_near* nh, int32_t* rowptr, int32_t* col, double* val, int32_t* ups_i, int32_t* ups_j,
                  int32_t* ups_p, int32_t* adp_i, int32_t* adp_j) {
    return guarded([&] {
        REQUIRE(nh, "null near");
        REQUIRE(!(val && nh->values_released), "near_copy: the block values were released (bie_near_release_values)");
        const bie::Near& n = nh->n;
        if (rowptr) std::copy(n.rowptr.begin(), n.rowptr.end(), rowptr);
        if (col) std::copy(n.col.begin(), n.col.end(), col);
        if (val) std::copy(n.val.begin(), n.val.end(), val);
        if (ups_i) std::copy(n.ups_i.begin(), n.ups_i.end(), ups_i);
        if (ups_j) std::copy(n.ups_j.begin(), n.ups_j.end(), ups_j);
        if (ups_p) std::copy(n.ups_p.begin(), n.ups_p.end(), ups_p);
        if (adp_i) std::copy(n.adp_i.begin(), n.adp_i.end(), adp_i);
        if (adp_j) std::copy(n.adp_j.begin(), n.adp_j.end(), adp_j);
    });
}

int bie_near_release_values(bie_near* n) {
    return guarded([&] {
        REQUIRE(n, "null near");
        std::vector<double>().swap(n->n.val);
        n->values_released = true;
    });
}

void bie_near_destroy(bie_near* n) { delete n; }

// ----------------------------- device geometry -----------------------------
int bie_geom_create(const double* pts, const double* nrm, const double* w, const double* diag, int64_t n,
                    int32_t npanels, int32_t nb, const int32_t* rowptr, const int32_t* col, const double* val,
                    int64_t nblocks, int device, bie_geom** out) {
    return guarded([&] {
        REQUIRE(out && pts && nrm && w && diag && n > 0, "geom_create: null array or n <= 0");
        REQUIRE(nblocks == 0 || (rowptr && col && val && nb > 0 && npanels > 0 && (int64_t)npanels * nb == n),
                "geom_create: BSR arrays need npanels * nb == n");
        *out = bie::geom_create(pts, nrm, w, diag, n, npanels, nb, rowptr, col, val, nblocks, device);
    });
}

int bie_geom_create_from_mesh(const bie_mesh* mh, const bie_near* nh, int device, bie_geom** out) {
    return guarded([&] {
        REQUIRE(mh && out, "null argument");
        REQUIRE(!(nh && nh->values_released), "geom_create_from_mesh: the near-field block values were released");
        const bie::Mesh& m = mh->m;
        const int64_t n = m.npoints();
        REQUIRE(n > 0, "empty mesh");
        std::vector<double> nrm((size_t)3 * n), diag(n);
        const int np = m.nq * m.nq;
        for (int p = 0; p < m.npanels; ++p)
            for (int t = 0; t < np; ++t)
                for (int c = 0; c < 3; ++c) nrm[3 * ((size_t)p * np + t) + c] = m.normals[3 * p + c];
        m.diag(diag.data());
        const bie::Near* nr = nh ? &nh->n : nullptr;
        *out = bie::geom_create(m.pts.data(), nrm.data(), m.w.data(), diag.data(), n, m.npanels, np,
                                nr ? nr->rowptr.data() : nullptr, nr ? nr->col.data() : nullptr,
                                nr ? nr->val.data() : nullptr, nr ? nr->nblocks() : 0, device);
    });
}

int bie_geom_info(const bie_geom* g, int64_t* n, int64_t* nblocks, size_t* bytes) {
    return guarded([&] {
        REQUIRE(g, "null geom");
        bie::geom_info(g, n, nblocks, bytes);
    });
}

void* bie_geom_stream(bie_geom* g) { return g ? bie::geom_stream(g) : nullptr; }

int bie_geom_near_values(bie_geom* g, double* val, int64_t len) {
    return guarded([&] {
        REQUIRE(g && (val || len == 0), "null argument");
        REQUIRE(bie::geom_near_values(g, val, len), "geom_near_values: len must be nblocks * nb * nb");
    });
}

void bie_geom_destroy(bie_geom* g) {
    if (g) bie::geom_destroy(g);
}

// ----------------------------- operators ----------------------------------
int bie_matvec(bie_geom* g, const double* X, double* Y, int32_t k, int32_t precision, uint32_t flags) {
    return guarded([&] {
        REQUIRE(g && X && Y && k >= 1, "matvec: bad argument");
        bie::matvec_host(g, X, Y, k, precision, flags);
    });
}

int bie_matvec_device(bie_geom* g, const double* dX, double* dY, int32_t k, int32_t precision, uint32_t flags,
                      void* stream) {
    return guarded([&] {
        REQUIRE(g && dX && dY && k >= 1, "matvec_device: bad argument");
        bie::matvec_device(g, dX, dY, k, precision, flags, (cudaStream_t)stream);
    });
}

int bie_tuning_read(bie_geom* g, int32_t family, int32_t columns, int32_t pieces, int32_t* nsplit,
                    int32_t* ctas_per_sm, double* ms) {
    return guarded([&] {
        REQUIRE(g && nsplit && ctas_per_sm && ms, "tuning_read: bad argument");
        int ns = 0, ct = 0;
        double t = 0.0;
        if (!bie::tuning_read(g, family, columns, pieces, &ns, &ct, &t))
            throw Error(BIE_EINVAL, "tuning_read: no tuned configuration for this key");
        *nsplit = ns;
        *ctas_per_sm = ct;
        *ms = t;
    });
}

int bie_peak_probe(int32_t device, int32_t which, double* per_second, double* ms) {
    return guarded([&] {
        REQUIRE(per_second && ms, "peak_probe: bad argument");
        int nd = 0;
        if (cudaGetDeviceCount(&nd) != cudaSuccess || device < 0 || device >= nd) {
            cudaGetLastError();
            throw Error(BIE_EINVAL, "peak_probe: no such device");
        }
        bie::peak_probe(device, which, per_second, ms);
    });
}

void bie_server_opts_default(bie_server_opts* o) {
    if (!o) return;
    o->max_slots = 4;
    o->max_batch_rhs = 128;
    o->hbm_fraction = 0.8;
    o->device = 0;
    o->max_group = 8;
}

int bie_server_create(const bie_server_opts* o, bie_server** out) {
    return guarded([&] {
        REQUIRE(out, "server_create: bad argument");
        bie_server_opts d;
        bie_server_opts_default(&d);
        *out = bie::server_create(o ? *o : d);
    });
}

int bie_server_submit(bie_server* s, bie_geom* g, const double* F, int32_t k, const bie_solve_opts* o,
                      uint64_t* ticket) {
    return guarded([&] {
        REQUIRE(s && g && F && ticket && k >= 1, "server_submit: bad argument");
        bie_solve_opts d;
        bie_solve_opts_default(&d);
        *ticket = bie::server_submit(s, g, F, k, o ? *o : d);
    });
}

int bie_server_submit_point(bie_server* s, bie_geom* g, const double* src, const double* q, const double* eps_src,
                            int32_t k, const bie_solve_opts* o, uint64_t* ticket) {
    return guarded([&] {
        REQUIRE(s && g && src && q && eps_src && ticket && k >= 1, "server_submit_point: bad argument");
        bie_solve_opts d;
        bie_solve_opts_default(&d);
        *ticket = bie::server_submit_point(s, g, src, q, eps_src, k, o ? *o : d);
    });
}

int bie_server_poll(bie_server* s, uint64_t ticket, int32_t timeout_ms, double* Sigma, bie_stats* st,
                    double* latency_ms, int* done) {
    int rc = BIE_OK;
    const int g = guarded([&] {
        REQUIRE(s && done, "server_poll: bad argument");
        std::string err;
        rc = bie::server_poll(s, ticket, timeout_ms, Sigma, st, latency_ms, done, &err);
        if (rc != BIE_OK) bie::g_last_error = err;
    });
    return g != BIE_OK ? g : rc;
}

int bie_server_counters_read(bie_server* s, bie_server_counters* out) {
    return guarded([&] {
        REQUIRE(s && out, "server_counters: bad argument");
        bie::server_counters(s, out);
    });
}

void bie_server_destroy(bie_server* s) {
    if (s) bie::server_destroy(s);
}

int bie_dt_apply_static(const double* x, const double* y, const double* z, const double* nx, const double* ny,
                        const double* nz, const double* w, int64_t n, const double* X, int32_t k, double* Y,
                        void* stream) {
    return guarded([&] { bie::dt_apply_static(x, y, z, nx, ny, nz, w, n, X, k, Y, (cudaStream_t)stream); });
}

int bie_rhs_point(bie_geom* g, const double* src, const double* q, const double* eps_src, int32_t k, double* F) {
    return guarded([&] {
        REQUIRE(g && src && q && eps_src && F && k >= 1, "rhs_point: bad argument");
        bie::rhs_point_host(g, src, q, eps_src, k, F);
    });
}

int bie_rhs_point_device(bie_geom* g, const double* d_src, const double* d_q, const double* d_eps, int32_t k,
                         double* dF, void* stream) {
    return guarded([&] {
        REQUIRE(g && d_src && d_q && d_eps && dF && k >= 1, "rhs_point_device: bad argument");
        bie::rhs_point_device(g, d_src, d_q, d_eps, k, dF, (cudaStream_t)stream);
    });
}

int bie_potential(bie_geom* g, const double* Sigma, int32_t k, const double* targets, int64_t M, double* phi) {
    return guarded([&] {
        REQUIRE(g && Sigma && targets && phi && k >= 1 && M >= 0, "potential: bad argument");
        bie::potential_host(g, Sigma, k, targets, M, phi);
    });
}

int bie_potential_device(bie_geom* g, const double* d_sigma, int32_t k, const double* d_targets, int64_t M,
                         double* d_phi, void* stream) {
    return guarded([&] {
        REQUIRE(g && d_sigma && d_targets && d_phi && k >= 1 && M >= 0, "potential_device: bad argument");
        bie::potential_device(g, d_sigma, k, d_targets, M, d_phi, (cudaStream_t)stream);
    });
}

int bie_probe_create(const bie_mesh* mh, const double* targets, int64_t M, double hcubature_atol,
                     double range_factor, int32_t device, bie_probe** out) {
    return guarded([&] {
        REQUIRE(mh && out && M >= 0 && (M == 0 || targets), "probe_create: bad argument");
        std::unique_ptr<bie_probe> p(new bie_probe());
        std::string err;
        if (bie::probe_setup(mh->m, targets, M, hcubature_atol, range_factor, 0, (int64_t)1 << 24, p->ps, err) != 0)
            throw Error(BIE_EINVAL, err);
        p->M = M;
        p->N = mh->m.npoints();
        if (device >= 0) {
            int nd = 0;
            if (cudaGetDeviceCount(&nd) != cudaSuccess || device >= nd) {
                cudaGetLastError();
                throw Error(BIE_ENODEVICE, "probe_create: no such CUDA device (libbie_b200 has no CPU fallback)");
            }
            p->dev = bie::probe_upload(p->ps, targets, M, p->N, device);
        }
        *out = p.release();
    });
}

int bie_probe_info(const bie_probe* p, int64_t* n_refined, int32_t* npanels_refined, int64_t* nnz_prolongation,
                   int64_t* nnz_corrections, int64_t* ncubatures, int64_t* capped) {
    return guarded([&] {
        REQUIRE(p, "probe_info: null handle");
        if (n_refined) *n_refined = p->ps.refined.npoints();
        if (npanels_refined) *npanels_refined = p->ps.refined.npanels;
        if (nnz_prolongation) *nnz_prolongation = (int64_t)p->ps.pcol.size();
        if (nnz_corrections) *nnz_corrections = (int64_t)p->ps.ccol.size();
        if (ncubatures) *ncubatures = p->ps.ncubatures;
        if (capped) *capped = p->ps.capped;
    });
}

int bie_probe_copy(const bie_probe* p, int32_t* parent, int32_t* from_split, double* refined_corners,
                   double* refined_pts, double* refined_w, int64_t* prow, int32_t* pcol, double* pval,
                   int64_t* crow, int32_t* ccol, double* cval) {
    return guarded([&] {
        REQUIRE(p, "probe_copy: null handle");
        const bie::ProbeSetup& s = p->ps;
        if (parent) std::copy(s.parent.begin(), s.parent.end(), parent);
        if (from_split) std::copy(s.from_split.begin(), s.from_split.end(), from_split);
        if (refined_corners) std::copy(s.refined.corners.begin(), s.refined.corners.end(), refined_corners);
        if (refined_pts) std::copy(s.refined.pts.begin(), s.refined.pts.end(), refined_pts);
        if (refined_w) std::copy(s.refined.w.begin(), s.refined.w.end(), refined_w);
        if (prow) std::copy(s.prow.begin(), s.prow.end(), prow);
        if (pcol) std::copy(s.pcol.begin(), s.pcol.end(), pcol);
        if (pval) std::copy(s.pval.begin(), s.pval.end(), pval);
        if (crow) std::copy(s.crow.begin(), s.crow.end(), crow);
        if (ccol) std::copy(s.ccol.begin(), s.ccol.end(), ccol);
        if (cval) std::copy(s.cval.begin(), s.cval.end(), cval);
    });
}

int bie_probe_apply(bie_probe* p, const double* Sigma, int32_t k, double* phi) {
    return guarded([&] {
        REQUIRE(p && Sigma && phi && k >= 1, "probe_apply: bad argument");
        REQUIRE(p->dev, "probe_apply: the probe operator was built without a device");
        bie::probe_apply(p->dev, Sigma, k, phi);
    });
}

void bie_probe_destroy(bie_probe* p) {
    if (!p) return;
    bie::probe_free(p->dev);
    delete p;
}

int bie_energy(bie_geom* g, const double* Sigma, int32_t k, const double* src, const double* q, double* W) {
    return guarded([&] {
        REQUIRE(g && Sigma && src && q && W && k >= 1, "energy: bad argument");
        bie::energy_host(g, Sigma, k, src, q, W);
    });
}

// ----------------------------- solvers -------------------------------------
void bie_solve_opts_default(bie_solve_opts* o) {
    if (!o) return;
    o->atol = 0.0;
    o->rtol = 1e-10;
    o->itmax = 500;
    o->restart = 200;
    o->precision = BIE_FP64;
    o->inner_rtol = 1e-6;
    o->max_outer = 8;
    o->precondition = 0;
    o->check_every = 1;
    o->flags = 0;
    o->block = 0;
}

int bie_solve(bie_geom* g, const double* F, double* Sigma, int32_t k, const bie_solve_opts* o, bie_stats* st) {
    int rc = BIE_OK;
    int grc = guarded([&] {
        REQUIRE(g && F && Sigma && k >= 1, "solve: bad argument");
        bie_solve_opts d;
        bie_solve_opts_default(&d);
        rc = bie::solve_host(g, F, Sigma, k, o ? *o : d, st);
    });
    return grc != BIE_OK ? grc : rc;
}

int bie_matvec_group_device(bie_geom* const* gs, int32_t G, const double* const* dX, double* const* dY,
                            const int32_t* ks, int32_t precision, uint32_t flags, void* stream) {
    return guarded([&] {
        REQUIRE(gs && dX && dY && ks && G >= 1 && G <= 4096, "matvec_group_device: bad argument");
        for (int i = 0; i < G; ++i) REQUIRE(dX[i] && dY[i], "matvec_group_device: null member array");
        bie::matvec_group_device(gs, G, dX, dY, ks, precision, flags, (cudaStream_t)stream);
    });
}

int bie_solve_group_device(bie_geom* const* gs, int32_t G, const double* const* dF, double* const* dSigma,
                           const int32_t* ks, const bie_solve_opts* o, bie_stats* st, void* stream) {
    int rc = BIE_OK;
    int grc = guarded([&] {
        REQUIRE(gs && dF && dSigma && ks && G >= 1 && G <= 4096, "solve_group_device: bad argument");
        for (int i = 0; i < G; ++i) REQUIRE(dF[i] && dSigma[i], "solve_group_device: null member array");
        bie_solve_opts d;
        bie_solve_opts_default(&d);
        rc = bie::solve_group(gs, G, dF, dSigma, ks, o ? *o : d, st, (cudaStream_t)stream);
        for (int i = 0; i < G; ++i) bie::geom_trim_if_short(gs[i]);
    });
    return grc != BIE_OK ? grc : rc;
}

int bie_solve_point(bie_geom* g, const double* src, const double* q, const double* eps_src, int32_t k, double* Sigma,
                    const bie_solve_opts* o, bie_stats* st) {
    int rc = BIE_OK;
    int grc = guarded([&] {
        REQUIRE(g && src && q && eps_src && Sigma && k >= 1, "solve_point: bad argument");
        bie_solve_opts d;
        bie_solve_opts_default(&d);
        rc = bie::solve_point_host(g, src, q, eps_src, k, Sigma, o ? *o : d, st);
    });
    return grc != BIE_OK ? grc : rc;
}

int bie_solve_device(bie_geom* g, const double* dF, double* dSigma, int32_t k, const bie_solve_opts* o, bie_stats* st,
                     void* stream) {
    int rc = BIE_OK;
    int grc = guarded([&] {
        REQUIRE(g && dF && dSigma && k >= 1, "solve_device: bad argument");
        bie_solve_opts d;
        bie_solve_opts_default(&d);
        rc = bie::solve_device(g, dF, dSigma, k, o ? *o : d, st, (cudaStream_t)stream);
        bie::geom_trim_if_short(g);
    });
    return grc != BIE_OK ? grc : rc;
}

// ----------------------------- kernel timing -------------------------------
int bie_profile_enable(bie_geom* g, int enable) {
    return guarded([&] {
        REQUIRE(g, "null geom");
        bie::profile_enable(g, enable);
    });
}

int bie_profile_read(bie_geom* g, int kind, bie_kernel_time* out) {
    return guarded([&] {
        REQUIRE(g && out && kind >= 0 && kind <= BIE_KERNEL_KINDS, "profile_read: bad argument");
        bie::profile_read(g, kind, out);
    });
}

}  // extern "C"

// Device-resident geometry, layer-potential operators and the device GMRES /
// iterative-refinement solvers of libbie_b200.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <memory>
#include <tuple>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <utility>
#include <vector>

#include "bgmres.cuh"
#include "kernels.cuh"
#include "solver.h"

struct bie_geom {
    int device = 0;
    cudaStream_t stream = nullptr;
    int sms = 148;
    int64_t n = 0;
    int32_t npanels = 0, nb = 0;
    int64_t nblocks = 0;
    size_t geom_bytes = 0;
    bie::Buf x, y, z, nx, ny, nz, w, diag, pinv, perm;
    bie::Buf rowptr, col, val;
    // operator workspace
    bie::Buf part, small, bpack, errflag, cpart, srcpack, glist;
    int max_row_blocks = 0;  // longest BSR block row (blocks of one target panel)
    // solver workspace
    bie::Buf V, W, R, gv, cs, sn, h, h2, hn, beta, eps, active, jlast, yv, resid, dpart, rr, xo, dd, io_a, io_b, sol;
    // block GMRES workspace: basis, Hessenberg matrix, right-hand sides, small factors
    bie::Buf bv, bq, bvj, bh, bgv, btau, br1, br2, br, bh2, bres, bidx, bflag, xa, ra, binv, bpart, btmp, bwy;
    cublasHandle_t blas = nullptr;  // created on the first block solve
    double* bres_host = nullptr;    // pinned copy of the block residual norms (64 doubles)
    cudaEvent_t ev_res = nullptr;   // marks that copy in the side stream
    cudaEvent_t ev_h = nullptr;     // marks a new Hessenberg block column in the solver's stream
    cudaStream_t s_ls = nullptr;    // side stream of the block least-squares updates
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // kernel timing
    struct ProfRec {
        int kind;
        cudaEvent_t a, b;
    };
    bool prof_on = false;
    std::vector<ProfRec> prof_pending;
    std::vector<cudaEvent_t> ev_pool;
    bie_kernel_time acc[BIE_KERNEL_KINDS] = {};
    // CUDA graphs of GMRES iterations: one executable per Arnoldi step index j for the
    // last two solver configurations (signature = sizes, options and buffer addresses)
    struct GraphCache {
        uint64_t sig = 0;
        bool warm = false;  // one eager solve finished with these buffers: safe to capture
        std::vector<cudaGraphExec_t> exec;
    };
    GraphCache gcache[2];
    int gcache_next = 0;
    bool graphs = true;  // off with the environment variable BIE_NO_GRAPHS
    // autotuned launch configurations of the direct sums, keyed by tune_key(family, columns, pieces)
    struct Tuned {
        int nsplit;
        int64_t chunk;
        int ctas;
        double ms;
    };
    std::map<std::tuple<int, int, int>, Tuned> tuned;
    bool autotune = true;  // off with the environment variable BIE_NO_AUTOTUNE
};

namespace bie {

// Relative errors of the reduced-precision operators (measured on the config boxes:
// ~4e-6 for the split-BF16 three-term contraction, ~1e-7 for the six-term one and
// the FP32 direct sum),
// used to decide when a residual update may run in reduced precision.
constexpr double kDeltaBF16X3 = 4e-6;
constexpr double kDeltaBF16X6 = 3e-7;
constexpr double kDeltaFP32 = 3e-7;
// Split-BF16 precisions run the tensor-core direct sum (K3, padded to 16 columns and
// bound by its kernel-tile generation, so its time hardly depends on k) unless the FP32
// CUDA-core sum (K2) covers k in one pass (k = 1, 2, 4), which is faster there.
inline bool use_tc(int prec, int k) {
    return (prec == BIE_BF16X3 || prec == BIE_BF16X6) && !(k == 1 || k == 2 || k == 4);
}

// The direct-sum operator apply_op runs for (prec, k): 0 FP32, 1 FP64, 2 split-BF16 x3, 3 x6.
inline int op_kind(int prec, int k) {
    return use_tc(prec, k) ? (prec == BIE_BF16X6 ? 3 : 2) : (prec == BIE_FP64 ? 1 : 0);
}

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) BIE_CK(cudaSetDevice(dev));
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

inline unsigned grid1(int64_t n, int bs = 256) { return (unsigned)((n + bs - 1) / bs); }

cudaEvent_t pool_event(bie_geom* g) {
    if (!g->ev_pool.empty()) {
        cudaEvent_t e = g->ev_pool.back();
        g->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    BIE_CK(cudaEventCreate(&e));
    return e;
}

void prof_drain(bie_geom* g) {
    for (auto& r : g->prof_pending) {
        BIE_CK(cudaEventSynchronize(r.b));
        float ms = 0.f;
        BIE_CK(cudaEventElapsedTime(&ms, r.a, r.b));
        g->acc[r.kind].ms += ms;
        g->ev_pool.push_back(r.a);
        g->ev_pool.push_back(r.b);
    }
    g->prof_pending.clear();
}

// Scope around the launches of one kernel kind: counts launches and algorithmic
// units always, and brackets them with CUDA events on `s` while timing is enabled.
struct Prof {
    bie_geom* g;
    int kind;
    cudaStream_t s;
    cudaEvent_t a = nullptr;
    // timed = false: launches counted but not timed (work overlapped with the solver's stream,
    // whose event span would include the wait for free SMs)
    Prof(bie_geom* g_, int kind_, cudaStream_t s_, int launches = 1, double pairs = 0, double pair_cols = 0,
         double bytes = 0, bool timed = true)
        : g(g_), kind(kind_), s(s_) {
        bie_kernel_time& t = g->acc[kind];
        t.launches += launches;
        t.pairs += pairs;
        t.pair_cols += pair_cols;
        t.bytes += bytes;
        if (g->prof_on && timed) {
            if (g->prof_pending.size() > 8192) prof_drain(g);
            a = pool_event(g);
            BIE_CK(cudaEventRecord(a, s));
        }
    }
    // further launches of this kind inside the scope (several kernels under one scope)
    void add(int n) { g->acc[kind].launches += n; }
    ~Prof() {
        if (!a) return;
        cudaEvent_t b = nullptr;
        if (!g->ev_pool.empty()) {
            b = g->ev_pool.back();
            g->ev_pool.pop_back();
        } else if (cudaEventCreate(&b) != cudaSuccess) {
            return;
        }
        cudaEventRecord(b, s);
        g->prof_pending.push_back({kind, a, b});
    }
};

GeomDev gdev(const bie_geom* g) {
    return GeomDev{g->x.as<double>(), g->y.as<double>(), g->z.as<double>(), g->nx.as<double>(),
                   g->ny.as<double>(), g->nz.as<double>(), g->w.as<double>(), g->n, g->perm.as<int32_t>()};
}

template <class T>
void upload(bie::Buf& b, const T* src, size_t count, cudaStream_t s) {
    b.ensure(sizeof(T) * std::max<size_t>(count, 1));
    if (count) BIE_CK(cudaMemcpyAsync(b.p, src, sizeof(T) * count, cudaMemcpyHostToDevice, s));
}

// --------------------------- direct-sum launchers --------------------------
enum class Kern { DT64, DT32, POT64 };

template <int C>
void* kern_ptr(Kern kind) {
    switch (kind) {
        case Kern::DT64: return (void*)k_dt_f64<C>;
        case Kern::DT32: return (void*)k_dt_f32<C>;
        default: return (void*)k_pot_f64<C>;
    }
}

template <int C>
size_t kern_smem(Kern kind) {
    return (size_t)(3 + C) * kTS * (kind == Kern::DT32 ? sizeof(float) : sizeof(double));
}

// occupancy (CTAs per SM) of one instantiation; also raises its dynamic smem limit
template <int C>
int kern_occ(Kern kind) {
    return occupancy(kern_ptr<C>(kind), kTB, kern_smem<C>(kind));
}

struct Split {
    int nsplit;
    int64_t chunk;
};

Split choose_split(int64_t rows, int64_t nsrc, int sms, int occ) {
    int64_t nblkx = (rows + kTB - 1) / kTB;
    int64_t want = (int64_t)sms * occ * 4;
    int64_t maxs = std::max<int64_t>(1, (nsrc + kTS - 1) / kTS);
    int64_t ns = std::min(maxs, std::max<int64_t>(1, (want + nblkx - 1) / nblkx));
    int64_t chunk = (nsrc + ns - 1) / ns;
    chunk = (chunk + kTS - 1) / kTS * kTS;
    ns = std::max<int64_t>(1, (nsrc + chunk - 1) / chunk);
    return Split{(int)ns, chunk};
}

template <int C>
void launch_direct(Kern kind, const GeomDev& g, const double* X, int ldx, int c0, const double* pre,
                   const double* T, int64_t M, Split sp, double* part, int ldp, cudaStream_t s) {
    size_t sm = kern_smem<C>(kind);
    kern_occ<C>(kind);  // sets the smem attribute
    int64_t rows = kind == Kern::POT64 ? M : g.n;
    dim3 grid((unsigned)((rows + kTB - 1) / kTB), (unsigned)sp.nsplit);
    if (kind == Kern::DT64)
        k_dt_f64<C><<<grid, kTB, sm, s>>>(g, X, ldx, c0, pre, sp.chunk, part, ldp);
    else if (kind == Kern::DT32)
        k_dt_f32<C><<<grid, kTB, sm, s>>>(g, X, ldx, c0, pre, sp.chunk, part, ldp);
    else
        k_pot_f64<C><<<grid, kTB, sm, s>>>(g, X, ldx, c0, T, M, sp.chunk, part, ldp);
    BIE_CK(cudaGetLastError());
}

int occ_for(Kern kind, int C) {
    switch (C) {
        case 64: return kern_occ<64>(kind);
        case 32: return kern_occ<32>(kind);
        case 16: return kern_occ<16>(kind);
        case 8: return kern_occ<8>(kind);
        case 4: return kern_occ<4>(kind);
        case 2: return kern_occ<2>(kind);
        default: return kern_occ<1>(kind);
    }
}

int pick_C(int rem) {
    static const int cs[] = {64, 32, 16, 8, 4, 2, 1};
    for (int c : cs)
        if (c <= rem) return c;
    return 1;
}

// Runs the direct sum for all k columns into g->part; returns the split used.
// K1 (FP64 tensor-core) split with ns source splits (chunks rounded up to kTS sources).
Split dt64_split_n(const bie_geom* g, int64_t ns) {
    ns = std::max<int64_t>(1, std::min<int64_t>(ns, (g->n + kTS - 1) / kTS));
    int64_t chunk = (g->n + ns - 1) / ns;
    chunk = (chunk + kTS - 1) / kTS * kTS;
    return Split{(int)((g->n + chunk - 1) / chunk), chunk};
}

// Autotuner key of a direct-sum family at a column width: the width is rounded up to the
// kernel instance the launch runs (K3: the MMA width, a multiple of 16, of the first block
// of at most 128 columns; K1: the 8/16/32/64-column template of the first block of at most
// 64), so that a server's batches of different widths share one tuning per instance.
std::tuple<int, int, int> tune_key(int family, int columns, int pieces) {
    if (family == 0) return std::make_tuple(0, tc_npad(std::min(columns, 128)), pieces);
    const int c = std::min(columns, 64);
    return std::make_tuple(1, c > 32 ? 64 : (c > 16 ? 32 : (c > 8 ? 16 : 8)), 0);
}

// Autotuning is allowed on an eager, unprofiled stream.
bool can_tune(const bie_geom* g, cudaStream_t s) {
    if (!g->autotune || g->prof_on) return false;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return false;
    }
    return true;
}

// Device time (ms) of one call of `run` on stream s.
template <class F>
double time_on(bie_geom* g, cudaStream_t s, F&& run) {
    if (!g->ev0) BIE_CK(cudaEventCreate(&g->ev0));
    if (!g->ev1) BIE_CK(cudaEventCreate(&g->ev1));
    BIE_CK(cudaEventRecord(g->ev0, s));
    run();
    BIE_CK(cudaEventRecord(g->ev1, s));
    BIE_CK(cudaEventSynchronize(g->ev1));
    float ms = 0.f;
    BIE_CK(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
    return ms;
}

// Autotuner: times the candidate launch configurations on the real operand once
// per (family, columns, pieces). Among the candidates within 1 % of the fastest it keeps
// the one with the fewest source splits (the reduction that follows reads one partial per
// split; near-ties would otherwise be decided by timing noise), then the wave model's
// choice (the first candidate).
template <class Launch>
bie_geom::Tuned tune(bie_geom* g, cudaStream_t s, const std::vector<bie_geom::Tuned>& cands, Launch&& launch) {
    launch(cands.front());  // warm-up (first-use costs)
    std::vector<double> t(cands.size());
    for (size_t i = 0; i < cands.size(); ++i) t[i] = time_on(g, s, [&] { launch(cands[i]); });
    size_t fast = 0;
    for (size_t i = 1; i < cands.size(); ++i)
        if (t[i] < t[fast]) fast = i;
    size_t best = fast;
    for (size_t i = 0; i < cands.size(); ++i)
        if (t[i] <= 1.01 * t[fast] &&
            (cands[i].nsplit < cands[best].nsplit || (cands[i].nsplit == cands[best].nsplit && i < best)))
            best = i;
    bie_geom::Tuned r = cands[best];
    r.ms = t[best];
    return r;
}

Split direct_sum(bie_geom* g, Kern kind, const double* X, int ldx, int k, const double* pre, const double* T,
                 int64_t M, cudaStream_t s) {
    GeomDev gd = gdev(g);
    if (kind == Kern::DT64 && k >= 8) {
        // FP64 tensor-core contraction, 64 columns per launch, 3 CTAs of 64 targets per SM;
        // the source split count is autotuned around the occupancy model's
        const double npairs = (double)g->n * (g->n - 1);
        auto run = [&](const Split& sp, bool prof) {
            g->part.ensure(sizeof(double) * (size_t)sp.nsplit * g->n * k);
            for (int c0 = 0; c0 < k; c0 += 64) {
                const int kc = std::min(64, k - c0);
                std::unique_ptr<Prof> pf;
                if (prof) pf.reset(new Prof(g, BIE_KERNEL_DIRECT_FP64, s, 1, npairs, npairs * kc));
                launch_dt_f64_mma(gd, X, ldx, c0, kc, pre, sp.nsplit, sp.chunk, g->part.as<double>(), k, s);
            }
        };
        // (the split model of 128-row tiles at two CTAs per SM, which gives the 64-target
        // CTAs about twice the source splits of a full wave: measured faster than the model
        // matched to 64-target CTAs at three per SM)
        const Split base = choose_split(g->n, g->n, g->sms, 2);
        const auto key = tune_key(1, k, 0);
        auto it = g->tuned.find(key);
        if (it == g->tuned.end() && can_tune(g, s)) {
            std::vector<bie_geom::Tuned> cands{{base.nsplit, base.chunk, 3, 0.0}};
            for (int64_t ns : {(int64_t)base.nsplit / 2, 2 * (int64_t)base.nsplit}) {
                const Split sp = dt64_split_n(g, ns);
                bool dup = false;
                for (auto& c : cands) dup = dup || c.nsplit == sp.nsplit;
                if (!dup) cands.push_back({sp.nsplit, sp.chunk, 3, 0.0});
            }
            it = g->tuned.emplace(key, tune(g, s, cands, [&](const bie_geom::Tuned& c) {
                                       run(Split{c.nsplit, c.chunk}, false);
                                   })).first;
        }
        const Split sp = it != g->tuned.end() ? Split{it->second.nsplit, it->second.chunk} : base;
        run(sp, true);
        return sp;
    }
    int64_t rows = kind == Kern::POT64 ? M : g->n;
    int Cmax = pick_C(k);
    Split sp = choose_split(rows, g->n, g->sms, occ_for(kind, Cmax));
    g->part.ensure(sizeof(double) * (size_t)sp.nsplit * std::max<int64_t>(rows, 1) * k);
    double* part = g->part.as<double>();
    const int pkind = kind == Kern::DT64 ? BIE_KERNEL_DIRECT_FP64
                      : (kind == Kern::DT32 ? BIE_KERNEL_DIRECT_FP32 : BIE_KERNEL_OTHER);
    const double npairs = kind == Kern::POT64 ? (double)M * g->n : (double)g->n * (g->n - 1);
    for (int c0 = 0; c0 < k;) {
        int C = pick_C(k - c0);
        Prof pf(g, pkind, s, 1, npairs, npairs * C);
        switch (C) {
            case 64: launch_direct<64>(kind, gd, X, ldx, c0, pre, T, M, sp, part, k, s); break;
            case 32: launch_direct<32>(kind, gd, X, ldx, c0, pre, T, M, sp, part, k, s); break;
            case 16: launch_direct<16>(kind, gd, X, ldx, c0, pre, T, M, sp, part, k, s); break;
            case 8: launch_direct<8>(kind, gd, X, ldx, c0, pre, T, M, sp, part, k, s); break;
            case 4: launch_direct<4>(kind, gd, X, ldx, c0, pre, T, M, sp, part, k, s); break;
            case 2: launch_direct<2>(kind, gd, X, ldx, c0, pre, T, M, sp, part, k, s); break;
            default: launch_direct<1>(kind, gd, X, ldx, c0, pre, T, M, sp, part, k, s); break;
        }
        c0 += C;
    }
    return sp;
}

// K3 launch plan: the number of source splits ns (<= 16, and at most 1024 chunks
// per split) that minimises the time of the wave-quantised grid, which is
// proportional to ceil(tiles ns / slots) / ns; ties go to fewer splits (each
// split adds an FP32 partial for the combine to read). force_ctas selects the CTA
// shape (0 = default).
Split tc_split(const bie_geom* g, int kc, int pieces, int force_ctas = 0) {
    const int64_t tiles = (g->n + kTcTileM - 1) / kTcTileM;
    const int64_t chunks = (g->n + kTcChunk - 1) / kTcChunk;
    const int64_t slots = (int64_t)g->sms * block_tc_ctas_per_sm(kc, pieces, force_ctas);
    const int64_t ns_min = std::min<int64_t>(chunks, std::max<int64_t>(1, (chunks + 1023) / 1024));
    const int64_t ns_max = std::min<int64_t>(chunks, std::max<int64_t>(ns_min, 16));
    int64_t ns = ns_min;
    double best = 1e300;
    for (int64_t t = ns_min; t <= ns_max; ++t) {
        const int64_t cps_t = (chunks + t - 1) / t;
        const int64_t nt = (chunks + cps_t - 1) / cps_t;  // splits actually launched
        const double waves = (double)((tiles * nt + slots - 1) / slots);
        const double cost = waves * (double)cps_t * (1.0 + 0.002 * (double)nt);
        if (cost < best - 1e-9) {
            best = cost;
            ns = t;
        }
    }
    int64_t cps = (chunks + ns - 1) / ns;
    ns = (chunks + cps - 1) / cps;
    return Split{(int)ns, cps};
}

// K3 split with ns source splits (chunks per split rounded up).
Split tc_split_n(const bie_geom* g, int64_t ns) {
    const int64_t chunks = (g->n + kTcChunk - 1) / kTcChunk;
    ns = std::max<int64_t>(std::max<int64_t>(1, (chunks + 1023) / 1024), std::min(ns, chunks));
    const int64_t cps = (chunks + ns - 1) / ns;
    return Split{(int)((chunks + cps - 1) / cps), cps};
}

Split direct_sum_tc(bie_geom* g, const double* X, int k, const double* pre, int pieces, cudaStream_t s) {
    GeomDev gd = gdev(g);
    const int kc0 = std::min(k, 128);
    const double npairs = (double)g->n * (g->n - 1);
    auto run = [&](const Split& sp, int ctas, bool prof) {
        g->part.ensure(sizeof(float) * (size_t)sp.nsplit * g->n * k);
        g->bpack.ensure(block_tc_pack_bytes(g->n, kc0, pieces));
        for (int c0 = 0; c0 < k; c0 += 128) {
            int kc = std::min(128, k - c0);
            std::unique_ptr<Prof> pf;
            if (prof) pf.reset(new Prof(g, BIE_KERNEL_DIRECT_TC, s, 2, npairs, npairs * tc_npad(kc)));
            launch_block_tc(gd, X, k, c0, kc, pre, sp.nsplit, sp.chunk, g->part.as<float>(), k,
                            g->bpack.as<uint8_t>(), g->errflag.as<int>(), pieces, ctas, s);
        }
    };
    const auto key = tune_key(0, kc0, pieces);
    auto it = g->tuned.find(key);
    if (it == g->tuned.end() && can_tune(g, s)) {
        std::vector<bie_geom::Tuned> cands;
        const int shape0 = block_tc_ctas_per_sm(kc0, pieces, 0);
        for (int ctas : {shape0, shape0 == 2 ? 1 : 0}) {
            if (ctas == 0) continue;
            const Split base = tc_split(g, kc0, pieces, ctas);
            for (int64_t ns : {(int64_t)base.nsplit, (int64_t)base.nsplit / 2, 2 * (int64_t)base.nsplit}) {
                const Split sp = ns == base.nsplit ? base : tc_split_n(g, ns);
                bool dup = false;
                for (auto& c : cands) dup = dup || (c.nsplit == sp.nsplit && c.ctas == ctas);
                if (!dup) cands.push_back({sp.nsplit, sp.chunk, ctas, 0.0});
            }
        }
        it = g->tuned.emplace(key, tune(g, s, cands, [&](const bie_geom::Tuned& c) {
                                   run(Split{c.nsplit, c.chunk}, c.ctas, false);
                               })).first;
    }
    Split sp;
    int ctas = 0;
    if (it != g->tuned.end()) {
        sp = Split{it->second.nsplit, it->second.chunk};
        ctas = it->second.ctas;
    } else {
        sp = tc_split(g, kc0, pieces);
    }
    run(sp, ctas, true);
    return sp;
}

// K4 launch for split partials of type TP (FP64 from K1/K2, FP32 from K3).
template <typename TP>
void combine(bie_geom* g, const TP* part, int nsplit, const double* X, double* Y, int k, const double* pre, bool corr,
             bool dg, cudaStream_t s) {
    const double* dgp = dg ? g->diag.as<double>() : nullptr;
    const int32_t* rp = corr ? g->rowptr.as<int32_t>() : nullptr;
    const int32_t* cl = corr ? g->col.as<int32_t>() : nullptr;
    const double* vl = corr ? g->val.as<double>() : nullptr;
    const int mt = (g->nb + 7) / 8;
    const bool panel_rows = g->nb > 0 && (int64_t)g->npanels * g->nb == g->n;
    if (panel_rows && mt <= 8) {
        // the block products on the FP64 tensor path, two pipeline stages
        const int nst = 2;
        const size_t sm = combine_smem_bytes(g->nb, std::min(k, kCombTile), nst);
        // narrow blocks of right-hand sides on meshes with enough block rows to fill the
        // GPU: the HBM-bound streaming form, where its layout conditions hold
        // (BIE_COMBINE_ROWS forces the block-row form, for comparisons)
        if (vl && g->npanels >= 4 * g->sms && !std::getenv("BIE_COMBINE_ROWS") &&
            launch_combine_bulk<TP>(g->n, k, g->nb, g->npanels, part, nsplit, X, pre, dgp, rp, cl, vl, Y,
                                    g->errflag.as<int>(), g->sms, s)) {
            BIE_CK(cudaGetLastError());
            return;
        }
        const int64_t ctas = (int64_t)g->npanels * ((k + kCombTile - 1) / kCombTile);
        // long block rows of few panels: split each row into groups of blocks so that
        // about 8 CTAs per SM run (summed by k_combine_groups)
        int ngroups = 1, bpg = 0;
        if (vl && g->max_row_blocks > 8) {
            const int64_t want = (8 * (int64_t)g->sms + ctas - 1) / ctas;
            ngroups = (int)std::min<int64_t>(want, (g->max_row_blocks + 3) / 4);
            ngroups = std::max(ngroups, 1);
            bpg = (g->max_row_blocks + ngroups - 1) / ngroups;
            ngroups = (g->max_row_blocks + bpg - 1) / bpg;
        }
        double* gsum = nullptr;
        if (ngroups > 1) {
            g->cpart.ensure(sizeof(double) * (size_t)ngroups * g->n * k);
            gsum = g->cpart.as<double>();
        }
        dim3 grid((unsigned)g->npanels, (unsigned)((k + kCombTile - 1) / kCombTile), (unsigned)ngroups);
#define BIE_COMB(MT, NST)                                       \
    ensure_smem_limit((const void*)k_combine_dmma<MT, NST, TP>, sm); \
    k_combine_dmma<MT, NST, TP><<<grid, 128, sm, s>>>(g->n, k, part, nsplit, X, pre, dgp, rp, cl, vl, g->nb, Y, bpg, \
                                                      gsum)
#define BIE_COMB_MT(NST)                      \
    switch (mt) {                             \
        case 1: BIE_COMB(1, NST); break;      \
        case 2: BIE_COMB(2, NST); break;      \
        case 3: BIE_COMB(3, NST); break;      \
        case 4: BIE_COMB(4, NST); break;      \
        case 5: BIE_COMB(5, NST); break;      \
        case 6: BIE_COMB(6, NST); break;      \
        case 7: BIE_COMB(7, NST); break;      \
        default: BIE_COMB(8, NST); break;     \
    }
        BIE_COMB_MT(2)
#undef BIE_COMB_MT
#undef BIE_COMB
        if (gsum) {
            BIE_CK(cudaGetLastError());
            const int64_t tot = g->n * (int64_t)k;
            const unsigned blocks = (unsigned)std::min<int64_t>((tot + 255) / 256, (int64_t)g->sms * 8);
            k_combine_groups<TP><<<blocks, 256, 0, s>>>(g->n, k, gsum, ngroups, part, nsplit, X, pre, dgp, Y);
        }
    } else {
        k_combine<TP><<<grid1(g->n * k), 256, 0, s>>>(g->n, k, part, nsplit, X, k, pre, dgp, rp, cl, vl, g->nb, Y, k);
    }
    BIE_CK(cudaGetLastError());
}

// Y = A(prec) (p .* X), node-major n x k (ldx = ldy = k).
void apply_op(bie_geom* g, const double* X, double* Y, int k, int prec, uint32_t flags, const double* pre,
              cudaStream_t s) {
    Split sp;
    const bool tc = use_tc(prec, k);
    if (tc) {
        sp = direct_sum_tc(g, X, k, pre, prec == BIE_BF16X6 ? 3 : 2, s);
    } else {
        Kern kind = prec == BIE_FP64 ? Kern::DT64 : Kern::DT32;  // split-BF16 with k = 1, 2, 4 runs K2 (FP32)
        sp = direct_sum(g, kind, X, k, k, pre, nullptr, 0, s);
    }
    const bool corr = g->nblocks > 0 && !(flags & BIE_NO_CORRECTIONS);
    const bool dg = !(flags & BIE_NO_DIAG);
    const double pbytes = tc ? 4.0 : 8.0;
    const double cbytes = (corr ? (double)g->nblocks * g->nb * g->nb * 8 + g->nblocks * 4.0 + (g->npanels + 1) * 4.0
                                : 0.0) +
                          (double)g->n * k * (16.0 + pbytes * sp.nsplit) + (dg ? g->n * 8.0 : 0.0);
    Prof pf(g, BIE_KERNEL_COMBINE, s, 1, 0, 0, cbytes);
    if (tc)
        combine(g, g->part.as<float>(), sp.nsplit, X, Y, k, pre, corr, dg, s);
    else
        combine(g, g->part.as<double>(), sp.nsplit, X, Y, k, pre, corr, dg, s);
}

// ------------------------------ reductions ---------------------------------
struct DotPlan {
    int bs, nblk;
    int64_t rows_per_blk;
};

// Row blocks of the column reductions: about 2048 CTAs over all vectors, each with
// at least 4 elements per thread.
DotPlan dot_plan(int64_t n, int k, int nv) {
    if (k > 256) throw Error(BIE_EUNSUPPORTED, "more than 256 right-hand sides per solve");
    int groups = 1;
    while (k * groups * 2 <= 256) groups *= 2;
    DotPlan p;
    p.bs = k * groups;
    const int64_t elems = n * (int64_t)k;
    int64_t nblk = std::min<int64_t>((2048 + nv - 1) / std::max(1, nv), (elems + 4 * p.bs - 1) / (4 * p.bs));
    nblk = std::max<int64_t>(1, std::min<int64_t>(nblk, n));
    p.rows_per_blk = (n + nblk - 1) / nblk;
    p.nblk = (int)((n + p.rows_per_blk - 1) / p.rows_per_blk);
    return p;
}

void dots_finish(bie_geom* g, int nblk, int64_t nout, double* out, int mode, cudaStream_t s) {
    k_dots_finish<<<(unsigned)((nout + 7) / 8), 256, 0, s>>>(g->dpart.as<double>(), nblk, nout, out, mode);
    BIE_CK(cudaGetLastError());
}

// out[v][c] = sum_i A_v[i][c] B[i][c] for v < nv (mode: 0 assign, 1 accumulate, 2 sqrt)
void dots(bie_geom* g, const double* A, int64_t strideA, int nv, const double* B, int k, double* out, int mode,
          cudaStream_t s) {
    DotPlan p = dot_plan(g->n, k, nv);
    g->dpart.ensure(sizeof(double) * (size_t)p.nblk * nv * k);
    Prof pf(g, BIE_KERNEL_KRYLOV, s, 2);
    k_dots_blk<<<dim3(p.nblk, nv), p.bs, p.bs * sizeof(double), s>>>(A, strideA, nv, B, g->n, k, p.rows_per_blk,
                                                                    g->dpart.as<double>());
    BIE_CK(cudaGetLastError());
    dots_finish(g, p.nblk, (int64_t)nv * k, out, mode, s);
}

// W -= sum_v V_v h[v] (columnwise), then out[c] = |W[:, c]|
void gs_update_norm(bie_geom* g, double* W, const double* V, int64_t strideV, int nv, const double* h, int k,
                    double* out, cudaStream_t s) {
    DotPlan p = dot_plan(g->n, k, 1);
    g->dpart.ensure(sizeof(double) * (size_t)p.nblk * k);
    Prof pf(g, BIE_KERNEL_KRYLOV, s, 2);
    k_gs_update_norm<<<p.nblk, p.bs, p.bs * sizeof(double), s>>>(W, V, strideV, nv, h, g->n, k, p.rows_per_blk,
                                                                g->dpart.as<double>());
    BIE_CK(cudaGetLastError());
    dots_finish(g, p.nblk, k, out, 2, s);
}

void col_norms(bie_geom* g, const double* X, int k, double* out, cudaStream_t s) {
    dots(g, X, 0, 1, X, k, out, 2, s);
}

template <class T>
void d2h(T* dst, const void* src, size_t count, cudaStream_t s) {
    BIE_CK(cudaMemcpyAsync(dst, src, sizeof(T) * count, cudaMemcpyDeviceToHost, s));
    BIE_CK(cudaStreamSynchronize(s));
}

// ------------------------------- GMRES -------------------------------------
struct GmresResult {
    int iters = 0;       // iterations (= operator applications inside the Arnoldi loop)
    int matvecs = 0;     // all operator applications incl. restart residuals
    bool all_converged = false;
    bool resid_written = false;  // bgmres: the residual r - A(p .* u) went to resid_out
    std::vector<int> col_iters;
};

// Solves A(prec) (p .* u) = r, x = p .* u for the columns flagged in `active0`;
// dx (node-major n x k) receives the solution (zeroed first). eps[c] is the
// absolute residual tolerance of column c. Each column runs its own Arnoldi
// process; converged columns are frozen. FP64 solves orthogonalise by classical
// Gram-Schmidt applied twice. The inner solves of iterative refinement (reduced
// precision operators) stop at a relative residual of about 1e-6, and the outer
// loop recomputes the true residual, so one classical Gram-Schmidt pass (fused with
// the new direction's norm) serves them and halves the passes over the basis.
GmresResult gmres(bie_geom* g, const double* dr, double* dx, int k, int prec, uint32_t flags, const double* pre,
                  const std::vector<double>& eps, const std::vector<char>& active0, int itmax, int m, int check_every,
                  cudaStream_t s, double* resid_out = nullptr, int resid_prec = -1) {
    const int64_t n = g->n;
    const int64_t nk = n * (int64_t)k;
    const bool one_pass = prec != BIE_FP64;  // see above
    // the residual r - A x into resid_out (may be dr) when the caller would form it with this
    // same operator: from the last cycle's Arnoldi relation, or the cycle-start residual
    const bool want_resid = resid_out && op_kind(prec, k) == op_kind(resid_prec, k);
    m = std::max(1, std::min(m, itmax));
    const int m1 = m + 1;
    g->V.ensure(sizeof(double) * (size_t)m1 * nk);
    g->W.ensure(sizeof(double) * nk);
    g->rr.ensure(sizeof(double) * nk);
    g->R.ensure(sizeof(double) * (size_t)m1 * m1 * k);
    g->gv.ensure(sizeof(double) * (size_t)m1 * k);
    g->cs.ensure(sizeof(double) * (size_t)m1 * k);
    g->sn.ensure(sizeof(double) * (size_t)m1 * k);
    g->h.ensure(sizeof(double) * (size_t)m1 * k);
    g->h2.ensure(sizeof(double) * (size_t)m1 * k);
    g->hn.ensure(sizeof(double) * k);
    g->beta.ensure(sizeof(double) * k);
    g->eps.ensure(sizeof(double) * k);
    g->active.ensure(sizeof(int) * k);
    g->jlast.ensure(sizeof(int) * k);
    g->yv.ensure(sizeof(double) * (size_t)m1 * k);
    g->resid.ensure(sizeof(double) * k);
    {
        // the column reductions' partials at their largest, so no iteration reallocates
        size_t need = 0;
        for (int nv = 1; nv <= m1; ++nv) {
            const DotPlan p = dot_plan(n, k, nv);
            need = std::max(need, (size_t)p.nblk * nv * k);
        }
        g->dpart.ensure(sizeof(double) * need);
    }
    double* V = g->V.as<double>();
    double* W = g->W.as<double>();
    BIE_CK(cudaMemsetAsync(dx, 0, sizeof(double) * nk, s));
    upload(g->eps, eps.data(), k, s);

    // Graph cache entry of this configuration. An iteration is captured once the same
    // configuration has completed one eager solve (every buffer it touches is sized), and
    // replayed afterwards; kernel timing (profiling) runs eagerly.
    auto signature = [&]() {
        uint64_t h = 1469598103934665603ull;
        auto mix = [&](uint64_t v) {
            h ^= v;
            h *= 1099511628211ull;
        };
        mix((uint64_t)k); mix((uint64_t)prec); mix(flags); mix((uint64_t)m); mix((uintptr_t)pre);
        const bie::Buf* bufs[] = {&g->V, &g->W, &g->part, &g->bpack, &g->cpart, &g->dpart, &g->h, &g->h2, &g->hn, &g->R,
                                  &g->cs, &g->sn, &g->gv, &g->active, &g->jlast, &g->eps, &g->resid, &g->errflag};
        for (const auto* b : bufs) {
            mix((uintptr_t)b->p);
            mix((uint64_t)b->bytes);
        }
        return h;
    };
    const uint64_t sig0 = signature();
    bie_geom::GraphCache* gc = nullptr;
    for (auto& c : g->gcache)
        if (c.sig == sig0 && !c.exec.empty()) gc = &c;
    if (!gc) {
        gc = &g->gcache[g->gcache_next];
        g->gcache_next ^= 1;
        for (auto ex : gc->exec)
            if (ex) cudaGraphExecDestroy(ex);
        gc->sig = sig0;
        gc->warm = false;
        gc->exec.assign(m, nullptr);
    }
    bool use_graph = g->graphs && !g->prof_on && gc->warm && s == g->stream;

    GmresResult res;
    res.col_iters.assign(k, 0);
    std::vector<double> hb(k), g0((size_t)k);
    std::vector<int> act(k), jl(k);
    bool first = true;
    int it = 0;
    while (true) {
        // residual of the current cycle
        const double* r = dr;
        if (!first) {
            apply_op(g, dx, W, k, prec, flags, nullptr, s);  // dx holds x = p .* u: the true residual
            ++res.matvecs;
            BIE_CK(cudaMemcpyAsync(g->rr.p, dr, sizeof(double) * nk, cudaMemcpyDeviceToDevice, s));
            {
                Prof pf(g, BIE_KERNEL_KRYLOV, s);
                k_axpby<<<grid1(nk), 256, 0, s>>>(-1.0, W, 1.0, g->rr.as<double>(), n, k, nullptr);
            }
            r = g->rr.as<double>();
        }
        col_norms(g, r, k, g->beta.as<double>(), s);
        d2h(hb.data(), g->beta.p, k, s);
        int nact = 0;
        for (int c = 0; c < k; ++c) {
            act[c] = active0[c] && hb[c] > eps[c] ? 1 : 0;
            nact += act[c];
        }
        if (nact == 0 || it >= itmax) {
            res.all_converged = nact == 0;
            if (want_resid) {  // nothing solved since r was formed
                if (resid_out != r)
                    BIE_CK(cudaMemcpyAsync(resid_out, r, sizeof(double) * nk, cudaMemcpyDeviceToDevice, s));
                res.resid_written = true;
            }
            break;
        }
        upload(g->active, act.data(), k, s);
        BIE_CK(cudaMemsetAsync(g->jlast.p, 0, sizeof(int) * k, s));
        BIE_CK(cudaMemsetAsync(g->gv.p, 0, sizeof(double) * m1 * k, s));
        BIE_CK(cudaMemcpyAsync(g->gv.p, g->beta.p, sizeof(double) * k, cudaMemcpyDeviceToDevice, s));
        {
            Prof pf(g, BIE_KERNEL_KRYLOV, s);
            k_scale_cols<<<grid1(nk), 256, 0, s>>>(r, g->beta.as<double>(), n, k, V);
        }
        int j = 0;
        bool any = true;
        for (; j < m && it < itmax; ++j) {
            auto iteration = [&]() {
                double* Vj = V + (size_t)j * nk;
                apply_op(g, Vj, W, k, prec, flags, pre, s);
                // classical Gram-Schmidt, twice for FP64 solves; the last pass is fused with the
                // norm of the new direction, and the second pass's coefficients are added to the
                // first pass's in the Givens step
                dots(g, V, nk, j + 1, W, k, g->h.as<double>(), 0, s);
                if (one_pass) {
                    gs_update_norm(g, W, V, nk, j + 1, g->h.as<double>(), k, g->hn.as<double>(), s);
                } else {
                    {
                        Prof pf(g, BIE_KERNEL_KRYLOV, s);
                        k_gs_update<<<grid1(nk), 256, 0, s>>>(W, V, nk, j + 1, g->h.as<double>(), n, k);
                    }
                    dots(g, V, nk, j + 1, W, k, g->h2.as<double>(), 0, s);
                    gs_update_norm(g, W, V, nk, j + 1, g->h2.as<double>(), k, g->hn.as<double>(), s);
                }
                {
                    Prof pf(g, BIE_KERNEL_KRYLOV, s);
                    k_scale_cols<<<grid1(nk), 256, 0, s>>>(W, g->hn.as<double>(), n, k, V + (size_t)(j + 1) * nk);
                }
                {
                    Prof pf(g, BIE_KERNEL_KRYLOV, s);
                    k_givens<<<grid1(k, 64), 64, 0, s>>>(g->R.as<double>(), g->h.as<double>(),
                                                        one_pass ? nullptr : g->h2.as<double>(),
                                                        g->hn.as<double>(), g->cs.as<double>(), g->sn.as<double>(),
                                                        g->gv.as<double>(), g->active.as<int>(), g->jlast.as<int>(),
                                                        g->eps.as<double>(), g->resid.as<double>(), j, m1, k);
                }
                BIE_CK(cudaGetLastError());
            };
            ++res.matvecs;
            if (use_graph && !gc->exec[j]) {
                // capture iteration j; on any failure fall back to eager iterations
                BIE_CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                bool ok = true;
                try {
                    iteration();
                } catch (...) {
                    ok = false;
                }
                cudaGraph_t graph = nullptr;
                const cudaError_t ec = cudaStreamEndCapture(s, &graph);
                cudaGraphExec_t ex = nullptr;
                if (ok && ec == cudaSuccess && graph && cudaGraphInstantiate(&ex, graph, 0) == cudaSuccess)
                    gc->exec[j] = ex;
                if (graph) cudaGraphDestroy(graph);
                if (!gc->exec[j]) {
                    cudaGetLastError();
                    use_graph = false;
                    g->graphs = false;
                }
            }
            if (use_graph)
                BIE_CK(cudaGraphLaunch(gc->exec[j], s));
            else
                iteration();
            BIE_CK(cudaGetLastError());
            ++it;
            if ((j + 1) % std::max(1, check_every) == 0 || j + 1 == m || it >= itmax) {
                d2h(act.data(), g->active.p, k, s);
                any = false;
                for (int c = 0; c < k; ++c) any = any || act[c];
                if (!any) {
                    ++j;
                    break;
                }
            }
        }
        {
            Prof pf(g, BIE_KERNEL_KRYLOV, s);
            k_backsolve<<<grid1(k, 64), 64, 0, s>>>(g->R.as<double>(), g->gv.as<double>(), g->jlast.as<int>(), m1, k,
            g->yv.as<double>());
        }
        {
            Prof pf(g, BIE_KERNEL_KRYLOV, s);
            k_update_solution<<<grid1(nk), 256, 0, s>>>(dx, V, nk, g->yv.as<double>(), g->jlast.as<int>(), m, pre, n, k);
        }
        BIE_CK(cudaGetLastError());
        d2h(jl.data(), g->jlast.p, k, s);
        for (int c = 0; c < k; ++c) res.col_iters[c] += jl[c];
        d2h(act.data(), g->active.p, k, s);
        any = false;
        for (int c = 0; c < k; ++c) any = any || act[c];
        if ((!any || it >= itmax) && want_resid) {
            // r - A(p .* u) = V z from the Arnoldi relation A P V_j = V_{j+1} H_j: equal to an
            // application of the operator to the correction up to FP64 rounding
            Prof pf(g, BIE_KERNEL_KRYLOV, s, 2);
            k_givens_resid<<<grid1(k, 64), 64, 0, s>>>(g->gv.as<double>(), g->cs.as<double>(), g->sn.as<double>(),
                                                       g->jlast.as<int>(), m1, k, g->yv.as<double>());
            k_basis_combine<<<grid1(nk), 256, 0, s>>>(resid_out, V, nk, g->yv.as<double>(), g->jlast.as<int>(), n, k);
            BIE_CK(cudaGetLastError());
            res.resid_written = true;
        }
        if (!any) {
            res.all_converged = true;
            break;
        }
        if (it >= itmax) break;
        first = false;  // restart from the true residual of the current iterate
    }
    if (signature() == gc->sig) gc->warm = true;
    res.iters = it;
    return res;
}

// ------------------------------ block GMRES ----------------------------------
void blas_ck(cublasStatus_t st, const char* what) {
    if (st != CUBLAS_STATUS_SUCCESS)
        throw Error(st == CUBLAS_STATUS_ALLOC_FAILED ? BIE_ENOMEM : BIE_ECUDA,
                    std::string("cuBLAS ") + what + " failed (status " + std::to_string((int)st) + ")");
}

cublasHandle_t blas_handle(bie_geom* g, cudaStream_t s) {
    if (!g->blas) blas_ck(cublasCreate(&g->blas), "create");
    blas_ck(cublasSetStream(g->blas, s), "set stream");
    return g->blas;
}

// G (ka x ka, ld ka) = Q Q^T for Q ka x n (ld ka): partial Gram matrices of up to 148 column
// chunks (one batched DGEMM, a second for the remainder), summed in a fixed order.
void gram(bie_geom* g, cublasHandle_t h, const double* Q, int ka, int64_t n, double* G, cudaStream_t s) {
    const double one = 1.0, zero = 0.0;
    const int64_t nb_want = std::max<int64_t>(1, std::min<int64_t>(148, n / 256));
    const int64_t c = (n + nb_want - 1) / nb_want;
    const int64_t nfull = n / c, rem = n - nfull * c;
    const int nb = (int)(nfull + (rem > 0 ? 1 : 0));
    const int64_t kk = (int64_t)ka * ka;
    g->bpart.ensure(sizeof(double) * (size_t)nb * kk);
    double* P = g->bpart.as<double>();
    if (nfull > 0)
        blas_ck(cublasDgemmStridedBatched(h, CUBLAS_OP_N, CUBLAS_OP_T, ka, ka, (int)c, &one, Q, ka, c * ka, Q, ka,
                                          c * ka, &zero, P, ka, kk, (int)nfull),
                "gemm (batched)");
    if (rem > 0)
        blas_ck(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, ka, ka, (int)rem, &one, Q + nfull * c * ka, ka,
                            Q + nfull * c * ka, ka, &zero, P + nfull * kk, ka),
                "gemm");
    k_sum_partials<<<(unsigned)((kk + 31) / 32), 256, 0, s>>>(P, nb, (int)kk, G);
    BIE_CK(cudaGetLastError());
}

// Orthonormalises the rows of Q (ka x n, column-major, ld ka: the transposed block of ka <= 64
// vectors) by Cholesky QR applied `passes` times (2: CholQR2, orthogonal to working precision
// for condition numbers up to about 1e8; 1: orthogonality error about cond^2 1e-16, enough
// for the reduced-precision inner solves that stop near 1e-6): Q_old = R^T Q_new, R = R2 R1
// (ka x ka upper) into Rout (ld ldr). The Gram matrix comes from chunked DGEMMs, is factored
// and inverted in shared memory and applied as a DGEMM with R^-T. Returns the number of this
// library's kernels it launched.
int cholqr2(bie_geom* g, cublasHandle_t h, double* Q, int ka, int64_t n, double* Rout, int ldr, cudaStream_t s,
            int passes = 2) {
    const double one = 1.0, zero = 0.0;
    double* R1 = g->br1.as<double>();
    double* R2 = g->br2.as<double>();
    g->binv.ensure(sizeof(double) * (size_t)ka * ka);
    g->btmp.ensure(sizeof(double) * (size_t)n * ka);
    double* Gm = g->br.as<double>();
    double* Ri = g->binv.as<double>();
    double* tmp = g->btmp.as<double>();
    const size_t sm = 2 * sizeof(double) * (size_t)ka * (ka + 1);
    ensure_smem_limit((const void*)k_chol_inv_smem<kCholThreads>, sm);
    for (int pass = 0; pass < passes; ++pass) {
        double* Rp = pass == 0 ? R1 : R2;
        gram(g, h, Q, ka, n, Gm, s);
        k_chol_inv_smem<kCholThreads><<<1, kCholThreads, sm, s>>>(Gm, ka, Rp, ka, Ri, g->bflag.as<int>());
        BIE_CK(cudaGetLastError());
        blas_ck(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, ka, (int)n, ka, &one, Ri, ka, Q, ka, &zero, tmp, ka), "gemm");
        BIE_CK(cudaMemcpyAsync(Q, tmp, sizeof(double) * (size_t)n * ka, cudaMemcpyDeviceToDevice, s));
    }
    const int per_pass = 2;  // k_sum_partials + k_chol_inv_smem
    if (passes == 1) {
        BIE_CK(cudaMemcpy2DAsync(Rout, sizeof(double) * (size_t)ldr, R1, sizeof(double) * (size_t)ka,
                                 sizeof(double) * (size_t)ka, (size_t)ka, cudaMemcpyDeviceToDevice, s));
        return per_pass;
    }
    k_trmm_upper<<<grid1((int64_t)ka * ka), 256, 0, s>>>(R2, ka, R1, ka, Rout, ldr, ka);
    BIE_CK(cudaGetLastError());
    return passes * per_pass + 1;
}

// Whether a solve of k columns runs block GMRES: the option is set and 2 <= k <= 64. Wider
// blocks run one Arnoldi process per column, which shares one operator application per
// iteration over all columns; block GMRES in chunks of 64 applies the operator once per chunk
// (cfg3 box, rtol 1e-10, bf16x3: 96 columns 85-88 ms per column-wise solve against 100-102 ms
// in chunks, 128 columns 98-99 ms against 104-114 ms).
inline bool use_block(const bie_solve_opts& o, int k) { return o.block && k > 1 && k <= 64; }

// The block solver's side stream, its two events and the pinned residual-norm buffer.
void ls_init(bie_geom* g) {
    if (!g->s_ls) BIE_CK(cudaStreamCreateWithFlags(&g->s_ls, cudaStreamNonBlocking));
    if (!g->ev_h) BIE_CK(cudaEventCreateWithFlags(&g->ev_h, cudaEventDisableTiming));
    if (!g->ev_res) BIE_CK(cudaEventCreateWithFlags(&g->ev_res, cudaEventDisableTiming));
    if (!g->bres_host) BIE_CK(cudaMallocHost(&g->bres_host, sizeof(double) * 64));
}

// One block Krylov space (the method of Krylov.block_gmres, src/solver/multi_rhs.jl:285) for
// the columns idx (at most 64) of dr. Block Arnoldi with classical Gram-Schmidt against the
// whole basis (two passes for FP64 solves, one for the reduced-precision inner solves), each
// new block orthonormalised by Cholesky QR (twice for FP64 solves, once for the inner
// solves); the block upper-Hessenberg least-squares problem is updated by Householder
// reflections one block column per iteration (kept in compact-WY form), which gives every
// column's residual norm. The tall-skinny products with the basis are cuBLAS DGEMMs. The
// basis is kept as the rows of M ((m + 1) ka x n, column-major: node i holds all basis values
// in a row of M's column i). The columns' solution goes to the same columns of dx, their
// residual r - A x to resid_out when it is not null (from the Arnoldi relation); iterations,
// operator applications and convergence are merged into res.
void bgmres_chunk(bie_geom* g, const double* dr, double* dx, int k, int prec, uint32_t flags, const double* pre,
                  const std::vector<int>& idx, const std::vector<double>& eps, int itmax, int m, cudaStream_t s,
                  double* resid_out, GmresResult& res) {
    const int64_t n = g->n;
    const bool one_pass = prec != BIE_FP64;
    const int ka = (int)idx.size();
    const bool want_resid = resid_out != nullptr;
    const int64_t L = (int64_t)(m + 1) * ka;  // rows of the basis and of the Hessenberg matrix
    const int64_t nka = n * ka;
    g->bv.ensure(sizeof(double) * (size_t)L * n);
    g->bq.ensure(sizeof(double) * nka);
    g->bvj.ensure(sizeof(double) * nka);
    g->bh.ensure(sizeof(double) * (size_t)L * m * ka);
    g->bgv.ensure(sizeof(double) * (size_t)L * ka);
    g->btau.ensure(sizeof(double) * (size_t)m * ka);
    g->bwy.ensure(sizeof(double) * (size_t)m * wy_stride(ka));
    g->br1.ensure(sizeof(double) * (size_t)ka * ka);
    g->br2.ensure(sizeof(double) * (size_t)ka * ka);
    g->br.ensure(sizeof(double) * (size_t)ka * ka);
    g->bh2.ensure(sizeof(double) * (size_t)L * ka);
    g->bres.ensure(sizeof(double) * ka);
    g->bidx.ensure(sizeof(int) * ka);
    g->bflag.ensure(sizeof(int));
    g->xa.ensure(sizeof(double) * nka);
    g->ra.ensure(sizeof(double) * nka);
    upload(g->bidx, idx.data(), ka, s);
    BIE_CK(cudaMemsetAsync(g->bflag.p, 0, sizeof(int), s));
    double* M = g->bv.as<double>();
    double* Q = g->bq.as<double>();
    double* Vj = g->bvj.as<double>();
    double* H = g->bh.as<double>();
    double* Gv = g->bgv.as<double>();
    double* Xa = g->xa.as<double>();
    double* Ra = g->ra.as<double>();
    BIE_CK(cudaMemsetAsync(Xa, 0, sizeof(double) * nka, s));
    std::vector<double> epsa(ka), rsd(ka);
    for (int a = 0; a < ka; ++a) epsa[a] = eps[idx[a]];
    const double one = 1.0, zero = 0.0, mone = -1.0;
    const size_t pitchL = sizeof(double) * (size_t)L, pitchK = sizeof(double) * (size_t)ka;
    int it = 0;
    bool first = true, conv = false;
    while (true) {
        // residual of the cycle: the right-hand side, or the true residual of the iterate
        {
            Prof pf(g, BIE_KERNEL_KRYLOV, s);
            k_gather_cols<<<grid1(nka), 256, 0, s>>>(dr, k, g->bidx.as<int>(), ka, n, Ra);
            BIE_CK(cudaGetLastError());
        }
        if (!first) {
            apply_op(g, Xa, Q, ka, prec, flags, nullptr, s);
            ++res.matvecs;
            Prof pf(g, BIE_KERNEL_KRYLOV, s);
            k_axpby<<<grid1(nka), 256, 0, s>>>(-1.0, Q, 1.0, Ra, n, ka, nullptr);
            BIE_CK(cudaGetLastError());
        }
        cublasHandle_t h = blas_handle(g, s);
        BIE_CK(cudaMemsetAsync(H, 0, sizeof(double) * (size_t)L * m * ka, s));
        BIE_CK(cudaMemsetAsync(Gv, 0, sizeof(double) * (size_t)L * ka, s));
        // V_0 S_0 = R (Cholesky QR); Gv = [S_0; 0]
        {
            Prof pf(g, BIE_KERNEL_KRYLOV, s, 0);
            pf.add(cholqr2(g, h, Ra, ka, n, Gv, (int)L, s, one_pass ? 1 : 2));
            BIE_CK(cudaMemcpy2DAsync(M, pitchL, Ra, pitchK, pitchK, (size_t)n, cudaMemcpyDeviceToDevice, s));
        }
        int jend = 0;
        bool queued = false;  // this iteration's operator application is already in the stream
        double worst = 0.0;   // max over the columns of residual / tolerance after an iteration
        auto queue_apply = [&](int jj) {  // W = A (p .* V_jj), held as Q = W^T
            BIE_CK(cudaMemcpy2DAsync(Vj, pitchK, M + (size_t)jj * ka, pitchL, pitchK, (size_t)n,
                                     cudaMemcpyDeviceToDevice, s));
            apply_op(g, Vj, Q, ka, prec, flags, pre, s);
            ++res.matvecs;
        };
        for (int j = 0; j < m && it < itmax; ++j) {
            const int64_t rows = (int64_t)(j + 1) * ka;  // basis vectors so far
            if (!queued) queue_apply(j);
            queued = false;
            {
                Prof pf(g, BIE_KERNEL_KRYLOV, s, 0);
                double* Hc = H + (size_t)j * ka * L;  // block column j
                // classical Gram-Schmidt: H = V^T W and W -= V H, i.e. H = M_j Q^T, Q -= H^T M_j
                blas_ck(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, (int)rows, ka, (int)n, &one, M, (int)L, Q, ka, &zero,
                                    Hc, (int)L),
                        "gemm");
                blas_ck(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, ka, (int)n, (int)rows, &mone, Hc, (int)L, M, (int)L,
                                    &one, Q, ka),
                        "gemm");
                if (!one_pass) {
                    double* H2 = g->bh2.as<double>();
                    blas_ck(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, (int)rows, ka, (int)n, &one, M, (int)L, Q, ka,
                                        &zero, H2, (int)rows),
                            "gemm");
                    blas_ck(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, ka, (int)n, (int)rows, &mone, H2, (int)rows, M,
                                        (int)L, &one, Q, ka),
                            "gemm");
                    blas_ck(cublasDgeam(h, CUBLAS_OP_N, CUBLAS_OP_N, (int)rows, ka, &one, Hc, (int)L, &one, H2,
                                        (int)rows, Hc, (int)L),
                            "geam");
                }
                // the new block: W = V_{j+1} R, R into H's block (j + 1, j)
                pf.add(cholqr2(g, h, Q, ka, n, Hc + rows, (int)L, s, one_pass ? 1 : 2));
                BIE_CK(cudaMemcpy2DAsync(M + (size_t)(j + 1) * ka, pitchL, Q, pitchK, pitchK, (size_t)n,
                                         cudaMemcpyDeviceToDevice, s));
            }
            // Least squares: the Householder QR of block column j and every column's residual,
            // on the side stream once the column is complete. Only the convergence test needs it:
            // the next operator application (queued below when convergence is still far) runs
            // beside it. The two streams touch disjoint data until the cycle's end, where the
            // solver's stream waits for the side stream (block column j, the right-hand sides,
            // tau and the WY blocks there; the basis block j + 1, Q and block column j + 1 here).
            ls_init(g);
            BIE_CK(cudaEventRecord(g->ev_h, s));
            BIE_CK(cudaStreamWaitEvent(g->s_ls, g->ev_h, 0));
            {
                Prof pf(g, BIE_KERNEL_KRYLOV, g->s_ls, 0, 0, 0, 0, false);
                double* wy = g->bwy.as<double>();  // each block column's compact-WY form (V, T^T)
                if (j > 0) {
                    const size_t sm = apply_prev_smem(ka);
                    ensure_smem_limit((const void*)k_bhess_apply_prev, sm);
                    k_bhess_apply_prev<<<(ka + kApplyCols - 1) / kApplyCols, 256, sm, g->s_ls>>>(H, (int)L, wy, ka,
                                                                                                j);
                    BIE_CK(cudaGetLastError());
                    pf.add(1);
                }
                pf.add(1);
                k_bhess_qr_tile<<<1, 512, 0, g->s_ls>>>(H, (int)L, g->btau.as<double>(), Gv, (int)L, ka, j,
                                                        g->bres.as<double>(), wy + (size_t)j * wy_stride(ka));
                BIE_CK(cudaGetLastError());
            }
            BIE_CK(cudaMemcpyAsync(g->bres_host, g->bres.p, sizeof(double) * ka, cudaMemcpyDeviceToHost, g->s_ls));
            BIE_CK(cudaEventRecord(g->ev_res, g->s_ls));
            ++it;
            jend = j + 1;
            // A GMRES iteration lowers a residual by a few times at most: while the previous one
            // left every column above 16 times its tolerance, the next iteration will run, and its
            // operator application is queued before the host waits for the norms (were the
            // columns to converge after all, that application is merely unused)
            if (j > 0 && worst > 16.0 && j + 1 < m && it < itmax) {
                queue_apply(j + 1);
                queued = true;
            }
            BIE_CK(cudaEventSynchronize(g->ev_res));
            bool all = true;
            worst = 0.0;
            for (int a = 0; a < ka; ++a) {
                rsd[a] = g->bres_host[a];
                all = all && rsd[a] <= epsa[a];
                worst = std::max(worst, rsd[a] / epsa[a]);
            }
            if (all) {
                conv = true;
                break;
            }
        }
        if (jend > 0) BIE_CK(cudaStreamWaitEvent(s, g->ev_res, 0));  // the cycle's last least-squares update
        // Y = R^-1 Gv[0 : jend ka], x += p .* (V Y)
        {
            Prof pf(g, BIE_KERNEL_KRYLOV, s);  // k_add_rows_scaled (TRSM and DGEMM are cuBLAS's)
            const int rows = jend * ka;
            blas_ck(cublasDtrsm(h, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, rows, ka,
                                &one, H, (int)L, Gv, (int)L),
                    "trsm");
            blas_ck(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, ka, (int)n, rows, &one, Gv, (int)L, M, (int)L, &zero, Q,
                                ka),
                    "gemm");
            k_add_rows_scaled<<<grid1(nka), 256, 0, s>>>(Xa, Q, pre, n, ka);
            BIE_CK(cudaGetLastError());
        }
        // The residual of the last cycle from the Arnoldi relation A P V_j = V_{j+1} H_j:
        // r - A(p .* u) = V (G - H Y) = V Q [0; g], g the last ka rows of the transformed right-hand
        // sides, Q the block reflectors. It equals an application of the inner operator to the
        // correction up to FP64 rounding, and replaces it when the caller would update its
        // residual with that same operator.
        if ((conv || it >= itmax) && want_resid && jend == 0) {
            // no iteration in this cycle: the residual is the cycle's own
            Prof pf(g, BIE_KERNEL_KRYLOV, s);
            k_scatter_cols<<<grid1(nka), 256, 0, s>>>(Ra, ka, g->bidx.as<int>(), k, n, resid_out);
            BIE_CK(cudaGetLastError());
        }
        if ((conv || it >= itmax) && want_resid && jend > 0) {
            Prof pf(g, BIE_KERNEL_KRYLOV, s, 0);
            double* Z = g->bh2.as<double>();  // (jend + 1) ka x ka, ld L
            BIE_CK(cudaMemsetAsync(Z, 0, sizeof(double) * (size_t)L * ka, s));
            BIE_CK(cudaMemcpy2DAsync(Z + (size_t)jend * ka, pitchL, Gv + (size_t)jend * ka, pitchL, pitchK, (size_t)ka,
                                     cudaMemcpyDeviceToDevice, s));
            const size_t sm = apply_q_smem(ka);
            ensure_smem_limit((const void*)k_bhess_apply_q, sm);
            k_bhess_apply_q<<<(ka + kApplyCols - 1) / kApplyCols, 256, sm, s>>>(g->bwy.as<double>(), ka, jend, Z,
                                                                                (int)L);
            BIE_CK(cudaGetLastError());
            blas_ck(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, ka, (int)n, (jend + 1) * ka, &one, Z, (int)L, M, (int)L,
                                &zero, Q, ka),
                    "gemm");
            k_scatter_cols<<<grid1(nka), 256, 0, s>>>(Q, ka, g->bidx.as<int>(), k, n, resid_out);
            BIE_CK(cudaGetLastError());
            pf.add(2);
        }
        if (conv || it >= itmax) break;
        first = false;
    }
    {
        Prof pf(g, BIE_KERNEL_KRYLOV, s);
        k_scatter_cols<<<grid1(nka), 256, 0, s>>>(Xa, ka, g->bidx.as<int>(), k, n, dx);
        BIE_CK(cudaGetLastError());
    }
    for (int a = 0; a < ka; ++a) res.col_iters[idx[a]] = it;
    res.iters = std::max(res.iters, it);
    res.all_converged = res.all_converged && conv;
}

// Block GMRES (the method of Krylov.block_gmres) over the active columns of dr that are above
// their tolerance, in balanced chunks of at most 64 columns, each its own block Krylov space
// (the least-squares and CholQR kernels hold up to 64 columns). Solves A(p .* u) = r, x = p .* u
// into dx (node-major n x k, zero in the other columns); m = block iterations per cycle
// (restart, at most 60). With resid_out (n x k, may be dr itself) and an operator for
// (resid_prec, k) equal to the one every chunk iterates with, the solved columns' residual
// r - A x is written there as well (GmresResult::resid_written).
GmresResult bgmres(bie_geom* g, const double* dr, double* dx, int k, int prec, uint32_t flags, const double* pre,
                   const std::vector<double>& eps, const std::vector<char>& active0, int itmax, int m, cudaStream_t s,
                   double* resid_out = nullptr, int resid_prec = -1) {
    const int64_t n = g->n;
    GmresResult res;
    res.col_iters.assign(k, 0);
    BIE_CK(cudaMemsetAsync(dx, 0, sizeof(double) * n * k, s));
    // columns that need work: active and above their tolerance
    g->beta.ensure(sizeof(double) * k);
    col_norms(g, dr, k, g->beta.as<double>(), s);
    std::vector<double> nr(k);
    d2h(nr.data(), g->beta.p, k, s);
    std::vector<int> idx;
    for (int c = 0; c < k; ++c)
        if (active0[c] && nr[c] > eps[c]) idx.push_back(c);
    const int ka = (int)idx.size();
    res.all_converged = true;
    if (ka == 0) return res;
    m = std::max(1, std::min({m, itmax, 60}));
    const int nch = (ka + 63) / 64, csz = (ka + nch - 1) / nch;
    bool want = resid_out != nullptr;
    for (int c0 = 0; c0 < ka; c0 += csz) want = want && op_kind(prec, std::min(csz, ka - c0)) == op_kind(resid_prec, k);
    for (int c0 = 0; c0 < ka; c0 += csz) {
        const std::vector<int> sub(idx.begin() + c0, idx.begin() + std::min(ka, c0 + csz));
        bgmres_chunk(g, dr, dx, k, prec, flags, pre, sub, eps, itmax, m, s, want ? resid_out : nullptr, res);
    }
    res.resid_written = want;
    return res;
}

// Raises BIE_ETIMEOUT if a kernel recorded an expired bounded wait (and clears the flag).
void check_device_error(bie_geom* g, cudaStream_t s) {
    int e = 0;
    BIE_CK(cudaMemcpyAsync(&e, g->errflag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    BIE_CK(cudaStreamSynchronize(s));
    if (e) {
        BIE_CK(cudaMemsetAsync(g->errflag.p, 0, sizeof(int), s));
        throw Error(BIE_ETIMEOUT, "a device wait ran out of its iteration limit (kernel returned early)");
    }
}

void check_prec(int prec) {
    if (prec != BIE_FP64 && prec != BIE_FP32 && prec != BIE_BF16X3 && prec != BIE_BF16X6)
        throw Error(BIE_EINVAL, "unknown precision");
}

}  // namespace

// ---------------------------------------------------------------------------
// geometry lifetime
// ---------------------------------------------------------------------------
bie_geom* geom_create(const double* pts, const double* nrm, const double* w, const double* diag, int64_t n,
                      int32_t npanels, int32_t nb, const int32_t* rowptr, const int32_t* col, const double* val,
                      int64_t nblocks, int device) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        throw Error(BIE_ENODEVICE, "no CUDA device available (libbie_b200 has no CPU fallback)");
    }
    if (device < 0 || device >= ndev) throw Error(BIE_EINVAL, "device ordinal out of range");
    if (n >= (int64_t)1 << 31) throw Error(BIE_EUNSUPPORTED, "at most 2^31 - 1 nodes per geometry");
    DeviceGuard dg(device);
    std::unique_ptr<bie_geom> g(new bie_geom());
    g->device = device;
    g->graphs = std::getenv("BIE_NO_GRAPHS") == nullptr;
    g->autotune = std::getenv("BIE_NO_AUTOTUNE") == nullptr;
    BIE_CK(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    BIE_CK(cudaEventCreate(&g->ev0));
    BIE_CK(cudaEventCreate(&g->ev1));
    BIE_CK(cudaDeviceGetAttribute(&g->sms, cudaDevAttrMultiProcessorCount, device));
    g->n = n;
    g->npanels = npanels;
    g->nb = nb;
    g->nblocks = nblocks;
    std::vector<double> col3((size_t)n);
    cudaStream_t s = g->stream;
    bie::Buf* xs[3] = {&g->x, &g->y, &g->z};
    bie::Buf* ns[3] = {&g->nx, &g->ny, &g->nz};
    for (int c = 0; c < 3; ++c) {
        for (int64_t i = 0; i < n; ++i) col3[i] = pts[3 * i + c];
        upload(*xs[c], col3.data(), n, s);
        BIE_CK(cudaStreamSynchronize(s));
        for (int64_t i = 0; i < n; ++i) col3[i] = nrm[3 * i + c];
        upload(*ns[c], col3.data(), n, s);
        BIE_CK(cudaStreamSynchronize(s));
    }
    upload(g->w, w, n, s);
    upload(g->diag, diag, n, s);
    // Morton (Z-order) permutation of the nodes: 21-bit quantised coordinates, bits interleaved
    {
        double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int64_t i = 0; i < n; ++i)
            for (int c = 0; c < 3; ++c) {
                lo[c] = std::min(lo[c], pts[3 * i + c]);
                hi[c] = std::max(hi[c], pts[3 * i + c]);
            }
        const double ext = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1e-300});
        auto spread = [](uint64_t v) {  // 21 bits -> every third bit of 63
            v &= 0x1FFFFFull;
            v = (v | v << 32) & 0x1F00000000FFFFull;
            v = (v | v << 16) & 0x1F0000FF0000FFull;
            v = (v | v << 8) & 0x100F00F00F00F00Full;
            v = (v | v << 4) & 0x10C30C30C30C30C3ull;
            v = (v | v << 2) & 0x1249249249249249ull;
            return v;
        };
        std::vector<std::pair<uint64_t, int32_t>> key((size_t)n);
        for (int64_t i = 0; i < n; ++i) {
            uint64_t q[3];
            for (int c = 0; c < 3; ++c)
                q[c] = (uint64_t)std::min(2097151.0, std::floor((pts[3 * i + c] - lo[c]) / ext * 2097151.0));
            key[i] = {spread(q[0]) | spread(q[1]) << 1 | spread(q[2]) << 2, (int32_t)i};
        }
        std::stable_sort(key.begin(), key.end(), [](auto& a, auto& b) { return a.first < b.first; });
        std::vector<int32_t> perm((size_t)n);
        for (int64_t i = 0; i < n; ++i) perm[i] = key[i].second;
        upload(g->perm, perm.data(), n, s);
        BIE_CK(cudaStreamSynchronize(s));
    }
    g->errflag.ensure(sizeof(int));
    BIE_CK(cudaMemsetAsync(g->errflag.p, 0, sizeof(int), s));
    for (int64_t i = 0; i < n; ++i) col3[i] = diag[i] != 0.0 ? 1.0 / diag[i] : 1.0;
    upload(g->pinv, col3.data(), n, s);
    if (nblocks > 0) {
        upload(g->rowptr, rowptr, (size_t)npanels + 1, s);
        for (int32_t p = 0; p < npanels; ++p) g->max_row_blocks = std::max(g->max_row_blocks, rowptr[p + 1] - rowptr[p]);
        upload(g->col, col, nblocks, s);
        upload(g->val, val, (size_t)nblocks * nb * nb, s);
    }
    BIE_CK(cudaStreamSynchronize(s));
    g->geom_bytes = sizeof(double) * (size_t)n * 9 + (nblocks > 0 ? (sizeof(int32_t) * ((size_t)npanels + 1 + nblocks) +
                                                                     sizeof(double) * (size_t)nblocks * nb * nb)
                                                                  : 0);
    return g.release();
}

bool tuning_read(bie_geom* g, int family, int columns, int pieces, int* nsplit, int* ctas, double* ms) {
    auto it = g->tuned.find(tune_key(family, columns, family == 0 ? pieces : 0));
    if (it == g->tuned.end()) return false;
    *nsplit = it->second.nsplit;
    *ctas = it->second.ctas;
    *ms = it->second.ms;
    return true;
}

// Releases a geometry's operator and solver workspace (direct-sum partials, Krylov
// basis, staging buffers) and the CUDA graphs that point into it; the geometry itself
// stays resident and the next call allocates again. solve_host and the device solve
// entry do this after a solve when less than a quarter of the device memory is free
// (or always, with the environment variable BIE_TRIM_WORKSPACE), so that many resident
// geometries solved in turn (a server's) do not keep a workspace each until the device
// runs out. The workspace is sized for the restart length: (restart + 1) N k doubles.
void geom_trim(bie_geom* g) {
    DeviceGuard dg(g->device);
    BIE_CK(cudaStreamSynchronize(g->stream));
    if (g->s_ls) BIE_CK(cudaStreamSynchronize(g->s_ls));  // block least-squares work in flight
    bie::Buf* ws[] = {&g->part, &g->bpack, &g->cpart, &g->V, &g->W, &g->R, &g->gv, &g->cs, &g->sn, &g->h, &g->h2,
                      &g->hn, &g->beta, &g->eps, &g->active, &g->jlast, &g->yv, &g->resid, &g->dpart, &g->rr,
                      &g->xo, &g->dd, &g->io_a, &g->io_b, &g->sol, &g->srcpack, &g->glist, &g->bv, &g->bq,
                      &g->bvj, &g->bh, &g->bgv, &g->btau, &g->br1, &g->br2, &g->br, &g->bh2, &g->bres, &g->bidx,
                      &g->bflag, &g->xa, &g->ra, &g->binv, &g->bpart, &g->btmp, &g->bwy};
    for (auto* b : ws) b->release();
    for (auto& c : g->gcache) {
        for (auto ex : c.exec)
            if (ex) cudaGraphExecDestroy(ex);
        c.exec.clear();
        c.sig = 0;
        c.warm = false;
    }
}

// The free-memory query runs only when the library allocated or released device memory
// since the last query that found enough free memory on this device (for at least this
// floor): cudaMemGetInfo can take milliseconds, and in steady state (the same solves
// again, buffers already sized) nothing the library holds has changed.
bool geom_trim_if_below(bie_geom* g, size_t free_floor) {
    DeviceGuard dg(g->device);
    bool trim = std::getenv("BIE_TRIM_WORKSPACE") != nullptr;
    if (!trim) {
        struct Verdict {
            uint64_t epoch = ~0ull;
            size_t floor = 0;
        };
        static std::mutex mu;
        static std::map<int, Verdict> ok;  // per device: last epoch and floor found clear
        const uint64_t ep = alloc_epoch();
        {
            std::lock_guard<std::mutex> lk(mu);
            auto it = ok.find(g->device);
            if (it != ok.end() && it->second.epoch == ep && free_floor <= it->second.floor) return false;
        }
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) {
            trim = fr < std::max(tot / 4, free_floor);
            if (!trim) {
                std::lock_guard<std::mutex> lk(mu);
                ok[g->device] = Verdict{ep, free_floor};
            }
        }
        cudaGetLastError();
    }
    if (trim) geom_trim(g);
    return trim;
}

void geom_trim_if_short(bie_geom* g) { geom_trim_if_below(g, 0); }

void geom_destroy(bie_geom* g) {
    {
        DeviceGuard dg(g->device);
        if (g->stream) cudaStreamSynchronize(g->stream);
        if (g->s_ls) cudaStreamSynchronize(g->s_ls);
        bie::Buf* all[] = {&g->x, &g->y, &g->z, &g->nx, &g->ny, &g->nz, &g->w, &g->diag, &g->pinv, &g->perm, &g->rowptr,
                           &g->col, &g->val, &g->part, &g->small, &g->bpack, &g->errflag, &g->cpart, &g->V, &g->W, &g->R, &g->gv, &g->cs, &g->sn,
                           &g->h, &g->h2, &g->hn, &g->beta, &g->eps, &g->active, &g->jlast, &g->yv, &g->resid,
                           &g->dpart, &g->rr, &g->xo, &g->dd, &g->io_a, &g->io_b, &g->sol, &g->srcpack, &g->glist,
                           &g->bv, &g->bq, &g->bvj, &g->bh, &g->bgv, &g->btau, &g->br1, &g->br2, &g->br, &g->bh2,
                           &g->bres, &g->bidx, &g->bflag, &g->xa, &g->ra, &g->binv, &g->bpart, &g->btmp, &g->bwy};
        for (auto* b : all) b->release();
        if (g->blas) cublasDestroy(g->blas);
        if (g->bres_host) cudaFreeHost(g->bres_host);
        if (g->ev_res) cudaEventDestroy(g->ev_res);
        if (g->ev_h) cudaEventDestroy(g->ev_h);
        if (g->s_ls) cudaStreamDestroy(g->s_ls);
        for (auto& r : g->prof_pending) {
            cudaEventDestroy(r.a);
            cudaEventDestroy(r.b);
        }
        for (auto e : g->ev_pool) cudaEventDestroy(e);
        for (auto& c : g->gcache)
            for (auto ex : c.exec)
                if (ex) cudaGraphExecDestroy(ex);
        if (g->ev0) cudaEventDestroy(g->ev0);
        if (g->ev1) cudaEventDestroy(g->ev1);
        if (g->stream) cudaStreamDestroy(g->stream);
    }
    delete g;
}

void geom_info(const bie_geom* g, int64_t* n, int64_t* nblocks, size_t* bytes) {
    if (n) *n = g->n;
    if (nblocks) *nblocks = g->nblocks;
    if (bytes) *bytes = g->geom_bytes;
}

void* geom_stream(bie_geom* g) { return (void*)g->stream; }

bool geom_near_values(bie_geom* g, double* val, int64_t len) {
    const int64_t want = g->nblocks * (int64_t)g->nb * g->nb;
    if (len != want) return false;
    if (want == 0) return true;
    DeviceGuard dg(g->device);
    BIE_CK(cudaMemcpyAsync(val, g->val.p, sizeof(double) * (size_t)want, cudaMemcpyDeviceToHost, g->stream));
    BIE_CK(cudaStreamSynchronize(g->stream));
    return true;
}

void profile_enable(bie_geom* g, int on) {
    DeviceGuard dg(g->device);
    prof_drain(g);
    if (on)
        for (auto& t : g->acc) t = bie_kernel_time{};
    g->prof_on = on != 0;
}

void profile_read(bie_geom* g, int kind, bie_kernel_time* out) {
    DeviceGuard dg(g->device);
    prof_drain(g);
    if (kind == BIE_KERNEL_KINDS) {
        bie_kernel_time t{};
        for (auto& a : g->acc) {
            t.ms += a.ms; t.launches += a.launches; t.pairs += a.pairs; t.pair_cols += a.pair_cols; t.bytes += a.bytes;
        }
        *out = t;
    } else {
        *out = g->acc[kind];
    }
}

// ---------------------------------------------------------------------------
// operators
// ---------------------------------------------------------------------------
void matvec_device(bie_geom* g, const double* dX, double* dY, int k, int precision, uint32_t flags, cudaStream_t s) {
    check_prec(precision);
    DeviceGuard dg(g->device);
    if (!s) s = g->stream;
    apply_op(g, dX, dY, k, precision, flags, nullptr, s);
}

void matvec_host(bie_geom* g, const double* X, double* Y, int k, int precision, uint32_t flags) {
    check_prec(precision);
    DeviceGuard dg(g->device);
    cudaStream_t s = g->stream;
    const int64_t nk = g->n * (int64_t)k;
    g->io_a.ensure(sizeof(double) * nk);
    g->io_b.ensure(sizeof(double) * nk);
    g->xo.ensure(sizeof(double) * nk);
    BIE_CK(cudaMemcpyAsync(g->io_a.p, X, sizeof(double) * nk, cudaMemcpyHostToDevice, s));
    {
        Prof pf(g, BIE_KERNEL_OTHER, s);
        k_colmajor_to_nodemajor<<<grid1(nk), 256, 0, s>>>(g->io_a.as<double>(), g->n, k, g->io_b.as<double>());
    }
    apply_op(g, g->io_b.as<double>(), g->xo.as<double>(), k, precision, flags, nullptr, s);
    {
        Prof pf(g, BIE_KERNEL_OTHER, s);
        k_nodemajor_to_colmajor<<<grid1(nk), 256, 0, s>>>(g->xo.as<double>(), g->n, k, g->io_a.as<double>());
    }
    BIE_CK(cudaGetLastError());
    BIE_CK(cudaMemcpyAsync(Y, g->io_a.p, sizeof(double) * nk, cudaMemcpyDeviceToHost, s));
    BIE_CK(cudaStreamSynchronize(s));
    check_device_error(g, s);
}

void rhs_point_device(bie_geom* g, const double* src, const double* q, const double* eps, int k, double* F,
                      cudaStream_t s) {
    DeviceGuard dg(g->device);
    if (!s) s = g->stream;
    {
        Prof pf(g, BIE_KERNEL_OTHER, s);
        k_rhs_point<<<grid1(g->n * k), 256, 0, s>>>(gdev(g), src, q, eps, k, F);
    }
    BIE_CK(cudaGetLastError());
}

void rhs_point_host(bie_geom* g, const double* src, const double* q, const double* eps, int k, double* F) {
    DeviceGuard dg(g->device);
    cudaStream_t s = g->stream;
    std::vector<double> packed((size_t)5 * k);
    std::copy(src, src + 3 * k, packed.begin());
    std::copy(q, q + k, packed.begin() + 3 * k);
    std::copy(eps, eps + k, packed.begin() + 4 * k);
    upload(g->small, packed.data(), packed.size(), s);
    const int64_t nk = g->n * (int64_t)k;
    g->io_a.ensure(sizeof(double) * nk);
    g->io_b.ensure(sizeof(double) * nk);
    const double* d = g->small.as<double>();
    {
        Prof pf(g, BIE_KERNEL_OTHER, s);
        k_rhs_point<<<grid1(nk), 256, 0, s>>>(gdev(g), d, d + 3 * k, d + 4 * k, k, g->io_b.as<double>());
    }
    {
        Prof pf(g, BIE_KERNEL_OTHER, s);
        k_nodemajor_to_colmajor<<<grid1(nk), 256, 0, s>>>(g->io_b.as<double>(), g->n, k, g->io_a.as<double>());
    }
    BIE_CK(cudaGetLastError());
    BIE_CK(cudaMemcpyAsync(F, g->io_a.p, sizeof(double) * nk, cudaMemcpyDeviceToHost, s));
    BIE_CK(cudaStreamSynchronize(s));
}

void potential_device(bie_geom* g, const double* S, int k, const double* T, int64_t M, double* phi, cudaStream_t s) {
    DeviceGuard dg(g->device);
    if (!s) s = g->stream;
    if (M == 0) return;
    Split sp = direct_sum(g, Kern::POT64, S, k, k, nullptr, T, M, s);
    {
        Prof pf(g, BIE_KERNEL_OTHER, s);
        k_reduce_parts<<<grid1(M * k), 256, 0, s>>>(g->part.as<double>(), sp.nsplit, M, k, kInv4Pi, phi);
    }
    BIE_CK(cudaGetLastError());
}

void potential_host(bie_geom* g, const double* S, int k, const double* T, int64_t M, double* phi) {
    DeviceGuard dg(g->device);
    cudaStream_t s = g->stream;
    if (M == 0) return;
    const int64_t nk = g->n * (int64_t)k;
    g->io_a.ensure(sizeof(double) * std::max<int64_t>(nk, M * k));
    g->io_b.ensure(sizeof(double) * nk);
    g->xo.ensure(sizeof(double) * M * k);
    upload(g->small, T, (size_t)3 * M, s);
    BIE_CK(cudaMemcpyAsync(g->io_a.p, S, sizeof(double) * nk, cudaMemcpyHostToDevice, s));
    {
        Prof pf(g, BIE_KERNEL_OTHER, s);
        k_colmajor_to_nodemajor<<<grid1(nk), 256, 0, s>>>(g->io_a.as<double>(), g->n, k, g->io_b.as<double>());
    }
    potential_device(g, g->io_b.as<double>(), k, g->small.as<double>(), M, g->xo.as<double>(), s);
    {
        Prof pf(g, BIE_KERNEL_OTHER, s);
        k_nodemajor_to_colmajor<<<grid1(M * k), 256, 0, s>>>(g->xo.as<double>(), M, k, g->io_a.as<double>());
    }
    BIE_CK(cudaGetLastError());
    BIE_CK(cudaMemcpyAsync(phi, g->io_a.p, sizeof(double) * M * k, cudaMemcpyDeviceToHost, s));
    BIE_CK(cudaStreamSynchronize(s));
}

void energy_host(bie_geom* g, const double* S, int k, const double* src, const double* q, double* W) {
    std::vector<double> phi((size_t)k * k);
    potential_host(g, S, k, src, k, phi.data());
    for (int c = 0; c < k; ++c) W[c] = 0.5 * q[c] * phi[(size_t)c * k + c];  // column c at target c
}

// ---------------------------------------------------------------------------
// solvers
// ---------------------------------------------------------------------------
int solve_device(bie_geom* g, const double* dF, double* dX, int k, const bie_solve_opts& o, bie_stats* st,
                 cudaStream_t s) {
    check_prec(o.precision);
    if (o.itmax < 1 || o.restart < 1 || !(o.rtol >= 0) || !(o.atol >= 0)) throw Error(BIE_EINVAL, "bad solver options");
    if (k > 256) throw Error(BIE_EUNSUPPORTED, "at most 256 right-hand sides per solve");
    DeviceGuard dg(g->device);
    if (!s) s = g->stream;
    const int64_t n = g->n, nk = n * (int64_t)k;
    const double* pre = o.precondition ? g->pinv.as<double>() : nullptr;
    BIE_CK(cudaEventRecord(g->ev0, s));
    // ||F_c|| and the per-column tolerance atol + rtol ||F_c|| (Krylov.jl stopping rule)
    g->small.ensure(sizeof(double) * (size_t)std::max(2 * k, 8));
    col_norms(g, dF, k, g->small.as<double>(), s);
    std::vector<double> fn(k), tol(k);
    d2h(fn.data(), g->small.p, k, s);
    for (int c = 0; c < k; ++c) tol[c] = o.atol + o.rtol * fn[c];
    std::vector<char> act(k, 1);
    int iters = 0, outer = 0, f64mv = 0, lpmv = 0;
    bool converged = false;
    std::vector<int> col_it(k, 0);
    std::vector<double> rel(k, 0.0);
    bool have_true_resid = false;
    g->rr.ensure(sizeof(double) * nk);
    g->dd.ensure(sizeof(double) * nk);
    g->xo.ensure(sizeof(double) * nk);
    double* rbuf = g->xo.as<double>();  // outer residual F - A x
    if (o.precision == BIE_FP64) {
        GmresResult r = use_block(o, k)
                            ? bgmres(g, dF, dX, k, BIE_FP64, o.flags, pre, tol, act, o.itmax, o.restart, s)
                            : gmres(g, dF, dX, k, BIE_FP64, o.flags, pre, tol, act, o.itmax, o.restart, o.check_every, s);
        iters = r.iters;
        outer = 1;
        f64mv = r.matvecs;
        converged = r.all_converged;
        col_it = r.col_iters;
    } else {
        BIE_CK(cudaMemsetAsync(dX, 0, sizeof(double) * nk, s));
        // FP64 iterative refinement. The residual r = F - A x is kept in FP64. After a
        // correction d it is refreshed either with the full FP64 operator
        // (r = F - A64 x) or, once the residual is small, updated with the
        // reduced-precision operator (r -= A_low d): that update errs by about
        // delta * ||A d|| ~ delta * ||r||, delta being the operator's relative error,
        // which is admitted only while it stays below half the tolerance.
        // Candidate operators for the residual update, cheapest first.
        const bool tc_ok = use_tc(o.precision == BIE_BF16X6 ? BIE_BF16X6 : BIE_BF16X3, k);
        struct Upd { int prec; double delta; };
        std::vector<Upd> upd;
        if (o.precision == BIE_BF16X3 && tc_ok) upd.push_back({BIE_BF16X3, kDeltaBF16X3});
        if ((o.precision == BIE_BF16X3 || o.precision == BIE_BF16X6) && tc_ok) upd.push_back({BIE_BF16X6, kDeltaBF16X6});
        upd.push_back({BIE_FP32, kDeltaFP32});
        std::vector<double> rn = fn, eps_in(k);
        const double inner_delta = (o.precision == BIE_BF16X3 && tc_ok)   ? kDeltaBF16X3
                                   : (o.precision == BIE_BF16X6 && tc_ok) ? kDeltaBF16X6
                                                                          : kDeltaFP32;
        BIE_CK(cudaMemcpyAsync(rbuf, dF, sizeof(double) * nk, cudaMemcpyDeviceToDevice, s));
        have_true_resid = true;
        for (int it_out = 0;; ++it_out) {
            int nact = 0;
            int upd_prec = BIE_FP64;  // cheapest admissible reduced-precision update, else FP64
            double worst = 0.0;       // max over active columns of ||r_c|| / tol_c
            for (int c = 0; c < k; ++c) {
                act[c] = rn[c] > tol[c] ? 1 : 0;
                nact += act[c];
                rel[c] = fn[c] > 0 ? rn[c] / fn[c] : 0.0;
                if (act[c]) worst = std::max(worst, rn[c] / tol[c]);
            }
            for (const Upd& u : upd)
                if (u.delta * worst <= 0.5) {
                    upd_prec = u.prec;
                    break;
                }
            if (std::getenv("BIE_TRACE")) {
                double mx = 0.0;
                for (int c = 0; c < k; ++c) mx = std::max(mx, rel[c]);
                std::fprintf(stderr, "[bie] outer %d: active %d, max |r|/|F| %.3e, worst |r|/tol %.3e, update %d\n",
                             it_out, nact, mx, worst, upd_prec);
            }
            if (nact == 0) {
                converged = true;
                break;
            }
            if (it_out >= o.max_outer || iters >= o.itmax) break;
            // inner tolerance: inner_rtol |r|, but not below half the outer tolerance nor
            // below twice the inner operator's own relative error (iterating past that
            // cannot lower the true residual of this pass)
            for (int c = 0; c < k; ++c)
                eps_in[c] = std::max({o.inner_rtol * rn[c], 0.5 * tol[c], 2.0 * inner_delta * rn[c]});
            // GMRES returns the updated residual r - A_low d itself (from its Arnoldi relation)
            // when A_low is its own operator
            GmresResult r = use_block(o, k)
                                ? bgmres(g, rbuf, g->dd.as<double>(), k, o.precision, o.flags, pre, eps_in, act,
                                         o.itmax - iters, o.restart, s, upd_prec != BIE_FP64 ? rbuf : nullptr,
                                         upd_prec)
                                : gmres(g, rbuf, g->dd.as<double>(), k, o.precision, o.flags, pre, eps_in, act,
                                        o.itmax - iters, o.restart, o.check_every, s,
                                        upd_prec != BIE_FP64 ? rbuf : nullptr, upd_prec);
            iters += r.iters;
            lpmv += r.matvecs;
            for (int c = 0; c < k; ++c) col_it[c] += r.col_iters[c];
            upload(g->active, std::vector<int>(act.begin(), act.end()).data(), k, s);
            {
                Prof pf(g, BIE_KERNEL_KRYLOV, s);
                k_axpby<<<grid1(nk), 256, 0, s>>>(1.0, g->dd.as<double>(), 1.0, dX, n, k, g->active.as<int>());
            }
            BIE_CK(cudaGetLastError());
            ++outer;
            if (upd_prec != BIE_FP64) {
                // r -= A_low d  (d = 0 in the frozen columns), unless GMRES returned it
                if (!r.resid_written) {
                    apply_op(g, g->dd.as<double>(), g->rr.as<double>(), k, upd_prec, o.flags, nullptr, s);
                    ++lpmv;
                    Prof pf(g, BIE_KERNEL_KRYLOV, s);
                    k_axpby<<<grid1(nk), 256, 0, s>>>(-1.0, g->rr.as<double>(), 1.0, rbuf, n, k, nullptr);
                }
                have_true_resid = false;
            } else {
                // r = F - A64 x
                apply_op(g, dX, rbuf, k, BIE_FP64, o.flags, nullptr, s);
                ++f64mv;
                Prof pf(g, BIE_KERNEL_KRYLOV, s);
                k_axpby<<<grid1(nk), 256, 0, s>>>(1.0, dF, -1.0, rbuf, n, k, nullptr);
                have_true_resid = true;
            }
            col_norms(g, rbuf, k, g->small.as<double>(), s);
            d2h(rn.data(), g->small.p, k, s);
        }
    }
    const bool verify = !(o.flags & 4u) && (st != nullptr);
    if (verify && !have_true_resid) {
        apply_op(g, dX, rbuf, k, BIE_FP64, o.flags, nullptr, s);
        ++f64mv;
        {
            Prof pf(g, BIE_KERNEL_KRYLOV, s);
            k_axpby<<<grid1(nk), 256, 0, s>>>(1.0, dF, -1.0, rbuf, n, k, nullptr);
        }
        std::vector<double> rn(k);
        col_norms(g, rbuf, k, g->small.as<double>(), s);
        d2h(rn.data(), g->small.p, k, s);
        bool all = true;
        for (int c = 0; c < k; ++c) {
            rel[c] = fn[c] > 0 ? rn[c] / fn[c] : 0.0;
            all = all && rn[c] <= tol[c] * (1.0 + 1e-6) + 1e-300;
        }
        if (o.precision == BIE_FP64) converged = converged && all;
    }
    BIE_CK(cudaEventRecord(g->ev1, s));
    BIE_CK(cudaEventSynchronize(g->ev1));
    check_device_error(g, s);
    float ms = 0.f;
    BIE_CK(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
    if (st) {
        st->iterations = iters;
        st->outer = outer;
        st->fp64_matvecs = f64mv;
        st->lowp_matvecs = lpmv;
        st->converged = converged ? 1 : 0;
        double mx = 0.0;
        for (int c = 0; c < k; ++c) mx = std::max(mx, rel[c]);
        st->max_rel_resid = mx;
        st->seconds = ms * 1e-3;
        if (st->col_iterations)
            for (int c = 0; c < k; ++c) st->col_iterations[c] = col_it[c];
        if (st->col_resid)
            for (int c = 0; c < k; ++c) st->col_resid[c] = rel[c];
    }
    return converged ? BIE_OK : BIE_ENOCONV;
}

// Right-hand sides of k point sources built on the device (rhs_dielectric_box3d,
// src/solver/dielectric_box3d.jl:95-104) and solved there (solve_dielectric_box3d_block,
// src/solver/multi_rhs.jl:270-286): only the 5 k source values go to the device and only
// Sigma comes back, so F never crosses the host link.
int solve_point_host(bie_geom* g, const double* src, const double* q, const double* eps, int k, double* Sigma,
                     const bie_solve_opts& o, bie_stats* st) {
    DeviceGuard dg(g->device);
    cudaStream_t s = g->stream;
    std::vector<double> packed((size_t)5 * k);
    std::copy(src, src + 3 * k, packed.begin());
    std::copy(q, q + k, packed.begin() + 3 * k);
    std::copy(eps, eps + k, packed.begin() + 4 * k);
    upload(g->srcpack, packed.data(), packed.size(), s);
    const int64_t nk = g->n * (int64_t)k;
    g->io_a.ensure(sizeof(double) * nk);
    g->io_b.ensure(sizeof(double) * nk);
    g->sol.ensure(sizeof(double) * nk);
    const double* d = g->srcpack.as<double>();
    {
        Prof pf(g, BIE_KERNEL_OTHER, s);
        k_rhs_point<<<grid1(nk), 256, 0, s>>>(gdev(g), d, d + 3 * k, d + 4 * k, k, g->io_b.as<double>());
    }
    BIE_CK(cudaGetLastError());
    int rc = solve_device(g, g->io_b.as<double>(), g->sol.as<double>(), k, o, st, s);
    {
        Prof pf(g, BIE_KERNEL_OTHER, s);
        k_nodemajor_to_colmajor<<<grid1(nk), 256, 0, s>>>(g->sol.as<double>(), g->n, k, g->io_a.as<double>());
    }
    BIE_CK(cudaGetLastError());
    BIE_CK(cudaMemcpyAsync(Sigma, g->io_a.p, sizeof(double) * nk, cudaMemcpyDeviceToHost, s));
    BIE_CK(cudaStreamSynchronize(s));
    geom_trim_if_short(g);
    return rc;
}

int solve_host(bie_geom* g, const double* F, double* Sigma, int k, const bie_solve_opts& o, bie_stats* st) {
    DeviceGuard dg(g->device);
    cudaStream_t s = g->stream;
    const int64_t nk = g->n * (int64_t)k;
    g->io_a.ensure(sizeof(double) * nk);
    g->io_b.ensure(sizeof(double) * nk);
    g->sol.ensure(sizeof(double) * nk);  // output buffer, never aliased by the solver's scratch
    BIE_CK(cudaMemcpyAsync(g->io_a.p, F, sizeof(double) * nk, cudaMemcpyHostToDevice, s));
    {
        Prof pf(g, BIE_KERNEL_OTHER, s);
        k_colmajor_to_nodemajor<<<grid1(nk), 256, 0, s>>>(g->io_a.as<double>(), g->n, k, g->io_b.as<double>());
    }
    int rc = solve_device(g, g->io_b.as<double>(), g->sol.as<double>(), k, o, st, s);
    {
        Prof pf(g, BIE_KERNEL_OTHER, s);
        k_nodemajor_to_colmajor<<<grid1(nk), 256, 0, s>>>(g->sol.as<double>(), g->n, k, g->io_a.as<double>());
    }
    BIE_CK(cudaGetLastError());
    BIE_CK(cudaMemcpyAsync(Sigma, g->io_a.p, sizeof(double) * nk, cudaMemcpyDeviceToHost, s));
    BIE_CK(cudaStreamSynchronize(s));
    geom_trim_if_short(g);
    return rc;
}


// ---------------------------------------------------------------------------
// Group solves: the block solves of several geometries in lockstep. Every
// reduced-precision operator application of the group is one work-list launch of the
// tensor-core direct sum over all members' (target tile, source split) items, followed by
// each member's correction apply; the Krylov kernels and host checks of all members are
// issued together on one stream, so a group of small geometries pays one set of
// per-iteration host round trips instead of one per geometry. The arithmetic of each
// member is that of its own solve (FP64 refinement around the split-BF16 operator, FP64
// Krylov), so each result matches the member solved alone within the refined tolerance.
// ---------------------------------------------------------------------------
namespace {

struct Member {
    bie_geom* g = nullptr;
    const double* dF = nullptr;  // node-major n x k
    double* dX = nullptr;
    int k = 0;
    int idx = 0;  // position in the caller's arrays
    // refinement
    std::vector<double> fn, tol, rn, eps_in, rel;
    std::vector<char> act;
    std::vector<int> col_it;
    int iters = 0, outer = 0, f64mv = 0, lpmv = 0;
    bool converged = false, have_true_resid = true;
    int upd_prec = BIE_FP64;
    // inner GMRES of the current refinement step
    double* dr = nullptr;        // right-hand side of the inner solve (the outer residual)
    double* dx = nullptr;        // its solution
    std::vector<char> in_act;    // columns the inner solve works on
    bool cycle = false;          // iterates in the current Arnoldi cycle
    bool done = false;           // inner solve finished (all columns converged or itmax)
    bool want_resid = false;     // the inner solve leaves r - A_low d in dr (its own operator)
    bool resid_written = false;
    int it = 0;                  // inner iterations
    std::vector<int> gact, jl;
    std::vector<double> hb;
};

// Y_m = A_low(X_m) for every member m (split-BF16, pieces 2 or 3): one K3 work-list launch,
// then each member's corrections and diagonal (combine).
void group_apply_tc(const std::vector<Member*>& ms, const std::vector<const double*>& X, const std::vector<double*>& Y,
                    int pieces, uint32_t flags, cudaStream_t s) {
    if (ms.empty()) return;
    std::vector<TcMember> tm;
    std::vector<Split> sp(ms.size());
    int64_t nitems = 0;
    for (size_t i = 0; i < ms.size(); ++i) {
        bie_geom* g = ms[i]->g;
        const int k = ms[i]->k;
        sp[i] = tc_split(g, k, pieces);
        g->part.ensure(sizeof(float) * (size_t)sp[i].nsplit * g->n * k);
        g->bpack.ensure(block_tc_pack_bytes(g->n, k, pieces));
        tm.push_back(TcMember{gdev(g), X[i], k, 0, k, nullptr, sp[i].nsplit, sp[i].chunk, g->part.as<float>(), k,
                              g->bpack.as<uint8_t>()});
        nitems += ((g->n + kTcTileM - 1) / kTcTileM) * sp[i].nsplit;
    }
    bie_geom* lead = ms.front()->g;
    const size_t need = block_tc_list_bytes((int)ms.size(), nitems);
    lead->glist.ensure(need);
    launch_block_tc_list(tm, pieces, lead->errflag.as<int>(), lead->glist.p, lead->glist.bytes, s);
    for (size_t i = 0; i < ms.size(); ++i) {
        bie_geom* g = ms[i]->g;
        const bool corr = g->nblocks > 0 && !(flags & BIE_NO_CORRECTIONS);
        const bool dg = !(flags & BIE_NO_DIAG);
        combine(g, g->part.as<float>(), sp[i].nsplit, X[i], Y[i], ms[i]->k, nullptr, corr, dg, s);
    }
}

// Copies k values of each member's device array to the host with one synchronisation.
template <class T, class Get>
void group_d2h(const std::vector<Member*>& ms, Get get, cudaStream_t s) {
    for (Member* m : ms) {
        std::pair<T*, const void*> p = get(m);
        BIE_CK(cudaMemcpyAsync(p.first, p.second, sizeof(T) * m->k, cudaMemcpyDeviceToHost, s));
    }
    BIE_CK(cudaStreamSynchronize(s));
}

// The inner solve of one refinement step for every member (restarted GMRES, one classical
// Gram-Schmidt pass: the reduced-precision inner solves stop near 1e-6 and the outer loop
// recomputes the residual), members in lockstep. Mirrors gmres() without graphs.
void group_gmres(const std::vector<Member*>& all, int pieces, uint32_t flags, int itmax, int m, int check_every,
                 cudaStream_t s) {
    m = std::max(1, std::min(m, itmax));
    const int m1 = m + 1;
    for (Member* M : all) {
        bie_geom* g = M->g;
        const int64_t nk = g->n * (int64_t)M->k;
        const int k = M->k;
        g->V.ensure(sizeof(double) * (size_t)m1 * nk);
        g->W.ensure(sizeof(double) * nk);
        g->rr.ensure(sizeof(double) * nk);
        g->R.ensure(sizeof(double) * (size_t)m1 * m1 * k);
        g->gv.ensure(sizeof(double) * (size_t)m1 * k);
        g->cs.ensure(sizeof(double) * (size_t)m1 * k);
        g->sn.ensure(sizeof(double) * (size_t)m1 * k);
        g->h.ensure(sizeof(double) * (size_t)m1 * k);
        g->hn.ensure(sizeof(double) * k);
        g->beta.ensure(sizeof(double) * k);
        g->eps.ensure(sizeof(double) * k);
        g->active.ensure(sizeof(int) * k);
        g->jlast.ensure(sizeof(int) * k);
        g->yv.ensure(sizeof(double) * (size_t)m1 * k);
        g->resid.ensure(sizeof(double) * k);
        size_t need = 0;
        for (int nv = 1; nv <= m1; ++nv) {
            const DotPlan p = dot_plan(g->n, k, nv);
            need = std::max(need, (size_t)p.nblk * nv * k);
        }
        g->dpart.ensure(sizeof(double) * need);
        BIE_CK(cudaMemsetAsync(M->dx, 0, sizeof(double) * nk, s));
        upload(g->eps, M->eps_in.data(), k, s);
        M->it = 0;
        M->done = false;
        M->gact.assign(k, 0);
        M->jl.assign(k, 0);
        M->hb.assign(k, 0.0);
    }
    bool first = true;
    for (;;) {
        // residual of the cycle: the right-hand side, or after a restart the true residual
        // of the current iterate
        std::vector<Member*> live;
        for (Member* M : all)
            if (!M->done) live.push_back(M);
        if (live.empty()) break;
        if (!first) {
            std::vector<const double*> X;
            std::vector<double*> Y;
            for (Member* M : live) {
                X.push_back(M->dx);
                Y.push_back(M->g->W.as<double>());
            }
            group_apply_tc(live, X, Y, pieces, flags, s);
            for (Member* M : live) {
                bie_geom* g = M->g;
                const int64_t nk = g->n * (int64_t)M->k;
                M->lpmv += 1;
                BIE_CK(cudaMemcpyAsync(g->rr.p, M->dr, sizeof(double) * nk, cudaMemcpyDeviceToDevice, s));
                k_axpby<<<grid1(nk), 256, 0, s>>>(-1.0, g->W.as<double>(), 1.0, g->rr.as<double>(), g->n, M->k,
                                                  nullptr);
            }
        }
        for (Member* M : live) col_norms(M->g, first ? M->dr : M->g->rr.as<double>(), M->k, M->g->beta.as<double>(), s);
        group_d2h<double>(live, [](Member* M) { return std::make_pair(M->hb.data(), (const void*)M->g->beta.p); }, s);
        std::vector<Member*> run;
        for (Member* M : live) {
            int nact = 0;
            for (int c = 0; c < M->k; ++c) {
                M->gact[c] = M->in_act[c] && M->hb[c] > M->eps_in[c] ? 1 : 0;
                nact += M->gact[c];
            }
            if (nact == 0 || M->it >= itmax) {
                M->done = true;
                if (M->want_resid) {  // nothing solved since the cycle's residual was formed
                    if (!first)
                        BIE_CK(cudaMemcpyAsync(M->dr, M->g->rr.p,
                                               sizeof(double) * M->g->n * (size_t)M->k, cudaMemcpyDeviceToDevice, s));
                    M->resid_written = true;
                }
                continue;
            }
            bie_geom* g = M->g;
            const int k = M->k;
            const int64_t nk = g->n * (int64_t)k;
            upload(g->active, M->gact.data(), k, s);
            BIE_CK(cudaMemsetAsync(g->jlast.p, 0, sizeof(int) * k, s));
            BIE_CK(cudaMemsetAsync(g->gv.p, 0, sizeof(double) * m1 * k, s));
            BIE_CK(cudaMemcpyAsync(g->gv.p, g->beta.p, sizeof(double) * k, cudaMemcpyDeviceToDevice, s));
            k_scale_cols<<<grid1(nk), 256, 0, s>>>(first ? M->dr : g->rr.as<double>(), g->beta.as<double>(), g->n, k,
                                                   g->V.as<double>());
            M->cycle = true;
            run.push_back(M);
        }
        if (run.empty()) break;
        for (int j = 0; j < m && !run.empty(); ++j) {
            std::vector<const double*> X;
            std::vector<double*> Y;
            for (Member* M : run) {
                const int64_t nk = M->g->n * (int64_t)M->k;
                X.push_back(M->g->V.as<double>() + (size_t)j * nk);
                Y.push_back(M->g->W.as<double>());
            }
            group_apply_tc(run, X, Y, pieces, flags, s);
            for (Member* M : run) {
                bie_geom* g = M->g;
                const int k = M->k;
                const int64_t nk = g->n * (int64_t)k;
                double* V = g->V.as<double>();
                double* W = g->W.as<double>();
                dots(g, V, nk, j + 1, W, k, g->h.as<double>(), 0, s);
                gs_update_norm(g, W, V, nk, j + 1, g->h.as<double>(), k, g->hn.as<double>(), s);
                k_scale_cols<<<grid1(nk), 256, 0, s>>>(W, g->hn.as<double>(), g->n, k, V + (size_t)(j + 1) * nk);
                k_givens<<<grid1(k, 64), 64, 0, s>>>(g->R.as<double>(), g->h.as<double>(), nullptr, g->hn.as<double>(),
                                                    g->cs.as<double>(), g->sn.as<double>(), g->gv.as<double>(),
                                                    g->active.as<int>(), g->jlast.as<int>(), g->eps.as<double>(),
                                                    g->resid.as<double>(), j, m1, k);
                BIE_CK(cudaGetLastError());
                M->lpmv += 1;
                M->it += 1;
            }
            if ((j + 1) % std::max(1, check_every) == 0 || j + 1 == m) {
                group_d2h<int>(run, [](Member* M) { return std::make_pair(M->gact.data(), (const void*)M->g->active.p); },
                               s);
                std::vector<Member*> still;
                for (Member* M : run) {
                    bool any = false;
                    for (int c = 0; c < M->k; ++c) any = any || M->gact[c];
                    if (any && M->it < itmax) still.push_back(M);
                }
                run.swap(still);
            }
        }
        // solution update of every member that iterated in this cycle
        std::vector<Member*> cyc;
        for (Member* M : live)
            if (M->cycle) cyc.push_back(M);
        for (Member* M : cyc) {
            bie_geom* g = M->g;
            const int k = M->k;
            const int64_t nk = g->n * (int64_t)k;
            k_backsolve<<<grid1(k, 64), 64, 0, s>>>(g->R.as<double>(), g->gv.as<double>(), g->jlast.as<int>(), m1, k,
                                                    g->yv.as<double>());
            k_update_solution<<<grid1(nk), 256, 0, s>>>(M->dx, g->V.as<double>(), nk, g->yv.as<double>(),
                                                        g->jlast.as<int>(), m, nullptr, g->n, k);
            BIE_CK(cudaGetLastError());
        }
        group_d2h<int>(cyc, [](Member* M) { return std::make_pair(M->jl.data(), (const void*)M->g->jlast.p); }, s);
        group_d2h<int>(cyc, [](Member* M) { return std::make_pair(M->gact.data(), (const void*)M->g->active.p); }, s);
        for (Member* M : cyc) {
            M->cycle = false;
            for (int c = 0; c < M->k; ++c) M->col_it[c] += M->jl[c];
            bool any = false;
            for (int c = 0; c < M->k; ++c) any = any || M->gact[c];
            if (!any || M->it >= itmax) {
                M->done = true;
                if (M->want_resid) {
                    // r - A_low d = V z from the Arnoldi relation (as in gmres), into dr
                    bie_geom* g = M->g;
                    const int64_t nk = g->n * (int64_t)M->k;
                    k_givens_resid<<<grid1(M->k, 64), 64, 0, s>>>(g->gv.as<double>(), g->cs.as<double>(),
                                                                  g->sn.as<double>(), g->jlast.as<int>(), m1, M->k,
                                                                  g->yv.as<double>());
                    k_basis_combine<<<grid1(nk), 256, 0, s>>>(M->dr, g->V.as<double>(), nk,
                                                              g->yv.as<double>(), g->jlast.as<int>(), g->n, M->k);
                    BIE_CK(cudaGetLastError());
                    M->resid_written = true;
                }
            }
        }
        first = false;
    }
}

}  // namespace

namespace {
void check_group(bie_geom* const* gs, int G, const int* ks) {
    if (G < 1) throw Error(BIE_EINVAL, "empty group");
    for (int i = 0; i < G; ++i) {
        if (!gs[i] || ks[i] < 1 || ks[i] > 128) throw Error(BIE_EINVAL, "group member needs 1..128 columns");
        for (int j = 0; j < i; ++j)
            if (gs[j] == gs[i]) throw Error(BIE_EINVAL, "a geometry appears twice in a group");
        if (gs[i]->device != gs[0]->device) throw Error(BIE_EINVAL, "group members on different devices");
    }
}
}  // namespace

void matvec_group_device(bie_geom* const* gs, int G, const double* const* dX, double* const* dY, const int* ks,
                         int prec, uint32_t flags, cudaStream_t s) {
    check_prec(prec);
    if (prec != BIE_BF16X3 && prec != BIE_BF16X6)
        throw Error(BIE_EUNSUPPORTED, "group operator applications run the split-BF16 precisions");
    check_group(gs, G, ks);
    DeviceGuard dg(gs[0]->device);
    if (!s) s = gs[0]->stream;
    for (int i = 0; i < G; ++i)
        if (gs[i]->stream != s) BIE_CK(cudaStreamSynchronize(gs[i]->stream));
    std::vector<Member> mem(G);
    std::vector<Member*> ms;
    std::vector<const double*> X;
    std::vector<double*> Y;
    for (int i = 0; i < G; ++i) {
        mem[i].g = gs[i];
        mem[i].k = ks[i];
        ms.push_back(&mem[i]);
    }
    std::stable_sort(ms.begin(), ms.end(), [](const Member* a, const Member* b) { return a->g->n > b->g->n; });
    for (Member* M : ms) {
        const int i = (int)(M - mem.data());
        X.push_back(dX[i]);
        Y.push_back(dY[i]);
    }
    group_apply_tc(ms, X, Y, prec == BIE_BF16X6 ? 3 : 2, flags, s);
    for (Member* M : ms) check_device_error(M->g, s);
}

int solve_group(bie_geom* const* gs, int G, const double* const* dF, double* const* dX, const int* ks,
                const bie_solve_opts& o, bie_stats* st, cudaStream_t s) {
    check_prec(o.precision);
    if (o.precision != BIE_BF16X3 && o.precision != BIE_BF16X6)
        throw Error(BIE_EUNSUPPORTED, "group solves run the split-BF16 precisions");
    if (o.precondition) throw Error(BIE_EUNSUPPORTED, "group solves run without the diagonal preconditioner");
    if (o.itmax < 1 || o.restart < 1 || !(o.rtol >= 0) || !(o.atol >= 0)) throw Error(BIE_EINVAL, "bad solver options");
    check_group(gs, G, ks);
    DeviceGuard dg(gs[0]->device);
    if (!s) s = gs[0]->stream;
    // the members' own streams finish their work before the group's stream starts
    for (int i = 0; i < G; ++i)
        if (gs[i]->stream != s) BIE_CK(cudaStreamSynchronize(gs[i]->stream));
    const int pieces = o.precision == BIE_BF16X6 ? 3 : 2;
    const double inner_delta = pieces == 3 ? kDeltaBF16X6 : kDeltaBF16X3;
    std::vector<Member> mem(G);
    std::vector<Member*> ms;
    for (int i = 0; i < G; ++i) {
        Member& M = mem[i];
        M.g = gs[i];
        M.dF = dF[i];
        M.dX = dX[i];
        M.k = ks[i];
        M.idx = i;
        ms.push_back(&M);
    }
    // largest members first: their items lead the work list
    std::stable_sort(ms.begin(), ms.end(), [](const Member* a, const Member* b) { return a->g->n > b->g->n; });
    BIE_CK(cudaEventRecord(ms.front()->g->ev0, s));
    for (Member* M : ms) {
        bie_geom* g = M->g;
        const int k = M->k;
        const int64_t nk = g->n * (int64_t)k;
        g->small.ensure(sizeof(double) * (size_t)std::max(2 * k, 8));
        col_norms(g, M->dF, k, g->small.as<double>(), s);
        g->rr.ensure(sizeof(double) * nk);
        g->dd.ensure(sizeof(double) * nk);
        g->xo.ensure(sizeof(double) * nk);
        BIE_CK(cudaMemsetAsync(M->dX, 0, sizeof(double) * nk, s));
        BIE_CK(cudaMemcpyAsync(g->xo.p, M->dF, sizeof(double) * nk, cudaMemcpyDeviceToDevice, s));
        M->fn.assign(k, 0.0);
        M->col_it.assign(k, 0);
        M->rel.assign(k, 0.0);
        M->act.assign(k, 1);
        M->eps_in.assign(k, 0.0);
        M->in_act.assign(k, 1);
    }
    group_d2h<double>(ms, [](Member* M) { return std::make_pair(M->fn.data(), (const void*)M->g->small.p); }, s);
    for (Member* M : ms) {
        M->tol.resize(M->k);
        for (int c = 0; c < M->k; ++c) M->tol[c] = o.atol + o.rtol * M->fn[c];
        M->rn = M->fn;
    }
    struct Upd { int prec; double delta; };
    std::vector<Upd> upd;
    if (o.precision == BIE_BF16X3) upd.push_back({BIE_BF16X3, kDeltaBF16X3});
    upd.push_back({BIE_BF16X6, kDeltaBF16X6});
    for (int it_out = 0;; ++it_out) {
        std::vector<Member*> act;
        for (Member* M : ms) {
            int nact = 0;
            double worst = 0.0;
            for (int c = 0; c < M->k; ++c) {
                M->act[c] = M->rn[c] > M->tol[c] ? 1 : 0;
                nact += M->act[c];
                M->rel[c] = M->fn[c] > 0 ? M->rn[c] / M->fn[c] : 0.0;
                if (M->act[c]) worst = std::max(worst, M->rn[c] / M->tol[c]);
            }
            if (nact == 0) {
                M->converged = true;
                continue;
            }
            if (it_out >= o.max_outer || M->iters >= o.itmax) continue;
            M->upd_prec = BIE_FP64;
            for (const Upd& u : upd)
                if (u.delta * worst <= 0.5) {
                    M->upd_prec = u.prec;
                    break;
                }
            for (int c = 0; c < M->k; ++c)
                M->eps_in[c] = std::max({o.inner_rtol * M->rn[c], 0.5 * M->tol[c], 2.0 * inner_delta * M->rn[c]});
            M->in_act = M->act;
            M->dr = M->g->xo.as<double>();
            M->dx = M->g->dd.as<double>();
            M->want_resid = (M->upd_prec == BIE_BF16X3 && pieces == 2) || (M->upd_prec == BIE_BF16X6 && pieces == 3);
            M->resid_written = false;
            act.push_back(M);
        }
        if (act.empty()) break;
        int budget = o.itmax;
        for (Member* M : act) budget = std::min(budget, o.itmax - M->iters);
        group_gmres(act, pieces, o.flags, std::max(1, budget), o.restart, o.check_every, s);
        // x += d, then the residual update: reduced precision (one work-list launch per
        // precision) or the FP64 operator
        std::vector<Member*> low[4];
        for (Member* M : act) {
            bie_geom* g = M->g;
            const int k = M->k;
            const int64_t nk = g->n * (int64_t)k;
            M->iters += M->it;
            upload(g->active, std::vector<int>(M->act.begin(), M->act.end()).data(), k, s);
            k_axpby<<<grid1(nk), 256, 0, s>>>(1.0, g->dd.as<double>(), 1.0, M->dX, g->n, k, g->active.as<int>());
            BIE_CK(cudaGetLastError());
            M->outer += 1;
            if (M->upd_prec != BIE_FP64) {
                if (M->resid_written)
                    M->have_true_resid = false;  // the inner solve left r - A_low d in xo
                else
                    low[M->upd_prec].push_back(M);
            } else {
                apply_op(g, M->dX, g->xo.as<double>(), k, BIE_FP64, o.flags, nullptr, s);
                M->f64mv += 1;
                k_axpby<<<grid1(nk), 256, 0, s>>>(1.0, M->dF, -1.0, g->xo.as<double>(), g->n, k, nullptr);
                M->have_true_resid = true;
            }
        }
        for (int p : {BIE_BF16X3, BIE_BF16X6}) {
            if (low[p].empty()) continue;
            std::vector<const double*> X;
            std::vector<double*> Y;
            for (Member* M : low[p]) {
                X.push_back(M->g->dd.as<double>());
                Y.push_back(M->g->rr.as<double>());
            }
            group_apply_tc(low[p], X, Y, p == BIE_BF16X6 ? 3 : 2, o.flags, s);
            for (Member* M : low[p]) {
                bie_geom* g = M->g;
                const int64_t nk = g->n * (int64_t)M->k;
                M->lpmv += 1;
                k_axpby<<<grid1(nk), 256, 0, s>>>(-1.0, g->rr.as<double>(), 1.0, g->xo.as<double>(), g->n, M->k,
                                                  nullptr);
                M->have_true_resid = false;
            }
        }
        for (Member* M : act) col_norms(M->g, M->g->xo.as<double>(), M->k, M->g->small.as<double>(), s);
        group_d2h<double>(act, [](Member* M) { return std::make_pair(M->rn.data(), (const void*)M->g->small.p); }, s);
    }
    const bool verify = !(o.flags & 4u) && (st != nullptr);
    if (verify) {
        std::vector<Member*> vm;
        for (Member* M : ms)
            if (!M->have_true_resid) vm.push_back(M);
        for (Member* M : vm) {
            bie_geom* g = M->g;
            const int64_t nk = g->n * (int64_t)M->k;
            apply_op(g, M->dX, g->xo.as<double>(), M->k, BIE_FP64, o.flags, nullptr, s);
            M->f64mv += 1;
            k_axpby<<<grid1(nk), 256, 0, s>>>(1.0, M->dF, -1.0, g->xo.as<double>(), g->n, M->k, nullptr);
            col_norms(g, g->xo.as<double>(), M->k, g->small.as<double>(), s);
        }
        group_d2h<double>(vm, [](Member* M) { return std::make_pair(M->rn.data(), (const void*)M->g->small.p); }, s);
        for (Member* M : vm)
            for (int c = 0; c < M->k; ++c) M->rel[c] = M->fn[c] > 0 ? M->rn[c] / M->fn[c] : 0.0;
    }
    bie_geom* lead = ms.front()->g;
    BIE_CK(cudaEventRecord(lead->ev1, s));
    BIE_CK(cudaEventSynchronize(lead->ev1));
    float msec = 0.f;
    BIE_CK(cudaEventElapsedTime(&msec, lead->ev0, lead->ev1));
    bool all = true;
    for (Member* M : ms) {
        check_device_error(M->g, s);
        all = all && M->converged;
        if (!st) continue;
        bie_stats& t = st[M->idx];
        t.iterations = M->iters;
        t.outer = M->outer;
        t.fp64_matvecs = M->f64mv;
        t.lowp_matvecs = M->lpmv;
        t.converged = M->converged ? 1 : 0;
        double mx = 0.0;
        for (int c = 0; c < M->k; ++c) mx = std::max(mx, M->rel[c]);
        t.max_rel_resid = mx;
        t.seconds = msec * 1e-3;
        if (t.col_iterations)
            for (int c = 0; c < M->k; ++c) t.col_iterations[c] = M->col_it[c];
        if (t.col_resid)
            for (int c = 0; c < M->k; ++c) t.col_resid[c] = M->rel[c];
    }
    return all ? BIE_OK : BIE_ENOCONV;
}

int solve_group_point_host(bie_geom* const* gs, int G, const double* const* src, const double* const* q,
                           const double* const* eps, const int* ks, double* const* Sigma, const bie_solve_opts& o,
                           bie_stats* st) {
    check_group(gs, G, ks);
    DeviceGuard dg(gs[0]->device);
    cudaStream_t s = gs[0]->stream;
    std::vector<const double*> dF(G);
    std::vector<double*> dX(G);
    for (int i = 0; i < G; ++i) {
        bie_geom* g = gs[i];
        const int k = ks[i];
        const int64_t nk = g->n * (int64_t)k;
        if (g->stream != s) BIE_CK(cudaStreamSynchronize(g->stream));
        std::vector<double> packed((size_t)5 * k);
        std::copy(src[i], src[i] + 3 * k, packed.begin());
        std::copy(q[i], q[i] + k, packed.begin() + 3 * k);
        std::copy(eps[i], eps[i] + k, packed.begin() + 4 * k);
        upload(g->srcpack, packed.data(), packed.size(), s);
        g->io_a.ensure(sizeof(double) * nk);
        g->io_b.ensure(sizeof(double) * nk);
        g->sol.ensure(sizeof(double) * nk);
        const double* d = g->srcpack.as<double>();
        k_rhs_point<<<grid1(nk), 256, 0, s>>>(gdev(g), d, d + 3 * k, d + 4 * k, k, g->io_b.as<double>());
        BIE_CK(cudaGetLastError());
        dF[i] = g->io_b.as<double>();
        dX[i] = g->sol.as<double>();
    }
    const int rc = solve_group(gs, G, dF.data(), dX.data(), ks, o, st, s);
    for (int i = 0; i < G; ++i) {
        bie_geom* g = gs[i];
        const int64_t nk = g->n * (int64_t)ks[i];
        k_nodemajor_to_colmajor<<<grid1(nk), 256, 0, s>>>(g->sol.as<double>(), g->n, ks[i], g->io_a.as<double>());
        BIE_CK(cudaGetLastError());
        BIE_CK(cudaMemcpyAsync(Sigma[i], g->io_a.p, sizeof(double) * nk, cudaMemcpyDeviceToHost, s));
    }
    BIE_CK(cudaStreamSynchronize(s));
    for (int i = 0; i < G; ++i) geom_trim_if_short(gs[i]);
    return rc;
}

}  // namespace bie

// Request server: the serving loop around the block solve
// (solve_dielectric_box3d_block, src/solver/multi_rhs.jl:270-286).
//
// Requests (a geometry handle, an N x k block of right-hand sides, solver
// options) are queued by bie_server_submit. A fixed number of worker threads
// ("slots") take admissible work from the queue: the oldest request whose
// geometry is not already being solved and whose estimated device workspace fits
// the HBM budget, merged with every later queued request for the same geometry
// and options up to max_batch_rhs columns — one block solve, one set of direct-sum
// launches for all of them. Batches on different geometries run at the same time,
// each on its geometry's CUDA stream, so their kernels overlap on the GPU; work
// that arrives while others run is admitted as slots and budget free up
// (continuous batching). Admission counts the estimated workspace of the batches in
// flight against the budget (a fraction of the device memory free when the server is
// created); a geometry keeps its workspace after a batch only while the budget not held by
// the other batches in flight is still free on the device, so that retained workspaces of
// idle geometries do not take memory that admission counts on. A batch whose device
// allocation fails anyway releases its own workspace and runs once more when every batch in
// flight is such a retry; retries run one at a time, and no new batch is admitted while one
// waits, so two batches that fail together do not wait for each other. A retry that fails
// again (memory held outside the server) backs off and tries again a bounded number of
// times. With the default solve options every column of a block solve runs its own Krylov
// process, so a request's result does not depend on what it was batched with beyond
// floating-point rounding; requests that ask for block GMRES share one Krylov space with
// their batch-mates and agree with a solo solve within the tolerance.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "solver.h"

namespace bie {
namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t ticket = 0;
    bie_geom* g = nullptr;
    int64_t n = 0;
    int k = 0;
    bie_solve_opts o{};
    std::vector<double> F, S;  // N x k column-major
    // point-source request: the sources only (x, y, z per column, charges, eps_src); its
    // right-hand sides are built on the device when its batch runs
    bool point = false;
    std::vector<double> src, q, eps;
    std::vector<int> col_it;
    std::vector<double> col_res;
    bie_stats st{};
    int rc = BIE_OK;
    std::string err;
    bool done = false;
    Clock::time_point t_submit, t_start, t_done;
};

bool same_opts(const bie_solve_opts& a, const bie_solve_opts& b) {
    return a.atol == b.atol && a.rtol == b.rtol && a.itmax == b.itmax && a.restart == b.restart &&
           a.precision == b.precision && a.inner_rtol == b.inner_rtol && a.max_outer == b.max_outer &&
           a.precondition == b.precondition && a.check_every == b.check_every && a.flags == b.flags &&
           a.block == b.block;
}

// Device workspace of a block solve of k columns: the Krylov basis (restart + 1
// vectors) plus about 32 more N x k blocks (residuals, split partials, I/O).
size_t footprint(int64_t n, int k, const bie_solve_opts& o) {
    const int64_t m = std::max(1, std::min(o.restart, o.itmax));
    return (size_t)(m + 1 + 32) * (size_t)n * (size_t)k * sizeof(double);
}

}  // namespace
}  // namespace bie

struct bie_server {
    bie_server_opts opt{};
    size_t budget = 0, in_use = 0, peak_use = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<bie::Request>> queue;
    std::unordered_map<uint64_t, std::shared_ptr<bie::Request>> table;
    std::unordered_map<bie_geom*, int> busy;
    uint64_t next_ticket = 1;
    bool stop = false;
    int inflight = 0;
    int retry_waiters = 0;    // batches in flight that released their workspace after ENOMEM
    std::mutex retry_mu;      // held by the one retry that runs
    std::atomic<int> inject_enomem{0};  // test hook: the next n solves fail with ENOMEM before any device work
    bie_server_counters cnt{};
    std::vector<std::thread> workers;
};

namespace bie {
namespace {

// Geometries of at most this many nodes join group solves: there one geometry's launches do
// not fill the GPU and per-iteration fixed costs dominate; a larger geometry runs alone.
constexpr int64_t kGroupMaxNodes = 24576;

// Attempts of a batch whose device allocation failed (the first run included); the waits
// between the later ones are 0.25, 0.5, 1, 2, 4, 8 s.
constexpr int kEnomemAttempts = 8;

// Whether a batch led by request r can join a group solve.
bool groupable(const Request& r) {
    return r.point && (r.o.precision == BIE_BF16X3 || r.o.precision == BIE_BF16X6) && !r.o.precondition &&
           r.n <= kGroupMaxNodes;
}

// Takes the next admissible batch off the queue (caller holds s->mu): the oldest request
// whose geometry is idle, merged with later ones for the same geometry and options up to
// kcap columns. like != null restricts it to batches that may join like's group solve;
// first says whether the batch would be the slot's first (admitted even over the budget
// when nothing runs).
bool take_batch(bie_server* s, std::vector<std::shared_ptr<Request>>& batch, size_t& fp, const Request* like,
                int kcap, bool first) {
    if (s->retry_waiters > 0) return false;  // a batch waits to retry after ENOMEM: let it have the device
    for (size_t i = 0; i < s->queue.size(); ++i) {
        const std::shared_ptr<Request> r = s->queue[i];
        if (s->busy.count(r->g)) continue;
        if (like && !(groupable(*r) && same_opts(r->o, like->o))) continue;
        if (r->k > kcap) continue;
        // gather the oldest request and later ones it can be merged with
        std::vector<size_t> pick{i};
        int K = r->k;
        for (size_t j = i + 1; j < s->queue.size(); ++j) {
            const auto& q = s->queue[j];
            if (q->g == r->g && q->point == r->point && same_opts(q->o, r->o) && K + q->k <= kcap) {
                pick.push_back(j);
                K += q->k;
            }
        }
        const size_t need = footprint(r->n, K, r->o);
        if (!(first && s->inflight == 0) && s->in_use + need > s->budget) continue;  // admitted later
        batch.clear();
        for (size_t j : pick) batch.push_back(s->queue[j]);
        for (size_t t = pick.size(); t-- > 0;) s->queue.erase(s->queue.begin() + (std::ptrdiff_t)pick[t]);
        s->busy[r->g] = 1;
        s->in_use += need;
        s->peak_use = std::max(s->peak_use, s->in_use);
        fp = need;
        return true;
    }
    return false;
}

void run_batch(bie_server* s, std::vector<std::shared_ptr<Request>>& batch) {
    const auto& r0 = batch.front();
    const int64_t n = r0->n;
    int K = 0;
    for (auto& r : batch) K += r->k;
    const bool point = r0->point;
    std::vector<double> F(point ? 0 : (size_t)n * K), S((size_t)n * K);
    std::vector<double> src(point ? 3 * (size_t)K : 0), q(point ? K : 0), eps(point ? K : 0);
    std::vector<int> col_it(K, 0);
    std::vector<double> col_res(K, 0.0);
    int off = 0;
    for (auto& r : batch) {
        if (point) {
            std::copy(r->src.begin(), r->src.end(), src.begin() + 3 * (size_t)off);
            std::copy(r->q.begin(), r->q.end(), q.begin() + off);
            std::copy(r->eps.begin(), r->eps.end(), eps.begin() + off);
        } else {
            std::memcpy(F.data() + (size_t)off * n, r->F.data(), sizeof(double) * (size_t)n * r->k);
            std::vector<double>().swap(r->F);  // the request's copy is not needed any more
        }
        off += r->k;
    }
    bie_stats st{};
    st.col_iterations = col_it.data();
    st.col_resid = col_res.data();
    auto solve = [&]() {
        int inj = s->inject_enomem.load();
        while (inj > 0 && !s->inject_enomem.compare_exchange_weak(inj, inj - 1)) {
        }
        if (inj > 0) throw Error(BIE_ENOMEM, "injected allocation failure (test hook)");
        return point ? solve_point_host(r0->g, src.data(), q.data(), eps.data(), K, S.data(), r0->o, &st)
                     : solve_host(r0->g, F.data(), S.data(), K, r0->o, &st);
    };
    int rc = BIE_OK;
    std::string err;
    const auto t_start = Clock::now();
    try {
        try {
            rc = solve();
        } catch (const Error& e) {
            if (e.code != BIE_ENOMEM) throw;
            // memory held by other batches in flight: release this geometry's workspace and
            // run once more when every batch in flight is a retry like this one (they hold no
            // workspace). Retries take turns under retry_mu; while any waits, take_batch admits
            // nothing new, so the running batches drain and the wait ends (bounded at 300 s).
            geom_trim(r0->g);
            struct Waiting {
                bie_server* s;
                explicit Waiting(bie_server* sv) : s(sv) {
                    std::lock_guard<std::mutex> lk(s->mu);
                    s->retry_waiters += 1;
                    s->cnt.enomem_retries += 1;
                }
                ~Waiting() {
                    {
                        std::lock_guard<std::mutex> lk(s->mu);
                        s->retry_waiters -= 1;
                    }
                    s->cv_done.notify_all();
                    s->cv_work.notify_all();
                }
            } waiting(s);
            s->cv_done.notify_all();  // a retry already waiting may now see only retries in flight
            std::lock_guard<std::mutex> turn(s->retry_mu);
            // Memory held outside the server (the caller's other threads building geometries,
            // other libraries) is released on its own schedule: a retry that meets ENOMEM again
            // backs off (0.25 s, doubling) and tries again, up to kEnomemAttempts runs in all.
            for (int attempt = 1;; ++attempt) {
                {
                    std::unique_lock<std::mutex> lk(s->mu);
                    s->cv_done.wait_for(lk, std::chrono::seconds(300),
                                        [&] { return s->inflight <= s->retry_waiters || s->stop; });
                }
                st = bie_stats{};
                st.col_iterations = col_it.data();
                st.col_resid = col_res.data();
                try {
                    rc = solve();
                    break;
                } catch (const Error& e2) {
                    if (e2.code != BIE_ENOMEM || attempt >= kEnomemAttempts - 1 || s->stop) throw;
                }
                geom_trim(r0->g);
                {
                    std::lock_guard<std::mutex> lk(s->mu);
                    s->cnt.enomem_retries += 1;
                }
                std::this_thread::sleep_for(std::chrono::milliseconds(250 << (attempt - 1)));
            }
        }
        if (rc != BIE_OK) err = "solver did not converge to the requested tolerance";
    } catch (const Error& e) {
        rc = e.code;
        err = e.what();
    } catch (const std::exception& e) {
        rc = BIE_EINVAL;
        err = e.what();
    }
    off = 0;
    for (auto& r : batch) {
        r->t_start = t_start;
        if (rc == BIE_OK || rc == BIE_ENOCONV) {
            r->S.assign(S.begin() + (size_t)off * n, S.begin() + (size_t)(off + r->k) * n);
            r->col_it.assign(col_it.begin() + off, col_it.begin() + off + r->k);
            r->col_res.assign(col_res.begin() + off, col_res.begin() + off + r->k);
        }
        r->st = st;
        r->st.col_iterations = nullptr;
        r->st.col_resid = nullptr;
        double mx = 0.0;
        for (double v : r->col_res) mx = std::max(mx, v);
        r->st.max_rel_resid = mx;
        r->rc = rc;
        r->err = err;
        off += r->k;
    }
}

// Batches of several geometries solved as one group (solve_group_point_host). If the group
// runs out of device memory, its members release their workspaces and run one by one
// (each with run_batch's own retry).
void run_group(bie_server* s, std::vector<std::vector<std::shared_ptr<Request>>>& group) {
    const int G = (int)group.size();
    std::vector<bie_geom*> gs(G);
    std::vector<int> ks(G, 0);
    std::vector<std::vector<double>> src(G), q(G), eps(G), S(G), col_res(G);
    std::vector<std::vector<int>> col_it(G);
    std::vector<bie_stats> st(G);
    std::vector<const double*> ps(G), pq(G), pe(G);
    std::vector<double*> pS(G);
    for (int m = 0; m < G; ++m) {
        gs[m] = group[m].front()->g;
        for (auto& r : group[m]) {
            ks[m] += r->k;
            src[m].insert(src[m].end(), r->src.begin(), r->src.end());
            q[m].insert(q[m].end(), r->q.begin(), r->q.end());
            eps[m].insert(eps[m].end(), r->eps.begin(), r->eps.end());
        }
        S[m].assign((size_t)group[m].front()->n * ks[m], 0.0);
        col_it[m].assign(ks[m], 0);
        col_res[m].assign(ks[m], 0.0);
        st[m] = bie_stats{};
        st[m].col_iterations = col_it[m].data();
        st[m].col_resid = col_res[m].data();
        ps[m] = src[m].data();
        pq[m] = q[m].data();
        pe[m] = eps[m].data();
        pS[m] = S[m].data();
    }
    int rc = BIE_OK;
    std::string err;
    const auto t_start = Clock::now();
    try {
        rc = solve_group_point_host(gs.data(), G, ps.data(), pq.data(), pe.data(), ks.data(), pS.data(),
                                    group.front().front()->o, st.data());
        if (rc != BIE_OK) err = "solver did not converge to the requested tolerance";
    } catch (const Error& e) {
        if (e.code == BIE_ENOMEM) {
            for (bie_geom* g : gs) {
                try {
                    geom_trim(g);
                } catch (...) {
                }
            }
            for (auto& b : group) run_batch(s, b);
            return;
        }
        rc = e.code;
        err = e.what();
    } catch (const std::exception& e) {
        rc = BIE_EINVAL;
        err = e.what();
    }
    for (int m = 0; m < G; ++m) {
        const int64_t n = group[m].front()->n;
        int off = 0;
        for (auto& r : group[m]) {
            r->t_start = t_start;
            if (rc == BIE_OK || rc == BIE_ENOCONV) {
                r->S.assign(S[m].begin() + (size_t)off * n, S[m].begin() + (size_t)(off + r->k) * n);
                r->col_it.assign(col_it[m].begin() + off, col_it[m].begin() + off + r->k);
                r->col_res.assign(col_res[m].begin() + off, col_res[m].begin() + off + r->k);
            }
            r->st = st[m];
            r->st.col_iterations = nullptr;
            r->st.col_resid = nullptr;
            double mx = 0.0;
            for (double v : r->col_res) mx = std::max(mx, v);
            r->st.max_rel_resid = mx;
            // a member's status: the group's ENOCONV applies to the members that missed
            r->rc = rc == BIE_ENOCONV ? (st[m].converged ? BIE_OK : BIE_ENOCONV) : rc;
            r->err = r->rc == BIE_OK ? std::string() : err;
            off += r->k;
        }
    }
}

void worker(bie_server* s) {
    for (;;) {
        std::vector<std::vector<std::shared_ptr<Request>>> group;
        std::vector<size_t> fps;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            for (;;) {
                if (s->stop) return;
                std::vector<std::shared_ptr<Request>> batch;
                size_t fp = 0;
                if (take_batch(s, batch, fp, nullptr, s->opt.max_batch_rhs, true)) {
                    group.push_back(std::move(batch));
                    fps.push_back(fp);
                    break;
                }
                s->cv_work.wait(lk);
            }
            // further geometries' batches for a group solve
            const Request& lead = *group.front().front();
            int Klead = 0;
            for (auto& r : group.front()) Klead += r->k;
            if (s->opt.max_group > 1 && groupable(lead) && Klead <= 128) {
                while ((int)group.size() < s->opt.max_group) {
                    std::vector<std::shared_ptr<Request>> batch;
                    size_t fp = 0;
                    if (!take_batch(s, batch, fp, &lead, std::min(128, s->opt.max_batch_rhs), false)) break;
                    group.push_back(std::move(batch));
                    fps.push_back(fp);
                }
            }
            ++s->inflight;
            s->cnt.batches += (int64_t)group.size();
            for (auto& b : group) s->cnt.merged_requests += (int64_t)b.size() - 1;
            if (group.size() > 1) {
                s->cnt.groups += 1;
                s->cnt.grouped_batches += (int64_t)group.size();
            }
            s->cnt.peak_inflight = std::max(s->cnt.peak_inflight, s->inflight);
        }
        if (group.size() == 1)
            run_batch(s, group.front());
        else
            run_group(s, group);
        // keep each geometry's workspace only while the part of the budget that the other
        // batches in flight do not hold stays free on the device (before the requests
        // complete: their caller may destroy the geometry once they are polled)
        size_t fp_all = 0;
        for (size_t f : fps) fp_all += f;
        size_t floor_b = 0;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            floor_b = s->budget > s->in_use - fp_all ? s->budget - (s->in_use - fp_all) : 0;
        }
        int64_t released = 0;
        for (auto& b : group) {
            try {
                released += geom_trim_if_below(b.front()->g, floor_b) ? 1 : 0;
            } catch (...) {
            }
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            const auto now = Clock::now();
            for (auto& b : group) {
                for (auto& r : b) {
                    r->t_done = now;
                    r->done = true;
                }
                s->busy.erase(b.front()->g);
                s->cnt.completed += (int64_t)b.size();
            }
            s->in_use -= fp_all;
            --s->inflight;
            s->cnt.workspace_releases += released;
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
}

}  // namespace

bie_server* server_create(const bie_server_opts& o) {
    if (o.max_slots < 1 || o.max_slots > 64 || o.max_batch_rhs < 1 || o.max_batch_rhs > 256 ||
        !(o.hbm_fraction > 0.0 && o.hbm_fraction <= 1.0) || o.max_group < 1 || o.max_group > 64)
        throw Error(BIE_EINVAL, "server_create: bad options");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        throw Error(BIE_ENODEVICE, "server_create: no CUDA device");
    }
    if (o.device < 0 || o.device >= ndev) throw Error(BIE_EINVAL, "server_create: bad device");
    int prev = 0;
    BIE_CK(cudaGetDevice(&prev));
    BIE_CK(cudaSetDevice(o.device));
    size_t free_b = 0, total_b = 0;
    const cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
    cudaSetDevice(prev);
    BIE_CK(e);
    auto s = std::make_unique<bie_server>();
    s->opt = o;
    s->budget = (size_t)(o.hbm_fraction * (double)free_b);
    s->cnt.hbm_budget = (int64_t)s->budget;
    if (const char* inj = std::getenv("BIE_TEST_SERVER_ENOMEM")) s->inject_enomem = std::atoi(inj);
    for (int i = 0; i < o.max_slots; ++i) s->workers.emplace_back(worker, s.get());
    return s.release();
}

void server_destroy(bie_server* s) {
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->workers) t.join();
    delete s;
}

namespace {
uint64_t enqueue(bie_server* s, const std::shared_ptr<Request>& r) {
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) throw Error(BIE_EINVAL, "server_submit: server is shutting down");
        r->ticket = s->next_ticket++;
        s->queue.push_back(r);
        s->table[r->ticket] = r;
        s->cnt.submitted += 1;
    }
    s->cv_work.notify_one();
    return r->ticket;
}

std::shared_ptr<Request> new_request(bie_server* s, bie_geom* g, int k, const bie_solve_opts& o) {
    int64_t n = 0, nblocks = 0;
    size_t bytes = 0;
    geom_info(g, &n, &nblocks, &bytes);
    if (k < 1 || k > s->opt.max_batch_rhs)
        throw Error(BIE_EINVAL, "server_submit: k must be in [1, max_batch_rhs]");
    auto r = std::make_shared<Request>();
    r->g = g;
    r->n = n;
    r->k = k;
    r->o = o;
    return r;
}
}  // namespace

uint64_t server_submit(bie_server* s, bie_geom* g, const double* F, int k, const bie_solve_opts& o) {
    auto r = new_request(s, g, k, o);
    r->F.assign(F, F + (size_t)r->n * k);
    return enqueue(s, r);
}

uint64_t server_submit_point(bie_server* s, bie_geom* g, const double* src, const double* q, const double* eps,
                             int k, const bie_solve_opts& o) {
    auto r = new_request(s, g, k, o);
    r->point = true;
    r->src.assign(src, src + 3 * (size_t)k);
    r->q.assign(q, q + k);
    r->eps.assign(eps, eps + k);
    return enqueue(s, r);
}

int server_poll(bie_server* s, uint64_t ticket, int timeout_ms, double* Sigma, bie_stats* st, double* latency_ms,
                int* done, std::string* err) {
    std::shared_ptr<Request> r;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->table.find(ticket);
        if (it == s->table.end()) throw Error(BIE_EINVAL, "server_poll: unknown ticket");
        r = it->second;
        auto ready = [&] { return r->done; };
        if (timeout_ms < 0)
            s->cv_done.wait(lk, ready);
        else
            s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
        if (!r->done) {
            *done = 0;
            return BIE_OK;
        }
        s->table.erase(it);
    }
    *done = 1;
    if (Sigma && !r->S.empty()) std::memcpy(Sigma, r->S.data(), sizeof(double) * r->S.size());
    if (st) {
        int* ci = st->col_iterations;
        double* cr = st->col_resid;
        *st = r->st;
        st->col_iterations = ci;
        st->col_resid = cr;
        if (ci)
            for (int c = 0; c < r->k && c < (int)r->col_it.size(); ++c) ci[c] = r->col_it[c];
        if (cr)
            for (int c = 0; c < r->k && c < (int)r->col_res.size(); ++c) cr[c] = r->col_res[c];
    }
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    *err = r->err;
    return r->rc;
}

void server_counters(bie_server* s, bie_server_counters* out) {
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->cnt;
    out->queued = (int64_t)s->queue.size();
    out->inflight = s->inflight;
    out->hbm_in_use = (int64_t)s->in_use;
    out->hbm_peak = (int64_t)s->peak_use;
}

}  // namespace bie

// Host set-up of near-accurate probe potentials, the operator of
// laplace3d_pottrg_fmm3d_corrected_hcubature (src/kernel/laplace3d_near_hcubature.jl:278-316):
//
//   phi = (S_refined + C) P sigma
//
// P interpolates sigma from the coarse panels onto an interface whose panels near the
// probes are split 4-way down to the smallest coarse panel size
// (_refine_interface_for_targets, _refined_interface_prolongation,
// src/kernel/laplace3d_near.jl:101-225); S_refined is the smooth-quadrature potential
// of the refined nodes (the GPU direct sum); C holds, for every probe within
// range_factor * l_panel / n_quad of a refined non-edge panel's centre
// (build_target_neighbor_list, src/kernel/laplace3d_near.jl:47-69), the adaptive
// integral of the panel's interpolated single layer minus its smooth-quadrature terms
// (laplace3d_pottrg_corrections_hcubature, laplace3d_near_hcubature.jl:122-192).
//
// The adaptive integrals restate the published algorithm behind HCubature.jl (the
// reference's un-vendored dependency, used with its default rule): the embedded
// Genz-Malik degree-7/degree-5 rule on rectangles (A. C. Genz and A. A. Malik, J.
// Comput. Appl. Math. 6 (1980) 295-302), the region with the largest error estimate
// bisected along the axis of the largest fourth difference until the total error
// estimate (2-norm over the nq^2 basis integrals) is at most atol.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <queue>
#include <string>
#include <unordered_map>
#include <vector>

#include <omp.h>

#include "host_setup.h"

namespace bie {
namespace {

struct P3 {
    double x, y, z;
};
inline P3 ld3(const double* p) { return {p[0], p[1], p[2]}; }
inline P3 add(P3 a, P3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline P3 sub(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline P3 mul(P3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot3(P3 a, P3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double len(P3 a) { return std::sqrt(dot3(a, a)); }

// laplace3d_pot (src/kernel/laplace3d.jl:1-7): 1 / (4 pi |src - trg|)
inline double lap_pot(P3 s, P3 t) {
    const P3 d = sub(s, t);
    const double r = std::sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
    return (1.0 / r) / (4.0 * M_PI);
}

// barycentric_row! (src/utils/barycentric.jl:19-42)
void bary_row_p(int n, const double* x, const double* lam, double xq, double* r) {
    const double rt = 1.4901161193847656e-08;
    for (int i = 0; i < n; ++i)
        if (xq == x[i] || std::fabs(xq - x[i]) <= rt * std::max(std::fabs(xq), std::fabs(x[i]))) {
            for (int k = 0; k < n; ++k) r[k] = 0.0;
            r[i] = 1.0;
            return;
        }
    double den = 0.0;
    for (int i = 0; i < n; ++i) {
        r[i] = lam[i] / (xq - x[i]);
        den += r[i];
    }
    const double inv = 1.0 / den;
    for (int i = 0; i < n; ++i) r[i] *= inv;
}

struct Panel {
    P3 a, b, c, d;
    P3 normal;
    int is_edge;
};
inline P3 centre(const Panel& p) { return mul(add(add(add(p.a, p.b), p.c), p.d), 0.25); }
// _panel_max_length (src/kernel/laplace3d_near.jl:77-79)
inline double max_len(const Panel& p) { return std::max(len(sub(p.a, p.b)), len(sub(p.b, p.c))); }

// Probes hashed into a uniform grid for the fixed-radius queries (KDTree inrange in
// the reference: every probe within distance r, boundary included).
struct Grid {
    double h = 1.0, lo[3] = {0, 0, 0};
    int64_t n[3] = {1, 1, 1};
    std::vector<int64_t> order;                                 // probes sorted by cell
    std::unordered_map<int64_t, std::pair<int64_t, int64_t>> cells;  // cell -> [begin, end) in order
    const double* T = nullptr;

    void build(const double* targets, int64_t M, double cell) {
        T = targets;
        h = cell > 0 ? cell : 1.0;
        double hi[3] = {0, 0, 0};
        for (int k = 0; k < 3; ++k) {
            lo[k] = M ? targets[k] : 0.0;
            hi[k] = lo[k];
        }
        for (int64_t m = 0; m < M; ++m)
            for (int k = 0; k < 3; ++k) {
                lo[k] = std::min(lo[k], targets[3 * m + k]);
                hi[k] = std::max(hi[k], targets[3 * m + k]);
            }
        for (int k = 0; k < 3; ++k) n[k] = (int64_t)std::floor((hi[k] - lo[k]) / h) + 1;
        std::vector<int64_t> key(M);
        for (int64_t m = 0; m < M; ++m) key[m] = cell_of(targets + 3 * m);
        order.resize(M);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return key[a] < key[b]; });
        for (int64_t i = 0; i < M;) {
            int64_t j = i;
            while (j < M && key[order[j]] == key[order[i]]) ++j;
            cells[key[order[i]]] = {i, j};
            i = j;
        }
    }
    int64_t coord(double v, int k) const {
        return std::min(n[k] - 1, std::max<int64_t>(0, (int64_t)std::floor((v - lo[k]) / h)));
    }
    int64_t cell_of(const double* p) const { return coord(p[0], 0) + n[0] * (coord(p[1], 1) + n[1] * coord(p[2], 2)); }
    // probes within distance r of c, ascending index
    void inrange(P3 c, double r, std::vector<int64_t>& out) const {
        out.clear();
        const double cv[3] = {c.x, c.y, c.z};
        int64_t a[3], b[3];
        for (int k = 0; k < 3; ++k) {
            const double l = (cv[k] - r - lo[k]) / h, u = (cv[k] + r - lo[k]) / h;
            if (u < 0 || l >= (double)n[k]) return;
            a[k] = std::max<int64_t>(0, (int64_t)std::floor(l));
            b[k] = std::min<int64_t>(n[k] - 1, (int64_t)std::floor(u));
        }
        for (int64_t z = a[2]; z <= b[2]; ++z)
            for (int64_t y = a[1]; y <= b[1]; ++y)
                for (int64_t x = a[0]; x <= b[0]; ++x) {
                    auto it = cells.find(x + n[0] * (y + n[1] * z));
                    if (it == cells.end()) continue;
                    for (int64_t i = it->second.first; i < it->second.second; ++i) {
                        const int64_t m = order[i];
                        if (len(sub(ld3(T + 3 * m), c)) <= r) out.push_back(m);
                    }
                }
        std::sort(out.begin(), out.end());
    }
};

// ------------------------- adaptive cubature (Genz-Malik) -------------------------
// Rule on [c - h, c + h] in 2-D: 17 points (centre, 4 at +-l2 on the axes, 4 at +-l4 on
// the axes, 4 at (+-l4, +-l4), 4 at (+-l5, +-l5)); weights of the degree-7 rule and of
// the embedded degree-5 rule (normalised to sum 1, times the region's area).
constexpr double kL2 = 0.35856858280031809;   // sqrt(9/70)
constexpr double kL4 = 0.94868329805051380;   // sqrt(9/10)
constexpr double kL5 = 0.68824720161168529;   // sqrt(9/19)
constexpr double kW1 = -3816.0 / 19683.0, kW2 = 980.0 / 6561.0, kW3 = 1020.0 / 19683.0, kW4 = 200.0 / 19683.0,
                 kW5 = 6859.0 / 19683.0 / 4.0;
constexpr double kV1 = -971.0 / 729.0, kV2 = 245.0 / 486.0, kV3 = 65.0 / 1458.0, kV4 = 25.0 / 729.0;
constexpr double kRatio = (kL2 * kL2) / (kL4 * kL4);  // of the fourth-difference estimate

struct Region {
    double c[2], h[2];
    double err;
    int kdiv;
    std::vector<double> I;
};

// Integrand: nq^2 values r_a(u) r_b(v) G(y(u, v), t) scale (the _pot_integrand_hcubature
// basis, src/kernel/laplace3d_near_hcubature.jl:58-85).
struct PotIntegrand {
    int nq;
    const double* glx;
    const double* bary;
    P3 cc, bma, dma, t;
    double scale;
    mutable std::vector<double> rx, ry;
    void operator()(double u, double v, double* out) const {
        bary_row_p(nq, glx, bary, u, rx.data());
        bary_row_p(nq, glx, bary, v, ry.data());
        const P3 p = add(add(cc, mul(bma, u / 2)), mul(dma, v / 2));
        const double k = lap_pot(p, t) * scale;
        int idx = 0;
        for (int i = 0; i < nq; ++i)
            for (int j = 0; j < nq; ++j) out[idx++] = k * rx[i] * ry[j];
    }
};

struct Cubature {
    int dim;                         // integrand values
    int64_t evals = 0, maxevals;
    std::vector<double> f0, fa, fb, fc, fd, tmp;  // scratch

    explicit Cubature(int d, int64_t maxev) : dim(d), maxevals(maxev), f0(d), fa(d), fb(d), fc(d), fd(d), tmp(d) {}

    double vnorm(const std::vector<double>& v) const {
        double s = 0.0;
        for (double x : v) s += x * x;
        return std::sqrt(s);
    }

    template <class F>
    void rule(const F& f, Region& R) {
        const int d = dim;
        std::vector<double> s7(d, 0.0), s5(d, 0.0);
        auto acc = [&](const std::vector<double>& v, double w7, double w5) {
            for (int i = 0; i < d; ++i) {
                s7[i] += w7 * v[i];
                s5[i] += w5 * v[i];
            }
        };
        f(R.c[0], R.c[1], f0.data());
        acc(f0, kW1, kV1);
        double divdiff[2];
        for (int k = 0; k < 2; ++k) {
            double o2[2] = {0, 0}, o4[2] = {0, 0};
            o2[k] = kL2 * R.h[k];
            o4[k] = kL4 * R.h[k];
            f(R.c[0] + o2[0], R.c[1] + o2[1], fa.data());
            f(R.c[0] - o2[0], R.c[1] - o2[1], fb.data());
            f(R.c[0] + o4[0], R.c[1] + o4[1], fc.data());
            f(R.c[0] - o4[0], R.c[1] - o4[1], fd.data());
            for (int i = 0; i < d; ++i) {
                s7[i] += kW2 * (fa[i] + fb[i]) + kW3 * (fc[i] + fd[i]);
                s5[i] += kV2 * (fa[i] + fb[i]) + kV3 * (fc[i] + fd[i]);
                tmp[i] = fa[i] + fb[i] - 2 * f0[i] - kRatio * (fc[i] + fd[i] - 2 * f0[i]);
            }
            divdiff[k] = vnorm(tmp);
        }
        for (int sx = -1; sx <= 1; sx += 2)
            for (int sy = -1; sy <= 1; sy += 2) {
                f(R.c[0] + sx * kL4 * R.h[0], R.c[1] + sy * kL4 * R.h[1], fa.data());
                acc(fa, kW4, kV4);
                f(R.c[0] + sx * kL5 * R.h[0], R.c[1] + sy * kL5 * R.h[1], fb.data());
                acc(fb, kW5, 0.0);
            }
        evals += 17;
        const double V = 4.0 * R.h[0] * R.h[1];
        R.I.assign(d, 0.0);
        for (int i = 0; i < d; ++i) {
            R.I[i] = V * s7[i];
            tmp[i] = V * (s7[i] - s5[i]);
        }
        R.err = vnorm(tmp);
        // bisect along the largest fourth difference; nearly equal ones: the wider axis
        if (std::fabs(divdiff[0] - divdiff[1]) <= 1e-12 * std::max(divdiff[0], divdiff[1]))
            R.kdiv = R.h[1] > R.h[0] ? 1 : 0;
        else
            R.kdiv = divdiff[1] > divdiff[0] ? 1 : 0;
    }

    // Integral over [-1, 1]^2 into out (dim values); returns false when maxevals ran out.
    template <class F>
    bool integrate(const F& f, double atol, double* out) {
        auto cmp = [](const Region& a, const Region& b) { return a.err < b.err; };
        std::priority_queue<Region, std::vector<Region>, decltype(cmp)> heap(cmp);
        Region r0;
        r0.c[0] = r0.c[1] = 0.0;
        r0.h[0] = r0.h[1] = 1.0;
        rule(f, r0);
        std::vector<double> I = r0.I;
        double E = r0.err;
        heap.push(std::move(r0));
        bool ok = true;
        while (E > atol && std::isfinite(E)) {
            if (evals >= maxevals) {
                ok = false;
                break;
            }
            Region R = heap.top();
            heap.pop();
            Region A = R, B = R;
            const int k = R.kdiv;
            A.h[k] = B.h[k] = R.h[k] / 2;
            A.c[k] = R.c[k] - R.h[k] / 2;
            B.c[k] = R.c[k] + R.h[k] / 2;
            rule(f, A);
            rule(f, B);
            for (int i = 0; i < dim; ++i) I[i] += (A.I[i] + B.I[i]) - R.I[i];
            E += (A.err + B.err) - R.err;
            heap.push(std::move(A));
            heap.push(std::move(B));
        }
        // re-sum the regions (the running totals accumulate rounding)
        std::fill(out, out + dim, 0.0);
        while (!heap.empty()) {
            const Region& R = heap.top();
            for (int i = 0; i < dim; ++i) out[i] += R.I[i];
            heap.pop();
        }
        return ok;
    }
};

// rect_panel3d_discretize children of a panel (_split_panel4, src/kernel/laplace3d_near.jl:81-99)
void split4(const Panel& p, Panel out[4]) {
    const P3 ab = mul(add(p.a, p.b), 0.5), bc = mul(add(p.b, p.c), 0.5), cd = mul(add(p.c, p.d), 0.5),
             da = mul(add(p.d, p.a), 0.5), cc = centre(p);
    out[0] = {p.a, ab, cc, da, p.normal, p.is_edge};
    out[1] = {ab, p.b, bc, cc, p.normal, p.is_edge};
    out[2] = {cc, bc, p.c, cd, p.normal, p.is_edge};
    out[3] = {da, cc, cd, p.d, p.normal, p.is_edge};
}

}  // namespace

int probe_setup(const Mesh& m, const double* targets, int64_t M, double atol, double range_factor, int nthreads,
                int64_t maxevals, ProbeSetup& out, std::string& err) {
    out = ProbeSetup();
    if (!(atol > 0) || !(range_factor > 0) || M < 0) {
        err = "probe set-up: hcubature_atol and range_factor must be positive";
        return -1;
    }
    const int nq = m.nq, np = nq * nq;
    const int P = m.npanels;
    std::vector<Panel> coarse(P);
    for (int p = 0; p < P; ++p) {
        const double* c = m.corners.data() + 12 * p;
        coarse[p] = {ld3(c), ld3(c + 3), ld3(c + 6), ld3(c + 9), ld3(m.normals.data() + 3 * p), m.is_edge[p]};
    }
    double size_limit = INFINITY, rmax = 0.0;
    for (const Panel& p : coarse) {
        size_limit = std::min(size_limit, max_len(p));
        rmax = std::max(rmax, range_factor * max_len(p) / nq);
    }
    Grid grid;
    grid.build(targets, M, rmax);
    std::vector<int64_t> near;

    // _refine_interface_for_targets: a stack of (parent, panel, split) popped from the back
    std::vector<Panel> refined;
    std::vector<std::pair<int, int>> stack_meta;  // (parent, from_split) of the stack entries
    std::vector<Panel> stack;
    for (int p = 0; p < P; ++p) {
        stack.push_back(coarse[p]);
        stack_meta.push_back({p, 0});
    }
    while (!stack.empty()) {
        const Panel pn = stack.back();
        const auto meta = stack_meta.back();
        stack.pop_back();
        stack_meta.pop_back();
        const double l = max_len(pn);
        grid.inrange(centre(pn), range_factor * l / nq, near);
        if (!near.empty() && l > size_limit && M > 0) {
            Panel ch[4];
            split4(pn, ch);
            for (int q = 0; q < 4; ++q) {
                stack.push_back(ch[q]);
                stack_meta.push_back({meta.first, 1});
            }
        } else {
            refined.push_back(pn);
            out.parent.push_back(meta.first);
            out.from_split.push_back(meta.second);
        }
    }
    const int R = (int)refined.size();
    {
        std::vector<double> corners((size_t)12 * R), normals((size_t)3 * R), ei(R), eo(R);
        std::vector<int> ie(R);
        for (int r = 0; r < R; ++r) {
            const Panel& pn = refined[r];
            const P3 cs[4] = {pn.a, pn.b, pn.c, pn.d};
            for (int q = 0; q < 4; ++q) {
                corners[12 * r + 3 * q] = cs[q].x;
                corners[12 * r + 3 * q + 1] = cs[q].y;
                corners[12 * r + 3 * q + 2] = cs[q].z;
            }
            normals[3 * r] = pn.normal.x;
            normals[3 * r + 1] = pn.normal.y;
            normals[3 * r + 2] = pn.normal.z;
            ie[r] = pn.is_edge;
            ei[r] = m.eps_in[out.parent[r]];
            eo[r] = m.eps_out[out.parent[r]];
        }
        if (mesh_from_panels(R, nq, corners.data(), normals.data(), ie.data(), ei.data(), eo.data(), out.refined,
                             err) != 0)
            return -1;
    }

    // _refined_interface_prolongation: unsplit panels copy their parent's nodes; nodes of
    // split panels interpolate the parent's tensor Lagrange basis at their (u, v)
    out.prow.assign(1, 0);
    std::vector<double> rx(nq), ry(nq);
    for (int r = 0; r < R; ++r) {
        const int par = out.parent[r];
        const int64_t col0 = (int64_t)par * np;
        if (!out.from_split[r]) {
            for (int t = 0; t < np; ++t) {
                out.pcol.push_back((int32_t)(col0 + t));
                out.pval.push_back(1.0);
                out.prow.push_back((int64_t)out.pcol.size());
            }
            continue;
        }
        const Panel& pp = coarse[par];
        const P3 cc = centre(pp), bma = sub(pp.b, pp.a), dma = sub(pp.d, pp.a);
        const double bb = dot3(bma, bma), bd = dot3(bma, dma), dd = dot3(dma, dma);
        const double det = bb * dd - bd * bd;
        const double i11 = dd / det, i12 = -bd / det, i22 = bb / det;
        for (int t = 0; t < np; ++t) {
            const P3 x = sub(ld3(out.refined.pts.data() + 3 * ((size_t)r * np + t)), cc);
            const double r1 = dot3(bma, x), r2 = dot3(dma, x);
            const double s = i11 * r1 + i12 * r2, tt = i12 * r1 + i22 * r2;
            bary_row_p(nq, m.glx.data(), m.bary.data(), 2 * s, rx.data());
            bary_row_p(nq, m.glx.data(), m.bary.data(), 2 * tt, ry.data());
            for (int ii = 0; ii < nq; ++ii)
                for (int jj = 0; jj < nq; ++jj) {
                    out.pcol.push_back((int32_t)(col0 + ii * nq + jj));
                    out.pval.push_back(rx[ii] * ry[jj]);
                }
            out.prow.push_back((int64_t)out.pcol.size());
        }
    }

    // build_target_neighbor_list on the refined interface, edge panels excluded
    std::vector<std::pair<int, std::vector<int64_t>>> entries;
    for (int r = 0; r < R; ++r) {
        const Panel& pn = refined[r];
        if (pn.is_edge) continue;
        grid.inrange(centre(pn), range_factor * max_len(pn) / nq, near);
        if (!near.empty()) entries.push_back({r, near});
    }

    // laplace3d_pottrg_corrections_hcubature: adaptive integral minus the smooth terms
    struct Trip {
        int64_t row;
        int32_t col;
        double v;
    };
    const int nent = (int)entries.size();
    std::vector<std::vector<Trip>> trips(nent);
    std::vector<int64_t> ncub(nent, 0), capped(nent, 0);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : omp_get_max_threads())
    for (int e = 0; e < nent; ++e) {
        const int r = entries[e].first;
        const Panel& pn = refined[r];
        PotIntegrand f;
        f.nq = nq;
        f.glx = m.glx.data();
        f.bary = m.bary.data();
        f.cc = centre(pn);
        f.bma = sub(pn.b, pn.a);
        f.dma = sub(pn.d, pn.a);
        f.scale = len(sub(pn.b, pn.a)) * len(sub(pn.d, pn.a)) / 4;
        f.rx.resize(nq);
        f.ry.resize(nq);
        std::vector<double> exact(np);
        for (int64_t tg : entries[e].second) {
            f.t = ld3(targets + 3 * tg);
            Cubature cub(np, maxevals);
            if (!cub.integrate(f, atol, exact.data())) ++capped[e];
            ++ncub[e];
            for (int c = 0; c < np; ++c) {
                const size_t node = (size_t)r * np + c;
                const double direct = out.refined.w[node] * lap_pot(ld3(out.refined.pts.data() + 3 * node), f.t);
                const double v = exact[c] - direct;
                if (v != 0.0) trips[e].push_back({tg, (int32_t)node, v});
            }
        }
    }
    std::vector<Trip> all;
    for (int e = 0; e < nent; ++e) {
        all.insert(all.end(), trips[e].begin(), trips[e].end());
        out.ncubatures += ncub[e];
        out.capped += capped[e];
    }
    std::sort(all.begin(), all.end(), [](const Trip& a, const Trip& b) { return a.row < b.row || (a.row == b.row && a.col < b.col); });
    out.crow.assign(M + 1, 0);
    out.ccol.resize(all.size());
    out.cval.resize(all.size());
    for (size_t i = 0; i < all.size(); ++i) {
        out.crow[all[i].row + 1]++;
        out.ccol[i] = all[i].col;
        out.cval[i] = all[i].v;
    }
    for (int64_t i = 0; i < M; ++i) out.crow[i + 1] += out.crow[i];
    out.nentries = nent;
    return 0;
}

}  // namespace bie

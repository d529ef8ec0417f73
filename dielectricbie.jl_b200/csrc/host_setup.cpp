// Host-side geometry setup: mesher, near-pair list, correction blocks (BSR).
// Each routine cites the reference (xuanzhaogao/DielectricBIE.jl) lines whose
// semantics it reproduces; node order, panel order and the correction-block
// formulas are part of the drop-in contract (sigma is compared node by node).
#include "host_setup.h"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <array>
#include <cfloat>
#include <climits>
#include <cmath>
#include <complex>
#include <cstring>
#include <deque>
#include <unordered_map>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace bie {

namespace {
constexpr double kFourPi = 4.0 * M_PI;

struct V3 {
    double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 ld(const double* p) { return {p[0], p[1], p[2]}; }
inline void st(double* p, V3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }
inline double comp(V3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
inline void setc(V3& v, int k, double s) { (k == 0 ? v.x : (k == 1 ? v.y : v.z)) = s; }

// laplace3d_grad (src/kernel/laplace3d.jl:9-15): n . (trg - src) / (4 pi |trg - src|^3)
inline double lap_grad(V3 src, V3 trg, V3 n) {
    V3 d = src - trg;
    double r2 = (d.x * d.x + d.y * d.y) + d.z * d.z;
    double ir = 1.0 / std::sqrt(r2);
    double i3 = ir * ir * ir;
    V3 e = trg - src;
    return ((n.x * (i3 * e.x) + n.y * (i3 * e.y)) + n.z * (i3 * e.z)) / kFourPi;
}
}  // namespace

// ---------------------------------------------------------------------------
// Gauss-Legendre rule (FastGaussQuadrature.jl 1.1.0): closed forms up to n = 5,
// Newton on the Legendre three-term recurrence beyond.
// ---------------------------------------------------------------------------
void gauss_legendre(int n, double* x, double* w) {
    switch (n) {
        case 1: x[0] = 0.0; w[0] = 2.0; return;
        case 2: x[0] = -1.0 / std::sqrt(3.0); x[1] = -x[0]; w[0] = w[1] = 1.0; return;
        case 3:
            x[0] = -std::sqrt(3.0 / 5.0); x[1] = 0.0; x[2] = -x[0];
            w[0] = w[2] = 5.0 / 9.0; w[1] = 8.0 / 9.0; return;
        case 4: {
            double a = 2.0 / 7.0 * std::sqrt(6.0 / 5.0);
            x[0] = -std::sqrt(3.0 / 7.0 + a); x[1] = -std::sqrt(3.0 / 7.0 - a); x[2] = -x[1]; x[3] = -x[0];
            w[0] = w[3] = (18.0 - std::sqrt(30.0)) / 36.0; w[1] = w[2] = (18.0 + std::sqrt(30.0)) / 36.0;
            return;
        }
        case 5: {
            double b = 2.0 * std::sqrt(10.0 / 7.0);
            x[0] = -std::sqrt(5.0 + b) / 3.0; x[1] = -std::sqrt(5.0 - b) / 3.0; x[2] = 0.0; x[3] = -x[1]; x[4] = -x[0];
            w[0] = w[4] = (322.0 - 13.0 * std::sqrt(70.0)) / 900.0;
            w[1] = w[3] = (322.0 + 13.0 * std::sqrt(70.0)) / 900.0;
            w[2] = 128.0 / 225.0;
            return;
        }
        default: break;
    }
    auto legendre = [n](long double z, long double& pn, long double& dpn) {
        long double p0 = 1.0L, p1 = z;
        for (int k = 2; k <= n; ++k) {
            long double p2 = ((2.0L * k - 1.0L) * z * p1 - (k - 1.0L) * p0) / k;
            p0 = p1; p1 = p2;
        }
        pn = p1;
        dpn = n * (z * p1 - p0) / (z * z - 1.0L);
    };
    for (int i = 0; i < (n + 1) / 2; ++i) {
        long double z = std::cos(M_PI * (i + 0.75L) / (n + 0.5L)), pn, dp;
        for (int it = 0; it < 100; ++it) {
            legendre(z, pn, dp);
            long double dz = pn / dp;
            z -= dz;
            if (std::fabs((double)dz) < 1e-19) break;
        }
        legendre(z, pn, dp);
        double wi = (double)(2.0L / ((1.0L - z * z) * dp * dp));
        x[i] = -(double)z; x[n - 1 - i] = (double)z;
        w[i] = wi; w[n - 1 - i] = wi;
    }
    if (n % 2) x[n / 2] = 0.0;
}

// ---------------------------------------------------------------------------
// best_grid (src/utils/best_grid.jl:8-118): continued-fraction convergents and
// semiconvergents of W/H, smallest m*n with aspect <= alpha.
// ---------------------------------------------------------------------------
int best_grid(double W, double H, double alpha, int* out_m, int* out_n) {
    if (!(W > 0 && H > 0) || alpha < 1) return -1;
    const long max_den = 1000000;
    bool swapped = W < H;
    if (swapped) std::swap(W, H);
    const double r = W / H;
    long bm = 0, bn = 0, bN = LONG_MAX;
    double brho = INFINITY;
    auto consider = [&](long m, long n) {
        if (m <= 0 || n <= 0 || m > max_den || n > max_den) return;
        double ratio = (W * (double)n) / (H * (double)m);
        double rho = ratio >= 1 ? ratio : 1 / ratio;
        if (rho > alpha) return;
        long N = m * n;
        if (N < bN || (N == bN && rho < brho)) { bm = m; bn = n; bN = N; brho = rho; }
    };
    long pmm = 0, pm = 1, qmm = 1, qm = 0;
    double x = r;
    for (int it = 0; it < 10000; ++it) {
        long a = (long)std::floor(x);
        long p = a * pm + pmm, q = a * qm + qmm;
        consider(p, q);
        if (a > 1) {
            long tmax = a - 1;
            if (pm > 0) tmax = std::min(tmax, (max_den - pmm) / pm);
            if (qm > 0) tmax = std::min(tmax, (max_den - qmm) / qm);
            for (long t = 1; t <= tmax; ++t) consider(t * pm + pmm, t * qm + qmm);
        }
        double frac = x - (double)a;
        if (std::fabs(frac) <= 1e-12) break;
        pmm = pm; pm = p; qmm = qm; qm = q;
        x = 1.0 / frac;
    }
    if (bm == 0) return -2;
    if (swapped) std::swap(bm, bn);
    *out_m = (int)bm; *out_n = (int)bn;
    return 0;
}

// ---------------------------------------------------------------------------
// Mesh
// ---------------------------------------------------------------------------
namespace {
struct Quad {
    V3 a, b, c, d, n;
    bool corner[4];  // a, b, c, d
    bool edge[4];    // ab, bc, cd, da
};

void init_rule(Mesh& m, int nq) {
    m.nq = nq;
    m.glx.resize(nq); m.glw.resize(nq); m.bary.resize(nq);
    gauss_legendre(nq, m.glx.data(), m.glw.data());
    // gl_barycentric_weights (src/utils/barycentric.jl:6-17)
    double mx = 0.0;
    for (int i = 0; i < nq; ++i) {
        double s = ((nq - 1 - i) % 2 == 0) ? 1.0 : -1.0;
        m.bary[i] = s * std::sqrt((1.0 - m.glx[i] * m.glx[i]) * m.glw[i] / 2.0);
        mx = std::max(mx, std::fabs(m.bary[i]));
    }
    for (auto& v : m.bary) v /= mx;
}

void push_panel(Mesh& m, const Quad& q, double ei, double eo) {
    double buf[12];
    st(buf, q.a); st(buf + 3, q.b); st(buf + 6, q.c); st(buf + 9, q.d);
    m.corners.insert(m.corners.end(), buf, buf + 12);
    m.normals.push_back(q.n.x); m.normals.push_back(q.n.y); m.normals.push_back(q.n.z);
    bool e = q.edge[0] || q.edge[1] || q.edge[2] || q.edge[3] || q.corner[0] || q.corner[1] || q.corner[2] ||
             q.corner[3];
    m.is_edge.push_back(e ? 1 : 0);
    m.eps_in.push_back(ei); m.eps_out.push_back(eo);
    m.npanels++;
}

// divide_temp_panel3d (src/shape/box3d.jl:66-98), children row-major in (i, j).
void subdivide(const Quad& t, int nx, int ny, std::vector<Quad>& out) {
    V3 bma = t.b - t.a, dma = t.d - t.a;
    for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= ny; ++j) {
            double u0 = (double)(i - 1) / nx, u1 = (double)i / nx, v0 = (double)(j - 1) / ny, v1 = (double)j / ny;
            Quad o;
            o.a = (t.a + bma * u0) + dma * v0;
            o.b = (t.a + bma * u1) + dma * v0;
            o.c = (t.a + bma * u1) + dma * v1;
            o.d = (t.a + bma * u0) + dma * v1;
            o.n = t.n;
            o.corner[0] = (i == 1 && j == 1) && t.corner[0];
            o.corner[1] = (i == nx && j == 1) && t.corner[1];
            o.corner[2] = (i == nx && j == ny) && t.corner[2];
            o.corner[3] = (i == 1 && j == ny) && t.corner[3];
            o.edge[0] = (j == 1) && t.edge[0];
            o.edge[1] = (i == nx) && t.edge[1];
            o.edge[2] = (j == ny) && t.edge[2];
            o.edge[3] = (i == 1) && t.edge[3];
            out.push_back(o);
        }
}

// rect_panel3d_adaptive_panels (src/shape/box3d.jl:101-133): coarse best_grid tiling,
// then breadth-first 2x2 splitting of edge/corner panels longer than l_ec.
int mesh_face(Mesh& m, const Quad& face, double alpha, double l_ec, double ei, double eo, std::string& err) {
    int nx, ny;
    int rc = best_grid(norm(face.b - face.a), norm(face.a - face.d), alpha, &nx, &ny);
    if (rc != 0) { err = "best_grid: no admissible (m, n) grid for a face"; return rc; }
    std::vector<Quad> tmp;
    subdivide(face, nx, ny, tmp);
    std::deque<Quad> queue(tmp.begin(), tmp.end());
    while (!queue.empty()) {
        Quad t = queue.front();
        queue.pop_front();
        bool ec = t.corner[0] || t.corner[1] || t.corner[2] || t.corner[3] || t.edge[0] || t.edge[1] ||
                  t.edge[2] || t.edge[3];
        if (ec && std::max(norm(t.b - t.a), norm(t.a - t.d)) > l_ec) {
            tmp.clear();
            subdivide(t, 2, 2, tmp);
            for (auto& c : tmp) queue.push_back(c);
        } else {
            push_panel(m, t, ei, eo);
        }
    }
    return 0;
}

// _box3d_faces_at_center (src/shape/box3d_multi.jl:4-30); with center 0 it is
// _box3d_geometry (src/shape/box3d_single.jl:1-34).
void box_faces(V3 c, double Lx, double Ly, double Lz, Quad f[6]) {
    double hx = Lx / 2, hy = Ly / 2, hz = Lz / 2;
    V3 v[8] = {{c.x + hx, c.y + hy, c.z + hz}, {c.x - hx, c.y + hy, c.z + hz}, {c.x - hx, c.y - hy, c.z + hz},
               {c.x + hx, c.y - hy, c.z + hz}, {c.x + hx, c.y + hy, c.z - hz}, {c.x - hx, c.y + hy, c.z - hz},
               {c.x - hx, c.y - hy, c.z - hz}, {c.x + hx, c.y - hy, c.z - hz}};
    static const int F[6][4] = {{0, 1, 2, 3}, {4, 7, 6, 5}, {7, 4, 0, 3}, {6, 2, 1, 5}, {5, 1, 0, 4}, {6, 7, 3, 2}};
    static const double N[6][3] = {{0, 0, 1}, {0, 0, -1}, {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}};
    for (int i = 0; i < 6; ++i) {
        f[i].a = v[F[i][0]]; f[i].b = v[F[i][1]]; f[i].c = v[F[i][2]]; f[i].d = v[F[i][3]];
        f[i].n = {N[i][0], N[i][1], N[i][2]};
        for (int k = 0; k < 4; ++k) f[i].corner[k] = f[i].edge[k] = true;
    }
}

void plane_axes(V3 n, int& a1, int& a2, int& an) {
    if (std::fabs(n.x) > 0.5) { a1 = 1; a2 = 2; an = 0; }
    else if (std::fabs(n.y) > 0.5) { a1 = 0; a2 = 2; an = 1; }
    else { a1 = 0; a2 = 1; an = 2; }
}

V3 plane_point(int a1, int a2, int an, double u, double v, double pc) {
    V3 p{0, 0, 0};
    setc(p, a1, u); setc(p, a2, v); setc(p, an, pc);
    return p;
}

// _rect_overlap_3d (src/shape/box3d_multi.jl:36-132)
bool rect_overlap(const Quad& f1, const V3 c2[4], V3 n2, V3 out[4]) {
    const double tol = 1e-10;
    if (norm(f1.n + n2) > tol) return false;
    for (int k = 0; k < 4; ++k)
        if (std::fabs(dot(f1.n, c2[k] - f1.a)) > tol) return false;
    int a1, a2, an;
    plane_axes(f1.n, a1, a2, an);
    V3 c1[4] = {f1.a, f1.b, f1.c, f1.d};
    double u1lo = INFINITY, u1hi = -INFINITY, v1lo = INFINITY, v1hi = -INFINITY;
    double u2lo = INFINITY, u2hi = -INFINITY, v2lo = INFINITY, v2hi = -INFINITY;
    for (int k = 0; k < 4; ++k) {
        u1lo = std::min(u1lo, comp(c1[k], a1)); u1hi = std::max(u1hi, comp(c1[k], a1));
        v1lo = std::min(v1lo, comp(c1[k], a2)); v1hi = std::max(v1hi, comp(c1[k], a2));
        u2lo = std::min(u2lo, comp(c2[k], a1)); u2hi = std::max(u2hi, comp(c2[k], a1));
        v2lo = std::min(v2lo, comp(c2[k], a2)); v2hi = std::max(v2hi, comp(c2[k], a2));
    }
    double lu = std::max(u1lo, u2lo), hu = std::min(u1hi, u2hi), lv = std::max(v1lo, v2lo), hv = std::min(v1hi, v2hi);
    if (hu - lu < tol || hv - lv < tol) return false;
    double pc = comp(f1.a, an);
    double eab0 = comp(f1.b, a1) - comp(f1.a, a1), eab1 = comp(f1.b, a2) - comp(f1.a, a2);
    double ead0 = comp(f1.d, a1) - comp(f1.a, a1), ead1 = comp(f1.d, a2) - comp(f1.a, a2);
    if (std::fabs(eab0) > tol) {
        double us = eab0 >= 0 ? lu : hu, ue = eab0 >= 0 ? hu : lu, vs = ead1 >= 0 ? lv : hv, ve = ead1 >= 0 ? hv : lv;
        out[0] = plane_point(a1, a2, an, us, vs, pc); out[1] = plane_point(a1, a2, an, ue, vs, pc);
        out[2] = plane_point(a1, a2, an, ue, ve, pc); out[3] = plane_point(a1, a2, an, us, ve, pc);
    } else {
        double us = ead0 >= 0 ? lu : hu, ue = ead0 >= 0 ? hu : lu, vs = eab1 >= 0 ? lv : hv, ve = eab1 >= 0 ? hv : lv;
        out[0] = plane_point(a1, a2, an, us, vs, pc); out[1] = plane_point(a1, a2, an, us, ve, pc);
        out[2] = plane_point(a1, a2, an, ue, ve, pc); out[3] = plane_point(a1, a2, an, ue, vs, pc);
    }
    return true;
}

// _subtract_rects_from_face_3d (src/shape/box3d_multi.jl:169-308): remaining cells of
// the face after removing shared rectangles, with physical edge/corner flags.
void subtract_rects(const Quad& f, const std::vector<std::array<V3, 4>>& sh, std::vector<Quad>& out) {
    const double tol = 1e-10;
    if (sh.empty()) { out.push_back(f); return; }
    int a1, a2, an;
    plane_axes(f.n, a1, a2, an);
    double pc = comp(f.a, an);
    V3 fc[4] = {f.a, f.b, f.c, f.d};
    double fu0 = INFINITY, fu1 = -INFINITY, fv0 = INFINITY, fv1 = -INFINITY;
    for (auto& p : fc) {
        fu0 = std::min(fu0, comp(p, a1)); fu1 = std::max(fu1, comp(p, a1));
        fv0 = std::min(fv0, comp(p, a2)); fv1 = std::max(fv1, comp(p, a2));
    }
    std::vector<double> us{fu0, fu1}, vs{fv0, fv1};
    for (auto& r : sh)
        for (auto& p : r) { us.push_back(comp(p, a1)); vs.push_back(comp(p, a2)); }
    auto uniq = [](std::vector<double>& v) {
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
    };
    uniq(us); uniq(vs);
    us.erase(std::remove_if(us.begin(), us.end(), [&](double u) { return !(fu0 - tol <= u && u <= fu1 + tol); }), us.end());
    vs.erase(std::remove_if(vs.begin(), vs.end(), [&](double v) { return !(fv0 - tol <= v && v <= fv1 + tol); }), vs.end());
    int nu = (int)us.size() - 1, nv = (int)vs.size() - 1;
    std::vector<char> cs((size_t)std::max(nu, 0) * std::max(nv, 0));
    auto CS = [&](int i, int j) -> char& { return cs[(size_t)i * nv + j]; };
    for (int i = 0; i < nu; ++i)
        for (int j = 0; j < nv; ++j) {
            double ulo = us[i], uhi = us[i + 1], vlo = vs[j], vhi = vs[j + 1];
            if (uhi - ulo < tol || vhi - vlo < tol) { CS(i, j) = 1; continue; }
            double um = (ulo + uhi) / 2, vm = (vlo + vhi) / 2;
            char hit = 0;
            for (auto& r : sh) {
                double r0 = INFINITY, r1 = -INFINITY, s0 = INFINITY, s1 = -INFINITY;
                for (auto& p : r) {
                    r0 = std::min(r0, comp(p, a1)); r1 = std::max(r1, comp(p, a1));
                    s0 = std::min(s0, comp(p, a2)); s1 = std::max(s1, comp(p, a2));
                }
                if (r0 - tol <= um && um <= r1 + tol && s0 - tol <= vm && vm <= s1 + tol) { hit = 1; break; }
            }
            CS(i, j) = hit;
        }
    auto physical = [&](int gi, int gj) {
        const int di[4] = {0, -1, 0, -1}, dj[4] = {0, 0, -1, -1};
        for (int t = 0; t < 4; ++t) {
            int ci = gi + di[t], cj = gj + dj[t];
            if (ci < 0 || ci >= nu || cj < 0 || cj >= nv || CS(ci, cj)) return true;
        }
        return false;
    };
    for (int i = 0; i < nu; ++i)
        for (int j = 0; j < nv; ++j) {
            if (CS(i, j)) continue;
            Quad q;
            q.a = plane_point(a1, a2, an, us[i], vs[j], pc);
            q.b = plane_point(a1, a2, an, us[i + 1], vs[j], pc);
            q.c = plane_point(a1, a2, an, us[i + 1], vs[j + 1], pc);
            q.d = plane_point(a1, a2, an, us[i], vs[j + 1], pc);
            q.n = f.n;
            q.edge[0] = (j == 0) || CS(i, j - 1);
            q.edge[1] = (i == nu - 1) || CS(i + 1, j);
            q.edge[2] = (j == nv - 1) || CS(i, j + 1);
            q.edge[3] = (i == 0) || CS(i - 1, j);
            q.corner[0] = physical(i, j);
            q.corner[1] = physical(i + 1, j);
            q.corner[2] = physical(i + 1, j + 1);
            q.corner[3] = physical(i, j + 1);
            out.push_back(q);
        }
}
}  // namespace

// rect_panel3d_discretize nodes/weights (src/shape/box3d.jl:44-59)
void Mesh::finalize() {
    const int np = nq * nq;
    pts.assign((size_t)npanels * np * 3, 0.0);
    w.assign((size_t)npanels * np, 0.0);
    for (int p = 0; p < npanels; ++p) {
        const double* cp = corners.data() + 12 * p;
        V3 a = ld(cp), b = ld(cp + 3), c = ld(cp + 6), d = ld(cp + 9);
        V3 cc = (((a + b) + c) + d) * 0.25;
        V3 bma = b - a, dma = d - a;
        double Lab = norm(bma), Lbc = norm(c - b);
        for (int i = 0; i < nq; ++i)
            for (int j = 0; j < nq; ++j) {
                size_t t = (size_t)p * np + i * nq + j;
                st(pts.data() + 3 * t, (cc + bma * (glx[i] / 2.0)) + dma * (glx[j] / 2.0));
                w[t] = glw[i] * glw[j] * Lab * Lbc / 4.0;
            }
    }
}

// t_P = (eps_out + eps_in) / (2 (eps_out - eps_in)) per node (src/solver/dielectric_box3d.jl:5-15)
void Mesh::diag(double* out) const {
    const int np = nq * nq;
    for (int p = 0; p < npanels; ++p) {
        double t = 0.5 * (eps_out[p] + eps_in[p]) / (eps_out[p] - eps_in[p]);
        for (int j = 0; j < np; ++j) out[(size_t)p * np + j] = t;
    }
}

int mesh_single_box(double Lx, double Ly, double Lz, int nq, double l_ec, double eps_in, double eps_out,
                    double alpha, Mesh& m, std::string& err) {
    if (nq < 1 || nq > 16) { err = "n_quad must be in [1, 16]"; return -1; }
    if (!(Lx > 0 && Ly > 0 && Lz > 0) || !(l_ec > 0)) { err = "box sides and l_ec must be positive"; return -1; }
    m = Mesh();
    init_rule(m, nq);
    Quad f[6];
    box_faces({0, 0, 0}, Lx, Ly, Lz, f);
    for (int i = 0; i < 6; ++i)
        if (int rc = mesh_face(m, f[i], alpha, l_ec, eps_in, eps_out, err)) return rc;
    m.finalize();
    return 0;
}

int mesh_multi_box(int nq, double l_ec, int nbox, const double* centers, const double* dims, const double* epses,
                   double eps_out, double alpha, Mesh& m, std::string& err) {
    if (nq < 1 || nq > 16) { err = "n_quad must be in [1, 16]"; return -1; }
    if (nbox < 1) { err = "at least one box is required"; return -1; }
    m = Mesh();
    init_rule(m, nq);
    struct Shared { std::array<V3, 4> r; int lo, hi; V3 n; };
    std::vector<Shared> shared;  // _detect_shared_faces_3d (src/shape/box3d_multi.jl:139-162)
    std::vector<std::array<Quad, 6>> faces(nbox);
    for (int b = 0; b < nbox; ++b)
        box_faces(ld(centers + 3 * b), dims[3 * b], dims[3 * b + 1], dims[3 * b + 2], faces[b].data());
    for (int i = 0; i < nbox; ++i)
        for (int j = i + 1; j < nbox; ++j)
            for (auto& f1 : faces[i])
                for (auto& f2 : faces[j]) {
                    V3 c2[4] = {f2.a, f2.b, f2.c, f2.d}, reg[4];
                    if (rect_overlap(f1, c2, f2.n, reg))
                        shared.push_back({{reg[0], reg[1], reg[2], reg[3]}, i, j, f1.n * -1.0});
                }
    // _multi_box3d_face_regions (src/shape/box3d_multi.jl:313-356)
    for (int b = 0; b < nbox; ++b)
        for (auto& f : faces[b]) {
            std::vector<std::array<V3, 4>> fs;
            for (auto& s : shared) {
                if (b != s.lo && b != s.hi) continue;
                V3 c2[4] = {s.r[0], s.r[1], s.r[2], s.r[3]}, reg[4];
                if (rect_overlap(f, c2, f.n * -1.0, reg)) fs.push_back({reg[0], reg[1], reg[2], reg[3]});
            }
            std::vector<Quad> rem;
            subtract_rects(f, fs, rem);
            for (auto& q : rem)
                if (int rc = mesh_face(m, q, alpha, l_ec, epses[b], eps_out, err)) return rc;
        }
    for (auto& s : shared) {
        Quad q;
        q.a = s.r[0]; q.b = s.r[1]; q.c = s.r[2]; q.d = s.r[3]; q.n = s.n;
        for (int k = 0; k < 4; ++k) q.corner[k] = q.edge[k] = true;
        if (int rc = mesh_face(m, q, alpha, l_ec, epses[s.hi], epses[s.lo], err)) return rc;
    }
    m.finalize();
    return 0;
}

int mesh_from_panels(int P, int nq, const double* corners, const double* normals, const int* is_edge,
                     const double* eps_in, const double* eps_out, Mesh& m, std::string& err) {
    if (nq < 1 || nq > 16 || P < 0) { err = "bad panel count or n_quad"; return -1; }
    m = Mesh();
    init_rule(m, nq);
    m.npanels = P;
    m.corners.assign(corners, corners + 12 * (size_t)P);
    m.normals.assign(normals, normals + 3 * (size_t)P);
    m.is_edge.assign(is_edge, is_edge + P);
    m.eps_in.assign(eps_in, eps_in + P);
    m.eps_out.assign(eps_out, eps_out + P);
    m.finalize();
    return 0;
}

// ---------------------------------------------------------------------------
// Near-field list and correction blocks
// ---------------------------------------------------------------------------
namespace {

// bernstein_rho_panel (src/utils/bernstein.jl:12-62)
double rho_pole(std::complex<double> z) {
    std::complex<double> s = std::sqrt(z * z - 1.0);
    return std::max(std::abs(z + s), std::abs(z - s));
}

struct PanelFrame {
    V3 cc, e1, e2, n, bma, dma;
    double L1, L2, lmax, scale;
};

PanelFrame frame(const Mesh& m, int p) {
    const double* c = m.corners.data() + 12 * p;
    V3 a = ld(c), b = ld(c + 3), cc3 = ld(c + 6), d = ld(c + 9);
    PanelFrame f;
    f.cc = (((a + b) + cc3) + d) * 0.25;
    f.bma = b - a; f.dma = d - a;
    double l1 = norm(f.bma), l2 = norm(f.dma);
    f.L1 = l1 / 2; f.L2 = l2 / 2;
    f.e1 = f.bma * (1.0 / l1); f.e2 = f.dma * (1.0 / l2);
    f.n = ld(m.normals.data() + 3 * p);
    f.lmax = std::max(norm(a - b), norm(b - cc3));
    f.scale = l1 * l2 / 4;
    return f;
}

double bernstein_rho(const PanelFrame& f, V3 trg) {
    V3 r = trg - f.cc;
    double xt = dot(r, f.e1), yt = dot(r, f.e2), zt = dot(r, f.n);
    double dy = yt - std::clamp(yt, -f.L2, f.L2);
    double rho1 = rho_pole(std::complex<double>(xt, std::sqrt(dy * dy + zt * zt)) / f.L1);
    double dx = xt - std::clamp(xt, -f.L1, f.L1);
    double rho2 = rho_pole(std::complex<double>(yt, std::sqrt(dx * dx + zt * zt)) / f.L2);
    return std::min(rho1, rho2);
}

// Uniform cell grid over points for range queries (replaces the KD-tree
// prefilter; the exact classification that follows decides).
struct Grid {
    double h;
    V3 lo;
    int nx, ny, nz;
    std::vector<int64_t> start, idx;
    void build(const double* p, int64_t n, double cell) {
        lo = {INFINITY, INFINITY, INFINITY};
        V3 hi{-INFINITY, -INFINITY, -INFINITY};
        for (int64_t i = 0; i < n; ++i) {
            lo.x = std::min(lo.x, p[3 * i]); lo.y = std::min(lo.y, p[3 * i + 1]); lo.z = std::min(lo.z, p[3 * i + 2]);
            hi.x = std::max(hi.x, p[3 * i]); hi.y = std::max(hi.y, p[3 * i + 1]); hi.z = std::max(hi.z, p[3 * i + 2]);
        }
        h = cell;
        auto dim = [&](double a, double b) { return std::max(1, std::min(1 << 10, (int)std::floor((b - a) / h) + 1)); };
        nx = dim(lo.x, hi.x); ny = dim(lo.y, hi.y); nz = dim(lo.z, hi.z);
        std::vector<int64_t> cnt((size_t)nx * ny * nz + 1, 0);
        std::vector<int64_t> cell_of(n);
        for (int64_t i = 0; i < n; ++i) {
            cell_of[i] = key(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
            cnt[cell_of[i] + 1]++;
        }
        for (size_t c = 1; c < cnt.size(); ++c) cnt[c] += cnt[c - 1];
        start = cnt;
        idx.assign(n, 0);
        for (int64_t i = 0; i < n; ++i) idx[cnt[cell_of[i]]++] = i;
    }
    int ci(double v, double l, int nmax) const { return std::clamp((int)std::floor((v - l) / h), 0, nmax - 1); }
    int64_t key(double x, double y, double z) const {
        return ((int64_t)ci(x, lo.x, nx) * ny + ci(y, lo.y, ny)) * nz + ci(z, lo.z, nz);
    }
    template <class F>
    void query(V3 c, double r, const double* p, F&& f) const {
        int x0 = ci(c.x - r, lo.x, nx), x1 = ci(c.x + r, lo.x, nx);
        int y0 = ci(c.y - r, lo.y, ny), y1 = ci(c.y + r, lo.y, ny);
        int z0 = ci(c.z - r, lo.z, nz), z1 = ci(c.z + r, lo.z, nz);
        for (int x = x0; x <= x1; ++x)
            for (int y = y0; y <= y1; ++y)
                for (int z = z0; z <= z1; ++z) {
                    int64_t k = ((int64_t)x * ny + y) * nz + z;
                    for (int64_t e = start[k]; e < start[k + 1]; ++e) {
                        int64_t i = idx[e];
                        V3 d = ld(p + 3 * i) - c;
                        if (std::sqrt(dot(d, d)) <= r) f(i);
                    }
                }
    }
};

// barycentric_row! (src/utils/barycentric.jl:19-42)
void bary_row(int n, const double* x, const double* lam, double xq, double* r) {
    const double rt = 1.4901161193847656e-08;  // isapprox default rtol = sqrt(eps)
    for (int i = 0; i < n; ++i)
        if (xq == x[i] || std::fabs(xq - x[i]) <= rt * std::max(std::fabs(xq), std::fabs(x[i]))) {
            for (int k = 0; k < n; ++k) r[k] = 0.0;
            r[i] = 1.0;
            return;
        }
    double den = 0.0;
    for (int i = 0; i < n; ++i) { r[i] = lam[i] / (xq - x[i]); den += r[i]; }
    double inv = 1.0 / den;
    for (int i = 0; i < n; ++i) r[i] *= inv;
}

// Direct block K[t, s] = grad(y_s, x_t, n_trg) w_s (laplace3d_DT_panel, src/kernel/laplace3d_near.jl:25-34).
void direct_block(const Mesh& m, int src, int trg, double* K) {
    const int np = m.nq * m.nq;
    V3 nt = ld(m.normals.data() + 3 * trg);
    for (int t = 0; t < np; ++t) {
        V3 xt = ld(m.pts.data() + 3 * ((size_t)trg * np + t));
        for (int s = 0; s < np; ++s) {
            size_t js = (size_t)src * np + s;
            K[t * np + s] = lap_grad(ld(m.pts.data() + 3 * js), xt, nt) * m.w[js];
        }
    }
}

// build_source_cache (src/kernel/laplace3d_near_upsampling.jl:8-50)
struct SourceCache {
    int n_up = 0;
    std::vector<V3> p_up;    // n_up^2, alpha = i_up * n_up + j_up
    std::vector<double> Mt;  // nq^2 x n_up^2
};

void source_cache(const Mesh& m, int src, int n_up, SourceCache& sc) {
    const int nq = m.nq, nu2 = n_up * n_up;
    std::vector<double> xu(n_up), wu(n_up), Ex((size_t)n_up * nq);
    gauss_legendre(n_up, xu.data(), wu.data());
    for (int i = 0; i < n_up; ++i) bary_row(nq, m.glx.data(), m.bary.data(), xu[i], Ex.data() + (size_t)i * nq);
    PanelFrame f = frame(m, src);
    sc.n_up = n_up;
    sc.p_up.resize(nu2);
    for (int i = 0; i < n_up; ++i)
        for (int j = 0; j < n_up; ++j) sc.p_up[i * n_up + j] = (f.cc + f.bma * (xu[i] / 2)) + f.dma * (xu[j] / 2);
    sc.Mt.assign((size_t)nq * nq * nu2, 0.0);
    for (int mx = 0; mx < nq; ++mx)
        for (int my = 0; my < nq; ++my)
            for (int i = 0; i < n_up; ++i)
                for (int j = 0; j < n_up; ++j)
                    sc.Mt[(size_t)(mx * nq + my) * nu2 + i * n_up + j] =
                        f.scale * wu[i] * wu[j] * Ex[(size_t)i * nq + mx] * Ex[(size_t)j * nq + my];
}

// Upsampled block (src/kernel/laplace3d_near_upsampling.jl:184-203): Kb[t, m] = sum_alpha Mt[m, alpha] K(alpha, t)
void upsampled_block(const Mesh& m, const SourceCache& sc, int trg, double* Kb, std::vector<double>& kmat) {
    const int np = m.nq * m.nq, nu2 = sc.n_up * sc.n_up;
    V3 nt = ld(m.normals.data() + 3 * trg);
    kmat.resize((size_t)nu2 * np);
    for (int t = 0; t < np; ++t) {
        V3 xt = ld(m.pts.data() + 3 * ((size_t)trg * np + t));
        for (int a = 0; a < nu2; ++a) kmat[(size_t)t * nu2 + a] = lap_grad(sc.p_up[a], xt, nt);
    }
    for (int t = 0; t < np; ++t)
        for (int mm = 0; mm < np; ++mm) {
            const double* mt = sc.Mt.data() + (size_t)mm * nu2;
            const double* kv = kmat.data() + (size_t)t * nu2;
            double acc = 0.0;
            for (int a = 0; a < nu2; ++a) acc += mt[a] * kv[a];
            Kb[t * np + mm] = acc;
        }
}

// Adaptive quadtree for touching pairs (src/kernel/laplace3d_near_adaptive.jl:119-224, 308-387).
struct Adaptive {
    const Mesh* m;
    PanelFrame f;
    int nGL;
    std::vector<double> xg, wg;
    double atol, rtol;
    int max_depth;
    bool hit = false;
    std::vector<std::array<double, 4>> leaves;

    void moments(V3 pt, V3 nt, double ulo, double uhi, double vlo, double vhi, double* out) const {
        const int nq = m->nq;
        double rx[16], ry[16];
        std::fill(out, out + nq * nq, 0.0);
        double hu = (uhi - ulo) / 2, hv = (vhi - vlo) / 2, mu = (uhi + ulo) / 2, mv = (vhi + vlo) / 2;
        double sc = hu * hv * f.scale;
        for (int gi = 0; gi < nGL; ++gi) {
            double u = mu + hu * xg[gi];
            bary_row(nq, m->glx.data(), m->bary.data(), u, rx);
            for (int gj = 0; gj < nGL; ++gj) {
                double v = mv + hv * xg[gj];
                bary_row(nq, m->glx.data(), m->bary.data(), v, ry);
                V3 y = (f.cc + f.bma * (u / 2)) + f.dma * (v / 2);
                double ww = wg[gi] * wg[gj] * sc * lap_grad(y, pt, nt);
                for (int a = 0; a < nq; ++a)
                    for (int b = 0; b < nq; ++b) out[a * nq + b] += ww * rx[a] * ry[b];
            }
        }
    }

    void walk(V3 pt, V3 nt, double ulo, double uhi, double vlo, double vhi, int depth) {
        const int n2 = m->nq * m->nq;
        double par[256], c[4][256];
        moments(pt, nt, ulo, uhi, vlo, vhi, par);
        double mu = (uhi + ulo) / 2, mv = (vhi + vlo) / 2;
        const double cell[4][4] = {{ulo, mu, vlo, mv}, {mu, uhi, vlo, mv}, {ulo, mu, mv, vhi}, {mu, uhi, mv, vhi}};
        for (int k = 0; k < 4; ++k) moments(pt, nt, cell[k][0], cell[k][1], cell[k][2], cell[k][3], c[k]);
        double err = -INFINITY, pmax = -INFINITY;
        for (int i = 0; i < n2; ++i) {
            double ch = ((c[0][i] + c[1][i]) + c[2][i]) + c[3][i];
            err = std::max(err, std::fabs(par[i] - ch));
            pmax = std::max(pmax, std::fabs(par[i]));
        }
        double tl = std::max(atol, rtol * pmax);
        if (err < tl || depth == max_depth) {
            for (int k = 0; k < 4; ++k) leaves.push_back({cell[k][0], cell[k][1], cell[k][2], cell[k][3]});
            if (depth == max_depth && err >= tl) hit = true;
            return;
        }
        for (int k = 0; k < 4; ++k) walk(pt, nt, cell[k][0], cell[k][1], cell[k][2], cell[k][3], depth + 1);
    }

    // Block moments for all targets of the target panel over the recorded leaves.
    void block(int trg, double* Kb) const {
        const int nq = m->nq, np = nq * nq;
        V3 nt = ld(m->normals.data() + 3 * trg);
        std::fill(Kb, Kb + np * np, 0.0);
        double rx[16], ry[16], kv[256];
        for (auto& L : leaves) {
            double hu = (L[1] - L[0]) / 2, hv = (L[3] - L[2]) / 2, mu = (L[1] + L[0]) / 2, mv = (L[3] + L[2]) / 2;
            double sc = hu * hv * f.scale;
            for (int gi = 0; gi < nGL; ++gi) {
                double u = mu + hu * xg[gi];
                bary_row(nq, m->glx.data(), m->bary.data(), u, rx);
                for (int gj = 0; gj < nGL; ++gj) {
                    double v = mv + hv * xg[gj];
                    bary_row(nq, m->glx.data(), m->bary.data(), v, ry);
                    V3 y = (f.cc + f.bma * (u / 2)) + f.dma * (v / 2);
                    double wuv = wg[gi] * wg[gj] * sc;
                    for (int t = 0; t < np; ++t) kv[t] = lap_grad(y, ld(m->pts.data() + 3 * ((size_t)trg * np + t)), nt);
                    for (int a = 0; a < nq; ++a)
                        for (int b = 0; b < nq; ++b) {
                            double wm = wuv * rx[a] * ry[b];
                            for (int t = 0; t < np; ++t) Kb[t * np + a * nq + b] += wm * kv[t];
                        }
                }
            }
        }
    }
};
}  // namespace

int near_build(const Mesh& m, const NearOpts& o, Near& out, std::string& err) {
    const int P = m.npanels, nq = m.nq, np = nq * nq;
    const int64_t N = m.npoints();
    if (o.max_order < 1 || o.max_order > 64) { err = "max_order must be in [1, 64]"; return -1; }
    if (!(o.up_tol > 0 && o.up_tol < 1)) { err = "up_tol must be in (0, 1)"; return -1; }
    out = Near();
    out.nb = np;
    std::vector<PanelFrame> fr(P);
    std::vector<double> offs(P);
    double Lmax = P > 0 ? -INFINITY : 1.0;
    for (int p = 0; p < P; ++p) {
        fr[p] = frame(m, p);
        offs[p] = dot(fr[p].n, ld(m.corners.data() + 12 * p));
        Lmax = std::max(Lmax, fr[p].lmax);
    }
    const double same_tol = std::sqrt(DBL_EPSILON);
    const double tol_corner = std::sqrt(DBL_EPSILON) * Lmax;
    const double rho_star = std::pow(o.up_tol, -1.0 / (2.0 * nq));
    const double As = (rho_star + 1.0 / rho_star) / 2, Bs = (rho_star - 1.0 / rho_star) / 2;
    const double rfac = 1.05 * std::sqrt(As * As + (1.0 + Bs) * (1.0 + Bs) + Bs * Bs);
    // prefilter radius r_i = 1.05 * L_half * sqrt(A*^2 + (1+B*)^2 + B*^2)  (laplace3d_near.jl:317-322)
    double rmed = 0.0;
    {
        std::vector<double> rs(P);
        for (int p = 0; p < P; ++p) rs[p] = rfac * fr[p].lmax / 2;
        if (P) { std::nth_element(rs.begin(), rs.begin() + P / 2, rs.end()); rmed = rs[P / 2]; }
    }
    Grid grid;
    if (N > 0) grid.build(m.pts.data(), N, std::max(rmed, 1e-12));
    // corner hash for touching detection (laplace3d_near.jl:282-298, 335-352)
    Grid cgrid;
    std::vector<double> cpts((size_t)4 * P * 3);
    for (int p = 0; p < P; ++p) std::copy(m.corners.begin() + 12 * p, m.corners.begin() + 12 * p + 12, cpts.begin() + 12 * p);
    if (P > 0) cgrid.build(cpts.data(), 4 * (int64_t)P, std::max(Lmax / 4, 1e-12));

    const auto t_start = std::chrono::steady_clock::now();
    const double log_atol = std::log(o.up_tol);
    std::vector<std::vector<std::pair<int, int>>> ups(P);  // per source: (target, p_up)
    std::vector<std::vector<int>> adp(P);
#ifdef _OPENMP
    int nth = o.nthreads > 0 ? o.nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nth)
#endif
    for (int i = 0; i < P; ++i) {
        if (!o.correct_edges && m.is_edge[i]) continue;
        const double r_i = rfac * fr[i].lmax / 2;
        std::unordered_map<int, double> rho_min;  // target panel -> min rho over in-range nodes
        grid.query(fr[i].cc, r_i, m.pts.data(), [&](int64_t t) {
            int j = (int)(t / np);
            if (j == i) return;
            double rho = bernstein_rho(fr[i], ld(m.pts.data() + 3 * t));
            auto it = rho_min.find(j);
            if (it == rho_min.end()) rho_min.emplace(j, rho);
            else if (rho < it->second) it->second = rho;
        });
        std::vector<int> touching;
        if (o.correct_edges)
            for (int ck = 0; ck < 4; ++ck) {
                V3 cp = ld(m.corners.data() + 12 * i + 3 * ck);
                cgrid.query(cp, tol_corner, cpts.data(), [&](int64_t e) {
                    int j = (int)(e / 4);
                    if (j != i) touching.push_back(j);
                });
            }
        std::sort(touching.begin(), touching.end());
        touching.erase(std::unique(touching.begin(), touching.end()), touching.end());
        std::vector<int> cand;
        for (auto& kv : rho_min) cand.push_back(kv.first);
        cand.insert(cand.end(), touching.begin(), touching.end());
        std::sort(cand.begin(), cand.end());
        cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
        for (int j : cand) {
            if (!o.correct_edges && m.is_edge[j]) continue;
            if (dot(fr[i].n, fr[j].n) > 1 - same_tol &&
                std::fabs(offs[i] - offs[j]) <= same_tol * std::max(1.0, fr[i].lmax))
                continue;  // same plane: the D^T kernel vanishes
            if (o.correct_edges && std::binary_search(touching.begin(), touching.end(), j)) {
                adp[i].push_back(j);
                continue;
            }
            auto it = rho_min.find(j);
            if (it == rho_min.end()) continue;
            double rmin = it->second;
            if (!(rmin <= rho_star)) continue;
            int p_up = rmin > 1.0 ? (int)std::ceil(-log_atol / (2.0 * std::log(rmin))) : o.max_order;
            p_up = std::clamp(p_up, nq, o.max_order);
            ups[i].push_back({j, p_up});
        }
    }
    for (int i = 0; i < P; ++i) {
        for (auto& e : ups[i]) { out.ups_i.push_back(i); out.ups_j.push_back(e.first); out.ups_p.push_back(e.second); }
        for (int j : adp[i]) { out.adp_i.push_back(i); out.adp_j.push_back(j); }
    }

    const auto t_list = std::chrono::steady_clock::now();
    double t_ups = 0.0, t_adp = 0.0, t_walk = 0.0;  // thread-seconds per block kind (BIE_TRACE)
    int64_t n_leaves = 0;
    // Blocks, computed per source panel (one upsampling order per source: the max
    // over its upsample neighbours, laplace3d_near_upsampling.jl:164-183).
    struct Blk { int row, col; std::vector<double> v; };
    std::vector<std::vector<Blk>> per_src(P);
    // adaptive pairs whose moment sums run on the GPU: (target, leaves) per source
    const bool gpu_adp = o.device >= 0 && nq <= 6;
    struct AdpJob { int j; std::vector<std::array<double, 4>> leaves; };
    std::vector<std::vector<AdpJob>> adp_jobs(gpu_adp ? P : 0);
    // upsampled blocks of sources whose order is at most 8 run on the GPU too
    const bool gpu_ups = o.device >= 0 && nq <= 6;
    std::vector<int> ups_order(P, 0);  // > 0: this source's upsampled blocks go to the GPU
    const int nGL = o.adaptive_n_GL == 0 ? nq : o.adaptive_n_GL;
    int hit_any = 0;
    const double aatol = o.adaptive_atol < 0 ? o.up_tol : o.adaptive_atol;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) num_threads(nth) reduction(| : hit_any) reduction(+ : t_ups, t_adp, t_walk, n_leaves)
#endif
    for (int i = 0; i < P; ++i) {
        if (ups[i].empty() && adp[i].empty()) continue;
        const auto t0 = std::chrono::steady_clock::now();
        std::vector<double> Kb((size_t)np * np), Kd((size_t)np * np), kmat;
        auto emit = [&](int j) {
            Blk b{j, i, std::vector<double>((size_t)np * np)};
            for (int s = 0; s < np; ++s)
                for (int r = 0; r < np; ++r) b.v[(size_t)s * np + r] = Kb[(size_t)r * np + s] - Kd[(size_t)r * np + s];
            per_src[i].push_back(std::move(b));
        };
        if (!ups[i].empty()) {
            int nup = 0;
            for (auto& e : ups[i]) nup = std::max(nup, e.second);
            if (gpu_ups && nup <= 8) {
                ups_order[i] = nup;
                nup = 0;  // nothing to do on the host
            }
        }
        if (!ups[i].empty() && ups_order[i] == 0) {
            int nup = 0;
            for (auto& e : ups[i]) nup = std::max(nup, e.second);
            SourceCache sc;
            source_cache(m, i, nup, sc);
            for (auto& e : ups[i]) {
                upsampled_block(m, sc, e.first, Kb.data(), kmat);
                direct_block(m, i, e.first, Kd.data());
                emit(e.first);
            }
        }
        const auto t1 = std::chrono::steady_clock::now();
        t_ups += std::chrono::duration<double>(t1 - t0).count();
        for (int j : adp[i]) {
            Adaptive A;
            A.m = &m; A.f = fr[i];
            A.nGL = o.adaptive_n_GL == 0 ? nq : o.adaptive_n_GL;
            A.xg.resize(A.nGL); A.wg.resize(A.nGL);
            gauss_legendre(A.nGL, A.xg.data(), A.wg.data());
            A.atol = aatol; A.rtol = o.adaptive_rtol; A.max_depth = o.adaptive_max_depth;
            // representative target: node of panel j nearest the first corner of panel i
            V3 c1 = ld(m.corners.data() + 12 * i);
            int rep = 0;
            double best = INFINITY;
            for (int t = 0; t < np; ++t) {
                double d = norm(ld(m.pts.data() + 3 * ((size_t)j * np + t)) - c1);
                if (d < best) { best = d; rep = t; }
            }
            const auto tw = std::chrono::steady_clock::now();
            A.walk(ld(m.pts.data() + 3 * ((size_t)j * np + rep)), ld(m.normals.data() + 3 * j), -1, 1, -1, 1, 0);
            t_walk += std::chrono::duration<double>(std::chrono::steady_clock::now() - tw).count();
            n_leaves += (int64_t)A.leaves.size();
            if (A.hit) hit_any = 1;
            if (gpu_adp) {
                adp_jobs[i].push_back({j, std::move(A.leaves)});
                continue;
            }
            A.block(j, Kb.data());
            direct_block(m, i, j, Kd.data());
            emit(j);
        }
        t_adp += std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
    }
    if (gpu_adp) {
        // one launch for every adaptive pair, then the direct blocks and the differences
        std::vector<int> trg;
        std::vector<double> frames, leaves;
        std::vector<int64_t> off{0};
        for (int i = 0; i < P; ++i)
            for (auto& jb : adp_jobs[i]) {
                trg.push_back(jb.j);
                const PanelFrame& f = fr[i];
                const double fv[10] = {f.cc.x, f.cc.y, f.cc.z, f.bma.x, f.bma.y, f.bma.z,
                                       f.dma.x, f.dma.y, f.dma.z, f.scale};
                frames.insert(frames.end(), fv, fv + 10);
                for (auto& L : jb.leaves) leaves.insert(leaves.end(), L.begin(), L.end());
                off.push_back((int64_t)leaves.size() / 4);
            }
        const int npairs = (int)trg.size();
        std::vector<double> Kball((size_t)npairs * np * np);
        std::vector<double> xg(nGL), wg(nGL);
        gauss_legendre(nGL, xg.data(), wg.data());
        if (adaptive_blocks_gpu(o.device, nq, nGL, m.glx.data(), m.bary.data(), xg.data(), wg.data(), m.pts.data(),
                                N, m.normals.data(), P, npairs, trg.data(), frames.data(), off.data(), leaves.data(),
                                Kball.data(), err) != 0)
            return -1;
        std::vector<int64_t> first(P + 1, 0);
        for (int i = 0; i < P; ++i) first[i + 1] = first[i] + (int64_t)adp_jobs[i].size();
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 4) num_threads(nth)
#endif
        for (int i = 0; i < P; ++i) {
            std::vector<double> Kd((size_t)np * np);
            for (size_t q = 0; q < adp_jobs[i].size(); ++q) {
                const int j = adp_jobs[i][q].j;
                const double* Kb = Kball.data() + (size_t)(first[i] + (int64_t)q) * np * np;
                direct_block(m, i, j, Kd.data());
                Blk b{j, i, std::vector<double>((size_t)np * np)};
                for (int s = 0; s < np; ++s)
                    for (int r = 0; r < np; ++r) b.v[(size_t)s * np + r] = Kb[(size_t)r * np + s] - Kd[(size_t)r * np + s];
                per_src[i].push_back(std::move(b));
            }
        }
    }
    if (gpu_ups) {
        // one launch for every source panel with GPU-side upsampled blocks
        std::vector<int> js, jn, tg;
        std::vector<double> jf;
        std::vector<int64_t> toff{0};
        for (int i = 0; i < P; ++i) {
            if (!ups_order[i]) continue;
            js.push_back(i);
            jn.push_back(ups_order[i]);
            const PanelFrame& f = fr[i];
            const double fv[10] = {f.cc.x, f.cc.y, f.cc.z, f.bma.x, f.bma.y, f.bma.z, f.dma.x, f.dma.y, f.dma.z, f.scale};
            jf.insert(jf.end(), fv, fv + 10);
            for (auto& e : ups[i]) tg.push_back(e.first);
            toff.push_back((int64_t)tg.size());
        }
        if (!js.empty()) {
            // Gauss nodes, weights and barycentric rows per order (as source_cache computes them)
            const int T = 9;
            std::vector<double> xu((size_t)T * T, 0.0), wu((size_t)T * T, 0.0), ex((size_t)T * T * nq, 0.0);
            for (int n = 1; n <= 8; ++n) {
                gauss_legendre(n, xu.data() + (size_t)n * T, wu.data() + (size_t)n * T);
                for (int a = 0; a < n; ++a)
                    bary_row(nq, m.glx.data(), m.bary.data(), xu[(size_t)n * T + a], ex.data() + ((size_t)n * T + a) * nq);
            }
            std::vector<double> blocks((size_t)tg.size() * np * np);
            if (upsampled_blocks_gpu(o.device, nq, m.pts.data(), N, m.w.data(), m.normals.data(), P, (int)js.size(),
                                     js.data(), jn.data(), jf.data(), toff.data(), tg.data(), xu.data(), wu.data(),
                                     ex.data(), blocks.data(), err) != 0)
                return -1;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 4) num_threads(nth)
#endif
            for (int q = 0; q < (int)js.size(); ++q) {
                const int i = js[q];
                for (int64_t p = toff[q]; p < toff[q + 1]; ++p) {
                    const double* b = blocks.data() + (size_t)p * np * np;
                    per_src[i].push_back(Blk{tg[p], i, std::vector<double>(b, b + (size_t)np * np)});
                }
            }
        }
    }
    out.hit_max = hit_any;
    if (std::getenv("BIE_TRACE")) {
        const double dl = std::chrono::duration<double>(t_list - t_start).count();
        const double db = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_list).count();
        std::fprintf(stderr,
                     "[bie] near_build: %d panels, neighbour lists %.3f s, blocks %.3f s (thread-seconds: "
                     "upsampled %.3f, adaptive %.3f of which tree walks %.3f; %zu upsampled and %zu adaptive pairs, "
                     "%lld leaves)\n",
                     P, dl, db, t_ups, t_adp, t_walk, out.ups_i.size(), out.adp_i.size(), (long long)n_leaves);
    }
    // assemble BSR (rows = target panels), columns sorted within each row
    std::vector<std::vector<std::pair<int, const Blk*>>> rows(P);
    for (int i = 0; i < P; ++i)
        for (auto& b : per_src[i]) rows[b.row].push_back({b.col, &b});
    out.rowptr.assign(P + 1, 0);
    for (int r = 0; r < P; ++r) {
        std::sort(rows[r].begin(), rows[r].end(), [](auto& a, auto& b) { return a.first < b.first; });
        out.rowptr[r + 1] = out.rowptr[r] + (int32_t)rows[r].size();
    }
    out.col.resize(out.rowptr[P]);
    out.val.resize((size_t)out.rowptr[P] * np * np);
    for (int r = 0; r < P; ++r)
        for (size_t e = 0; e < rows[r].size(); ++e) {
            size_t b = (size_t)out.rowptr[r] + e;
            out.col[b] = rows[r][e].first;
            std::copy(rows[r][e].second->v.begin(), rows[r][e].second->v.end(), out.val.begin() + b * np * np);
        }
    return 0;
}

}  // namespace bie

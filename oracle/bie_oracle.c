/*
 * bie_oracle.c -- CPU restatement (FP64, plain C99 + OpenMP) of the reference's
 * layer-potential hot path, used ONLY as test infrastructure: the parity checker
 * for the CUDA library and the timed CPU baseline of the benchmark. Nothing in the
 * product links, imports or calls this file.
 *
 * Reference: xuanzhaogao/DielectricBIE.jl (Julia). The Julia toolchain is absent,
 * so the reference cannot be executed; this file follows its source line by line,
 * with each function citing the file:line it restates. Third-party arithmetic
 * restated here:
 *   - FastGaussQuadrature.jl 1.1.0 `gausslegendre` (closed forms for n <= 5,
 *     Newton iteration on the three-term Legendre recurrence for n > 5);
 *   - NearestNeighbors.jl 0.4.20 `KDTree/inrange`: a candidate prefilter only,
 *     replaced by an exact brute-force range test (same result set);
 *   - Krylov.jl 0.10.2 `gmres`: full (unrestarted) GMRES with modified Gram-Schmidt
 *     and Givens rotations, x0 = 0, stop when the residual estimate drops to
 *     atol + rtol*||b||;
 *   - FMM3D.jl `lfmm3d`: replaced by the exact direct sum it approximates.
 *
 * Pinned by the reference's own known-answer tests (tests/test_oracle_*.py):
 * best_grid values, Gauss flux, total polarisation charge, panel D^T vs loop,
 * corrections == explicit blocks, n_up == n_quad => zero correction, neighbour
 * classification, adaptive moments vs cubature, touching-pair regression.
 */
#include <complex.h>
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define FOUR_PI (4.0 * M_PI)

/* ------------------------------------------------------------------------- */
/* Gauss-Legendre nodes/weights (FastGaussQuadrature.jl 1.1.0 gausslegendre). */
/* Called at src/shape/box3d_single.jl:50 and                                 */
/* src/kernel/laplace3d_near_upsampling.jl:9. Ascending nodes.                */
/* ------------------------------------------------------------------------- */
void orc_gausslegendre(int n, double* x, double* w) {
    if (n <= 0) return;
    if (n == 1) { x[0] = 0.0; w[0] = 2.0; return; }
    if (n == 2) {
        x[0] = -1.0 / sqrt(3.0); x[1] = 1.0 / sqrt(3.0);
        w[0] = 1.0; w[1] = 1.0; return;
    }
    if (n == 3) {
        x[0] = -sqrt(3.0 / 5.0); x[1] = 0.0; x[2] = sqrt(3.0 / 5.0);
        w[0] = 5.0 / 9.0; w[1] = 8.0 / 9.0; w[2] = 5.0 / 9.0; return;
    }
    if (n == 4) {
        double a = 2.0 / 7.0 * sqrt(6.0 / 5.0);
        x[0] = -sqrt(3.0 / 7.0 + a); x[1] = -sqrt(3.0 / 7.0 - a);
        x[2] = sqrt(3.0 / 7.0 - a);  x[3] = sqrt(3.0 / 7.0 + a);
        w[0] = (18.0 - sqrt(30.0)) / 36.0; w[1] = (18.0 + sqrt(30.0)) / 36.0;
        w[2] = w[1]; w[3] = w[0]; return;
    }
    if (n == 5) {
        double b = 2.0 * sqrt(10.0 / 7.0);
        x[0] = -sqrt(5.0 + b) / 3.0; x[1] = -sqrt(5.0 - b) / 3.0; x[2] = 0.0;
        x[3] = sqrt(5.0 - b) / 3.0;  x[4] = sqrt(5.0 + b) / 3.0;
        w[0] = (322.0 - 13.0 * sqrt(70.0)) / 900.0; w[1] = (322.0 + 13.0 * sqrt(70.0)) / 900.0;
        w[2] = 128.0 / 225.0; w[3] = w[1]; w[4] = w[0]; return;
    }
    /* Newton on P_n from the Tricomi-type initial guess; evaluate P_n and P_n'
     * through the three-term recurrence in long double; symmetrise. */
    int m = (n + 1) / 2;
    for (int i = 0; i < m; ++i) {
        long double z = cosl(M_PI * ((long double)i + 0.75L) / ((long double)n + 0.5L));
        long double dp = 0.0L;
        for (int it = 0; it < 100; ++it) {
            long double p0 = 1.0L, p1 = z;
            for (int k = 2; k <= n; ++k) {
                long double p2 = ((2.0L * k - 1.0L) * z * p1 - (k - 1.0L) * p0) / (long double)k;
                p0 = p1; p1 = p2;
            }
            dp = (long double)n * (z * p1 - p0) / (z * z - 1.0L);
            long double dz = p1 / dp;
            z -= dz;
            if (fabsl(dz) < 1e-19L) break;
        }
        {
            long double p0 = 1.0L, p1 = z;
            for (int k = 2; k <= n; ++k) {
                long double p2 = ((2.0L * k - 1.0L) * z * p1 - (k - 1.0L) * p0) / (long double)k;
                p0 = p1; p1 = p2;
            }
            dp = (long double)n * (z * p1 - p0) / (z * z - 1.0L);
        }
        long double wi = 2.0L / ((1.0L - z * z) * dp * dp);
        x[i] = -(double)z;          /* z ~ cos(small angle) is the largest node */
        x[n - 1 - i] = (double)z;
        w[i] = (double)wi;
        w[n - 1 - i] = (double)wi;
    }
    if (n % 2 == 1) x[n / 2] = 0.0;
}

/* ------------------------------------------------------------------------- */
/* best_grid  (src/utils/best_grid.jl:8-118)                                 */
/* returns 0 on success, -1 for an ArgumentError on inputs, -2 if not found  */
/* ------------------------------------------------------------------------- */
static double bg_aspect(double W, double H, long m, long n) {
    double ratio = (W * (double)n) / (H * (double)m);
    return ratio >= 1.0 ? ratio : 1.0 / ratio;
}

int orc_best_grid(double W, double H, double alpha, int* out_m, int* out_n) {
    const long max_den = 1000000; const int max_iter = 10000; const double frac_tol = 1e-12;
    if (!(W > 0 && H > 0)) return -1;
    if (alpha < 1) return -1;
    int swapped = 0;
    if (W < H) { double t = W; W = H; H = t; swapped = 1; }
    double r = W / H;
    long best_m = 0, best_n = 0, best_N = LONG_MAX; double best_rho = INFINITY;
#define BG_CONSIDER(MM, NN) do { long _m = (MM), _n = (NN);                        \
        if (_m > 0 && _n > 0 && _m <= max_den && _n <= max_den) {                \
            double _rho = bg_aspect(W, H, _m, _n);                                \
            if (_rho <= alpha) { long _N = _m * _n;                               \
                if (_N < best_N || (_N == best_N && _rho < best_rho)) {           \
                    best_m = _m; best_n = _n; best_N = _N; best_rho = _rho; } } } \
    } while (0)
    long pmm = 0, pm = 1, qmm = 1, qm = 0;
    double xx = r;
    for (int it = 0; it < max_iter; ++it) {
        long a = (long)floor(xx);
        long p = a * pm + pmm, q = a * qm + qmm;
        BG_CONSIDER(p, q);
        if (a > 1) {
            long t_max = a - 1;
            if (pm > 0) { long c = (max_den - pmm) / pm; if (c < t_max) t_max = c; }
            if (qm > 0) { long c = (max_den - qmm) / qm; if (c < t_max) t_max = c; }
            for (long t = 1; t <= t_max; ++t) BG_CONSIDER(t * pm + pmm, t * qm + qmm);
        }
        double frac = xx - (double)a;
        if (fabs(frac) <= frac_tol) break;
        pmm = pm; pm = p; qmm = qm; qm = q;
        xx = 1.0 / frac;
    }
#undef BG_CONSIDER
    if (best_m == 0) return -2;
    if (swapped) { long t = best_m; best_m = best_n; best_n = t; }
    *out_m = (int)best_m; *out_n = (int)best_n;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Panels and the interface (src/core/panels.jl:5-22, 64-68, 87-118)         */
/* ------------------------------------------------------------------------- */
typedef struct {
    int npanels, nq, cap;
    double* corners;  /* P x 4 x 3 (a, b, c, d) */
    double* normals;  /* P x 3 */
    int* is_edge;     /* P */
    double* eps_in;   /* P */
    double* eps_out;  /* P */
    double glx[64], glw[64], bary[64];
} orc_mesh;

static void mesh_push(orc_mesh* m, const double* a, const double* b, const double* c, const double* d,
                      const double* nrm, int is_edge, double ei, double eo) {
    if (m->npanels == m->cap) {
        m->cap = m->cap ? 2 * m->cap : 64;
        m->corners = (double*)realloc(m->corners, sizeof(double) * 12 * m->cap);
        m->normals = (double*)realloc(m->normals, sizeof(double) * 3 * m->cap);
        m->is_edge = (int*)realloc(m->is_edge, sizeof(int) * m->cap);
        m->eps_in = (double*)realloc(m->eps_in, sizeof(double) * m->cap);
        m->eps_out = (double*)realloc(m->eps_out, sizeof(double) * m->cap);
    }
    int p = m->npanels++;
    memcpy(m->corners + 12 * p + 0, a, 3 * sizeof(double));
    memcpy(m->corners + 12 * p + 3, b, 3 * sizeof(double));
    memcpy(m->corners + 12 * p + 6, c, 3 * sizeof(double));
    memcpy(m->corners + 12 * p + 9, d, 3 * sizeof(double));
    memcpy(m->normals + 3 * p, nrm, 3 * sizeof(double));
    m->is_edge[p] = is_edge; m->eps_in[p] = ei; m->eps_out[p] = eo;
}

/* gl_barycentric_weights  (src/utils/barycentric.jl:6-17) */
static void gl_bary_weights(int n, const double* x, const double* w, double* lam) {
    double mx = 0.0;
    for (int i = 0; i < n; ++i) {
        double s = ((n - (i + 1)) % 2 == 0) ? 1.0 : -1.0;
        lam[i] = s * sqrt((1.0 - x[i] * x[i]) * w[i] / 2.0);
        if (fabs(lam[i]) > mx) mx = fabs(lam[i]);
    }
    for (int i = 0; i < n; ++i) lam[i] /= mx;
}

static orc_mesh* mesh_new(int nq) {
    orc_mesh* m = (orc_mesh*)calloc(1, sizeof(orc_mesh));
    m->nq = nq;
    orc_gausslegendre(nq, m->glx, m->glw);
    gl_bary_weights(nq, m->glx, m->glw, m->bary);
    return m;
}

void orc_mesh_free(orc_mesh* m) {
    if (!m) return;
    free(m->corners); free(m->normals); free(m->is_edge); free(m->eps_in); free(m->eps_out);
    free(m);
}

int orc_mesh_npanels(const orc_mesh* m) { return m->npanels; }
int orc_mesh_nq(const orc_mesh* m) { return m->nq; }
int64_t orc_mesh_npoints(const orc_mesh* m) { return (int64_t)m->npanels * m->nq * m->nq; }

/* rect_panel3d_discretize nodes and weights (src/shape/box3d.jl:44-59):
 * p = cc + (b-a)*(ns[i]/2) + (d-a)*(ns[j]/2), i outer, j inner;
 * w = ws[i]*ws[j]*|b-a|*|c-b|/4. */
static void panel_nodes(const orc_mesh* m, int p, double* pts, double* wts) {
    const double* a = m->corners + 12 * p; const double* b = a + 3; const double* c = a + 6; const double* d = a + 9;
    int nq = m->nq;
    double cc[3], bma[3], dma[3], cmb[3];
    for (int k = 0; k < 3; ++k) {
        cc[k] = (((a[k] + b[k]) + c[k]) + d[k]) / 4.0;
        bma[k] = b[k] - a[k]; dma[k] = d[k] - a[k]; cmb[k] = c[k] - b[k];
    }
    double Lab = sqrt(bma[0] * bma[0] + bma[1] * bma[1] + bma[2] * bma[2]);
    double Lbc = sqrt(cmb[0] * cmb[0] + cmb[1] * cmb[1] + cmb[2] * cmb[2]);
    int t = 0;
    for (int i = 0; i < nq; ++i)
        for (int j = 0; j < nq; ++j, ++t) {
            for (int k = 0; k < 3; ++k)
                pts[3 * t + k] = (cc[k] + bma[k] * (m->glx[i] / 2.0)) + dma[k] * (m->glx[j] / 2.0);
            wts[t] = m->glw[i] * m->glw[j] * Lab * Lbc / 4.0;
        }
}

/* all points/normals/weights in the interface iteration order (panels.jl:87-118) */
void orc_mesh_copy(const orc_mesh* m, double* corners, double* normals, int* is_edge, double* eps_in,
                   double* eps_out, double* pts, double* nrm, double* w) {
    int P = m->npanels, np = m->nq * m->nq;
    if (corners) memcpy(corners, m->corners, sizeof(double) * 12 * P);
    if (normals) memcpy(normals, m->normals, sizeof(double) * 3 * P);
    if (is_edge) memcpy(is_edge, m->is_edge, sizeof(int) * P);
    if (eps_in) memcpy(eps_in, m->eps_in, sizeof(double) * P);
    if (eps_out) memcpy(eps_out, m->eps_out, sizeof(double) * P);
    for (int p = 0; p < P; ++p) {
        if (pts && w) panel_nodes(m, p, pts + 3 * (int64_t)p * np, w + (int64_t)p * np);
        if (nrm)
            for (int t = 0; t < np; ++t)
                for (int k = 0; k < 3; ++k) nrm[3 * ((int64_t)p * np + t) + k] = m->normals[3 * p + k];
    }
}

/* interface from explicit panels (rect_panel3d_discretize for hand-built test interfaces) */
orc_mesh* orc_mesh_from_panels(int P, int nq, const double* corners, const double* normals, const int* is_edge,
                               const double* eps_in, const double* eps_out) {
    orc_mesh* m = mesh_new(nq);
    for (int p = 0; p < P; ++p)
        mesh_push(m, corners + 12 * p, corners + 12 * p + 3, corners + 12 * p + 6, corners + 12 * p + 9,
                  normals + 3 * p, is_edge[p], eps_in[p], eps_out[p]);
    return m;
}

/* TempPanel3D and divide_temp_panel3d (src/shape/box3d.jl:2-19, 66-98) */
typedef struct {
    double a[3], b[3], c[3], d[3];
    int ca, cb, cc, cd;   /* corner flags */
    int eab, ebc, ecd, eda; /* edge flags */
    double n[3];
} tpanel;

static int divide_tpanel(const tpanel* t, int nx, int ny, tpanel* out) {
    for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= ny; ++j) {
            double u0 = (double)(i - 1) / (double)nx, u1 = (double)i / (double)nx;
            double v0 = (double)(j - 1) / (double)ny, v1 = (double)j / (double)ny;
            tpanel* o = out + (i - 1) * ny + (j - 1);
            for (int k = 0; k < 3; ++k) {
                double bma = t->b[k] - t->a[k], dma = t->d[k] - t->a[k];
                o->a[k] = (t->a[k] + bma * u0) + dma * v0;
                o->b[k] = (t->a[k] + bma * u1) + dma * v0;
                o->c[k] = (t->a[k] + bma * u1) + dma * v1;
                o->d[k] = (t->a[k] + bma * u0) + dma * v1;
                o->n[k] = t->n[k];
            }
            o->ca = (i == 1 && j == 1) ? t->ca : 0;
            o->cb = (i == nx && j == 1) ? t->cb : 0;
            o->cc = (i == nx && j == ny) ? t->cc : 0;
            o->cd = (i == 1 && j == ny) ? t->cd : 0;
            o->eab = (j == 1) ? t->eab : 0;
            o->ebc = (i == nx) ? t->ebc : 0;
            o->ecd = (j == ny) ? t->ecd : 0;
            o->eda = (i == 1) ? t->eda : 0;
        }
    return nx * ny;
}

static double vnorm3(const double* a, const double* b) { /* norm(b - a) */
    double x = b[0] - a[0], y = b[1] - a[1], z = b[2] - a[2];
    return sqrt(x * x + y * y + z * z);
}

/* rect_panel3d_adaptive_panels (src/shape/box3d.jl:101-133): breadth-first 2x2
 * splitting (popfirst!/append!) of edge/corner panels longer than l_ec. */
static int adaptive_panels(orc_mesh* m, const double* a, const double* b, const double* c, const double* d,
                           const double* nrm, const int* is_edge4, const int* is_corner4, double alpha, double l_ec,
                           double ei, double eo) {
    int nx, ny;
    int rc = orc_best_grid(vnorm3(a, b), vnorm3(d, a), alpha, &nx, &ny);
    if (rc != 0) return rc;
    tpanel root;
    memcpy(root.a, a, 24); memcpy(root.b, b, 24); memcpy(root.c, c, 24); memcpy(root.d, d, 24);
    memcpy(root.n, nrm, 24);
    root.ca = is_corner4[0]; root.cb = is_corner4[1]; root.cc = is_corner4[2]; root.cd = is_corner4[3];
    root.eab = is_edge4[0]; root.ebc = is_edge4[1]; root.ecd = is_edge4[2]; root.eda = is_edge4[3];
    size_t cap = (size_t)nx * ny + 64, head = 0, tail = 0;
    tpanel* q = (tpanel*)malloc(sizeof(tpanel) * cap);
    tail = divide_tpanel(&root, nx, ny, q);
    while (head < tail) {
        tpanel t = q[head++];
        int has_ec = t.ca || t.cb || t.cc || t.cd || t.eab || t.ebc || t.ecd || t.eda;
        double Lab = vnorm3(t.a, t.b), Lda = vnorm3(t.d, t.a);
        double mx = Lab > Lda ? Lab : Lda;
        if (has_ec && mx > l_ec) {
            if (tail + 4 > cap) { cap *= 2; q = (tpanel*)realloc(q, sizeof(tpanel) * cap); }
            tail += divide_tpanel(&t, 2, 2, q + tail);
        } else {
            int ie = t.eab || t.ebc || t.ecd || t.eda || t.ca || t.cb || t.cc || t.cd;
            mesh_push(m, t.a, t.b, t.c, t.d, t.n, ie, ei, eo);
        }
    }
    free(q);
    return 0;
}

/* _box3d_geometry / single_dielectric_box3d (src/shape/box3d_single.jl:1-70) */
orc_mesh* orc_mesh_single_box(double Lx, double Ly, double Lz, int nq, double l_ec, double eps_in, double eps_out,
                              double alpha) {
    double V[8][3] = {{Lx / 2, Ly / 2, Lz / 2},   {-Lx / 2, Ly / 2, Lz / 2},  {-Lx / 2, -Ly / 2, Lz / 2},
                      {Lx / 2, -Ly / 2, Lz / 2},  {Lx / 2, Ly / 2, -Lz / 2},  {-Lx / 2, Ly / 2, -Lz / 2},
                      {-Lx / 2, -Ly / 2, -Lz / 2}, {Lx / 2, -Ly / 2, -Lz / 2}};
    int F[6][4] = {{1, 2, 3, 4}, {5, 8, 7, 6}, {8, 5, 1, 4}, {7, 3, 2, 6}, {6, 2, 1, 5}, {7, 8, 4, 3}};
    double N[6][3] = {{0, 0, 1}, {0, 0, -1}, {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}};
    int all4[4] = {1, 1, 1, 1};
    orc_mesh* m = mesh_new(nq);
    for (int f = 0; f < 6; ++f)
        if (adaptive_panels(m, V[F[f][0] - 1], V[F[f][1] - 1], V[F[f][2] - 1], V[F[f][3] - 1], N[f], all4, all4, alpha,
                            l_ec, eps_in, eps_out) != 0) {
            orc_mesh_free(m); return NULL;
        }
    return m;
}

/* --- multi-box (src/shape/box3d_multi.jl:4-30, 36-132, 139-162, 169-308, 313-386) --- */
static void box_faces_at_center(const double* ctr, double Lx, double Ly, double Lz, double f[6][5][3]) {
    double cx = ctr[0], cy = ctr[1], cz = ctr[2], hx = Lx / 2, hy = Ly / 2, hz = Lz / 2;
    double v[8][3] = {{cx + hx, cy + hy, cz + hz}, {cx - hx, cy + hy, cz + hz}, {cx - hx, cy - hy, cz + hz},
                      {cx + hx, cy - hy, cz + hz}, {cx + hx, cy + hy, cz - hz}, {cx - hx, cy + hy, cz - hz},
                      {cx - hx, cy - hy, cz - hz}, {cx + hx, cy - hy, cz - hz}};
    int F[6][4] = {{1, 2, 3, 4}, {5, 8, 7, 6}, {8, 5, 1, 4}, {7, 3, 2, 6}, {6, 2, 1, 5}, {7, 8, 4, 3}};
    double N[6][3] = {{0, 0, 1}, {0, 0, -1}, {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}};
    for (int i = 0; i < 6; ++i) {
        for (int k = 0; k < 4; ++k) memcpy(f[i][k], v[F[i][k] - 1], 24);
        memcpy(f[i][4], N[i], 24);
    }
}

static void tang_axes(const double* n, int* ax1, int* ax2, int* nax) {
    if (fabs(n[0]) > 0.5) { *ax1 = 1; *ax2 = 2; *nax = 0; }
    else if (fabs(n[1]) > 0.5) { *ax1 = 0; *ax2 = 2; *nax = 1; }
    else { *ax1 = 0; *ax2 = 1; *nax = 2; }
}

static void mkpt(int ax1, int ax2, int nax, double u, double v, double pc, double* p) {
    p[ax1] = u; p[ax2] = v; p[nax] = pc;
}

/* _rect_overlap_3d: face1 (a1..d1, n1) vs face2 (corners c2[4], n2) */
static int rect_overlap(double f1[5][3], double c2[4][3], const double* n2, double out[4][3]) {
    const double tol = 1e-10;
    const double* n1 = f1[4];
    double s0 = n1[0] + n2[0], s1 = n1[1] + n2[1], s2 = n1[2] + n2[2];
    if (sqrt(s0 * s0 + s1 * s1 + s2 * s2) > tol) return 0;
    for (int k = 0; k < 4; ++k) {
        double dd = n1[0] * (c2[k][0] - f1[0][0]) + n1[1] * (c2[k][1] - f1[0][1]) + n1[2] * (c2[k][2] - f1[0][2]);
        if (fabs(dd) > tol) return 0;
    }
    int ax1, ax2, nax; tang_axes(n1, &ax1, &ax2, &nax);
    double min1u = INFINITY, max1u = -INFINITY, min1v = INFINITY, max1v = -INFINITY;
    double min2u = INFINITY, max2u = -INFINITY, min2v = INFINITY, max2v = -INFINITY;
    for (int k = 0; k < 4; ++k) {
        min1u = fmin(min1u, f1[k][ax1]); max1u = fmax(max1u, f1[k][ax1]);
        min1v = fmin(min1v, f1[k][ax2]); max1v = fmax(max1v, f1[k][ax2]);
        min2u = fmin(min2u, c2[k][ax1]); max2u = fmax(max2u, c2[k][ax1]);
        min2v = fmin(min2v, c2[k][ax2]); max2v = fmax(max2v, c2[k][ax2]);
    }
    double lou = fmax(min1u, min2u), hiu = fmin(max1u, max2u), lov = fmax(min1v, min2v), hiv = fmin(max1v, max2v);
    if (hiu - lou < tol || hiv - lov < tol) return 0;
    double pc = f1[0][nax];
    double eab0 = f1[1][ax1] - f1[0][ax1], eab1 = f1[1][ax2] - f1[0][ax2];
    double ead0 = f1[3][ax1] - f1[0][ax1], ead1 = f1[3][ax2] - f1[0][ax2];
    if (fabs(eab0) > tol) {
        double us = eab0 >= 0 ? lou : hiu, ue = eab0 >= 0 ? hiu : lou;
        double vs = ead1 >= 0 ? lov : hiv, ve = ead1 >= 0 ? hiv : lov;
        mkpt(ax1, ax2, nax, us, vs, pc, out[0]); mkpt(ax1, ax2, nax, ue, vs, pc, out[1]);
        mkpt(ax1, ax2, nax, ue, ve, pc, out[2]); mkpt(ax1, ax2, nax, us, ve, pc, out[3]);
    } else {
        double us = ead0 >= 0 ? lou : hiu, ue = ead0 >= 0 ? hiu : lou;
        double vs = eab1 >= 0 ? lov : hiv, ve = eab1 >= 0 ? hiv : lov;
        mkpt(ax1, ax2, nax, us, vs, pc, out[0]); mkpt(ax1, ax2, nax, us, ve, pc, out[1]);
        mkpt(ax1, ax2, nax, ue, ve, pc, out[2]); mkpt(ax1, ax2, nax, ue, vs, pc, out[3]);
    }
    return 1;
}

typedef struct { double r[4][3]; int lo, hi; double n[3]; } shared_face;

static int dcmp(const void* a, const void* b) {
    double x = *(const double*)a, y = *(const double*)b;
    return (x > y) - (x < y);
}

static int uniq_sorted(double* v, int n) { /* sort!(unique!(v)) on exact values */
    qsort(v, n, sizeof(double), dcmp);
    int k = 0;
    for (int i = 0; i < n; ++i) if (k == 0 || v[i] != v[k - 1]) v[k++] = v[i];
    return k;
}

/* _subtract_rects_from_face_3d + region push; returns number of regions pushed */
static int subtract_and_mesh(orc_mesh* m, double f[5][3], double (*sh)[4][3], int nsh, double alpha, double l_ec,
                             double ei, double eo) {
    const double tol = 1e-10;
    int all4[4] = {1, 1, 1, 1};
    if (nsh == 0) return adaptive_panels(m, f[0], f[1], f[2], f[3], f[4], all4, all4, alpha, l_ec, ei, eo);
    int ax1, ax2, nax; tang_axes(f[4], &ax1, &ax2, &nax);
    double pc = f[0][nax];
    double fu0 = INFINITY, fu1 = -INFINITY, fv0 = INFINITY, fv1 = -INFINITY;
    for (int k = 0; k < 4; ++k) {
        fu0 = fmin(fu0, f[k][ax1]); fu1 = fmax(fu1, f[k][ax1]);
        fv0 = fmin(fv0, f[k][ax2]); fv1 = fmax(fv1, f[k][ax2]);
    }
    int cap = 2 + 4 * nsh;
    double* uc = (double*)malloc(sizeof(double) * cap); double* vc = (double*)malloc(sizeof(double) * cap);
    int nu_ = 0, nv_ = 0;
    uc[nu_++] = fu0; uc[nu_++] = fu1; vc[nv_++] = fv0; vc[nv_++] = fv1;
    for (int s = 0; s < nsh; ++s) for (int k = 0; k < 4; ++k) { uc[nu_++] = sh[s][k][ax1]; vc[nv_++] = sh[s][k][ax2]; }
    nu_ = uniq_sorted(uc, nu_); nv_ = uniq_sorted(vc, nv_);
    int ku = 0, kv = 0;
    for (int i = 0; i < nu_; ++i) if (fu0 - tol <= uc[i] && uc[i] <= fu1 + tol) uc[ku++] = uc[i];
    for (int i = 0; i < nv_; ++i) if (fv0 - tol <= vc[i] && vc[i] <= fv1 + tol) vc[kv++] = vc[i];
    int nu = ku - 1, nv = kv - 1;
    int* cs = (int*)malloc(sizeof(int) * (nu > 0 ? nu : 1) * (nv > 0 ? nv : 1));
#define CS(i, j) cs[(i) * nv + (j)]
    for (int i = 0; i < nu; ++i)
        for (int j = 0; j < nv; ++j) {
            double ulo = uc[i], uhi = uc[i + 1], vlo = vc[j], vhi = vc[j + 1];
            if (uhi - ulo < tol || vhi - vlo < tol) { CS(i, j) = 1; continue; }
            double um = (ulo + uhi) / 2, vm = (vlo + vhi) / 2;
            int hit = 0;
            for (int s = 0; s < nsh && !hit; ++s) {
                double ru0 = INFINITY, ru1 = -INFINITY, rv0 = INFINITY, rv1 = -INFINITY;
                for (int k = 0; k < 4; ++k) {
                    ru0 = fmin(ru0, sh[s][k][ax1]); ru1 = fmax(ru1, sh[s][k][ax1]);
                    rv0 = fmin(rv0, sh[s][k][ax2]); rv1 = fmax(rv1, sh[s][k][ax2]);
                }
                if (ru0 - tol <= um && um <= ru1 + tol && rv0 - tol <= vm && vm <= rv1 + tol) hit = 1;
            }
            CS(i, j) = hit;
        }
    int rc = 0;
    for (int i = 0; i < nu && rc == 0; ++i)
        for (int j = 0; j < nv && rc == 0; ++j) {
            if (CS(i, j)) continue;
            double ra[3], rb[3], rcc[3], rd[3];
            mkpt(ax1, ax2, nax, uc[i], vc[j], pc, ra); mkpt(ax1, ax2, nax, uc[i + 1], vc[j], pc, rb);
            mkpt(ax1, ax2, nax, uc[i + 1], vc[j + 1], pc, rcc); mkpt(ax1, ax2, nax, uc[i], vc[j + 1], pc, rd);
            int ie[4], ic[4];
            ie[0] = (j == 0) || CS(i, j - 1);
            ie[1] = (i == nu - 1) || CS(i + 1, j);
            ie[2] = (j == nv - 1) || CS(i, j + 1);
            ie[3] = (i == 0) || CS(i - 1, j);
            int gi[4] = {i, i + 1, i + 1, i}, gj[4] = {j, j, j + 1, j + 1};
            for (int q = 0; q < 4; ++q) {
                int phys = 0;
                int di[4] = {0, -1, 0, -1}, dj[4] = {0, 0, -1, -1};
                for (int t = 0; t < 4 && !phys; ++t) {
                    int ci = gi[q] + di[t], cj = gj[q] + dj[t];
                    if (ci < 0 || ci >= nu || cj < 0 || cj >= nv) phys = 1;
                    else if (CS(ci, cj)) phys = 1;
                }
                ic[q] = phys;
            }
            rc = adaptive_panels(m, ra, rb, rcc, rd, f[4], ie, ic, alpha, l_ec, ei, eo);
        }
#undef CS
    free(uc); free(vc); free(cs);
    return rc;
}

orc_mesh* orc_mesh_multi_box(int nq, double l_ec, int nbox, const double* centers, const double* dims,
                             const double* epses, double eps_out, double alpha) {
    orc_mesh* m = mesh_new(nq);
    /* _detect_shared_faces_3d */
    int nshared = 0, capsh = 16;
    shared_face* sh = (shared_face*)malloc(sizeof(shared_face) * capsh);
    for (int i = 0; i < nbox; ++i) {
        double fi[6][5][3]; box_faces_at_center(centers + 3 * i, dims[3 * i], dims[3 * i + 1], dims[3 * i + 2], fi);
        for (int j = i + 1; j < nbox; ++j) {
            double fj[6][5][3]; box_faces_at_center(centers + 3 * j, dims[3 * j], dims[3 * j + 1], dims[3 * j + 2], fj);
            for (int a = 0; a < 6; ++a)
                for (int b = 0; b < 6; ++b) {
                    double reg[4][3];
                    if (rect_overlap(fi[a], fj[b], fj[b][4], reg)) {
                        if (nshared == capsh) { capsh *= 2; sh = (shared_face*)realloc(sh, sizeof(shared_face) * capsh); }
                        memcpy(sh[nshared].r, reg, sizeof(reg));
                        sh[nshared].lo = i; sh[nshared].hi = j;
                        for (int k = 0; k < 3; ++k) sh[nshared].n[k] = -fi[a][4][k];
                        ++nshared;
                    }
                }
        }
    }
    int rc = 0;
    double (*fs)[4][3] = (double (*)[4][3])malloc(sizeof(double) * 12 * (nshared > 0 ? nshared : 1));
    for (int bid = 0; bid < nbox && rc == 0; ++bid) {
        double f[6][5][3]; box_faces_at_center(centers + 3 * bid, dims[3 * bid], dims[3 * bid + 1], dims[3 * bid + 2], f);
        for (int a = 0; a < 6 && rc == 0; ++a) {
            int nfs = 0;
            for (int s = 0; s < nshared; ++s) {
                if (bid != sh[s].lo && bid != sh[s].hi) continue;
                double mn[3] = {-f[a][4][0], -f[a][4][1], -f[a][4][2]};
                double reg[4][3];
                if (rect_overlap(f[a], sh[s].r, mn, reg)) memcpy(fs[nfs++], reg, sizeof(reg));
            }
            rc = subtract_and_mesh(m, f[a], fs, nfs, alpha, l_ec, epses[bid], eps_out);
        }
    }
    int all4[4] = {1, 1, 1, 1};
    for (int s = 0; s < nshared && rc == 0; ++s)
        rc = adaptive_panels(m, sh[s].r[0], sh[s].r[1], sh[s].r[2], sh[s].r[3], sh[s].n, all4, all4, alpha, l_ec,
                             epses[sh[s].hi], epses[sh[s].lo]);
    free(fs); free(sh);
    if (rc != 0) { orc_mesh_free(m); return NULL; }
    return m;
}

/* ------------------------------------------------------------------------- */
/* Pointwise kernels (src/kernel/laplace3d.jl:1-15)                          */
/* ------------------------------------------------------------------------- */
double orc_pot(const double* src, const double* trg) {
    double d0 = src[0] - trg[0], d1 = src[1] - trg[1], d2 = src[2] - trg[2];
    double r2 = (d0 * d0 + d1 * d1) + d2 * d2;
    double inv_r = 1.0 / sqrt(r2);
    return inv_r / FOUR_PI;
}

double orc_grad(const double* src, const double* trg, const double* n) {
    double d0 = src[0] - trg[0], d1 = src[1] - trg[1], d2 = src[2] - trg[2];
    double r2 = (d0 * d0 + d1 * d1) + d2 * d2;
    double inv_r = 1.0 / sqrt(r2);
    double i3 = inv_r * inv_r * inv_r;
    double dot = (n[0] * (i3 * (trg[0] - src[0])) + n[1] * (i3 * (trg[1] - src[1]))) + n[2] * (i3 * (trg[2] - src[2]));
    return dot / FOUR_PI;
}

/* ------------------------------------------------------------------------- */
/* Dense operators (src/kernel/laplace3d.jl:18-40; solver/dielectric_box3d.jl:1-17) */
/* Column-major N x N output.                                                */
/* ------------------------------------------------------------------------- */
static void mesh_arrays(const orc_mesh* m, double** pts, double** nrm, double** w) {
    int64_t N = orc_mesh_npoints(m);
    *pts = (double*)malloc(sizeof(double) * 3 * N);
    *nrm = (double*)malloc(sizeof(double) * 3 * N);
    *w = (double*)malloc(sizeof(double) * N);
    orc_mesh_copy(m, NULL, NULL, NULL, NULL, NULL, *pts, *nrm, *w);
}

void orc_diag(const orc_mesh* m, double* diag) {
    int np = m->nq * m->nq;
    for (int p = 0; p < m->npanels; ++p) {
        double t = 0.5 * (m->eps_out[p] + m->eps_in[p]) / (m->eps_out[p] - m->eps_in[p]);
        for (int j = 0; j < np; ++j) diag[(int64_t)p * np + j] = t;
    }
}

void orc_DT_dense(const orc_mesh* m, double* A, int with_diag) {
    int64_t N = orc_mesh_npoints(m);
    double *pts, *nrm, *w; mesh_arrays(m, &pts, &nrm, &w);
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < N; ++j)
        for (int64_t i = 0; i < N; ++i)
            A[i + j * N] = (i == j) ? 0.0 : orc_grad(pts + 3 * j, pts + 3 * i, nrm + 3 * i) * w[j];
    if (with_diag) {
        double* dg = (double*)malloc(sizeof(double) * N);
        orc_diag(m, dg);
        for (int64_t i = 0; i < N; ++i) A[i + i * N] += dg[i];
        free(dg);
    }
    free(pts); free(nrm); free(w);
}

void orc_S_dense(const orc_mesh* m, double* A) {
    int64_t N = orc_mesh_npoints(m);
    double *pts, *nrm, *w; mesh_arrays(m, &pts, &nrm, &w);
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < N; ++j)
        for (int64_t i = 0; i < N; ++i)
            A[i + j * N] = (i == j) ? 0.0 : orc_pot(pts + 3 * j, pts + 3 * i) * w[j];
    free(pts); free(nrm); free(w);
}

/* Matrix-free direct sums. X, Y column-major (N x k); pts/nrm 3 x N (Julia SoA,
 * src/kernel/laplace3d.jl:85-97). Y[i,c] = sum_{j != i} grad(y_j, x_i, n_i) w_j X[j,c]. */
void orc_DT_apply(int64_t N, const double* pts, const double* nrm, const double* w, const double* X, double* Y,
                  int k, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < N; ++i) {
        for (int c = 0; c < k; ++c) {
            double acc = 0.0;
            for (int64_t j = 0; j < N; ++j) {
                if (j == i) continue;
                acc += orc_grad(pts + 3 * j, pts + 3 * i, nrm + 3 * i) * w[j] * X[j + c * N];
            }
            Y[i + c * N] = acc;
        }
    }
}

/* S[sigma](x_m) = sum_j pot(y_j, x_m) w_j X[j,c]   (src/kernel/laplace3d.jl:69-82) */
void orc_pottrg_apply(int64_t N, const double* pts, const double* w, int64_t M, const double* trg, const double* X,
                      double* Y, int k, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(static)
    for (int64_t m = 0; m < M; ++m)
        for (int c = 0; c < k; ++c) {
            double acc = 0.0;
            for (int64_t j = 0; j < N; ++j) acc += orc_pot(pts + 3 * j, trg + 3 * m) * w[j] * X[j + c * N];
            Y[m + c * M] = acc;
        }
}

/* rhs_dielectric_box3d(::PointSource)  (src/solver/dielectric_box3d.jl:95-104) */
void orc_rhs_point(int64_t N, const double* pts, const double* nrm, const double* src, double q, double eps_src,
                   double* out) {
    for (int64_t i = 0; i < N; ++i) out[i] = -q * orc_grad(src, pts + 3 * i, nrm + 3 * i) / eps_src;
}

/* ------------------------------------------------------------------------- */
/* Bernstein radius (src/utils/bernstein.jl:12-62)                           */
/* ------------------------------------------------------------------------- */
static double rho_from_pole(double complex z) {
    double complex s = csqrt(z * z - 1.0);
    double a1 = cabs(z + s), a2 = cabs(z - s);
    return a1 > a2 ? a1 : a2;
}

double orc_bernstein_rho_panel(const double* corners, const double* normal, const double* trg) {
    const double *a = corners, *b = corners + 3, *c = corners + 6, *d = corners + 9;
    double cc[3], u1[3], u2[3], e1[3], e2[3], r[3];
    for (int k = 0; k < 3; ++k) {
        cc[k] = (((a[k] + b[k]) + c[k]) + d[k]) / 4.0;
        u1[k] = b[k] - a[k]; u2[k] = d[k] - a[k];
    }
    double len1 = sqrt(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
    double len2 = sqrt(u2[0] * u2[0] + u2[1] * u2[1] + u2[2] * u2[2]);
    double L1 = len1 / 2, L2 = len2 / 2;
    for (int k = 0; k < 3; ++k) { e1[k] = u1[k] / len1; e2[k] = u2[k] / len2; r[k] = trg[k] - cc[k]; }
    double xt = r[0] * e1[0] + r[1] * e1[1] + r[2] * e1[2];
    double yt = r[0] * e2[0] + r[1] * e2[1] + r[2] * e2[2];
    double zt = r[0] * normal[0] + r[1] * normal[1] + r[2] * normal[2];
    double cy = yt < -L2 ? -L2 : (yt > L2 ? L2 : yt);
    double dy = yt - cy;
    double complex t1 = (xt + I * sqrt(dy * dy + zt * zt)) / L1;
    double rho1 = rho_from_pole(t1);
    double cx = xt < -L1 ? -L1 : (xt > L1 ? L1 : xt);
    double dx = xt - cx;
    double complex t2 = (yt + I * sqrt(dx * dx + zt * zt)) / L2;
    double rho2 = rho_from_pole(t2);
    return rho1 < rho2 ? rho1 : rho2;
}

/* ------------------------------------------------------------------------- */
/* build_neighbor_list  (src/kernel/laplace3d_near.jl:240-392)               */
/* Output: upsample triples (i, j, p_up) and adaptive pairs (i, j), 0-based  */
/* source panel i, target panel j, in (i ascending, j ascending) order.       */
/* ------------------------------------------------------------------------- */
typedef struct {
    int n_ups, n_adp;
    int *ups_i, *ups_j, *ups_p;
    int *adp_i, *adp_j;
} orc_nbr;

void orc_nbr_free(orc_nbr* n) {
    if (!n) return;
    free(n->ups_i); free(n->ups_j); free(n->ups_p); free(n->adp_i); free(n->adp_j); free(n);
}
int orc_nbr_counts(const orc_nbr* n, int* n_ups, int* n_adp) { *n_ups = n->n_ups; *n_adp = n->n_adp; return 0; }
void orc_nbr_copy(const orc_nbr* n, int* ups_i, int* ups_j, int* ups_p, int* adp_i, int* adp_j) {
    memcpy(ups_i, n->ups_i, sizeof(int) * n->n_ups); memcpy(ups_j, n->ups_j, sizeof(int) * n->n_ups);
    memcpy(ups_p, n->ups_p, sizeof(int) * n->n_ups);
    memcpy(adp_i, n->adp_i, sizeof(int) * n->n_adp); memcpy(adp_j, n->adp_j, sizeof(int) * n->n_adp);
}

orc_nbr* orc_build_neighbor_list(const orc_mesh* m, int max_order, double atol, int correct_edges) {
    int P = m->npanels, nq = m->nq, np = nq * nq;
    int64_t N = (int64_t)P * np;
    double *pts, *nrm, *w; mesh_arrays(m, &pts, &nrm, &w);
    double* centers = (double*)malloc(sizeof(double) * 3 * P);
    double* lengths = (double*)malloc(sizeof(double) * P);
    double* offs = (double*)malloc(sizeof(double) * P);
    for (int p = 0; p < P; ++p) {
        const double* c = m->corners + 12 * p;
        for (int k = 0; k < 3; ++k) centers[3 * p + k] = (((c[k] + c[3 + k]) + c[6 + k]) + c[9 + k]) / 4.0;
        double l1 = vnorm3(c + 3, c), l2 = vnorm3(c + 6, c + 3);
        lengths[p] = l1 > l2 ? l1 : l2;
        const double* n = m->normals + 3 * p;
        offs[p] = n[0] * c[0] + n[1] * c[1] + n[2] * c[2];
    }
    const double same_tol = sqrt(DBL_EPSILON);
    double Lmax = 1.0;
    if (P > 0) { Lmax = -INFINITY; for (int p = 0; p < P; ++p) if (lengths[p] > Lmax) Lmax = lengths[p]; }
    const double tol_corner = sqrt(DBL_EPSILON) * Lmax;
    const double log_atol = log(atol);

    int cap_u = 1024, cap_a = 256;
    orc_nbr* out = (orc_nbr*)calloc(1, sizeof(orc_nbr));
    out->ups_i = (int*)malloc(sizeof(int) * cap_u); out->ups_j = (int*)malloc(sizeof(int) * cap_u);
    out->ups_p = (int*)malloc(sizeof(int) * cap_u);
    out->adp_i = (int*)malloc(sizeof(int) * cap_a); out->adp_j = (int*)malloc(sizeof(int) * cap_a);

    double* rho_min = (double*)malloc(sizeof(double) * P);  /* per target panel, INF = not in panel_dict */
    char* in_dict = (char*)malloc(P);
    char* touching = (char*)malloc(P);
    for (int i = 0; i < P; ++i) {
        if (!correct_edges && m->is_edge[i]) continue;
        double l_i = lengths[i];
        double rho_star = pow(atol, -1.0 / (2.0 * nq));
        double L_half = l_i / 2;
        double As = (rho_star + 1.0 / rho_star) / 2, Bs = (rho_star - 1.0 / rho_star) / 2;
        double r_i = 105.0 / 100.0 * L_half * sqrt(As * As + (1.0 + Bs) * (1.0 + Bs) + Bs * Bs);
        memset(in_dict, 0, P); memset(touching, 0, P);
        for (int j = 0; j < P; ++j) rho_min[j] = INFINITY;
        const double* ci = centers + 3 * i;
        /* nearby nodes (inrange over the node KD-tree; exact brute force here) */
        for (int64_t t = 0; t < N; ++t) {
            double dx = pts[3 * t] - ci[0], dy = pts[3 * t + 1] - ci[1], dz = pts[3 * t + 2] - ci[2];
            if (sqrt(dx * dx + dy * dy + dz * dz) > r_i) continue;
            int j = (int)(t / np);
            if (j == i) continue;
            in_dict[j] = 1;
            double rho = orc_bernstein_rho_panel(m->corners + 12 * i, m->normals + 3 * i, pts + 3 * t);
            if (rho < rho_min[j]) rho_min[j] = rho;
        }
        if (correct_edges) {
            for (int ck = 0; ck < 4; ++ck) {
                const double* cp = m->corners + 12 * i + 3 * ck;
                for (int j = 0; j < P; ++j) {
                    if (j == i) continue;
                    for (int cj = 0; cj < 4; ++cj) {
                        const double* q = m->corners + 12 * j + 3 * cj;
                        double dx = q[0] - cp[0], dy = q[1] - cp[1], dz = q[2] - cp[2];
                        if (sqrt(dx * dx + dy * dy + dz * dz) <= tol_corner) { touching[j] = 1; break; }
                    }
                }
            }
            for (int j = 0; j < P; ++j) if (touching[j]) in_dict[j] = 1;
        }
        for (int j = 0; j < P; ++j) {
            if (!in_dict[j]) continue;
            if (!correct_edges && m->is_edge[j]) continue;
            const double *ni = m->normals + 3 * i, *nj = m->normals + 3 * j;
            double dn = ni[0] * nj[0] + ni[1] * nj[1] + ni[2] * nj[2];
            if (dn > 1 - same_tol) {
                if (fabs(offs[i] - offs[j]) <= same_tol * (l_i > 1.0 ? l_i : 1.0)) continue;
            }
            if (correct_edges && touching[j]) {
                if (out->n_adp == cap_a) {
                    cap_a *= 2;
                    out->adp_i = (int*)realloc(out->adp_i, sizeof(int) * cap_a);
                    out->adp_j = (int*)realloc(out->adp_j, sizeof(int) * cap_a);
                }
                out->adp_i[out->n_adp] = i; out->adp_j[out->n_adp] = j; out->n_adp++;
                continue;
            }
            if (!(rho_min[j] < INFINITY)) continue;  /* points_j empty */
            if (!(rho_min[j] <= rho_star)) continue;
            int p_up;
            if (rho_min[j] > 1.0) p_up = (int)ceil(-log_atol / (2.0 * log(rho_min[j])));
            else p_up = max_order;
            if (p_up < nq) p_up = nq;
            if (p_up > max_order) p_up = max_order;
            if (out->n_ups == cap_u) {
                cap_u *= 2;
                out->ups_i = (int*)realloc(out->ups_i, sizeof(int) * cap_u);
                out->ups_j = (int*)realloc(out->ups_j, sizeof(int) * cap_u);
                out->ups_p = (int*)realloc(out->ups_p, sizeof(int) * cap_u);
            }
            out->ups_i[out->n_ups] = i; out->ups_j[out->n_ups] = j; out->ups_p[out->n_ups] = p_up; out->n_ups++;
        }
    }
    free(rho_min); free(in_dict); free(touching);
    free(centers); free(lengths); free(offs); free(pts); free(nrm); free(w);
    return out;
}

/* ------------------------------------------------------------------------- */
/* Barycentric interpolation (src/utils/barycentric.jl:19-42, 87-95)         */
/* ------------------------------------------------------------------------- */
static void bary_row(int n, const double* x, const double* lam, double xq, double* r) {
    for (int i = 0; i < n; ++i) {
        /* isapprox(xq, x[i]) with rtol = sqrt(eps), atol = 0 */
        double ax = fabs(xq), ay = fabs(x[i]);
        double mx = ax > ay ? ax : ay;
        if (xq == x[i] || fabs(xq - x[i]) <= sqrt(DBL_EPSILON) * mx) {
            for (int k = 0; k < n; ++k) r[k] = 0.0;
            r[i] = 1.0;
            return;
        }
    }
    double denom = 0.0;
    for (int i = 0; i < n; ++i) { double t = lam[i] / (xq - x[i]); r[i] = t; denom += t; }
    double inv = 1.0 / denom;
    for (int i = 0; i < n; ++i) r[i] *= inv;
}

/* ------------------------------------------------------------------------- */
/* Panel-level blocks                                                          */
/* ------------------------------------------------------------------------- */
/* laplace3d_DT_panel (src/kernel/laplace3d_near.jl:1-34): K[t, s] = grad(p_s, x_t, n_trg) * w_s,
 * row-major out[t * np_src + s]. */
void orc_DT_panel(const orc_mesh* m, int src, int trg, double* out) {
    int np = m->nq * m->nq;
    double* ps = (double*)malloc(sizeof(double) * 3 * np); double* ws = (double*)malloc(sizeof(double) * np);
    double* pt = (double*)malloc(sizeof(double) * 3 * np); double* wt = (double*)malloc(sizeof(double) * np);
    panel_nodes(m, src, ps, ws); panel_nodes(m, trg, pt, wt);
    const double* nt = m->normals + 3 * trg;
    for (int t = 0; t < np; ++t)
        for (int s = 0; s < np; ++s) out[t * np + s] = orc_grad(ps + 3 * s, pt + 3 * t, nt) * ws[s];
    free(ps); free(ws); free(pt); free(wt);
}

/* SourceCache (src/kernel/laplace3d_near_upsampling.jl:8-50): upsampled points
 * p_up[alpha] (alpha = i_up*n_up + j_up) and Mt[m, alpha] (m = m_x*nq + m_y). */
static void source_cache(const orc_mesh* m, int src, int n_up, double* p_up, double* Mt) {
    int nq = m->nq, nq2 = nq * nq, nu2 = n_up * n_up;
    double xu[64], wu[64], Ex[64 * 64];
    orc_gausslegendre(n_up, xu, wu);
    for (int i = 0; i < n_up; ++i) bary_row(nq, m->glx, m->bary, xu[i], Ex + i * nq); /* Ex[i_up, m] */
    const double* a = m->corners + 12 * src; const double *b = a + 3, *c = a + 6, *d = a + 9;
    double cc[3], bma[3], dma[3];
    for (int k = 0; k < 3; ++k) { cc[k] = (((a[k] + b[k]) + c[k]) + d[k]) / 4.0; bma[k] = b[k] - a[k]; dma[k] = d[k] - a[k]; }
    double Lx = sqrt(bma[0] * bma[0] + bma[1] * bma[1] + bma[2] * bma[2]);
    double Ly = sqrt(dma[0] * dma[0] + dma[1] * dma[1] + dma[2] * dma[2]);
    double scale = Lx * Ly / 4;
    for (int iu = 0; iu < n_up; ++iu) {
        double x = xu[iu] / 2;
        for (int ju = 0; ju < n_up; ++ju) {
            double y = xu[ju] / 2;
            int al = iu * n_up + ju;
            for (int k = 0; k < 3; ++k) p_up[3 * al + k] = (cc[k] + bma[k] * x) + dma[k] * y;
        }
    }
    for (int mx = 0; mx < nq; ++mx)
        for (int my = 0; my < nq; ++my) {
            int mm = mx * nq + my;
            for (int iu = 0; iu < n_up; ++iu)
                for (int ju = 0; ju < n_up; ++ju)
                    Mt[(int64_t)mm * nu2 + iu * n_up + ju] = scale * wu[iu] * wu[ju] * Ex[iu * nq + mx] * Ex[ju * nq + my];
        }
    (void)nq2;
}

/* Upsampled block K_up[t, m] = sum_alpha Mt[m, alpha] grad(p_up[alpha], x_t, n_trg), row-major out[t*nq2+m]
 * (src/kernel/laplace3d_near_upsampling.jl:184-203; equal to laplace3d_DT_panel_upsampled, :52-119) */
void orc_DT_panel_upsampled(const orc_mesh* m, int src, int trg, int n_up, double* out) {
    int nq2 = m->nq * m->nq, nu2 = n_up * n_up;
    double* p_up = (double*)malloc(sizeof(double) * 3 * nu2);
    double* Mt = (double*)malloc(sizeof(double) * nq2 * nu2);
    double* pt = (double*)malloc(sizeof(double) * 3 * nq2); double* wt = (double*)malloc(sizeof(double) * nq2);
    double* kv = (double*)malloc(sizeof(double) * nu2);
    source_cache(m, src, n_up, p_up, Mt);
    panel_nodes(m, trg, pt, wt);
    const double* nt = m->normals + 3 * trg;
    for (int t = 0; t < nq2; ++t) {
        for (int al = 0; al < nu2; ++al) kv[al] = orc_grad(p_up + 3 * al, pt + 3 * t, nt);
        for (int mm = 0; mm < nq2; ++mm) {
            double acc = 0.0;
            for (int al = 0; al < nu2; ++al) acc += Mt[(int64_t)mm * nu2 + al] * kv[al];
            out[t * nq2 + mm] = acc;
        }
    }
    free(p_up); free(Mt); free(pt); free(wt); free(kv);
}

/* Adaptive quadtree (src/kernel/laplace3d_near_adaptive.jl:17-224, 308-387) */
typedef struct {
    const orc_mesh* m; int src;
    double cc[3], bma[3], dma[3], scale_panel;
    int nGL; double xg[64], wg[64];
    double atol, rtol; int max_depth;
    const double* pt; const double* nt;
    double* leaves; int nleaves, capl; int hit_max;
} adp_ctx;

static void cell_moments(adp_ctx* C, double ulo, double uhi, double vlo, double vhi, double* out) {
    int nq = C->m->nq, nq2 = nq * nq;
    double rx[64], ry[64];
    for (int mm = 0; mm < nq2; ++mm) out[mm] = 0.0;
    double hu = (uhi - ulo) / 2, hv = (vhi - vlo) / 2, mu = (uhi + ulo) / 2, mv = (vhi + vlo) / 2;
    double sc = hu * hv * C->scale_panel;
    for (int gi = 0; gi < C->nGL; ++gi) {
        double u = mu + hu * C->xg[gi], wu = C->wg[gi];
        bary_row(nq, C->m->glx, C->m->bary, u, rx);
        for (int gj = 0; gj < C->nGL; ++gj) {
            double v = mv + hv * C->xg[gj], wv = C->wg[gj];
            bary_row(nq, C->m->glx, C->m->bary, v, ry);
            double y[3];
            for (int k = 0; k < 3; ++k) y[k] = (C->cc[k] + C->bma[k] * (u / 2)) + C->dma[k] * (v / 2);
            double kval = orc_grad(y, C->pt, C->nt);
            double ww = wu * wv * sc * kval;
            int mm = 0;
            for (int mx = 0; mx < nq; ++mx)
                for (int my = 0; my < nq; ++my, ++mm) out[mm] += ww * rx[mx] * ry[my];
        }
    }
}

static void push_leaf(adp_ctx* C, double a, double b, double c, double d) {
    if (C->nleaves == C->capl) {
        C->capl = C->capl ? 2 * C->capl : 64;
        C->leaves = (double*)realloc(C->leaves, sizeof(double) * 4 * C->capl);
    }
    double* L = C->leaves + 4 * C->nleaves++;
    L[0] = a; L[1] = b; L[2] = c; L[3] = d;
}

static void recurse_walk(adp_ctx* C, double ulo, double uhi, double vlo, double vhi, int depth) {
    int nq2 = C->m->nq * C->m->nq;
    double par[256], c1[256], c2[256], c3[256], c4[256];
    cell_moments(C, ulo, uhi, vlo, vhi, par);
    double mu = (uhi + ulo) / 2, mv = (vhi + vlo) / 2;
    cell_moments(C, ulo, mu, vlo, mv, c1);
    cell_moments(C, mu, uhi, vlo, mv, c2);
    cell_moments(C, ulo, mu, mv, vhi, c3);
    cell_moments(C, mu, uhi, mv, vhi, c4);
    double err = -INFINITY, pmax = -INFINITY;
    for (int mm = 0; mm < nq2; ++mm) {
        double ch = ((c1[mm] + c2[mm]) + c3[mm]) + c4[mm];
        double e = fabs(par[mm] - ch);
        if (e > err) err = e;
        if (fabs(par[mm]) > pmax) pmax = fabs(par[mm]);
    }
    double tl = C->rtol * pmax;
    if (C->atol > tl) tl = C->atol;
    if (err < tl || depth == C->max_depth) {
        push_leaf(C, ulo, mu, vlo, mv);
        push_leaf(C, mu, uhi, vlo, mv);
        push_leaf(C, ulo, mu, mv, vhi);
        push_leaf(C, mu, uhi, mv, vhi);
        if (depth == C->max_depth && err >= tl) C->hit_max = 1;
        return;
    }
    recurse_walk(C, ulo, mu, vlo, mv, depth + 1);
    recurse_walk(C, mu, uhi, vlo, mv, depth + 1);
    recurse_walk(C, ulo, mu, mv, vhi, depth + 1);
    recurse_walk(C, mu, uhi, mv, vhi, depth + 1);
}

static void adp_init(adp_ctx* C, const orc_mesh* m, int src, double atol, double rtol, int nGL, int max_depth) {
    memset(C, 0, sizeof(*C));
    C->m = m; C->src = src; C->atol = atol; C->rtol = rtol; C->max_depth = max_depth;
    C->nGL = nGL == 0 ? m->nq : nGL;
    orc_gausslegendre(C->nGL, C->xg, C->wg);
    const double* a = m->corners + 12 * src; const double *b = a + 3, *c = a + 6, *d = a + 9;
    for (int k = 0; k < 3; ++k) { C->cc[k] = (((a[k] + b[k]) + c[k]) + d[k]) / 4.0; C->bma[k] = b[k] - a[k]; C->dma[k] = d[k] - a[k]; }
    double Lx = sqrt(C->bma[0] * C->bma[0] + C->bma[1] * C->bma[1] + C->bma[2] * C->bma[2]);
    double Ly = sqrt(C->dma[0] * C->dma[0] + C->dma[1] * C->dma[1] + C->dma[2] * C->dma[2]);
    C->scale_panel = Lx * Ly / 4;
}

/* adaptive_panel_moments_inplace! equivalent for one target (leaves accumulated by children sums):
 * used by the cubature known-answer test (test/kernel/laplace3d_near_adaptive.jl:21-59). */
static int recurse_acc(adp_ctx* C, double* K, double ulo, double uhi, double vlo, double vhi, int depth) {
    int nq2 = C->m->nq * C->m->nq;
    double par[256], c1[256], c2[256], c3[256], c4[256], ch[256];
    cell_moments(C, ulo, uhi, vlo, vhi, par);
    double mu = (uhi + ulo) / 2, mv = (vhi + vlo) / 2;
    cell_moments(C, ulo, mu, vlo, mv, c1); cell_moments(C, mu, uhi, vlo, mv, c2);
    cell_moments(C, ulo, mu, mv, vhi, c3); cell_moments(C, mu, uhi, mv, vhi, c4);
    double err = -INFINITY, pmax = -INFINITY;
    for (int mm = 0; mm < nq2; ++mm) {
        ch[mm] = ((c1[mm] + c2[mm]) + c3[mm]) + c4[mm];
        double e = fabs(par[mm] - ch[mm]); if (e > err) err = e;
        if (fabs(par[mm]) > pmax) pmax = fabs(par[mm]);
    }
    double tl = C->rtol * pmax; if (C->atol > tl) tl = C->atol;
    if (err < tl || depth == C->max_depth) {
        for (int mm = 0; mm < nq2; ++mm) K[mm] += ch[mm];
        return depth == C->max_depth && err >= tl;
    }
    int h1 = recurse_acc(C, K, ulo, mu, vlo, mv, depth + 1);
    int h2 = recurse_acc(C, K, mu, uhi, vlo, mv, depth + 1);
    int h3 = recurse_acc(C, K, ulo, mu, mv, vhi, depth + 1);
    int h4 = recurse_acc(C, K, mu, uhi, mv, vhi, depth + 1);
    return h1 || h2 || h3 || h4;
}

int orc_adaptive_panel_moments(const orc_mesh* m, int src, const double* pt, const double* nt, double atol,
                               double rtol, int nGL, int max_depth, double* K) {
    adp_ctx C; adp_init(&C, m, src, atol, rtol, nGL, max_depth);
    C.pt = pt; C.nt = nt;
    for (int mm = 0; mm < m->nq * m->nq; ++mm) K[mm] = 0.0;
    return recurse_acc(&C, K, -1.0, 1.0, -1.0, 1.0, 0);
}

/* Touching-pair block (src/kernel/laplace3d_near_upsampling.jl:219-249 + adaptive_block_moments_inplace!):
 * K_block[t, m], row-major out[t * nq2 + m]. Returns hit_max. */
int orc_DT_panel_adaptive(const orc_mesh* m, int src, int trg, double atol, double rtol, int nGL, int max_depth,
                          double* out, int* nleaves) {
    int nq = m->nq, nq2 = nq * nq;
    double* pt = (double*)malloc(sizeof(double) * 3 * nq2); double* wt = (double*)malloc(sizeof(double) * nq2);
    panel_nodes(m, trg, pt, wt);
    const double* nt = m->normals + 3 * trg;
    const double* c1s = m->corners + 12 * src;
    int rep = 0; double best = INFINITY;
    for (int t = 0; t < nq2; ++t) {
        double dd = vnorm3(c1s, pt + 3 * t);
        if (dd < best) { best = dd; rep = t; }
    }
    adp_ctx C; adp_init(&C, m, src, atol, rtol, nGL, max_depth);
    C.pt = pt + 3 * rep; C.nt = nt;
    recurse_walk(&C, -1.0, 1.0, -1.0, 1.0, 0);
    for (int i = 0; i < nq2 * nq2; ++i) out[i] = 0.0;
    double rx[64], ry[64];
    double* kv = (double*)malloc(sizeof(double) * nq2);
    for (int l = 0; l < C.nleaves; ++l) {
        const double* L = C.leaves + 4 * l;
        double hu = (L[1] - L[0]) / 2, hv = (L[3] - L[2]) / 2, mu = (L[1] + L[0]) / 2, mv = (L[3] + L[2]) / 2;
        double sc = hu * hv * C.scale_panel;
        for (int gi = 0; gi < C.nGL; ++gi) {
            double u = mu + hu * C.xg[gi], wu = C.wg[gi];
            bary_row(nq, m->glx, m->bary, u, rx);
            for (int gj = 0; gj < C.nGL; ++gj) {
                double v = mv + hv * C.xg[gj], wv = C.wg[gj];
                bary_row(nq, m->glx, m->bary, v, ry);
                double y[3];
                for (int k = 0; k < 3; ++k) y[k] = (C.cc[k] + C.bma[k] * (u / 2)) + C.dma[k] * (v / 2);
                double wuv = wu * wv * sc;
                for (int t = 0; t < nq2; ++t) kv[t] = orc_grad(y, pt + 3 * t, nt);
                for (int mx = 0; mx < nq; ++mx) {
                    double rxm = rx[mx];
                    for (int my = 0; my < nq; ++my) {
                        int mm = mx * nq + my;
                        double wm = wuv * rxm * ry[my];
                        for (int t = 0; t < nq2; ++t) out[t * nq2 + mm] += wm * kv[t];
                    }
                }
            }
        }
    }
    if (nleaves) *nleaves = C.nleaves;
    int hm = C.hit_max;
    free(C.leaves); free(pt); free(wt); free(kv);
    return hm;
}

/* _laplace3d_corrections  (src/kernel/laplace3d_near_upsampling.jl:127-270):
 * COO triplets (0-based row = target node, col = source node). Each source panel
 * uses ONE upsampling order, the max over its upsample neighbours (:164-183). */
typedef struct { int64_t nnz, cap; int64_t *rows, *cols; double* vals; int hit_max; } orc_coo;

void orc_coo_free(orc_coo* c) { if (!c) return; free(c->rows); free(c->cols); free(c->vals); free(c); }
int64_t orc_coo_nnz(const orc_coo* c) { return c->nnz; }
int orc_coo_hit_max(const orc_coo* c) { return c->hit_max; }
void orc_coo_copy(const orc_coo* c, int64_t* rows, int64_t* cols, double* vals) {
    memcpy(rows, c->rows, sizeof(int64_t) * c->nnz); memcpy(cols, c->cols, sizeof(int64_t) * c->nnz);
    memcpy(vals, c->vals, sizeof(double) * c->nnz);
}

static void coo_push_block(orc_coo* C, const double* Kb, const double* Kd, int nq2, int64_t row_off, int64_t col_off) {
    for (int cl = 0; cl < nq2; ++cl)
        for (int rl = 0; rl < nq2; ++rl) {
            double v = Kb[rl * nq2 + cl] - Kd[rl * nq2 + cl];
            if (v == 0.0) continue;
            if (C->nnz == C->cap) {
                C->cap = C->cap ? 2 * C->cap : 4096;
                C->rows = (int64_t*)realloc(C->rows, sizeof(int64_t) * C->cap);
                C->cols = (int64_t*)realloc(C->cols, sizeof(int64_t) * C->cap);
                C->vals = (double*)realloc(C->vals, sizeof(double) * C->cap);
            }
            C->rows[C->nnz] = row_off + rl; C->cols[C->nnz] = col_off + cl; C->vals[C->nnz] = v; C->nnz++;
        }
}

orc_coo* orc_DT_corrections(const orc_mesh* m, const orc_nbr* nb, double adp_atol, double adp_rtol, int adp_nGL,
                            int adp_max_depth, int nthreads) {
    int P = m->npanels, nq2 = m->nq * m->nq;
    int* nup_max = (int*)calloc(P, sizeof(int));
    for (int e = 0; e < nb->n_ups; ++e) if (nb->ups_p[e] > nup_max[nb->ups_i[e]]) nup_max[nb->ups_i[e]] = nb->ups_p[e];
    orc_coo* res = (orc_coo*)calloc(1, sizeof(orc_coo));
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    /* per-source work, assembled in source order so the triplet list is deterministic */
    orc_coo* parts = (orc_coo*)calloc(P, sizeof(orc_coo));
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < P; ++i) {
        orc_coo* C = parts + i;
        double* Kb = (double*)malloc(sizeof(double) * nq2 * nq2);
        double* Kd = (double*)malloc(sizeof(double) * nq2 * nq2);
        for (int e = 0; e < nb->n_ups; ++e) {
            if (nb->ups_i[e] != i) continue;
            int j = nb->ups_j[e];
            orc_DT_panel_upsampled(m, i, j, nup_max[i], Kb);
            orc_DT_panel(m, i, j, Kd);
            coo_push_block(C, Kb, Kd, nq2, (int64_t)j * nq2, (int64_t)i * nq2);
        }
        for (int e = 0; e < nb->n_adp; ++e) {
            if (nb->adp_i[e] != i) continue;
            int j = nb->adp_j[e];
            if (orc_DT_panel_adaptive(m, i, j, adp_atol, adp_rtol, adp_nGL, adp_max_depth, Kb, NULL)) C->hit_max = 1;
            orc_DT_panel(m, i, j, Kd);
            coo_push_block(C, Kb, Kd, nq2, (int64_t)j * nq2, (int64_t)i * nq2);
        }
        free(Kb); free(Kd);
    }
    for (int i = 0; i < P; ++i) {
        orc_coo* C = parts + i;
        if (C->nnz) {
            if (res->nnz + C->nnz > res->cap) {
                res->cap = (res->nnz + C->nnz) * 2;
                res->rows = (int64_t*)realloc(res->rows, sizeof(int64_t) * res->cap);
                res->cols = (int64_t*)realloc(res->cols, sizeof(int64_t) * res->cap);
                res->vals = (double*)realloc(res->vals, sizeof(double) * res->cap);
            }
            memcpy(res->rows + res->nnz, C->rows, sizeof(int64_t) * C->nnz);
            memcpy(res->cols + res->nnz, C->cols, sizeof(int64_t) * C->nnz);
            memcpy(res->vals + res->nnz, C->vals, sizeof(double) * C->nnz);
            res->nnz += C->nnz;
        }
        if (C->hit_max) res->hit_max = 1;
        free(C->rows); free(C->cols); free(C->vals);
    }
    free(parts); free(nup_max);
    return res;
}

/* ------------------------------------------------------------------------- */
/* The corrected operator  A x = D^T_direct x + C x + diag .* x               */
/* (src/kernel/laplace3d_near.jl:395-419; src/solver/dielectric_box3d.jl:48-92)*/
/* C given as CSC (Julia SparseMatrixCSC, 0-based here). Vectors length N.    */
/* ------------------------------------------------------------------------- */
typedef struct {
    int64_t N; const double *pts, *nrm, *w, *diag;
    const int64_t *colptr, *rowidx; const double* cval;  /* may be NULL */
    int nthreads;
} orc_op;

static void op_apply(const orc_op* op, const double* x, double* y) {
    orc_DT_apply(op->N, op->pts, op->nrm, op->w, x, y, 1, op->nthreads);
    if (op->colptr)
        for (int64_t c = 0; c < op->N; ++c)
            for (int64_t e = op->colptr[c]; e < op->colptr[c + 1]; ++e) y[op->rowidx[e]] += op->cval[e] * x[c];
    for (int64_t i = 0; i < op->N; ++i) y[i] += op->diag[i] * x[i];
}

void orc_op_apply(int64_t N, const double* pts, const double* nrm, const double* w, const double* diag,
                  const int64_t* colptr, const int64_t* rowidx, const double* cval, const double* x, double* y,
                  int nthreads) {
    orc_op op = {N, pts, nrm, w, diag, colptr, rowidx, cval, nthreads};
    op_apply(&op, x, y);
}

static double dnrm2(int64_t n, const double* x) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += x[i] * x[i];
    return sqrt(s);
}

/* Full GMRES with MGS + Givens, x0 = 0 (Krylov.jl 0.10.2 gmres as called by
 * solve_gmres, src/utils/linear_algebra.jl:3-5). Returns iterations; *resid =
 * final residual-norm estimate. */
int orc_gmres(int64_t N, const double* pts, const double* nrm, const double* w, const double* diag,
              const int64_t* colptr, const int64_t* rowidx, const double* cval, const double* b, double* x,
              double atol, double rtol, int itmax, int nthreads, double* resid) {
    orc_op op = {N, pts, nrm, w, diag, colptr, rowidx, cval, nthreads};
    int mcap = itmax + 1;
    double bn = dnrm2(N, b);
    for (int64_t i = 0; i < N; ++i) x[i] = 0.0;
    if (bn == 0.0) { *resid = 0.0; return 0; }
    double eps = atol + rtol * bn;
    double* V = (double*)malloc(sizeof(double) * N * (size_t)(mcap < 2 ? 2 : (mcap > 2000 ? 2000 : mcap)));
    int vcap = mcap > 2000 ? 2000 : mcap;
    double* H = (double*)calloc((size_t)vcap * vcap, sizeof(double)); /* H[i + j*vcap] */
    double* cs = (double*)malloc(sizeof(double) * vcap); double* sn = (double*)malloc(sizeof(double) * vcap);
    double* g = (double*)calloc(vcap + 1, sizeof(double));
    double* wv = (double*)malloc(sizeof(double) * N);
    for (int64_t i = 0; i < N; ++i) V[i] = b[i] / bn;
    g[0] = bn;
    double rnorm = bn;
    int j = 0;
    while (j < itmax && j + 1 < vcap && rnorm > eps) {
        op_apply(&op, V + (size_t)j * N, wv);
        for (int i = 0; i <= j; ++i) {
            double h = 0.0; const double* vi = V + (size_t)i * N;
            for (int64_t t = 0; t < N; ++t) h += vi[t] * wv[t];
            H[i + j * vcap] = h;
            for (int64_t t = 0; t < N; ++t) wv[t] -= h * vi[t];
        }
        double hn = dnrm2(N, wv);
        H[(j + 1) + j * vcap] = hn;
        if (hn != 0.0) for (int64_t t = 0; t < N; ++t) V[(size_t)(j + 1) * N + t] = wv[t] / hn;
        for (int i = 0; i < j; ++i) {
            double a = H[i + j * vcap], bb = H[(i + 1) + j * vcap];
            H[i + j * vcap] = cs[i] * a + sn[i] * bb;
            H[(i + 1) + j * vcap] = -sn[i] * a + cs[i] * bb;
        }
        double a = H[j + j * vcap], bb = H[(j + 1) + j * vcap];
        double r = hypot(a, bb);
        cs[j] = a / r; sn[j] = bb / r;
        H[j + j * vcap] = r; H[(j + 1) + j * vcap] = 0.0;
        g[j + 1] = -sn[j] * g[j]; g[j] = cs[j] * g[j];
        rnorm = fabs(g[j + 1]);
        ++j;
        if (hn == 0.0) break;
    }
    /* back substitution */
    double* yv = (double*)malloc(sizeof(double) * (j > 0 ? j : 1));
    for (int i = j - 1; i >= 0; --i) {
        double s = g[i];
        for (int l = i + 1; l < j; ++l) s -= H[i + l * vcap] * yv[l];
        yv[i] = s / H[i + i * vcap];
    }
    for (int i = 0; i < j; ++i) {
        const double* vi = V + (size_t)i * N;
        for (int64_t t = 0; t < N; ++t) x[t] += yv[i] * vi[t];
    }
    *resid = rnorm;
    free(V); free(H); free(cs); free(sn); free(g); free(wv); free(yv);
    return j;
}

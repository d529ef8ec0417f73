// Host-side geometry setup of the B200 library: panel mesher, near-pair list and
// near-field correction blocks (block-sparse, one nq^2 x nq^2 block per near
// panel pair). This is setup work the reference also runs on the host; the hot
// path (direct sums, correction apply, GMRES) runs on the GPU.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace bie {

struct Mesh {
    int nq = 0;
    int npanels = 0;
    std::vector<double> corners;  // P x 4 x 3, corners (a, b, c, d) anti-clockwise
    std::vector<double> normals;  // P x 3 outward unit normals
    std::vector<int> is_edge;     // P
    std::vector<double> eps_in, eps_out;  // P
    std::vector<double> glx, glw, bary;   // Gauss-Legendre nodes/weights, barycentric weights
    std::vector<double> pts;  // N x 3 (== 3 x N column-major)
    std::vector<double> w;    // N
    int64_t npoints() const { return (int64_t)npanels * nq * nq; }
    void finalize();           // fills pts/w from the panels
    void diag(double* out) const;
};

// FastGaussQuadrature.jl gausslegendre (ascending nodes).
void gauss_legendre(int n, double* x, double* w);
// best_grid_mn (src/utils/best_grid.jl:8-126); returns 0, -1 (bad argument) or -2 (none found).
int best_grid(double W, double H, double alpha, int* m, int* n);

// single_dielectric_box3d (src/shape/box3d_single.jl:49-70).
int mesh_single_box(double Lx, double Ly, double Lz, int nq, double l_ec, double eps_in, double eps_out,
                    double alpha, Mesh& out, std::string& err);
// multi_dielectric_box3d (src/shape/box3d_multi.jl:358-386), including shared-face subtraction.
int mesh_multi_box(int nq, double l_ec, int nbox, const double* centers, const double* dims, const double* epses,
                   double eps_out, double alpha, Mesh& out, std::string& err);
// DielectricInterface from explicit rect_panel3d_discretize panels (src/shape/box3d.jl:22-64).
int mesh_from_panels(int P, int nq, const double* corners, const double* normals, const int* is_edge,
                     const double* eps_in, const double* eps_out, Mesh& out, std::string& err);

struct NearOpts {
    int max_order = 8;
    double up_tol = 1e-9;
    int correct_edges = 1;
    double adaptive_atol = -1.0;  // < 0 => up_tol
    double adaptive_rtol = 1.4901161193847656e-08;
    int adaptive_n_GL = 0;
    int adaptive_max_depth = 20;
    int nthreads = 0;
    int device = -1;  // >= 0: the adaptive blocks' moment sums and the upsampled blocks (n_up <= 8)
                      // run on this CUDA device (n_quad <= 6)
};

// Moment blocks of the adaptive (touching) pairs on a CUDA device (near_gpu.cu):
// pair p has target panel trg[p], source frame frames[10 p ..] = (cc, b - a, d - a, scale)
// and the quadtree leaves leaves[4 l ..], l in [leaf_off[p], leaf_off[p + 1]); Kb receives
// npairs x (nq^2 x nq^2) blocks in the host's layout, bitwise equal to the host sums.
// Returns 0, or -1 with err set.
int adaptive_blocks_gpu(int device, int nq, int ngl, const double* glx, const double* bary, const double* xg,
                        const double* wg, const double* pts, int64_t npts, const double* normals, int npanels,
                        int npairs, const int* trg, const double* frames, const int64_t* leaf_off,
                        const double* leaves, double* Kb, std::string& err);

// Upsampled blocks on a CUDA device (near_gpu.cu), bitwise equal to the host's: job q is
// source panel job_src[q] at order job_nup[q] (<= 8) with frame job_frame[10 q ..], its
// target panels tgt[tgt_off[q] .. tgt_off[q + 1]); xu/wu/ex are the Gauss nodes, weights and
// barycentric rows of each order n at [n * 9 + i] (ex: [(n * 9 + i) * nq + m]). out receives
// one nq^2 x nq^2 block per pair in the BSR value layout (column-major), upsampled minus
// direct. Returns 0, or -1 with err set.
int upsampled_blocks_gpu(int device, int nq, const double* pts, int64_t npts, const double* w, const double* normals,
                         int npanels, int njobs, const int* job_src, const int* job_nup, const double* job_frame,
                         const int64_t* tgt_off, const int* tgt, const double* xu, const double* wu, const double* ex,
                         double* out, std::string& err);

// Near-field corrections in block-sparse-row form: block rows = target panels,
// block columns = source panels, each block nb x nb (nb = nq^2) stored
// column-major: val[b*nb*nb + s*nb + r] = C[target node r, source node s].
struct Near {
    int nb = 0;
    std::vector<int32_t> rowptr;  // P + 1
    std::vector<int32_t> col;     // nblocks
    std::vector<double> val;      // nblocks * nb * nb
    std::vector<int32_t> ups_i, ups_j, ups_p;  // upsample pairs (source i, target j, order)
    std::vector<int32_t> adp_i, adp_j;         // touching (adaptive) pairs
    int hit_max = 0;
    int64_t nblocks() const { return (int64_t)col.size(); }
};

// build_neighbor_list (src/kernel/laplace3d_near.jl:240-392) + laplace3d_DT_corrections
// (src/kernel/laplace3d_near_upsampling.jl:127-276).
int near_build(const Mesh& m, const NearOpts& o, Near& out, std::string& err);
// Near-accurate probe potentials (laplace3d_pottrg_fmm3d_corrected_hcubature,
// src/kernel/laplace3d_near_hcubature.jl:278-316): phi = (S_refined + C) P sigma.
struct ProbeSetup {
    Mesh refined;                          // interface refined near the probes
    std::vector<int> parent, from_split;   // per refined panel: coarse panel, split or not
    std::vector<int64_t> prow;             // P: refined nodes x coarse nodes, CSR
    std::vector<int32_t> pcol;
    std::vector<double> pval;
    std::vector<int64_t> crow;             // C: probes x refined nodes, CSR
    std::vector<int32_t> ccol;
    std::vector<double> cval;
    int64_t nentries = 0;                  // (refined panel, near probes) entries
    int64_t ncubatures = 0;                // adaptive integrals evaluated
    int64_t capped = 0;                    // of which stopped at maxevals before reaching atol
};
// targets: 3 x M (column-major, as the reference's targets matrix); maxevals bounds each
// adaptive integral's integrand evaluations. Returns 0, or -1 with err set.
int probe_setup(const Mesh& m, const double* targets, int64_t M, double atol, double range_factor, int nthreads,
                int64_t maxevals, ProbeSetup& out, std::string& err);

}  // namespace bie

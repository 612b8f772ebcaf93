// sdot_internal.h -- context layout and shared device helpers of libsdot_cuda.
//
// Data layout in HBM (all FP64 unless noted, internal orderings):
//   source cells are sorted by the Morton code of their centres; quadrature
//   points follow their cell (cell-major, uniform points per cell).  Source
//   blocks = SBLK_CELLS consecutive cells, each with a bounding sphere.
//   targets are sorted by Morton code of their position; target blocks =
//   TBLK consecutive targets with a bounding sphere.
// Per evaluation:
//   tpack[j] = {A_j, B_j(dim), nu_j, y_j(dim)} padded to 8 doubles, where the
//     scaled exponent is b_qj = A_j + B_j.xt_q + C_q = kappa*(psi_j-|x_q-y_j|^2/2)/eps,
//     kappa = 16/ln 2 (units of 2^(1/16)), xt = x - origin;
//   Lq[q] = log of the reference's total_sum_exp at q (natural units, +inf if
//     the point is skipped), written by the value sweep and read by the
//     gradient sweep.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/sdot.h"

namespace sdot {

constexpr int SBLK_CELLS = 8;        // cells per source block (value sweep, one warp per cell)
constexpr int TBLK = 64;             // targets per target block (gradient sweep CTA)
constexpr int DENSE_A_THREADS = 128; // dense value sweep: threads per CTA
constexpr int DENSE_A_QT = 4;        // dense value sweep: quadrature points per thread
constexpr int DENSE_B_THREADS = 128; // dense gradient sweep: threads per CTA
constexpr int DENSE_B_TT = 2;        // dense gradient sweep: targets per thread
constexpr int TPACK = 8;             // doubles per packed target
constexpr int MAX_QPC = 64;          // quadrature points per cell supported
constexpr double KAPPA = 23.083120654223414;  // 16 / ln 2
constexpr double LOG2E = 1.4426950408889634;

// Scalars produced by one evaluation (device buffer, read back in one copy).
enum ScalarSlot {
    SC_VALUE = 0,      // J(psi)
    SC_C = 1,          // C_global
    SC_DOT_GP = 2,     // g . p  (line search)
    SC_L1 = 3,         // ||g||_1
    SC_LINF = 4,       // max |g_j|
    SC_COMP = 5,       // max_j (|g_j| - nu_j * tol)
    SC_L2SQ = 6,       // ||g||_2^2
    SC_PSINU = 7,      // sum psi_j nu_j
    SC_SKIPPED = 8,    // number of skipped quadrature points
    SC_MAXPSI = 9,
    SC_MINPSI = 10,
    SC_PSIBAD = 11,    // 1 if psi has a non-finite entry
    SC_R = 12,         // threshold used
    SC_SSTAR = 13,     // squared-distance bound equivalent to sqrt_rn(d2) <= r
    SC_NONFINITE = 14, // 1 if value or gradient not finite
    SC_PAIRS = 15,     // candidate pairs of the evaluation
    SC_VALSRC = 16,    // source part of J (before the linear term)
    SC_COUNT = 20
};

template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t alloc(size_t count) {
        if (count <= n && p) return cudaSuccess;
        release();
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e == cudaSuccess) n = count;
        else p = nullptr;
        return e;
    }
    size_t bytes() const { return n * sizeof(T); }
};

struct EvalPlan {
    bool dense = true;         // every (cell, target) pair is a candidate
    int64_t n_dense_ablk = 0;  // CTAs of the dense value sweep
    int n_ksplit = 1;          // q-slices of the dense gradient sweep
};

}  // namespace sdot

struct sdot_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int precision = SDOT_PREC_HYBRID;
    size_t budget = 0;
    int verbose = 0;
    std::string err;

    // ---- source (internal order) ----
    int dim = 0;
    int64_t nq = 0, ncells = 0;
    int qpc = 0;                       // quadrature points per cell (uniform)
    bool w_nonneg = true;              // all rho*JxW >= 0
    sdot::DevBuf<double> x, rho, jxw, w, lw;  // x: nq*dim
    sdot::DevBuf<double> cell_ctr;     // ncells*dim
    int64_t nsblk = 0;                 // value-sweep blocks (8 warp units each)
    sdot::DevBuf<double> sblk_sph;     // 4 per block: centre(3), radius
    int64_t ncblk = 0;                 // gradient-sweep cell blocks (SBLK_CELLS cells)
    sdot::DevBuf<double> cblk_sph;
    int ql = 0, ngroups = 1;           // quadrature points per warp unit, units per cell
    std::vector<double> cell_ctr_host; // internal order, for the covering radius
    double src_lo[3] = {0, 0, 0}, src_hi[3] = {0, 0, 0};

    // ---- target (internal order) ----
    int64_t nt = 0;
    sdot::DevBuf<double> y, nu;        // y: nt*dim
    sdot::DevBuf<int64_t> perm;        // internal index -> caller index
    int64_t ntblk = 0;
    sdot::DevBuf<double> tblk_sph;     // 4 per block
    std::vector<double> nu_host;       // caller order
    std::vector<double> y_host;        // caller order
    double tgt_lo[3] = {0, 0, 0}, tgt_hi[3] = {0, 0, 0};

    double origin[3] = {0, 0, 0};      // centring point of the value sweep
    double diam = 0;                   // diameter bound of cells U targets

    // ---- per-evaluation buffers ----
    sdot::DevBuf<double> psi, grad, tpack, Lq, gpart, blkpart, scal, redpart;
    sdot::DevBuf<double> io_a, io_b;   // caller-order staging
    double *scal_host = nullptr;       // pinned, SC_COUNT doubles

    // ---- parameters and reference-like persistent state ----
    sdot_solver_params prm{};
    double global_functional = 0.0;
    double C_global = 0.0;
    double covering_radius = 0.0;
    double min_target_density = 0.0;
    double current_distance_threshold = 1e-1;
    unsigned last_iterations = 0;
    int last_converged = 0;
    bool have_solve = false;

    // ---- solver buffers ----
    sdot::DevBuf<double> x0, pdir, sk, yk, hist_s, hist_y, gtmp;

    int64_t last_pairs = 0;

    // ---- measurement ----
    bool profiling = false;
    cudaEvent_t pev[8] = {};
    double kms[6] = {0, 0, 0, 0, 0, 0};
    int64_t klaunch[6] = {0, 0, 0, 0, 0, 0};
};

namespace sdot {

// Internal entry points shared between translation units.
sdot_status set_error(sdot_ctx *c, sdot_status s, const std::string &msg);
sdot_status cuda_error(sdot_ctx *c, cudaError_t e, const char *where);

// Evaluate J and grad at c->psi (internal order, device).  p_dir (device,
// internal order) may be null; when given, g.p is computed too.  Fills
// c->scal_host and updates the persistent state.  r_host: threshold computed
// on the host (integral/geometric) or NaN to let the device compute the
// pointwise threshold.
sdot_status evaluate_internal(sdot_ctx *c, const double *p_dir, double comp_tol,
                              double *ms_out, bool partial = false);

// Threshold for the current psi (host computation mirroring
// SotSolver::compute_distance_threshold), using device reductions for max/min.
double host_threshold(sdot_ctx *c, double maxpsi, double minpsi);

// largest double s with sqrt_rn(s) <= r
double sstar_of(double r);

sdot_status launch_gather(sdot_ctx *c, double *dst, const double *src, int64_t n);
sdot_status launch_scatter(sdot_ctx *c, double *dst, const double *src, int64_t n);
sdot_status launch_minmax(sdot_ctx *c, const double *v, int64_t n, double *mx, double *mn);

// L-BFGS helpers (device vector kernels)
void k_axpy_launch(cudaStream_t s, double *x, const double *x0, double a, const double *p, int64_t n);

}  // namespace sdot

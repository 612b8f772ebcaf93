// sdot_internal.h -- context layout and shared device helpers of libsdot_cuda.
//
// Data layout in HBM (all FP64 unless noted, internal orderings):
//   source cells are ordered by a k-d tree over their centres (leaves of at
//   most SBLK_UNITS warp units = source blocks); quadrature points follow
//   their cell (cell-major, uniform points per cell).  Targets are ordered by
//   a k-d tree over their positions (leaves of at most TBLK_KD = target
//   blocks).  Every block has a bounding sphere (FP64 and conservative FP32).
// Per evaluation:
//   tpack[j], 8 doubles: dense path {A_j, B_j(dim), nu_j, y_j(dim)} where the
//     scaled exponent is b_qj = A_j + B_j.xt_q + C_q = kappa*(psi_j-|x_q-y_j|^2/2)/eps,
//     kappa = 16/ln 2 (units of 2^(1/16)), xt = x - origin; truncated path
//     {y_j(3), nu_j, log2 nu_j, kappa psi_j / eps};
//   Lq[q] = log of the reference's total_sum_exp at q (natural units, +inf if
//     the point is skipped), written by the value sweep and read by the
//     gradient sweep.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include <string>
#include <vector>

#include "../../include/sdot.h"

namespace sdot {

constexpr int SBLK_UNITS = 8;        // warp units (cell, q-group) per source block
constexpr int TBLK_KD = 32;          // max targets per target block (k-d tree leaf)
constexpr int DENSE_A_THREADS = 128; // dense value sweep: threads per CTA
constexpr int DENSE_A_QT = 1;        // dense value sweep: quadrature points per thread (1: the most CTAs for small sources)
constexpr int DENSE_B_THREADS = 128; // dense gradient sweep: threads per CTA
constexpr int DENSE_B_TT = 2;        // dense gradient sweep: targets per thread
constexpr int DENSE_B_QG = 4;        // dense gradient sweep: point groups per CTA (single-problem path)
constexpr int DENSE_B_CTA = DENSE_B_THREADS * DENSE_B_QG;  // its threads per CTA

// Quadrature slices of the single-problem dense gradient sweep for nq points
// and nt targets: the (target block, slice) CTAs fill two CTAs per SM of a
// 148-SM part (rounded down, so that they run as one wave), slices of at
// least 256 points, at most DENSE_B_MAXKS.  Two CTAs of DENSE_B_CTA threads
// per SM (32 warps) measured faster than three with registers capped at 40
// (spills) and than 256-thread CTAs.
constexpr int DENSE_B_MAXKS = 128;
constexpr int DENSE_B_PER_SM = 2;
inline int dense_grad_slices(int64_t nq, int64_t nt)
{
    const int64_t tb = (nt + DENSE_B_THREADS * DENSE_B_TT - 1) / (DENSE_B_THREADS * DENSE_B_TT);
    int64_t k = (int64_t)148 * DENSE_B_PER_SM / (tb > 0 ? tb : 1);
    const int64_t maxks = (nq + 255) / 256;
    if (k > maxks) k = maxks;
    if (k > DENSE_B_MAXKS) k = DENSE_B_MAXKS;
    return (int)(k < 1 ? 1 : k);
}
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

// Allocation-failure injection for tests (sdot_debug_fail_allocation): when
// the countdown is >= 0, every device allocation made through DevBuf counts
// it down, and the one that finds it at 0 fails with
// cudaErrorMemoryAllocation without calling cudaMalloc.  -1: off.  The
// counter counts the allocations that reached cudaMalloc or were failed.
inline std::atomic<long long> g_alloc_countdown{-1};
inline std::atomic<long long> g_alloc_count{0};

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
        g_alloc_count.fetch_add(1);
        long long left = g_alloc_countdown.load();
        while (left >= 0 && !g_alloc_countdown.compare_exchange_weak(left, left - 1)) {
        }
        if (left == 0) return cudaErrorMemoryAllocation;
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
    sdot::DevBuf<double> x, rho, jxw, w;  // x: nq*dim
    sdot::DevBuf<double> cell_ctr;     // ncells*dim
    int64_t nsblk = 0;                 // source blocks (k-d leaves)
    sdot::DevBuf<int64_t> sblk_cell;   // first cell of each block (nsblk + 1)
    sdot::DevBuf<double> sblk_sph;     // 4 per block: centre(3), radius (FP64)
    sdot::DevBuf<float4> sblk_sph32;   // conservative FP32 spheres
    int ql = 0, ngroups = 1;           // quadrature points per warp unit, units per cell
    std::vector<double> cell_ctr_host; // internal order, for the covering radius
    std::vector<double> src_sph_host, tgt_sph_host;  // FP64 block spheres (4 per block)
    double src_lo[3] = {0, 0, 0}, src_hi[3] = {0, 0, 0};

    // ---- target (internal order) ----
    int64_t nt = 0;
    sdot::DevBuf<double> y, nu;        // y: nt*dim
    sdot::DevBuf<int64_t> perm;        // internal index -> caller index
    int64_t ntblk = 0;                 // target blocks (k-d leaves)
    sdot::DevBuf<int64_t> tblk_off;    // first target of each block (ntblk + 1)
    sdot::DevBuf<double> tblk_sph;     // 4 per block
    sdot::DevBuf<float4> tblk_sph32;
    std::vector<double> nu_host;       // caller order
    double nu_min = 0.0;               // min of nu_host (set with the targets)
    std::vector<double> y_host;        // caller order
    double tgt_lo[3] = {0, 0, 0}, tgt_hi[3] = {0, 0, 0};

    double origin[3] = {0, 0, 0};      // centring point of the dense value sweep
    double diam = 0;                   // diameter bound of cells U targets
    double coord_scale = 1.0;          // max |coordinate|, for FP32 cull margins
    double delta_max = 0.0;            // max distance of a quadrature point to its cell centre
    int tensor_m = 0;                  // > 0: points form an m^dim tensor grid symmetric about the cell centre
    double tensor_amax = 0.0;          // largest per-dimension offset of that grid
    bool tensor_uniform = false;       // the same offset per dimension in every cell (within 1e-13)
    double tensor_a[3] = {0, 0, 0};    // that offset

    // ---- truncated path: block-pair lists and gradient partials ----
    sdot::DevBuf<int64_t> fwd_cnt, fwd_off, inv_cnt, inv_off, fwd2inv;
    sdot::DevBuf<int> fwd_t, inv_b, shit, spidx, scount, pmpre, inv_tmpb;
    sdot::DevBuf<int64_t> inv_tmpk;    // inverse-list scatter (forward position per entry)
    sdot::DevBuf<unsigned> pmask;
    sdot::DevBuf<unsigned char> superpair;
    sdot::DevBuf<float4> ssup_sph32, tsup_sph32;  // super-block spheres (32 blocks each)
    sdot::DevBuf<double> part;
    size_t part_cap_bytes = (size_t)4 << 30;

    // ---- per-evaluation buffers ----
    sdot::DevBuf<double> psi, grad, tpack, Lq, gpart, blkpart, scal, redpart;
    sdot::DevBuf<double> vpart;        // dense value sweep: per (target slice, point) largest exponent and sum
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

    // ---- tensor-core Hessian (sdot_hessian_tc.cu) and Newton solver ----
    sdot::DevBuf<double> htc_tdat, htc_diag, htc_blk, htc_scr;
    sdot::DevBuf<float> htc_qa, htc_qb;
    sdot::DevBuf<int> htc_tiles, htc_err;
    sdot::DevBuf<float> htc_cd, htc_qw;  // factored generation: per-chunk cell data, per-point factors
    bool hess_factored = true;         // factored generation where the source allows it (sdot_set_hessian_generation)
    bool hess_last_factored = false;   // the last tensor Hessian used it
    int hess_pair_mode = 2;            // whole tensor Hessians: 0 single SMs, 1 SM pairs, 2 SM pairs with two
                                       // generation groups (sdot_set_hessian_pairs)
    int hess_last_pair = 0;            // the mode the last tensor Hessian ran in
    double hess_kernel_ms = 0.0;
    int64_t hess_tiles = 0;
    int distance = 0;                  // distance function: 0 euclidean, 1 spherical (sdot_set_distance_function)
    int hess_chunk = 64;               // stages (x 64 points) per FP32 accumulation chunk
    long long hess_wait_limit = 0;     // SM clocks per stage-loop mbarrier wait (<= 0: the default, ~1 s)
    double newton_reuse = 0.1;         // lagged-Hessian contraction threshold (0: recompute every step)
    sdot::DevBuf<float> nt_H32;        // Newton: tensor-core Hessian (caller order)
    sdot::DevBuf<double> nt_H64;       // Newton: FP64 Hessian when the tensor method does not apply
    sdot::DevBuf<double> nt_vec;       // Newton/CG vectors (caller order)

    // ---- measurement ----
    bool profiling = false;
    cudaEvent_t pev[8] = {};
    // phases: threshold, target prep, value sweep, gradient sweep, finalize,
    // layout (gather/scatter), block-pair lists
    double kms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t klaunch[8] = {0, 0, 0, 0, 0, 0, 0, 0};

    // ---- CUDA graph of the untruncated evaluation (sdot_eval.cu) ----
    // Captured on the second consecutive evaluation with the same launch key
    // (sizes, parameters, buffer addresses), replayed while the key holds.
    cudaGraphExec_t dg_exec = nullptr;
    std::vector<unsigned char> dg_key;
    bool dg_armed = false;
    bool graphs_off = false;           // set when capture failed: every evaluation runs eagerly
    int64_t dg_launches[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};

namespace sdot {

// Internal entry points shared between translation units.
sdot_status set_error(sdot_ctx *c, sdot_status s, const std::string &msg);
sdot_status cuda_error(sdot_ctx *c, cudaError_t e, const char *where);

// Evaluate J and grad at c->psi (internal order, device).  p_dir (device,
// internal order) may be null; when given, g.p is computed too.  Fills
// c->scal_host and updates the persistent state.
sdot_status evaluate_internal(sdot_ctx *c, const double *p_dir, double comp_tol,
                              double *ms_out, bool partial = false);
// The same in two halves, so that a caller can queue more work (the
// gradient's scatter, its copy to the host) before the one wait for the
// stream: evaluate_enqueue queues the evaluation and the copy of its scalars
// to c->scal_host; after the caller has synchronised c->stream,
// evaluate_complete reads them (and the timing events) and updates the state.
struct EvalPending {
    double r = 0.0;
    bool dense = false;
    bool ranged = false;   // the ψ range was computed (for the threshold)
};
sdot_status evaluate_enqueue(sdot_ctx *c, const double *p_dir, double comp_tol, bool partial, EvalPending &pend);
sdot_status evaluate_complete(sdot_ctx *c, const EvalPending &pend, double *ms_out);

// Threshold for the current psi (host computation mirroring
// SotSolver::compute_distance_threshold), using device reductions for max/min.
double host_threshold(sdot_ctx *c, double maxpsi, double minpsi);

// largest double s with sqrt_rn(s) <= r
double sstar_of(double r);

sdot_status launch_gather(sdot_ctx *c, double *dst, const double *src, int64_t n);
sdot_status launch_scatter(sdot_ctx *c, double *dst, const double *src, int64_t n);
sdot_status launch_minmax(sdot_ctx *c, const double *v, int64_t n, double *mx, double *mn);

struct EvalArgs;
// truncated evaluation (block-pair lists, fused sweeps, partial reduction)
sdot_status run_trunc(sdot_ctx *c, const EvalArgs &a, double r);
// value and gradient sweeps with the spherical distance (sdot_spherical.cu);
// *nval: the value blocks whose partials k_finalize_scalars sums
sdot_status run_spherical(sdot_ctx *c, const EvalArgs &a, double r, int64_t *nval);
// dense-layout tpack for the current psi (used by the Hessian)
void launch_target_prep_dense(sdot_ctx *c, const EvalArgs &a);

// Tensor-core Hessian (BF16 hi+lo on tcgen05, FP64 drains) at the potential of
// the last untruncated evaluation; H_dev n x n row-major in the caller's order.
// Tiles [tile_begin, tile_end) of the upper-triangle tile list only (tile_end < 0: all); entries of other tiles
// are left untouched.
sdot_status hessian_tc(sdot_ctx *c, void *H_dev, bool out_f32, int chunk_stages, double *ms_out,
                       int64_t tile_begin = 0, int64_t tile_end = -1);
// Number of 128 x 256 tiles of the upper triangle for n targets.
int64_t hessian_tc_tiles(int64_t n);
// Evaluation at psi_dev (caller order) followed by the Hessian by `method`.
sdot_status hessian_device(sdot_ctx *c, const double *psi_dev, void *H_dev, int method, int out_f32,
                           sdot_hessian_info *info);
sdot_status ensure_eval_buffers(sdot_ctx *c);
// VerboseSolverControl::check on the last evaluation's scalars: 1 converged,
// 0 iterate, -1 failure (max_iterations reached or NaN).
int solver_control_check(sdot_ctx *c, unsigned step, double *value);

// L-BFGS helpers (device vector kernels)
void k_axpy_launch(cudaStream_t s, double *x, const double *x0, double a, const double *p, int64_t n);

}  // namespace sdot

// sdot_newton.cu -- Newton solver for the entropic dual with the tensor-core Hessian.
//
// The reference declares SotSolver::compute_hessian (include/SemiDiscreteOT/
// solvers/SotSolver.h:343-344) but only ever drives the functional with
// deal.II's SolverBFGS (SotSolver::solve, src/solvers/SotSolver.cc:105-215).
// This file adds the second-order method that the Hessian is for, with the
// same parameters, convergence control (VerboseSolverControl l1norm /
// componentwise / linf) and in-place potential update as SotSolver::solve:
//
//   repeat:  evaluate J(psi), g(psi) in FP64              (sdot_eval.cu)
//            H(psi) on tcgen05, BF16 hi+lo, stored FP32   (sdot_hessian_tc.cu)
//            solve H p = -g by Jacobi-preconditioned CG: FP64 vectors and
//              recurrences, the constant null vector projected out of every
//              residual, the true residual b - H x recomputed in FP64 every
//              RESTART iterations (residual replacement);
//            Armijo backtracking on J in FP64 (c1 = 1e-4, halving);
// until the control's check value is below the tolerance.
//
// All vectors stay on the device in the caller's target order (the Hessian's
// order); the host reads one scalar block per CG check and per trial step.
// CG reductions run in one CTA with a fixed order, so a solve is bitwise
// repeatable.
#include <float.h>
#include <math.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "sdot_device.cuh"
#include "sdot_internal.h"

namespace sdot {

sdot_status hessian_fp64_to(sdot_ctx *c, double *H_dev);
bool hessian_tensor_ok(const sdot_ctx *c);

namespace {

constexpr int CG_THREADS = 1024;
constexpr int CG_CHECK = 8;        // CG iterations between host convergence checks
constexpr int CG_RESTART = 64;     // iterations between residual replacements
constexpr int MAX_HALVINGS = 40;

// CG scalar slots (device)
enum { S_RZ = 0, S_RR = 1, S_BB = 2, S_PAP = 3, S_GP = 4, S_COUNT = 8 };

// Fixed-order block sum (all threads get the result).
__device__ double block_sum(double v, double *sh)
{
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double t = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
    if (w == 0) t = warp_sum(t);
    if (threadIdx.x == 0) sh[32] = t;
    __syncthreads();
    return sh[32];
}

// y = H x, H row-major n x n (float or double), FP64 accumulation; one warp per row.
template <typename T>
__global__ void __launch_bounds__(256) k_matvec(const T *__restrict__ H, const double *__restrict__ x,
                                                double *__restrict__ y, int64_t n)
{
    const int lane = threadIdx.x & 31;
    const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t r = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); r < n; r += nw) {
        const T *row = H + r * n;
        double acc = 0.0;
        for (int64_t j = lane; j < n; j += 32) acc = fma((double)__ldg(row + j), x[j], acc);
        acc = warp_sum(acc);
        if (lane == 0) y[r] = acc;
    }
}

template <typename T>
__global__ void k_diag(const T *__restrict__ H, double *__restrict__ D, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double d = (double)H[i * n + i];
        D[i] = d > 0.0 ? d : 1.0;
    }
}

// r = b - mean(b) with b = -g (or b - Ax when Ax != null); z = r / D; p = z;
// x = 0 unless keep_x; sc[RZ] = r.z, sc[RR] = r.r, sc[BB] = |b|^2 (first call).
__global__ void __launch_bounds__(CG_THREADS) k_cg_start(int64_t n, const double *__restrict__ g,
                                                         const double *__restrict__ Ax, const double *__restrict__ D,
                                                         double *__restrict__ x, double *__restrict__ r,
                                                         double *__restrict__ z, double *__restrict__ p,
                                                         double *__restrict__ sc, int keep_x)
{
    __shared__ double sh[33];
    double s = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double b = -g[i] - (Ax ? Ax[i] : 0.0);
        r[i] = b;
        s += b;
    }
    const double mean = block_sum(s, sh) / (double)n;
    double rz = 0.0, rr = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double ri = r[i] - mean;
        r[i] = ri;
        const double zi = ri / D[i];
        z[i] = zi;
        p[i] = zi;
        if (!keep_x) x[i] = 0.0;
        rz = fma(ri, zi, rz);
        rr = fma(ri, ri, rr);
    }
    rz = block_sum(rz, sh);
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) {
        sc[S_RZ] = rz;
        sc[S_RR] = rr;
        if (!keep_x) sc[S_BB] = rr;
    }
}

// One PCG step after Ap = H p.
__global__ void __launch_bounds__(CG_THREADS) k_cg_step(int64_t n, const double *__restrict__ Ap,
                                                        const double *__restrict__ D, double *__restrict__ x,
                                                        double *__restrict__ r, double *__restrict__ z,
                                                        double *__restrict__ p, double *__restrict__ sc)
{
    __shared__ double sh[33];
    double pap = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) pap = fma(p[i], Ap[i], pap);
    pap = block_sum(pap, sh);
    const double rz = sc[S_RZ];
    if (!(pap > 0.0)) {
        // H p = 0 numerically: nothing left to reduce in this direction
        if (threadIdx.x == 0) { sc[S_PAP] = pap; sc[S_RR] = 0.0; }
        return;
    }
    const double alpha = rz / pap;
    double s = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        x[i] = fma(alpha, p[i], x[i]);
        const double ri = fma(-alpha, Ap[i], r[i]);
        r[i] = ri;
        s += ri;
    }
    const double mean = block_sum(s, sh) / (double)n;
    double rz2 = 0.0, rr = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double ri = r[i] - mean;
        r[i] = ri;
        const double zi = ri / D[i];
        z[i] = zi;
        rz2 = fma(ri, zi, rz2);
        rr = fma(ri, ri, rr);
    }
    rz2 = block_sum(rz2, sh);
    rr = block_sum(rr, sh);
    const double beta = rz2 / rz;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) p[i] = fma(beta, p[i], z[i]);
    if (threadIdx.x == 0) {
        sc[S_RZ] = rz2;
        sc[S_RR] = rr;
        sc[S_PAP] = pap;
    }
}

__global__ void __launch_bounds__(CG_THREADS) k_dot(int64_t n, const double *__restrict__ a,
                                                    const double *__restrict__ b, double *__restrict__ out)
{
    __shared__ double sh[33];
    double s = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s = fma(a[i], b[i], s);
    s = block_sum(s, sh);
    if (threadIdx.x == 0) *out = s;
}

__global__ void k_neg(int64_t n, const double *__restrict__ a, double *__restrict__ b)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = -a[i];
}

struct Vecs {
    double *gc, *x, *r, *z, *p, *Ap, *D, *sc;
};

template <typename T>
void launch_matvec(sdot_ctx *c, const T *H, const double *x, double *y, int64_t n)
{
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    const int64_t blocks = std::min<int64_t>((n + 7) / 8, (int64_t)sms * 8);
    k_matvec<T><<<(unsigned)blocks, 256, 0, c->stream>>>(H, x, y, n);
}

// PCG on H x = -g (caller order).  Returns iterations; *rel = final |r| / |b|.
template <typename T>
sdot_status pcg(sdot_ctx *c, const T *H, const Vecs &v, int64_t n, double eta, int max_it, int *iters, double *rel)
{
    k_diag<T><<<(unsigned)std::min<int64_t>((n + 255) / 256, 1184), 256, 0, c->stream>>>(H, v.D, n);
    k_cg_start<<<1, CG_THREADS, 0, c->stream>>>(n, v.gc, nullptr, v.D, v.x, v.r, v.z, v.p, v.sc, 0);
    double hs[S_COUNT];
    cudaError_t e = cudaMemcpyAsync(hs, v.sc, sizeof(hs), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_error(c, e, "cg start");
    const double bb = hs[S_BB];
    *iters = 0;
    *rel = 0.0;
    if (!(bb > 0.0)) return SDOT_OK;
    int it = 0;
    while (it < max_it) {
        launch_matvec<T>(c, H, v.p, v.Ap, n);
        k_cg_step<<<1, CG_THREADS, 0, c->stream>>>(n, v.Ap, v.D, v.x, v.r, v.z, v.p, v.sc);
        ++it;
        if (it % CG_RESTART == 0) {
            // residual replacement: r = b - H x in FP64, restart the directions
            launch_matvec<T>(c, H, v.x, v.Ap, n);
            k_cg_start<<<1, CG_THREADS, 0, c->stream>>>(n, v.gc, v.Ap, v.D, v.x, v.r, v.z, v.p, v.sc, 1);
        }
        if (it % CG_CHECK == 0 || it == max_it) {
            e = cudaMemcpyAsync(hs, v.sc, sizeof(hs), cudaMemcpyDeviceToHost, c->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
            if (e != cudaSuccess) return cuda_error(c, e, "cg");
            if (!std::isfinite(hs[S_RR])) return set_error(c, SDOT_ENONFINITE, "non-finite CG residual");
            *rel = std::sqrt(hs[S_RR] / bb);
            if (*rel <= eta) break;
        }
    }
    *iters = it;
    return cuda_error(c, cudaGetLastError(), "cg");
}

float elapsed(cudaEvent_t a, cudaEvent_t b)
{
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

}  // namespace
}  // namespace sdot

using namespace sdot;

extern "C" sdot_status sdot_solve_newton(sdot_ctx *c, double *psi, const sdot_solver_params *params,
                                         int hessian_method, sdot_newton_info *info)
{
    if (!c || !psi) return SDOT_EINVAL;
    if (c->distance != 0) return sdot::set_error(c, SDOT_EINVAL, "Newton supports the euclidean distance only");
    if (hessian_method != SDOT_HESS_AUTO && hessian_method != SDOT_HESS_FP64 && hessian_method != SDOT_HESS_TENSOR)
        return set_error(c, SDOT_EINVAL, "unknown Hessian method");
    if (params) {
        sdot_status s = sdot_configure(c, params);
        if (s != SDOT_OK) return s;
    }
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    struct Restore {
        int p, d;
        ~Restore() { if (p >= 0 && p != d) cudaSetDevice(p); }
    } restore{prev, c->device};
    if (c->nq == 0 || c->nt == 0) return set_error(c, SDOT_ESTATE, "Invalid measures configuration");
    sdot_status s = ensure_eval_buffers(c);
    if (s != SDOT_OK) return s;
    const int64_t n = c->nt;
    if (n > 46340) return set_error(c, SDOT_EBUDGET, "Newton with a dense Hessian is limited to n_targets <= 46340");
    cudaError_t e = c->nt_vec.alloc((size_t)n * 7 + 16);
    if (e == cudaSuccess) e = c->x0.alloc(n);
    if (e == cudaSuccess) e = c->pdir.alloc(n);
    if (e != cudaSuccess) return cuda_error(c, e, "alloc newton");
    Vecs v{};
    v.gc = c->nt_vec.p;
    v.x = v.gc + n;
    v.r = v.x + n;
    v.z = v.r + n;
    v.p = v.z + n;
    v.Ap = v.p + n;
    v.D = v.Ap + n;
    v.sc = v.D + n;

    // solve() prologue (SotSolver.cc:131-133): covering radius and min density
    double cov = 0.0;
    if ((s = sdot_compute_covering_radius(c, &cov)) != SDOT_OK) return s;
    c->covering_radius = cov * 1.1;
    c->min_target_density = c->nu_min;
    c->have_solve = true;

    e = cudaMemcpyAsync(c->io_a.p, psi, n * 8, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return cuda_error(c, e, "copy psi");
    if ((s = launch_gather(c, c->psi.p, c->io_a.p, n)) != SDOT_OK) return s;

    cudaEvent_t t0 = nullptr, t1 = nullptr;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    struct Ev {
        cudaEvent_t a, b;
        ~Ev() { cudaEventDestroy(a); cudaEventDestroy(b); }
    } evs{t0, t1};

    double eval_ms = 0, hess_ms = 0, cg_ms = 0, ms = 0;
    int64_t evals = 0, cg_total = 0, pairs = 0;
    int used_method = 0;
    const double tol = c->prm.tolerance;
    s = evaluate_internal(c, nullptr, tol, &ms);
    ++evals;
    eval_ms += ms;
    pairs += (int64_t)c->scal_host[SC_PAIRS];
    if (s != SDOT_OK) return s;
    double J = c->scal_host[SC_VALUE], check = 0.0;
    unsigned k = 0;
    int conv = solver_control_check(c, k, &check);
    sdot_status result = SDOT_OK;
    bool have_H = false;             // a Hessian of an earlier step is in nt_H32 / nt_H64
    double g2_prev = 0.0, alpha_prev = 0.0;
    int64_t n_hess = 0;
    bool tensor = false;
    while (conv == 0) {
        const double g2 = std::sqrt(c->scal_host[SC_L2SQ]);
        // keep the previous Hessian after a full step that contracted |g|_2 by newton_reuse
        const bool reuse = have_H && c->newton_reuse > 0.0 && alpha_prev == 1.0 && g2 <= c->newton_reuse * g2_prev;
        // Hessian at psi (uses L_q, g and the threshold of the evaluation just made)
        if (!reuse) tensor = hessian_method != SDOT_HESS_FP64 && hessian_tensor_ok(c);
        if (hessian_method == SDOT_HESS_TENSOR && !tensor) {
            result = set_error(c, SDOT_EINVAL,
                               "tensor-core Hessian needs an untruncated evaluation (tau <= 0 or a threshold above "
                               "the domain diameter) and rho*JxW >= 0");
            break;
        }
        used_method = tensor ? SDOT_HESS_TENSOR : SDOT_HESS_FP64;
        if ((s = launch_scatter(c, v.gc, c->grad.p, n)) != SDOT_OK) { result = s; break; }
        if (!reuse) {
            cudaEventRecord(t0, c->stream);
            if (tensor) {
                if ((e = c->nt_H32.alloc((size_t)n * n)) != cudaSuccess) { result = cuda_error(c, e, "alloc Hessian"); break; }
                s = hessian_tc(c, c->nt_H32.p, true, c->hess_chunk, nullptr);
            } else {
                if ((e = c->nt_H64.alloc((size_t)n * n)) != cudaSuccess) { result = cuda_error(c, e, "alloc Hessian"); break; }
                s = hessian_fp64_to(c, c->nt_H64.p);
            }
            cudaEventRecord(t1, c->stream);
            if (s != SDOT_OK) { result = s; break; }
            cudaEventSynchronize(t1);
            hess_ms += elapsed(t0, t1);
            have_H = true;
            ++n_hess;
        }
        g2_prev = g2;

        // inexact Newton forcing term: eta = min(0.5, sqrt(|g|_2)), floored at 1e-10
        const double gnorm = std::sqrt(c->scal_host[SC_L2SQ]);
        const double eta = std::max(1e-10, std::min(0.5, std::sqrt(gnorm)));
        int it = 0;
        double rel = 0.0;
        cudaEventRecord(t0, c->stream);
        s = tensor ? pcg<float>(c, c->nt_H32.p, v, n, eta, 4 * (int)std::min<int64_t>(n, 2500), &it, &rel)
                   : pcg<double>(c, c->nt_H64.p, v, n, eta, 4 * (int)std::min<int64_t>(n, 2500), &it, &rel);
        cudaEventRecord(t1, c->stream);
        if (s != SDOT_OK) { result = s; break; }
        cg_total += it;
        // direction: x (caller order) -> pdir (internal); g.p must be negative
        k_dot<<<1, CG_THREADS, 0, c->stream>>>(n, v.gc, v.x, v.sc + S_GP);
        double gp = 0.0;
        e = cudaMemcpyAsync(&gp, v.sc + S_GP, 8, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) { result = cuda_error(c, e, "newton direction"); break; }
        cg_ms += elapsed(t0, t1);
        if (!(gp < 0.0)) {
            // not a descent direction (CG stopped on a numerically singular H): steepest descent
            k_neg<<<(unsigned)std::min<int64_t>((n + 255) / 256, 1184), 256, 0, c->stream>>>(n, v.gc, v.x);
            gp = -c->scal_host[SC_L2SQ];
        }
        if ((s = launch_gather(c, c->pdir.p, v.x, n)) != SDOT_OK) { result = s; break; }
        e = cudaMemcpyAsync(c->x0.p, c->psi.p, n * 8, cudaMemcpyDeviceToDevice, c->stream);
        if (e != cudaSuccess) { result = cuda_error(c, e, "copy x0"); break; }

        // Armijo backtracking on J (FP64)
        double alpha = 1.0;
        bool accepted = false;
        for (int h = 0; h < MAX_HALVINGS; ++h) {
            k_axpy_launch(c->stream, c->psi.p, c->x0.p, alpha, c->pdir.p, n);
            s = evaluate_internal(c, nullptr, tol, &ms);
            ++evals;
            eval_ms += ms;
            pairs += (int64_t)c->scal_host[SC_PAIRS];
            if (s != SDOT_OK && s != SDOT_ENONFINITE) break;
            const double Jn = c->scal_host[SC_VALUE];
            if (s == SDOT_OK && std::isfinite(Jn) && Jn <= J + 1e-4 * alpha * gp) {
                J = Jn;
                accepted = true;
                break;
            }
            s = SDOT_OK;
            alpha *= 0.5;
        }
        if (s != SDOT_OK) { result = s; break; }
        if (!accepted) {
            result = set_error(c, SDOT_ELINESEARCH, "Newton: no sufficient decrease after 40 step halvings");
            break;
        }
        alpha_prev = alpha;
        ++k;
        conv = solver_control_check(c, k, &check);
        if (c->verbose)
            printf("Newton %u: J = %.15e, step %.3g, CG %d its (rel. residual %.2e)\n", k, J, alpha, it, rel);
    }
    c->last_iterations = k;
    c->last_converged = (conv == 1);
    sdot_status s2 = launch_scatter(c, c->io_b.p, c->psi.p, n);
    if (s2 == SDOT_OK) {
        e = cudaMemcpyAsync(psi, c->io_b.p, n * 8, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) s2 = cuda_error(c, e, "copy psi");
    }
    if (info) {
        info->iterations = k;
        info->converged = (conv == 1);
        info->n_evaluations = evals;
        info->cg_iterations = cg_total;
        info->last_value = J;
        info->last_check_value = check;
        info->total_pairs = pairs;
        info->eval_ms = eval_ms;
        info->hessian_ms = hess_ms;
        info->cg_ms = cg_ms;
        info->hessian_method = used_method;
        info->n_hessians = n_hess;
    }
    if (result != SDOT_OK) return result;
    return s2;
}

extern "C" sdot_status sdot_set_newton_hessian_reuse(sdot_ctx *c, double contraction)
{
    if (!c) return SDOT_EINVAL;
    if (!(contraction >= 0.0 && contraction < 1.0))
        return set_error(c, SDOT_EINVAL, "Hessian reuse contraction must be in [0, 1)");
    c->newton_reuse = contraction;
    return SDOT_OK;
}

extern "C" sdot_status sdot_hessian_matvec_device(sdot_ctx *c, const void *H_dev, int f32, const double *x_dev,
                                                  double *y_dev)
{
    if (!c || !H_dev || !x_dev || !y_dev) return SDOT_EINVAL;
    if (c->nt == 0) return set_error(c, SDOT_ESTATE, "targets not set");
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    if (f32) launch_matvec<float>(c, static_cast<const float *>(H_dev), x_dev, y_dev, c->nt);
    else launch_matvec<double>(c, static_cast<const double *>(H_dev), x_dev, y_dev, c->nt);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (prev >= 0 && prev != c->device) cudaSetDevice(prev);
    return cuda_error(c, e, "Hessian matvec");
}

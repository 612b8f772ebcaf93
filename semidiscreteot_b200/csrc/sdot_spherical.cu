// sdot_spherical.cu -- the spherical distance on the evaluation path and the
// spherical weighted-barycenter iteration.
//
// Replaces SotSolver with distance_name == "spherical" (src/solvers/
// SotSolver.cc:22-41): every use of distance_function -- the candidate
// predicate d(y_j, c_K) <= r of find_nearest_target_points (:553-570) and the
// cost d(x_q, y_j)^2 / 2 of local_assemble (:769-869) -- takes the great-circle
// distance of Distance.h, acos(clamp(a.b / (|a| |b|), -1, 1)).  The value and
// gradient kernels follow local_assemble's two passes (largest exponent, then
// the sum of shifted exponentials) in FP64 per point; the gradient is gathered
// per target over the points in a fixed order (no atomics).  The barycenter
// iteration restates evaluate_weighted_barycenters / compute_weighted_
// barycenters_non_euclidean (:612-650, :662-767): per iteration the
// accumulator G_j = sum_q w_q pi_qj grad_b d^2(b_j, x_q) (spherical_distance_
// gradient), its 2-norm against the tolerance, and the exponential-map step
// b_j <- exp_{b_j}(-G_j).
//
// These kernels visit every (point, target) pair, O(Q N) per evaluation: the
// spherical cost is an option of the reference beside the euclidean hot path.
#include <float.h>
#include <math.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "sdot_device.cuh"
#include "sdot_internal.h"

namespace sdot {

constexpr int SPH_THREADS = 128;
constexpr int SPH_TILE = 256;

// spherical_distance (Distance.h): norms as Point::norm, the cosine clamped.
template <int DIM>
__device__ __forceinline__ double sph_dist(const double *a, const double *b)
{
    double dot = 0.0, na = 0.0, nb = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) dot += a[d] * b[d];
#pragma unroll
    for (int d = 0; d < DIM; ++d) na += a[d] * a[d];
#pragma unroll
    for (int d = 0; d < DIM; ++d) nb += b[d] * b[d];
    double c = dot / (sqrt(na) * sqrt(nb));
    c = fmin(1.0, fmax(-1.0, c));
    return acos(c);
}

// Value sweep: thread <-> point q (cell-major, qpc points per cell).  Pass 1
// takes the largest exponent over the cell's candidates, pass 2 sums the
// shifted exponentials (LSE) or the plain ones; the epilogue gives the point's
// part of J, of C_global and L_q = log of its total (+inf when skipped).
template <int DIM>
__global__ void __launch_bounds__(SPH_THREADS)
k_sph_value(int64_t nq, int qpc, const double *__restrict__ x, const double *__restrict__ rho,
            const double *__restrict__ jxw, const double *__restrict__ cell_ctr, int64_t nt,
            const double *__restrict__ y, const double *__restrict__ nu, const double *__restrict__ psi, double r,
            double eps, int lse, double *__restrict__ Lq, double *__restrict__ part)
{
    __shared__ double sy[SPH_TILE][DIM];
    __shared__ double spsi[SPH_TILE], snu[SPH_TILE];
    const int64_t q = blockIdx.x * (int64_t)SPH_THREADS + threadIdx.x;
    const bool have = q < nq;
    double xq[DIM], cq[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        xq[d] = have ? x[q * DIM + d] : 0.0;
        cq[d] = have ? cell_ctr[(q / qpc) * DIM + d] : 0.0;
    }
    const double einv = 1.0 / eps;
    double m = -DBL_MAX, total = 0.0, ncand = 0.0;
    const int npass = lse ? 2 : 1;
    for (int pass = 0; pass < npass; ++pass) {
        for (int64_t t0 = 0; t0 < nt; t0 += SPH_TILE) {
            const int tn = (int)min((int64_t)SPH_TILE, nt - t0);
            __syncthreads();
            for (int i = threadIdx.x; i < tn; i += SPH_THREADS) {
#pragma unroll
                for (int d = 0; d < DIM; ++d) sy[i][d] = y[(t0 + i) * DIM + d];
                spsi[i] = psi[t0 + i];
                snu[i] = nu[t0 + i];
            }
            __syncthreads();
            if (!have) continue;
            for (int i = 0; i < tn; ++i) {
                if (!(sph_dist<DIM>(sy[i], cq) <= r)) continue;
                const double dd = sph_dist<DIM>(xq, sy[i]);
                const double e = (spsi[i] - 0.5 * (dd * dd)) * einv;
                if (lse && pass == 0) {
                    m = fmax(m, e);
                    ncand += 1.0;
                } else {
                    total += snu[i] * exp(lse ? e - m : e);
                    if (!lse) ncand += 1.0;
                }
            }
        }
    }
    double tv = 0.0, tc = 0.0, ts = 0.0;
    if (have) {
        double L = CUDART_INF;
        ts = 1.0;   // no candidate, or a total <= 0 (SotSolver.cc:802, :846)
        if (ncand > 0.0 && total > 0.0) {
            const double lt = lse ? m + log(total) : log(total);
            tv = rho[q] * eps * lt * jxw[q];
            tc = rho[q] * jxw[q] / total;
            L = lt;
            ts = 0.0;
        }
        Lq[q] = L;
    }
    block_partials(tv, tc, ts, have ? ncand : 0.0, part);
}

// Gradient sweep: thread <-> target j, the points streamed in tiles; the
// candidates' w_q nu_j e^(t_qj - L_q) summed in point order.
template <int DIM>
__global__ void __launch_bounds__(SPH_THREADS)
k_sph_grad(int64_t nq, int qpc, const double *__restrict__ x, const double *__restrict__ w,
           const double *__restrict__ Lq, const double *__restrict__ cell_ctr, int64_t nt,
           const double *__restrict__ y, const double *__restrict__ nu, const double *__restrict__ psi, double r,
           double eps, const double *__restrict__ bary, double *__restrict__ out)
{
    __shared__ double sx[SPH_TILE][DIM], sc[SPH_TILE][DIM];
    __shared__ double sw[SPH_TILE], sL[SPH_TILE];
    const int64_t j = blockIdx.x * (int64_t)SPH_THREADS + threadIdx.x;
    const bool have = j < nt;
    double yj[DIM], bj[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        yj[d] = have ? y[j * DIM + d] : 0.0;
        bj[d] = (have && bary) ? bary[j * DIM + d] : 0.0;
    }
    const double pj = have ? psi[j] : 0.0, nj = have ? nu[j] : 0.0;
    const double einv = 1.0 / eps;
    double acc = 0.0, ag[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) ag[d] = 0.0;
    for (int64_t q0 = 0; q0 < nq; q0 += SPH_TILE) {
        const int qn = (int)min((int64_t)SPH_TILE, nq - q0);
        __syncthreads();
        for (int i = threadIdx.x; i < qn; i += SPH_THREADS) {
            const int64_t q = q0 + i;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                sx[i][d] = x[q * DIM + d];
                sc[i][d] = cell_ctr[(q / qpc) * DIM + d];
            }
            sw[i] = w[q];
            sL[i] = Lq[q];
        }
        __syncthreads();
        if (!have) continue;
        for (int i = 0; i < qn; ++i) {
            if (!(sL[i] < CUDART_INF)) continue;            // skipped point
            if (!(sph_dist<DIM>(yj, sc[i]) <= r)) continue;
            const double dd = sph_dist<DIM>(sx[i], yj);
            const double p = sw[i] * nj * exp((pj - 0.5 * (dd * dd)) * einv - sL[i]);
            if (!bary) {
                acc += p;
            } else {
                // spherical_distance_gradient(b_j, x_q): -2 (d / sin d)(x - (b.x) b)
                const double db = sph_dist<DIM>(bj, sx[i]);
                double dot = 0.0;
#pragma unroll
                for (int d = 0; d < DIM; ++d) dot += bj[d] * sx[i][d];
                const double f = db > 0.0 ? db / sin(db) : 1.0;
#pragma unroll
                for (int d = 0; d < DIM; ++d) ag[d] += p * (-2.0 * f * (sx[i][d] - dot * bj[d]));
            }
        }
    }
    if (!have) return;
    if (!bary) {
        out[j] = acc;
    } else {
#pragma unroll
        for (int d = 0; d < DIM; ++d) out[j * DIM + d] = ag[d];
    }
}

template <int DIM>
static void launch_sph_value(sdot_ctx *c, const EvalArgs &a, double r, int64_t nval)
{
    k_sph_value<DIM><<<(unsigned)nval, SPH_THREADS, 0, c->stream>>>(c->nq, c->qpc, c->x.p, c->rho.p, c->jxw.p,
                                                                    c->cell_ctr.p, c->nt, c->y.p, c->nu.p, c->psi.p,
                                                                    r, a.eps, a.lse, c->Lq.p, c->blkpart.p);
}

template <int DIM>
static void launch_sph_grad(sdot_ctx *c, const EvalArgs &a, double r, const double *bary, double *out)
{
    const unsigned g = (unsigned)((c->nt + SPH_THREADS - 1) / SPH_THREADS);
    k_sph_grad<DIM><<<g, SPH_THREADS, 0, c->stream>>>(c->nq, c->qpc, c->x.p, c->w.p, c->Lq.p, c->cell_ctr.p, c->nt,
                                                      c->y.p, c->nu.p, c->psi.p, r, a.eps, bary, out);
}

// Value and gradient sweeps of an evaluation with the spherical distance:
// L_q, the block partials of J / C_global / skipped / pairs (nval blocks),
// and the source part of the gradient in c->gpart (one slice).
sdot_status run_spherical(sdot_ctx *c, const EvalArgs &a, double r, int64_t *nval_out)
{
    const int64_t nval = (c->nq + SPH_THREADS - 1) / SPH_THREADS;
    if (c->blkpart.n < (size_t)(4 * nval)) {
        const cudaError_t e = c->blkpart.alloc((size_t)4 * nval);
        if (e != cudaSuccess) return cuda_error(c, e, "spherical evaluation buffers");
    }
    if (c->dim == 2) {
        launch_sph_value<2>(c, a, r, nval);
        launch_sph_grad<2>(c, a, r, nullptr, c->gpart.p);
    } else {
        launch_sph_value<3>(c, a, r, nval);
        launch_sph_grad<3>(c, a, r, nullptr, c->gpart.p);
    }
    *nval_out = nval;
    return cuda_error(c, cudaGetLastError(), "spherical evaluation");
}

}  // namespace sdot

extern "C" sdot_status sdot_weighted_barycenters_spherical(sdot_ctx *c, const double *psi, double *bary,
                                                           unsigned max_iterations, double tolerance,
                                                           unsigned *iterations, double *grad_norm)
{
    using namespace sdot;
    if (!c || !psi || !bary) return SDOT_EINVAL;
    if (c->distance != 1) return set_error(c, SDOT_EINVAL, "spherical barycenters need the spherical distance");
    if (c->nq == 0 || c->nt == 0) return set_error(c, SDOT_ESTATE, "measures not set");
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    struct Restore {
        int dev;
        ~Restore() {
            if (dev >= 0) cudaSetDevice(dev);
        }
    } restore{prev != c->device ? prev : -1};
    const int64_t n = c->nt;
    const int D = c->dim;
    // the evaluation at psi fixes L_q and the threshold (the reference's
    // compute_distance_threshold and local_assemble inside every iteration
    // give the same values, psi being fixed)
    std::vector<double> g((size_t)n);
    double J = 0.0;
    sdot_status s = sdot_evaluate(c, psi, g.data(), &J, nullptr);
    if (s != SDOT_OK) return s;
    const double r = c->current_distance_threshold;
    std::vector<int64_t> perm((size_t)n);   // internal index -> caller index
    cudaError_t e = cudaMemcpy(perm.data(), c->perm.p, n * sizeof(int64_t), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_error(c, e, "spherical barycenters");
    DevBuf<double> db, dg;
    e = db.alloc((size_t)n * D);
    if (e == cudaSuccess) e = dg.alloc((size_t)n * D);
    if (e != cudaSuccess) return cuda_error(c, e, "spherical barycenters");
    EvalArgs a{};
    a.eps = c->prm.epsilon;
    a.lse = c->prm.use_log_sum_exp;
    std::vector<double> hb((size_t)n * D), hg((size_t)n * D);
    unsigned it = 0;
    double l2 = 0.0;
    for (it = 0; it < max_iterations;) {
        for (int64_t i = 0; i < n; ++i)
            for (int d = 0; d < D; ++d) hb[i * D + d] = bary[perm[i] * D + d];
        e = cudaMemcpyAsync(db.p, hb.data(), hb.size() * 8, cudaMemcpyHostToDevice, c->stream);
        if (e != cudaSuccess) return cuda_error(c, e, "spherical barycenters");
        if (D == 2) launch_sph_grad<2>(c, a, r, db.p, dg.p);
        else launch_sph_grad<3>(c, a, r, db.p, dg.p);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(hg.data(), dg.p, hg.size() * 8, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) return cuda_error(c, e, "spherical barycenters");
        ++it;
        // ||G||_2 in the caller's target order, as the reference's Vector::l2_norm
        double s2 = 0.0;
        std::vector<double> Gc((size_t)n * D);
        for (int64_t i = 0; i < n; ++i)
            for (int d = 0; d < D; ++d) Gc[perm[i] * D + d] = hg[i * D + d];
        for (double v : Gc) s2 += v * v;
        l2 = std::sqrt(s2);
        if (l2 < tolerance) break;
        // exp map at b_j of the step -G_j: cos|v| b + sin|v| v / |v|
        for (int64_t j = 0; j < n; ++j) {
            double nv = 0.0;
            for (int d = 0; d < D; ++d) nv += Gc[j * D + d] * Gc[j * D + d];
            nv = std::sqrt(nv);
            if (!(nv > 0.0)) continue;
            const double cs = std::cos(nv), sn = std::sin(nv);
            for (int d = 0; d < D; ++d) bary[j * D + d] = cs * bary[j * D + d] + sn * (-Gc[j * D + d] / nv);
        }
    }
    if (iterations) *iterations = it;
    if (grad_norm) *grad_norm = l2;
    return SDOT_OK;
}

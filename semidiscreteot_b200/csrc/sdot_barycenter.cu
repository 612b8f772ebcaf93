// sdot_barycenter.cu -- weighted barycenters of the transport cells and the
// potential-conditioned source densities.
//
// Replaces SotSolver::compute_weighted_barycenters_euclidean
// (src/solvers/SotSolver.cc:871-971, through evaluate_weighted_barycenters,
// :584-660) and SotSolver::get_potential_conditioned_density (:973-1046):
//   barycenter_j = sum_q rho_q JxW_q pi_qj x_q / nu_j, with pi_qj =
//     nu_j e^(t_qj - L_q) over the candidates of cell(q) (the evaluation's
//     candidate sets, skipped points excluded), divided by the target density
//     as the reference does;
//   conditioned_k(x) = rho(x) e^(t_k(x) - m(x)) / sum_i nu_i e^(t_i(x) - m(x))
//     over the targets within the threshold of the query point x itself, for
//     each requested target k that is such a candidate (0 otherwise).
// The barycenters run after an FP64 evaluation at psi, which fixes L_q, the
// threshold and (truncated) the block-pair lists; the conditioned densities
// take epsilon and the threshold from the caller, as the reference reads its
// current members.  No atomics: fixed-order sums.
#include <float.h>
#include <math.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "sdot_device.cuh"
#include "sdot_internal.h"

namespace sdot {
namespace {

constexpr int BY_WARPS = 8;

struct BaryArgs {
    const double *x, *w, *Lq, *cell_ctr, *y, *nu, *psi;  // internal orders
    const int64_t *sblk_cell, *tblk_off, *inv_off, *perm;
    const int *inv_b;
    int64_t nsblk;
    int qpc;
    double sstar, eps_inv;
    int trunc;
    double *out;          // n_t x dim, caller order
};

// CTA <-> target block, lane <-> target, warp w <-> paired source blocks
// w, w + 8, ...; per (cell, target) the exact candidate test, per point the
// FP64 weight w_q nu_j e^(t - L_q) times x_q.
template <int DIM>
__global__ void __launch_bounds__(BY_WARPS * 32) k_bary(BaryArgs a)
{
    __shared__ double red[BY_WARPS][32][DIM];
    const int tb = blockIdx.x, lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int64_t j0 = a.tblk_off[tb], j1 = a.tblk_off[tb + 1];
    const int64_t j = j0 + lane;
    const bool has = j < j1;
    double yj[3] = {0.0, 0.0, 0.0}, psij = 0.0, nuj = 0.0;
    if (has) {
        for (int d = 0; d < DIM; ++d) yj[d] = a.y[j * DIM + d];
        psij = a.psi[j];
        nuj = a.nu[j];
    }
    double acc[3] = {0.0, 0.0, 0.0};
    const int64_t nlist = a.trunc ? a.inv_off[tb + 1] - a.inv_off[tb] : a.nsblk;
    for (int64_t e = wp; e < nlist; e += BY_WARPS) {
        const int64_t b = a.trunc ? a.inv_b[a.inv_off[tb] + e] : e;
        for (int64_t c = a.sblk_cell[b]; c < a.sblk_cell[b + 1]; ++c) {
            if (!has) continue;
            if (a.trunc && !(dist2_exact<DIM>(yj, a.cell_ctr + c * DIM) <= a.sstar)) continue;
            for (int i = 0; i < a.qpc; ++i) {
                const int64_t q = c * a.qpc + i;
                const double L = a.Lq[q];
                if (!isfinite(L)) continue;
                const double *xq = a.x + q * DIM;
                const double dd = sqrt(dist2_exact<DIM>(xq, yj));
                const double t = (psij - 0.5 * (dd * dd)) * a.eps_inv;
                const double v = a.w[q] * nuj * exp(t - L);
                if (v > 0.0)
                    for (int d = 0; d < DIM; ++d) acc[d] += v * xq[d];
            }
        }
    }
    for (int d = 0; d < DIM; ++d) red[wp][lane][d] = acc[d];
    __syncthreads();
    if (wp == 0 && has) {
        double s[3] = {0.0, 0.0, 0.0};
        for (int u = 0; u < BY_WARPS; ++u)
            for (int d = 0; d < DIM; ++d) s[d] += red[u][lane][d];
        const int64_t jc = a.perm[j];
        for (int d = 0; d < DIM; ++d) a.out[jc * DIM + d] = s[d] / nuj;
    }
}

struct CondArgs {
    const double *y, *nu;                  // internal order
    const double *psi;                     // caller order
    const int64_t *tblk_off, *perm;
    const double *tblk_sph;                // FP64 target-block spheres (centre, radius)
    int64_t ntblk;
    const double *px, *prho;               // query points, source density there
    int64_t np;
    const double *yreq, *psireq;           // requested targets' points (nidx x dim), potentials
    int64_t nidx;
    double r, sstar, eps_inv;
    double *out;                           // nidx x np
};

// warp <-> query point: online log-sum-exp of nu_i e^(t_i - m) over the
// targets within the threshold of the point (lanes over the targets of the
// target blocks whose sphere reaches it), merged over the lanes in a fixed
// tree; then e^(t_k - m) / sum for the requested targets that are candidates.
template <int DIM>
__global__ void __launch_bounds__(256) k_cond_density(CondArgs a)
{
    const int lane = threadIdx.x & 31;
    const int64_t p = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (p >= a.np) return;
    double xp[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < DIM; ++d) xp[d] = a.px[p * DIM + d];
    double M = -CUDART_INF, S = 0.0;
    for (int64_t tb = 0; tb < a.ntblk; ++tb) {
        const double *sp = a.tblk_sph + tb * 4;
        double s2 = 0.0;
        for (int d = 0; d < DIM; ++d) {
            const double t = xp[d] - sp[d];
            s2 += t * t;
        }
        const double rc = (a.r + sp[3]) * (1.0 + 1e-12) + 1e-300;
        if (!(s2 <= rc * rc)) continue;
        const int64_t j = a.tblk_off[tb] + lane;
        if (j >= a.tblk_off[tb + 1]) continue;
        const double *yj = a.y + j * DIM;
        const double d2 = dist2_exact<DIM>(yj, xp);
        if (!(d2 <= a.sstar)) continue;
        const double dd = sqrt(d2);
        const double e = (a.psi[a.perm[j]] - 0.5 * (dd * dd)) * a.eps_inv;
        if (e > M) {
            S = (M == -CUDART_INF ? 0.0 : S * exp(M - e)) + a.nu[j];
            M = e;
        } else {
            S += a.nu[j] * exp(e - M);
        }
    }
    for (int o = 1; o < 32; o <<= 1) {
        const double Mo = __shfl_xor_sync(0xffffffffu, M, o);
        const double So = __shfl_xor_sync(0xffffffffu, S, o);
        const bool low = (lane & o) == 0;
        const double Ma = low ? M : Mo, Sa = low ? S : So, Mb = low ? Mo : M, Sb = low ? So : S;
        const double Mn = fmax(Ma, Mb);
        S = Mn == -CUDART_INF ? 0.0
                              : (Ma == -CUDART_INF ? 0.0 : Sa * exp(Ma - Mn)) +
                                    (Mb == -CUDART_INF ? 0.0 : Sb * exp(Mb - Mn));
        M = Mn;
    }
    for (int64_t k = lane; k < a.nidx; k += 32) {
        double v = 0.0;
        if (S > 0.0) {
            const double d2 = dist2_exact<DIM>(a.yreq + k * DIM, xp);
            if (d2 <= a.sstar) {
                const double dd = sqrt(d2);
                const double e = (a.psireq[k] - 0.5 * (dd * dd)) * a.eps_inv;
                v = a.prho[p] * (exp(e - M) / S);
            }
        }
        a.out[k * a.np + p] = v;
    }
}

// FP64 evaluation at psi (caller order, host) for L_q, the threshold and the
// block-pair lists.  The reference's barycenter pass recomputes the threshold
// but leaves global_functional and C_global as they were: restore them.
sdot_status eval_fp64_at(sdot_ctx *c, const double *psi_host)
{
    struct Keep {
        sdot_ctx *c;
        double f, C;
        ~Keep() { c->global_functional = f; c->C_global = C; }
    } keep{c, c->global_functional, c->C_global};
    cudaError_t e = cudaMemcpyAsync(c->io_a.p, psi_host, c->nt * 8, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return cuda_error(c, e, "copy psi");
    sdot_status s = launch_gather(c, c->psi.p, c->io_a.p, c->nt);
    if (s != SDOT_OK) return s;
    const int prec = c->precision;
    c->precision = SDOT_PREC_FP64;
    double ms = 0;
    s = evaluate_internal(c, nullptr, c->prm.tolerance, &ms);
    c->precision = prec;
    return s;
}

}  // namespace
}  // namespace sdot

using namespace sdot;

extern "C" sdot_status sdot_weighted_barycenters(sdot_ctx *c, const double *psi, double *barycenters)
{
    if (!c || !psi || !barycenters) return SDOT_EINVAL;
    if (c->nq == 0 || c->nt == 0) return set_error(c, SDOT_ESTATE, "Invalid measures configuration");
    if (c->distance != 0)
        return set_error(c, SDOT_EINVAL,
                         "with the spherical distance use sdot_weighted_barycenters_spherical (an iteration)");
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    struct Restore {
        int p, d;
        ~Restore() { if (p >= 0 && p != d) cudaSetDevice(p); }
    } restore{prev, c->device};
    sdot_status s = ensure_eval_buffers(c);
    if (s == SDOT_OK) s = eval_fp64_at(c, psi);
    if (s != SDOT_OK) return s;
    const double r = c->current_distance_threshold;
    const bool dense = std::isinf(r) || !(r < c->diam * (1.0 + 1e-12));
    DevBuf<double> out;
    cudaError_t e = out.alloc((size_t)c->nt * c->dim);
    if (e != cudaSuccess) return cuda_error(c, e, "barycenter alloc");
    BaryArgs a{};
    a.x = c->x.p; a.w = c->w.p; a.Lq = c->Lq.p; a.cell_ctr = c->cell_ctr.p;
    a.y = c->y.p; a.nu = c->nu.p; a.psi = c->psi.p;
    a.sblk_cell = c->sblk_cell.p; a.tblk_off = c->tblk_off.p;
    a.inv_off = c->inv_off.p; a.inv_b = c->inv_b.p; a.perm = c->perm.p;
    a.nsblk = c->nsblk;
    a.qpc = c->qpc;
    a.sstar = sstar_of(r);
    a.eps_inv = 1.0 / c->prm.epsilon;
    a.trunc = (dense || std::isnan(r)) ? 0 : 1;
    a.out = out.p;
    if (std::isnan(r)) a.sstar = NAN;
    if (c->dim == 2) k_bary<2><<<(unsigned)c->ntblk, BY_WARPS * 32, 0, c->stream>>>(a);
    else k_bary<3><<<(unsigned)c->ntblk, BY_WARPS * 32, 0, c->stream>>>(a);
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(barycenters, out.p, (size_t)c->nt * c->dim * 8, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return cuda_error(c, e, "barycenters");
}

extern "C" sdot_status sdot_conditioned_densities(sdot_ctx *c, const double *psi, double epsilon, double threshold,
                                                 int64_t n_points, const double *points,
                                                 const double *density_at_points, int64_t n_indices,
                                                 const int64_t *indices, double *out)
{
    if (c && c->distance != 0)
        return set_error(c, SDOT_EINVAL, "conditioned densities support the euclidean distance only");
    if (!c || !psi || !points || !density_at_points || !indices || !out || n_points < 0 || n_indices < 0)
        return SDOT_EINVAL;
    if (c->nt == 0 || c->dim == 0) return set_error(c, SDOT_ESTATE, "Invalid measures configuration");
    if (!(epsilon > 0.0)) return set_error(c, SDOT_EINVAL, "epsilon must be positive");
    for (int64_t k = 0; k < n_indices; ++k)
        if (indices[k] < 0 || indices[k] >= c->nt) return set_error(c, SDOT_EINVAL, "target index out of range");
    if (n_points == 0 || n_indices == 0) return SDOT_OK;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    struct Restore {
        int p, d;
        ~Restore() { if (p >= 0 && p != d) cudaSetDevice(p); }
    } restore{prev, c->device};
    const int D = c->dim;
    std::vector<double> yreq((size_t)n_indices * D), preq((size_t)n_indices);
    for (int64_t k = 0; k < n_indices; ++k) {
        for (int d = 0; d < D; ++d) yreq[k * D + d] = c->y_host[indices[k] * D + d];
        preq[k] = psi[indices[k]];
    }
    DevBuf<double> px, pr, o, ps, yr, pq;
    cudaError_t e = px.alloc(n_points * D);
    if (e == cudaSuccess) e = pr.alloc(n_points);
    if (e == cudaSuccess) e = o.alloc((size_t)n_points * n_indices);
    if (e == cudaSuccess) e = ps.alloc(c->nt);
    if (e == cudaSuccess) e = yr.alloc(n_indices * D);
    if (e == cudaSuccess) e = pq.alloc(n_indices);
    if (e != cudaSuccess) return cuda_error(c, e, "conditioned density alloc");
    const cudaMemcpyKind h2d = cudaMemcpyHostToDevice;
    e = cudaMemcpyAsync(px.p, points, n_points * D * 8, h2d, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(pr.p, density_at_points, n_points * 8, h2d, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ps.p, psi, c->nt * 8, h2d, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(yr.p, yreq.data(), n_indices * D * 8, h2d, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(pq.p, preq.data(), n_indices * 8, h2d, c->stream);
    if (e != cudaSuccess) return cuda_error(c, e, "conditioned density upload");
    CondArgs a{};
    a.y = c->y.p; a.nu = c->nu.p; a.psi = ps.p;
    a.tblk_off = c->tblk_off.p; a.perm = c->perm.p; a.tblk_sph = c->tblk_sph.p;
    a.ntblk = c->ntblk;
    a.px = px.p; a.prho = pr.p; a.np = n_points;
    a.yreq = yr.p; a.psireq = pq.p; a.nidx = n_indices;
    a.r = std::isnan(threshold) ? 0.0 : std::min(threshold, 1e300);
    a.sstar = sstar_of(threshold);
    a.eps_inv = 1.0 / epsilon;
    a.out = o.p;
    const unsigned g = (unsigned)((n_points * 32 + 255) / 256);
    if (D == 2) k_cond_density<2><<<g, 256, 0, c->stream>>>(a);
    else k_cond_density<3><<<g, 256, 0, c->stream>>>(a);
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, o.p, (size_t)n_points * n_indices * 8, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return cuda_error(c, e, "conditioned densities");
}

// sdot_hessian.cu -- dense Hessian of the entropic dual functional.
//
// SotSolver declares compute_hessian(potential, LAPACKFullMatrix&) but never
// defines it (include/SemiDiscreteOT/solvers/SotSolver.h:343-344).  This file
// provides it:
//     H = (1/eps) [ diag(sum_q w_q pi_q) - sum_q w_q pi_q pi_q^T ],
//     pi_qj = nu_j exp(t_qj - L_q)   (0 outside the candidate set of cell(q)),
// which is d(grad)/d(psi) of the evaluation in sdot_eval.cu.  The diagonal
// term equals (g_j + nu_j)/eps and is taken from the evaluation; the
// contraction P_w^T P (P_w = diag(w) P) is accumulated here in FP64 on
// 64x64 output tiles (upper triangle, mirrored), P regenerated on the fly
// from the L_q of the value sweep and never stored.
#include <float.h>
#include <math.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "sdot_device.cuh"
#include "sdot_internal.h"

namespace sdot {

constexpr int HT = 64;        // output tile edge
constexpr int HQ = 16;        // quadrature points per smem chunk

template <int DIM, bool TRUNC>
__global__ void __launch_bounds__(256)
k_hessian_simt(const double *__restrict__ x, const double *__restrict__ w, const double *__restrict__ Lq,
               const double *__restrict__ cell_ctr, const double *__restrict__ tpack, const double *__restrict__ grad,
               const double *__restrict__ nu, EvalArgs a, double *__restrict__ H)
{
    const int tb = blockIdx.x, ta = blockIdx.y;
    if (tb < ta) return;  // upper triangle of tiles
    __shared__ double tab[16];
    __shared__ double PA[HQ][HT + 1];   // w_q pi_qa
    __shared__ double PB[HQ][HT + 1];   // pi_qb
    __shared__ double tgt[2][HT][8];
    const int tid = threadIdx.x;
    if (tid < 16) tab[tid] = c_exp2_tab[tid];
    for (int i = tid; i < 2 * HT * 8; i += 256) {
        const int side = i / (HT * 8), r = (i / 8) % HT, f = i % 8;
        const int64_t j = (int64_t)(side == 0 ? ta : tb) * HT + r;
        tgt[side][r][f] = j < a.nt ? tpack[j * TPACK + f] : 0.0;
    }
    const int tr = tid / 16, tc = tid % 16;  // thread owns rows tr*4.., cols tc*4..
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[i][k] = 0.0;
    __syncthreads();
    for (int64_t q0 = 0; q0 < a.nq; q0 += HQ) {
        // fill PA/PB: HQ x 2*HT entries, 256 threads -> 8 each
        for (int i = tid; i < HQ * 2 * HT; i += 256) {
            const int qi = i / (2 * HT), col = i % (2 * HT);
            const int side = col / HT, r = col % HT;
            const int64_t q = q0 + qi;
            const int64_t j = (int64_t)(side == 0 ? ta : tb) * HT + r;
            double val = 0.0;
            if (q < a.nq && j < a.nt) {
                const double Lv = Lq[q];
                bool in = isfinite(Lv);
                const double *tp = tgt[side][r];
                if (TRUNC && in) {
                    const int64_t cell = q / a.qpc;
                    in = dist2_exact<DIM>(tp + 2 + DIM, cell_ctr + cell * DIM) <= a.sstar;
                }
                if (in) {
                    double xt[3], xsq = 0.0;
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        xt[d] = x[q * DIM + d] - a.o[d];
                        xsq += xt[d] * xt[d];
                    }
                    double u = fma(tp[1], xt[0], tp[0] + (-a.halfs * xsq - KAPPA * Lv));
#pragma unroll
                    for (int d = 1; d < DIM; ++d) u = fma(tp[1 + d], xt[d], u);
                    val = tp[1 + DIM] * exp2_16(u, tab);
                    if (side == 0) val *= w[q];
                }
            }
            if (side == 0) PA[qi][r] = val;
            else PB[qi][r] = val;
        }
        __syncthreads();
#pragma unroll 4
        for (int qi = 0; qi < HQ; ++qi) {
            double av[4], bv[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) av[i] = PA[qi][tr * 4 + i];
#pragma unroll
            for (int k = 0; k < 4; ++k) bv[k] = PB[qi][tc * 4 + k];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int k = 0; k < 4; ++k) acc[i][k] = fma(av[i], bv[k], acc[i][k]);
        }
        __syncthreads();
    }
    const double einv = 1.0 / a.eps;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int64_t ja = (int64_t)ta * HT + tr * 4 + i;
        if (ja >= a.nt) continue;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int64_t jb = (int64_t)tb * HT + tc * 4 + k;
            if (jb >= a.nt) continue;
            double h = -acc[i][k];
            if (ja == jb) h += grad[ja] + nu[ja];
            h *= einv;
            H[ja * a.nt + jb] = h;
            if (tb != ta) H[jb * a.nt + ja] = h;
        }
    }
}

// Hu[perm[a], perm[b]] = Hi[a, b]
__global__ void k_permute_matrix(const double *__restrict__ Hi, double *__restrict__ Hu, const int64_t *__restrict__ perm,
                                 int64_t n)
{
    for (int64_t a = blockIdx.y; a < n; a += gridDim.y) {
        const int64_t pa = perm[a];
        for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < n; b += (int64_t)gridDim.x * blockDim.x)
            Hu[pa * n + perm[b]] = Hi[a * n + b];
    }
}

// FP64 Hessian at the potential of the last evaluation into H_dev (device,
// n x n row-major, caller order).
sdot_status hessian_fp64_to(sdot_ctx *c, double *H_dev)
{
    const int64_t n = c->nt;
    if (n > 46340) return set_error(c, SDOT_EBUDGET, "dense Hessian limited to n_targets <= 46340");
    const double r = c->current_distance_threshold;
    EvalArgs a{};
    a.qpc = c->qpc;
    a.nq = c->nq;
    a.ncells = c->ncells;
    a.nt = n;
    a.eps = c->prm.epsilon;
    a.s = KAPPA / c->prm.epsilon;
    a.halfs = 0.5 * a.s;
    for (int d = 0; d < 3; ++d) a.o[d] = c->origin[d];
    a.sstar = sstar_of(r);
    const bool trunc = std::isnan(r) || r < c->diam;
    launch_target_prep_dense(c, a);  // the truncated evaluation leaves another layout in tpack
    DevBuf<double> Hi;
    cudaError_t e = Hi.alloc((size_t)n * n);
    if (e != cudaSuccess) return cuda_error(c, e, "hessian alloc");
    const unsigned nb = (unsigned)((n + HT - 1) / HT);
    dim3 g(nb, nb);
    if (c->dim == 2) {
        if (trunc) k_hessian_simt<2, true><<<g, 256, 0, c->stream>>>(c->x.p, c->w.p, c->Lq.p, c->cell_ctr.p, c->tpack.p, c->grad.p, c->nu.p, a, Hi.p);
        else k_hessian_simt<2, false><<<g, 256, 0, c->stream>>>(c->x.p, c->w.p, c->Lq.p, c->cell_ctr.p, c->tpack.p, c->grad.p, c->nu.p, a, Hi.p);
    } else {
        if (trunc) k_hessian_simt<3, true><<<g, 256, 0, c->stream>>>(c->x.p, c->w.p, c->Lq.p, c->cell_ctr.p, c->tpack.p, c->grad.p, c->nu.p, a, Hi.p);
        else k_hessian_simt<3, false><<<g, 256, 0, c->stream>>>(c->x.p, c->w.p, c->Lq.p, c->cell_ctr.p, c->tpack.p, c->grad.p, c->nu.p, a, Hi.p);
    }
    k_permute_matrix<<<dim3(std::max<unsigned>(1, (unsigned)std::min<int64_t>((n + 255) / 256, 64)),
                            (unsigned)std::min<int64_t>(n, 65535)), 256, 0,
                       c->stream>>>(Hi.p, H_dev, c->perm.p, n);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);  // Hi is released on return
    return cuda_error(c, e, "hessian");
}

sdot_status hessian_internal(sdot_ctx *c, double *H_host)
{
    // an evaluation at c->psi provides L_q, the gradient and the threshold
    double ms = 0;
    sdot_status s = evaluate_internal(c, nullptr, c->prm.tolerance, &ms);
    if (s != SDOT_OK) return s;
    const int64_t n = c->nt;
    if (n > 46340) return set_error(c, SDOT_EBUDGET, "dense Hessian limited to n_targets <= 46340");
    DevBuf<double> Hu;
    cudaError_t e = Hu.alloc((size_t)n * n);
    if (e != cudaSuccess) return cuda_error(c, e, "hessian alloc");
    if ((s = hessian_fp64_to(c, Hu.p)) != SDOT_OK) return s;
    e = cudaMemcpyAsync(H_host, Hu.p, (size_t)n * n * 8, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return cuda_error(c, e, "hessian");
}

// The tensor-core path needs every (q, j) pair in the sum (no truncation) and
// w_q >= 0 (its log2 w_q is folded into the exponent).
static bool tensor_ok(const sdot_ctx *c)
{
    const double r = c->current_distance_threshold;
    const bool dense = std::isinf(r) || !(r < c->diam * (1.0 + 1e-12));
    return dense && !std::isnan(r) && c->w_nonneg;
}

bool hessian_tensor_ok(const sdot_ctx *c) { return tensor_ok(c); }

sdot_status hessian_device(sdot_ctx *c, const double *psi_dev, void *H_dev, int method, int out_f32,
                           sdot_hessian_info *info)
{
    if (method != SDOT_HESS_AUTO && method != SDOT_HESS_FP64 && method != SDOT_HESS_TENSOR)
        return set_error(c, SDOT_EINVAL, "unknown Hessian method");
    if (c->distance != 0) return set_error(c, SDOT_EINVAL, "the Hessian supports the euclidean distance only");
    sdot_status s = launch_gather(c, c->psi.p, psi_dev, c->nt);
    if (s != SDOT_OK) return s;
    double ems = 0, hms = 0;
    s = evaluate_internal(c, nullptr, c->prm.tolerance, &ems);
    if (s != SDOT_OK) return s;
    int used = method;
    if (method == SDOT_HESS_AUTO) used = tensor_ok(c) ? SDOT_HESS_TENSOR : SDOT_HESS_FP64;
    if (used == SDOT_HESS_TENSOR) {
        if (!tensor_ok(c))
            return set_error(c, SDOT_EINVAL,
                             "tensor-core Hessian needs an untruncated evaluation (tau <= 0 or a threshold above the "
                             "domain diameter) and rho*JxW >= 0");
        s = hessian_tc(c, H_dev, out_f32 != 0, c->hess_chunk, &hms);
    } else {
        if (out_f32) return set_error(c, SDOT_EINVAL, "the FP64 Hessian writes doubles (out_f32 must be 0)");
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, c->stream);
        s = hessian_fp64_to(c, static_cast<double *>(H_dev));
        cudaEventRecord(e1, c->stream);
        cudaEventSynchronize(e1);
        float f = 0.f;
        cudaEventElapsedTime(&f, e0, e1);
        hms = f;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    if (info) {
        info->method = used;
        info->eval_ms = ems;
        info->hessian_ms = hms;
        info->tiles = used == SDOT_HESS_TENSOR ? c->hess_tiles : 0;
        info->kernel_ms = used == SDOT_HESS_TENSOR ? c->hess_kernel_ms : hms;
    }
    return s;
}

}  // namespace sdot

extern "C" sdot_status sdot_hessian_device(sdot_ctx *c, const double *psi_dev, void *H_dev, int method, int out_f32,
                                           sdot_hessian_info *info)
{
    if (!c || !psi_dev || !H_dev) return SDOT_EINVAL;
    if (c->nq == 0 || c->nt == 0) return sdot::set_error(c, SDOT_ESTATE, "measures not set");
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    sdot_status s = sdot::ensure_eval_buffers(c);
    if (s == SDOT_OK) s = sdot::hessian_device(c, psi_dev, H_dev, method, out_f32, info);
    if (prev >= 0 && prev != c->device) cudaSetDevice(prev);
    return s;
}

extern "C" sdot_status sdot_hessian_tile_count(sdot_ctx *c, int64_t *count)
{
    if (!c || !count) return SDOT_EINVAL;
    if (c->nt == 0) return sdot::set_error(c, SDOT_ESTATE, "targets not set");
    *count = sdot::hessian_tc_tiles(c->nt);
    return SDOT_OK;
}

extern "C" sdot_status sdot_hessian_tiles_device(sdot_ctx *c, const double *psi_dev, void *H_dev, int out_f32,
                                                 int64_t tile_begin, int64_t tile_end, sdot_hessian_info *info)
{
    if (!c || !psi_dev || !H_dev) return SDOT_EINVAL;
    if (c->nq == 0 || c->nt == 0) return sdot::set_error(c, SDOT_ESTATE, "measures not set");
    if (c->distance != 0) return sdot::set_error(c, SDOT_EINVAL, "the Hessian supports the euclidean distance only");
    const int64_t nt = sdot::hessian_tc_tiles(c->nt);
    if (tile_begin < 0 || tile_end < tile_begin || tile_end > nt)
        return sdot::set_error(c, SDOT_EINVAL, "tile range outside [0, sdot_hessian_tile_count]");
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    sdot_status s = sdot::ensure_eval_buffers(c);
    double ems = 0, hms = 0;
    if (s == SDOT_OK) s = sdot::launch_gather(c, c->psi.p, psi_dev, c->nt);
    if (s == SDOT_OK) s = sdot::evaluate_internal(c, nullptr, c->prm.tolerance, &ems);
    if (s == SDOT_OK && !sdot::tensor_ok(c))
        s = sdot::set_error(c, SDOT_EINVAL,
                            "tensor-core Hessian needs an untruncated evaluation (tau <= 0 or a threshold above the "
                            "domain diameter) and rho*JxW >= 0");
    if (s == SDOT_OK) s = sdot::hessian_tc(c, H_dev, out_f32 != 0, c->hess_chunk, &hms, tile_begin, tile_end);
    if (s == SDOT_OK && info) {
        info->method = SDOT_HESS_TENSOR;
        info->eval_ms = ems;
        info->hessian_ms = hms;
        info->tiles = c->hess_tiles;
        info->kernel_ms = c->hess_kernel_ms;
    }
    if (prev >= 0 && prev != c->device) cudaSetDevice(prev);
    return s;
}

extern "C" sdot_status sdot_set_hessian_chunk(sdot_ctx *c, int stages)
{
    if (!c || stages < 1) return SDOT_EINVAL;
    c->hess_chunk = stages;
    return SDOT_OK;
}

extern "C" sdot_status sdot_set_hessian_generation(sdot_ctx *c, int factored, int *last_factored)
{
    if (!c) return SDOT_EINVAL;
    if (factored >= 0) c->hess_factored = factored != 0;
    if (last_factored) *last_factored = c->hess_last_factored ? 1 : 0;
    return SDOT_OK;
}

extern "C" sdot_status sdot_set_hessian_pairs(sdot_ctx *c, int pairs, int *last_pairs)
{
    if (!c) return SDOT_EINVAL;
    if (pairs > 2) return sdot::set_error(c, SDOT_EINVAL, "sdot_set_hessian_pairs: mode 0, 1 or 2");
    if (pairs >= 0) c->hess_pair_mode = pairs;
    if (last_pairs) *last_pairs = c->hess_last_pair;
    return SDOT_OK;
}

extern "C" sdot_status sdot_set_hessian_wait_limit(sdot_ctx *c, int64_t clocks)
{
    if (!c) return SDOT_EINVAL;
    c->hess_wait_limit = clocks > 0 ? (long long)clocks : 0;
    return SDOT_OK;
}

extern "C" sdot_status sdot_hessian(sdot_ctx *c, const double *psi, double *H)
{
    if (!c || !psi || !H) return SDOT_EINVAL;
    if (c->nq == 0 || c->nt == 0) return sdot::set_error(c, SDOT_ESTATE, "measures not set");
    if (c->distance != 0) return sdot::set_error(c, SDOT_EINVAL, "the Hessian supports the euclidean distance only");
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    double dummy = 0;
    // reuse the public evaluation to stage psi and the per-evaluation buffers
    std::vector<double> g((size_t)c->nt);
    sdot_status s = sdot_evaluate(c, psi, g.data(), &dummy, nullptr);
    if (s == SDOT_OK) s = sdot::hessian_internal(c, H);
    if (prev >= 0 && prev != c->device) cudaSetDevice(prev);
    return s;
}

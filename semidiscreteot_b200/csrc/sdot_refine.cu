// sdot_refine.cu -- softmax transfer of potentials from a coarse target level
// to its children (the multilevel warm start).
//
// Replaces SoftmaxRefinement::compute_refinement
// (src/solvers/SoftmaxRefinement.cc:61-280, called from
// SemiDiscreteOT::assign_potentials_by_hierarchy, SemiDiscreteOT.cc:748-828):
//   for every cell K, its coarse candidates {i : |y_i - c_K| <= r} and, per
//   quadrature point x_q, the log-sum-exp over the candidates within r of x_q
//     m_q = max (psi_i - d2_qi / 2) / lambda,  S_q = sum nu_i e^((psi_i - d2_qi / 2) / lambda - m_q),
//   scale_q = rho_q JxW_q e^(-m_q) / S_q (S_q and no shift when the
//   log-sum-exp trick is off; points with S_q <= 0 contribute nothing); every
//   fine child k of a candidate of K, within r of x_q, receives
//   scale_q e^(-d2_qk / (2 lambda)), and psi_fine_k = -lambda log(sum) when the
//   sum is positive (0 otherwise).  Distances are rounded like the reference
//   (pow(|x - y|, 2)); the candidate test at the cell centre is the exact one
//   of the evaluation (sqrt_rn(d2) <= r).
//
// Two kernels, both deterministic (no atomics):
//   k_refine_scale : CTA <-> source block; coarse targets culled against the
//                    block sphere and staged in smem chunk by chunk; warp <->
//                    cell, lane <-> (quadrature point, candidate group), online
//                    log-sum-exp per lane, groups merged in a fixed xor tree;
//                    scale_q to global;
//   k_refine_fine  : CTA <-> coarse target; threads scan the source blocks
//                    (sphere cull) and then (block, cell) items with the exact
//                    centre test, each summing its items for every child; the
//                    CTA adds the thread sums in thread order.
#include <float.h>
#include <math.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "sdot_device.cuh"
#include "sdot_internal.h"

namespace sdot {
namespace {

constexpr int RF_WARPS = 8;
constexpr int RF_CHUNK = 1024;     // coarse targets staged per chunk
constexpr int RF_THREADS = 256;
constexpr int RF_MAXQ = 32;        // quadrature points per cell supported
constexpr int RF_MAXCHILD = 32;    // children of one coarse target per pass of k_refine_fine

struct RefineArgs {
    const double *x, *rho, *jxw, *cell_ctr;  // source, internal order
    const int64_t *sblk_cell;                 // source block -> first cell
    const double *sblk_sph;                   // FP64 block spheres (centre, radius of the cell centres)
    int64_t nsblk;
    int qpc;
    int64_t nc;                               // coarse targets
    const double *yc, *nuc, *psic;            // coarse targets (caller order)
    double r, r2, sstar, lam_inv;
    int lse;
    double *scale;                            // per q (internal order)
    // fine pass
    const double *yf;                         // fine targets (caller order)
    const int64_t *coff, *cidx;               // children CSR of the coarse targets
    double *acc;                              // per fine target: sum (caller order)
};

// pow(|a - b|, 2) as the reference rounds it
template <int DIM>
__device__ __forceinline__ double pow_dist2(const double *a, const double *b)
{
    const double d = sqrt(dist2_exact<DIM>(a, b));
    return d * d;
}

template <int DIM>
__global__ void __launch_bounds__(RF_WARPS * 32) k_refine_scale(RefineArgs a)
{
    __shared__ double sy[RF_CHUNK][DIM];
    __shared__ double sv[RF_CHUNK][2];       // nu, psi
    __shared__ int wcnt[RF_WARPS], wbase[RF_WARPS], nst;
    const int b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    const int64_t c0 = a.sblk_cell[b], c1 = a.sblk_cell[b + 1];
    const int ncell = (int)(c1 - c0);
    const double *bs = a.sblk_sph + (int64_t)b * 4;
    const double rc = (a.r + bs[3]) * (1.0 + 1e-12) + 1e-300;
    int QP = 1;
    while (QP < a.qpc) QP <<= 1;                 // lanes per group
    const int G = 32 / QP;                       // candidate groups per warp
    const int q = lane % QP, grp = lane / QP;
    const bool valid = wp < ncell;
    const bool qok = valid && q < a.qpc;
    const int64_t cell = c0 + wp;
    double cc[3] = {0.0, 0.0, 0.0}, xq[3] = {0.0, 0.0, 0.0};
    if (valid)
        for (int d = 0; d < DIM; ++d) cc[d] = a.cell_ctr[cell * DIM + d];
    if (qok)
        for (int d = 0; d < DIM; ++d) xq[d] = a.x[(cell * a.qpc + q) * DIM + d];
    double M = -CUDART_INF, S = 0.0;            // online state of (q, group); LSE: S relative to M
    for (int64_t j0 = 0; j0 < a.nc; j0 += RF_CHUNK) {
        __syncthreads();
        if (tid == 0) nst = 0;
        __syncthreads();
        const int64_t j1 = min(a.nc, j0 + RF_CHUNK);
        for (int64_t jb = j0; jb < j1; jb += RF_WARPS * 32) {
            const int64_t j = jb + tid;
            bool keep = false;
            if (j < j1) {
                double s = 0.0;
                for (int d = 0; d < DIM; ++d) {
                    const double t = a.yc[j * DIM + d] - bs[d];
                    s += t * t;
                }
                keep = s <= rc * rc;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            if (lane == 0) wcnt[wp] = __popc(bal);
            __syncthreads();
            if (tid == 0) {
                int acc = nst;
                for (int w = 0; w < RF_WARPS; ++w) {
                    wbase[w] = acc;
                    acc += wcnt[w];
                }
                nst = acc;
            }
            __syncthreads();
            if (keep) {
                const int pos = wbase[wp] + __popc(bal & ((1u << lane) - 1u));
                for (int d = 0; d < DIM; ++d) sy[pos][d] = a.yc[j * DIM + d];
                sv[pos][0] = a.nuc[j];
                sv[pos][1] = a.psic[j];
            }
            __syncthreads();
        }
        const int n = nst;
        if (!qok) continue;
        for (int t = grp; t < n; t += G) {
            const double y[3] = {sy[t][0], sy[t][1], DIM == 3 ? sy[t][2] : 0.0};
            if (!(dist2_exact<DIM>(y, cc) <= a.sstar)) continue;     // candidate of the cell
            const double d2 = pow_dist2<DIM>(xq, y);
            if (!(d2 <= a.r2)) continue;
            const double e = (sv[t][1] - 0.5 * d2) * a.lam_inv;
            if (a.lse) {
                if (e > M) {
                    S = (M == -CUDART_INF ? 0.0 : S * exp(M - e)) + sv[t][0];
                    M = e;
                } else {
                    S += sv[t][0] * exp(e - M);
                }
            } else {
                S += sv[t][0] * exp(e);
            }
        }
    }
    if (!valid) return;
    // merge the candidate groups of each q (fixed xor tree over the group bits)
    for (int o = QP; o < 32; o <<= 1) {
        const double Mo = __shfl_xor_sync(0xffffffffu, M, o);
        const double So = __shfl_xor_sync(0xffffffffu, S, o);
        if (a.lse) {
            const double Mn = fmax(M, Mo);
            if (Mn == -CUDART_INF) {
                S = 0.0;
            } else {
                // combine in a fixed operand order (lower group first) so every lane agrees
                const bool low = (lane & o) == 0;
                const double Ma = low ? M : Mo, Sa = low ? S : So, Mb = low ? Mo : M, Sb = low ? So : S;
                S = (Ma == -CUDART_INF ? 0.0 : Sa * exp(Ma - Mn)) + (Mb == -CUDART_INF ? 0.0 : Sb * exp(Mb - Mn));
            }
            M = Mn;
        } else {
            const bool low = (lane & o) == 0;
            S = low ? S + So : So + S;
        }
    }
    if (qok && grp == 0) {
        const int64_t qi = cell * a.qpc + q;
        double sc = 0.0;
        if (S > 0.0) {
            sc = a.rho[qi] * a.jxw[qi] / S;
            if (a.lse) sc *= exp(-M);
        }
        a.scale[qi] = sc;
    }
}

// CTA <-> coarse target p: every cell K with p as candidate, every point q of
// K and every child k of p within r of x_q adds scale_q e^(-d2 / (2 lambda)).
template <int DIM>
__global__ void __launch_bounds__(RF_THREADS) k_refine_fine(RefineArgs a)
{
    __shared__ int sblk[4096];
    __shared__ int nb;
    __shared__ double red[RF_THREADS];
    const int64_t p = blockIdx.x;
    const int tid = threadIdx.x;
    const int64_t k0 = a.coff[p], k1 = a.coff[p + 1];
    if (k1 <= k0) return;
    double yp[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < DIM; ++d) yp[d] = a.yc[p * DIM + d];
    for (int64_t kb = k0; kb < k1; kb += RF_MAXCHILD) {
        const int nk = (int)min((int64_t)RF_MAXCHILD, k1 - kb);
        double accv[RF_MAXCHILD];
#pragma unroll
        for (int i = 0; i < RF_MAXCHILD; ++i) accv[i] = 0.0;
        // source blocks in chunks of 4096: cull, compact (order by thread, then pass)
        for (int64_t b0 = 0; b0 < a.nsblk; b0 += 4096) {
            __syncthreads();
            if (tid == 0) nb = 0;
            __syncthreads();
            const int64_t b1 = min(a.nsblk, b0 + 4096);
            // ordered compaction: each pass of RF_THREADS blocks
            for (int64_t bb = b0; bb < b1; bb += RF_THREADS) {
                const int64_t bi = bb + tid;
                bool keep = false;
                if (bi < b1) {
                    const double *bs = a.sblk_sph + bi * 4;
                    double s = 0.0;
                    for (int d = 0; d < DIM; ++d) {
                        const double t = yp[d] - bs[d];
                        s += t * t;
                    }
                    const double rc = (a.r + bs[3]) * (1.0 + 1e-12) + 1e-300;
                    keep = s <= rc * rc;
                }
                // prefix over the CTA in thread order
                red[tid] = keep ? 1.0 : 0.0;
                __syncthreads();
                if (tid == 0) {
                    int acc = nb;
                    for (int i = 0; i < RF_THREADS; ++i) {
                        const int v = red[i] != 0.0;
                        red[i] = acc;
                        acc += v;
                    }
                    nb = acc;
                }
                __syncthreads();
                if (keep) sblk[(int)red[tid]] = (int)bi;
                __syncthreads();
            }
            const int n = nb;
            // items (block, cell): thread-strided
            for (int it = tid; it < n * 8; it += RF_THREADS) {
                const int bi = sblk[it >> 3];
                const int64_t cell = a.sblk_cell[bi] + (it & 7);
                if (cell >= a.sblk_cell[bi + 1]) continue;
                double cc[3] = {0.0, 0.0, 0.0};
                for (int d = 0; d < DIM; ++d) cc[d] = a.cell_ctr[cell * DIM + d];
                if (!(dist2_exact<DIM>(yp, cc) <= a.sstar)) continue;
                for (int qq = 0; qq < a.qpc; ++qq) {
                    const int64_t qi = cell * a.qpc + qq;
                    const double sc = a.scale[qi];
                    if (sc == 0.0) continue;
                    const double *xq = a.x + qi * DIM;
#pragma unroll
                    for (int i = 0; i < RF_MAXCHILD; ++i) {
                        if (i < nk) {
                            const int64_t f = a.cidx[kb + i];
                            const double d2 = pow_dist2<DIM>(xq, a.yf + f * DIM);
                            if (d2 <= a.r2) accv[i] += sc * exp((-0.5 * d2) * a.lam_inv);
                        }
                    }
                }
            }
        }
        // CTA sum of each child's thread partials, in thread order
#pragma unroll
        for (int i = 0; i < RF_MAXCHILD; ++i) {
            if (i >= nk) break;
            __syncthreads();
            red[tid] = accv[i];
            __syncthreads();
            if (tid == 0) {
                double s = 0.0;
                for (int t = 0; t < RF_THREADS; ++t) s += red[t];
                a.acc[a.cidx[kb + i]] = s;
            }
        }
    }
}

}  // namespace
}  // namespace sdot

using namespace sdot;

extern "C" sdot_status sdot_softmax_refinement(sdot_ctx *c, const double *psi_coarse, double epsilon, double threshold,
                                              int use_log_sum_exp, int64_t n_fine, const double *y_fine,
                                              const int64_t *child_offsets, const int64_t *child_indices,
                                              double *psi_fine)
{
    if (c && c->distance != 0)
        return sdot::set_error(c, SDOT_EINVAL, "the softmax refinement supports the euclidean distance only");
    if (!c || !psi_coarse || !y_fine || !child_offsets || !child_indices || !psi_fine || n_fine <= 0)
        return SDOT_EINVAL;
    if (c->nq == 0 || c->nt == 0) return set_error(c, SDOT_ESTATE, "measures not set (the targets are the coarse level)");
    if (!(epsilon > 0.0) || !(threshold >= 0.0)) return set_error(c, SDOT_EINVAL, "epsilon > 0 and threshold >= 0 required");
    if (c->qpc > RF_MAXQ) return set_error(c, SDOT_EINVAL, "softmax refinement supports up to 32 quadrature points per cell");
    const int64_t nc = c->nt;
    if (child_offsets[0] != 0) return set_error(c, SDOT_EINVAL, "child_offsets must start at 0");
    std::vector<char> seen((size_t)n_fine, 0);
    for (int64_t i = 0; i < nc; ++i) {
        if (child_offsets[i + 1] < child_offsets[i]) return set_error(c, SDOT_EINVAL, "child_offsets must be non-decreasing");
        for (int64_t k = child_offsets[i]; k < child_offsets[i + 1]; ++k) {
            const int64_t f = child_indices[k];
            if (f < 0 || f >= n_fine) return set_error(c, SDOT_EINVAL, "child index out of range");
            if (seen[f]) return set_error(c, SDOT_EINVAL, "a fine target listed as the child of two coarse targets");
            seen[f] = 1;
        }
    }
    const int64_t nchild = child_offsets[nc];
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    struct Restore {
        int p, d;
        ~Restore() { if (p >= 0 && p != d) cudaSetDevice(p); }
    } restore{prev, c->device};
    const int D = c->dim;
    DevBuf<double> yc, nuc, psic, yf, scale, acc;
    DevBuf<int64_t> coff, cidx;
    cudaError_t e = yc.alloc(nc * D);
    if (e == cudaSuccess) e = nuc.alloc(nc);
    if (e == cudaSuccess) e = psic.alloc(nc);
    if (e == cudaSuccess) e = yf.alloc(n_fine * D);
    if (e == cudaSuccess) e = scale.alloc(c->nq);
    if (e == cudaSuccess) e = acc.alloc(n_fine);
    if (e == cudaSuccess) e = coff.alloc(nc + 1);
    if (e == cudaSuccess) e = cidx.alloc(std::max<int64_t>(1, nchild));
    if (e != cudaSuccess) return cuda_error(c, e, "refinement alloc");
    cudaStream_t st = c->stream;
    e = cudaMemcpyAsync(yc.p, c->y_host.data(), nc * D * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(nuc.p, c->nu_host.data(), nc * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(psic.p, psi_coarse, nc * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(yf.p, y_fine, n_fine * D * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(coff.p, child_offsets, (nc + 1) * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nchild > 0)
        e = cudaMemcpyAsync(cidx.p, child_indices, nchild * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(acc.p, 0, n_fine * 8, st);
    if (e != cudaSuccess) return cuda_error(c, e, "refinement upload");
    RefineArgs a{};
    a.x = c->x.p;
    a.rho = c->rho.p;
    a.jxw = c->jxw.p;
    a.cell_ctr = c->cell_ctr.p;
    a.sblk_cell = c->sblk_cell.p;
    a.sblk_sph = c->sblk_sph.p;
    a.nsblk = c->nsblk;
    a.qpc = c->qpc;
    a.nc = nc;
    a.yc = yc.p;
    a.nuc = nuc.p;
    a.psic = psic.p;
    a.r = threshold;
    a.r2 = threshold * threshold;
    a.sstar = sstar_of(threshold);
    a.lam_inv = 1.0 / epsilon;
    a.lse = use_log_sum_exp ? 1 : 0;
    a.scale = scale.p;
    a.yf = yf.p;
    a.coff = coff.p;
    a.cidx = cidx.p;
    a.acc = acc.p;
    if (D == 2) {
        k_refine_scale<2><<<(unsigned)c->nsblk, RF_WARPS * 32, 0, st>>>(a);
        k_refine_fine<2><<<(unsigned)nc, RF_THREADS, 0, st>>>(a);
    } else {
        k_refine_scale<3><<<(unsigned)c->nsblk, RF_WARPS * 32, 0, st>>>(a);
        k_refine_fine<3><<<(unsigned)nc, RF_THREADS, 0, st>>>(a);
    }
    e = cudaGetLastError();
    std::vector<double> h((size_t)n_fine);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), acc.p, n_fine * 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_error(c, e, "refinement");
    for (int64_t f = 0; f < n_fine; ++f) psi_fine[f] = h[f] > 0.0 ? -epsilon * std::log(h[f]) : 0.0;
    return SDOT_OK;
}

// sdot_eval.cu -- evaluation of the entropic semi-discrete dual functional
// and its gradient on B200 (sm_100a).
//
// Replaces SotSolver::evaluate_functional / local_assemble / the value-grad
// lambda / find_nearest_target_points (src/solvers/SotSolver.cc:217-377,
// 769-869, 267-296, 553-570).  One evaluation is two sweeps over the
// (quadrature point, target) pairs plus two small reductions:
//
//   value sweep  (source-centric): per q the reference's max exponent m_q and
//     shifted sum S_q, accumulated online in FP64 with a hand-written exp2
//     (sdot_device.cuh) -> L_q = m_q + log S_q, value and C_global partials.
//   gradient sweep (target-centric, pull): g_j = sum_q w_q nu_j e^{t_qj - L_q}
//     accumulated per target without atomics; exponentials in FP32 ex2 with
//     FP64 accumulation (HYBRID/MIXED) or FP64 (FP64 precision).
//
// Truncation: a (cell, target) pair is a candidate iff
// sqrt_rn(d2(y_j, c_K)) <= r, evaluated as d2 <= s* where s* is the largest
// double with sqrt_rn(s*) <= r (sqrt_rn is monotone, so the two tests are
// identical); d2 is rounded exactly like the reference.  Both sweeps apply
// the same test, after a conservative bounding-sphere cull of whole blocks.
#include <float.h>
#include <math.h>
#include <stdio.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>

#include "sdot_dense.cuh"
#include "sdot_device.cuh"
#include "sdot_internal.h"

namespace sdot {

// ---------------------------------------------------------------------------
// small kernels
// ---------------------------------------------------------------------------

__global__ void k_gather(double *dst, const double *src, const int64_t *perm, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = src[perm[i]];
}

__global__ void k_scatter(double *dst, const double *src, const int64_t *perm, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[perm[i]] = src[i];
}

__global__ void k_axpy(double *x, const double *x0, double a, const double *p, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = x0[i] + a * p[i];
}

// max/min/non-finite flag of a vector: out[0]=max, out[1]=min, out[2]=1 if non-finite.
__global__ void k_minmax(const double *v, int64_t n, double *out)
{
    __shared__ double smx[32], smn[32];
    __shared__ int sbad[32];
    double mx = -DBL_MAX, mn = DBL_MAX;
    int bad = 0;
    // sixteen independent loads in flight per thread (max, min and the flag do
    // not depend on the order): the single CTA is bound by load latency
    constexpr int U = 16;
    const int64_t step = blockDim.x;
    int64_t i = threadIdx.x;
    for (; i + (U - 1) * step < n; i += U * step) {
        double a[U];
#pragma unroll
        for (int u = 0; u < U; ++u) a[u] = v[i + u * step];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (!isfinite(a[u])) bad = 1;
            mx = a[u] > mx ? a[u] : mx;
            mn = a[u] < mn ? a[u] : mn;
        }
    }
    for (; i < n; i += step) {
        const double a = v[i];
        if (!isfinite(a)) bad = 1;
        mx = a > mx ? a : mx;
        mn = a < mn ? a : mn;
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { smx[w] = mx; smn[w] = mn; sbad[w] = bad; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < (int)(blockDim.x >> 5); ++i) {
            mx = fmax(mx, smx[i]);
            mn = fmin(mn, smn[i]);
            bad |= sbad[i];
        }
        out[0] = mx;
        out[1] = mn;
        out[2] = bad;
    }
}

// tpack[j] = {A_j, B_j(DIM), nu_j, y_j(DIM)}: scaled exponent coefficients.
template <int DIM>
__global__ void k_target_prep(int64_t nt, const double *__restrict__ y, const double *__restrict__ nu,
                              const double *__restrict__ psi, EvalArgs a, double *__restrict__ tpack)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nt; j += (int64_t)gridDim.x * blockDim.x) {
        double yt[3], ysq = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            yt[d] = y[j * DIM + d] - a.o[d];
            ysq += yt[d] * yt[d];
        }
        double *t = tpack + j * TPACK;
        t[0] = a.s * psi[j] - a.halfs * ysq;
#pragma unroll
        for (int d = 0; d < DIM; ++d) t[1 + d] = a.s * yt[d];
        t[1 + DIM] = nu[j];
#pragma unroll
        for (int d = 0; d < DIM; ++d) t[2 + DIM + d] = y[j * DIM + d];
    }
}

// truncated-path layout: {y(3), nu, log2 nu, kappa psi / eps}
template <int DIM>
__global__ void k_target_prep_kd(int64_t nt, const double *__restrict__ y, const double *__restrict__ nu,
                                 const double *__restrict__ psi, EvalArgs a, double *__restrict__ tpack)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nt; j += (int64_t)gridDim.x * blockDim.x) {
        double *t = tpack + j * TPACK;
#pragma unroll
        for (int d = 0; d < 3; ++d) t[d] = d < DIM ? y[j * DIM + d] : 0.0;
        t[3] = nu[j];
        t[4] = log2(nu[j]);
        t[5] = a.s * psi[j];
    }
}

template <int DIM>
__global__ void __launch_bounds__(DENSE_A_THREADS)
k_value_dense(const double *__restrict__ x, const double *__restrict__ rho, const double *__restrict__ jxw,
              const double *__restrict__ tpack, EvalArgs a, double *__restrict__ Lq, double *__restrict__ part)
{
    dense_value_block<DIM>(x, rho, jxw, tpack, a, blockIdx.x, Lq, part + (int64_t)blockIdx.x * 4);
}

static_assert(DENSE_A_QT == 1, "the sliced dense value sweep keeps one point per thread");

template <int DIM>
__global__ void __launch_bounds__(DENSE_A_THREADS)
k_value_dense_slice(const double *__restrict__ x, const double *__restrict__ tpack, EvalArgs a, int64_t tslice,
                    double *__restrict__ ms)
{
    const int64_t t0 = blockIdx.y * tslice;
    const int64_t t1 = min(a.nt, t0 + tslice);
    dense_value_slice<DIM>(x, tpack, a, blockIdx.x, t0, t1, ms + (int64_t)blockIdx.y * 2 * a.nq);
}

constexpr int MERGE_THREADS = DENSE_A_THREADS * DENSE_MERGE_SPLIT;

template <int DIM>
__global__ void __launch_bounds__(MERGE_THREADS)
k_value_dense_merge(const double *__restrict__ x, const double *__restrict__ rho, const double *__restrict__ jxw,
                    const double *__restrict__ ms, int nslice, EvalArgs a, double *__restrict__ Lq,
                    double *__restrict__ part)
{
    dense_value_merge<DIM>(x, rho, jxw, ms, nslice, a, blockIdx.x, Lq, part + (int64_t)blockIdx.x * 4);
}

// Dense value sweep over cells whose points form a TM^DIM tensor grid
// symmetric about the cell centre (point i = i_0 + TM i_1 (+ TM^2 i_2)):
// thread <-> cell, one slice of the targets per blockIdx.y, with the same
// output as k_value_dense_slice (per point: its largest scaled exponent mx
// and the sum relative to it), merged by k_value_dense_merge.  The exponent
// of point q and target j, b_qj = A_j + B_j.(c - o) + sum_d B_jd delta_qd,
// factors per dimension: with G_d = B_jd a_d and the lowest point's
// exponent b_0 = B0 - sum_d G_d, b_qj = b_0 + sum_d i_d h_d G_d (h = 2 for
// TM = 2, 1 for TM = 3), so one exponential 2^((b_0 - M)/16) and one per
// dimension serve the cell's TM^DIM points.  M is a common shift per cell,
// an upper bound of every exponent so far (raised lazily, as in
// lse_update).  The per-point maxima are exact: a target updates them only
// when its upper bound B0 + sum |G_d| reaches the largest lower bound
// B0 - sum |G_d| seen so far, below which it cannot be any point's maximum.
// UNI (every cell has the offsets ua_d): G_d, its factor 2^(H G_d / 16) and
// the sums of G_d and |G_d| depend on the target alone, so they are computed
// once per staged target instead of once per (cell, target), leaving one
// exponential per (cell, target).
struct Spacing {
    double a[3];
};

template <int DIM, int TM, bool UNI>
__global__ void __launch_bounds__(DENSE_A_THREADS)
k_value_dense_tensor(const double *__restrict__ x, const double *__restrict__ tpack, EvalArgs a, int64_t ncells,
                     int64_t tslice, Spacing ua, double *__restrict__ ms)
{
    constexpr int NQ = DIM == 3 ? TM * TM * TM : TM * TM;
    // staged per target: A, B(DIM), nu; UNI adds G(DIM), 2^(H G / 16) (DIM), sum G, sum |G|
    constexpr int TSZ = UNI ? 3 * DIM + 4 : DIM + 2;
    constexpr double H = TM == 2 ? 2.0 : 1.0;
    __shared__ double tab[16];
    __shared__ double stg[DA_CHUNK * TSZ];
    if (threadIdx.x < 16) tab[threadIdx.x] = c_exp2_tab[threadIdx.x];
    const int64_t cell = blockIdx.x * (int64_t)DENSE_A_THREADS + threadIdx.x;
    const bool valid = cell < ncells;
    const int64_t q0 = (valid ? cell : 0) * NQ;
    // cell centre (relative to o) and half spacing per dimension, from the extreme points along d
    double cp[DIM], ah[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        const int stride = d == 0 ? 1 : (d == 1 ? TM : TM * TM);
        const double lo = x[q0 * DIM + d], hi = x[(q0 + (int64_t)(TM - 1) * stride) * DIM + d];
        const double cd = 0.5 * (lo + hi);
        cp[d] = cd - a.o[d];
        ah[d] = hi - cd;
    }
    const int64_t t0 = blockIdx.y * tslice;
    const int64_t t1 = min(a.nt, t0 + tslice);
    double S[NQ], mx[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        S[q] = 0.0;
        mx[q] = -CUDART_INF;
    }
    double M = -CUDART_INF, lbmax = -CUDART_INF;
    for (int64_t c0 = t0; c0 < t1; c0 += DA_CHUNK) {
        const int cn = (int)min((int64_t)DA_CHUNK, t1 - c0);
        __syncthreads();
        if constexpr (UNI) {
            for (int t = threadIdx.x; t < cn; t += DENSE_A_THREADS) {
                const double *src = tpack + (c0 + t) * TPACK;
                double *dst = stg + t * TSZ;
                double sg = 0.0, ag = 0.0;
#pragma unroll
                for (int f = 0; f < DIM + 2; ++f) dst[f] = src[f];
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    const double G = src[1 + d] * ua.a[d];
                    dst[DIM + 2 + d] = G;
                    dst[2 * DIM + 2 + d] = exp2_16(H * G, tab);
                    sg += G;
                    ag += fabs(G);
                }
                dst[3 * DIM + 2] = sg;
                dst[3 * DIM + 3] = ag;
            }
        } else {
            for (int i = threadIdx.x; i < cn * TSZ; i += DENSE_A_THREADS) {
                const int t = i / TSZ, f = i - t * TSZ;
                stg[i] = tpack[(c0 + t) * TPACK + f];
            }
        }
        __syncthreads();
        for (int t = 0; t < cn; ++t) {
            const double *tp = stg + t * TSZ;
            double B0 = tp[0], G[DIM], sg = 0.0, ag = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                B0 = fma(tp[1 + d], cp[d], B0);
                if constexpr (UNI) {
                    G[d] = tp[DIM + 2 + d];
                } else {
                    G[d] = tp[1 + d] * ah[d];
                    sg += G[d];
                    ag += fabs(G[d]);
                }
            }
            if constexpr (UNI) {
                sg = tp[3 * DIM + 2];
                ag = tp[3 * DIM + 3];
            }
            const double ub = B0 + ag;
            if (ub - M > LSE_THR) {   // raise the shift (the first target sets it)
                if (M > -CUDART_INF) {
                    const double sc = exp2_16(M - ub, tab);
#pragma unroll
                    for (int q = 0; q < NQ; ++q) S[q] *= sc;
                }
                M = ub;
            }
            const double P = tp[1 + DIM] * exp2_16(B0 - sg - M, tab);
            double r[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) r[d] = UNI ? tp[2 * DIM + 2 + d] : exp2_16(H * G[d], tab);
#pragma unroll
            for (int i0 = 0; i0 < TM; ++i0) {
                const double f0 = i0 == 0 ? P : (i0 == 1 ? P * r[0] : P * r[0] * r[0]);
#pragma unroll
                for (int i1 = 0; i1 < TM; ++i1) {
                    const double f1 = i1 == 0 ? f0 : (i1 == 1 ? f0 * r[1] : f0 * r[1] * r[1]);
                    if constexpr (DIM == 2) {
                        S[i0 + TM * i1] += f1;
                    } else {
#pragma unroll
                        for (int i2 = 0; i2 < TM; ++i2) {
                            const double f2 = i2 == 0 ? f1 : (i2 == 1 ? f1 * r[2] : f1 * r[2] * r[2]);
                            S[i0 + TM * i1 + TM * TM * i2] += f2;
                        }
                    }
                }
            }
            if (ub >= lbmax) {
                lbmax = fmax(lbmax, B0 - ag);
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    double b = B0;
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        const int id = (d == 0 ? q : (d == 1 ? q / TM : q / (TM * TM))) % TM;
                        const double sd = TM == 2 ? (id == 0 ? -1.0 : 1.0) : (double)(id - 1);
                        b = fma(sd, G[d], b);
                    }
                    mx[q] = fmax(mx[q], b);
                }
            }
        }
    }
    if (valid) {
        double *out = ms + (int64_t)blockIdx.y * 2 * a.nq + 2 * q0;
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            out[2 * q] = mx[q];
            out[2 * q + 1] = (mx[q] == -CUDART_INF) ? 0.0 : S[q] * exp2_16(M - mx[q], tab);
        }
    }
}

// Sum over a tensor-grid cell's points of W_q prod_d r_d^(i_d) (point
// q = i_0 + TM i_1 (+ TM^2 i_2)), by Horner's scheme along each dimension.
template <typename R>
__device__ __forceinline__ R fma_r(R x, R y, R z)
{
    if constexpr (sizeof(R) == 4) return fmaf(x, y, z);
    else return fma(x, y, z);
}

template <int DIM, int TM, typename R>
__device__ __forceinline__ R cell_sum(const R *W, const R *r)
{
    R t2 = R(0);
#pragma unroll
    for (int i2 = (DIM == 3 ? TM - 1 : 0); i2 >= 0; --i2) {
        R t1 = R(0);
#pragma unroll
        for (int i1 = TM - 1; i1 >= 0; --i1) {
            const R *Wr = W + TM * i1 + TM * TM * i2;
            R t0 = Wr[TM - 1];
#pragma unroll
            for (int i0 = TM - 2; i0 >= 0; --i0) t0 = fma_r(t0, r[0], Wr[i0]);
            t1 = (i1 == TM - 1) ? t0 : fma_r(t1, r[1], t0);
        }
        t2 = (DIM == 2 || i2 == TM - 1) ? t1 : fma_r(t2, r[DIM == 3 ? 2 : 0], t1);
    }
    return t2;
}

// Dense gradient sweep over the tensor-grid cells of k_value_dense_tensor:
// thread lane <-> DENSE_B_TT targets, the CTA's slice of cells staged in
// shared memory, DENSE_B_QG groups taking every QG-th staged cell, the
// groups' sums added in group order.  With the cell centre C, the half
// spacing a_d and point offsets delta_qd = (H i_d - 1) a_d,
// |x_q - y|^2 = |C - y|^2 + sum_d (2 delta_qd (C_d - y_d) + delta_qd^2), so a
// (point, target) term is a cell factor times one factor per dimension
// raised to i_d times a per-point weight that does not depend on the target:
//   FP32: 2^(alpha_j + beta_q - c |x_q - y_j|^2)
//       = 2^(alpha_j + bref - c |C - y_j|^2 - sum_d v_d) prod_d 2^(H v_d i_d) W_q,
//         v_d = -2 c a_d (C_d - y_d),  W_q = w_q 2^(beta_q - c |delta_q|^2 - bref);
//   FP64: 2^(u_qj / 16), u_qj = A_j + B_j . (x_q - o) + D_q
//       = 2^((A_j + B_j . (C - o) - sum_d G_d + Dref) / 16) prod_d 2^(H G_d i_d / 16) W_q,
//         G_d = B_jd a_d,  W_q = w_q 2^((D_q - Dref) / 16),
// where bref / Dref is the largest per-point part in the cell (W_q <= w_q).
// One exponential per cell and one per dimension replace TM^DIM.  The
// caller admits the FP32 form only when the factors of a cell span less
// than 2^60 (dense_grad_tensor), so no factor or Horner sum leaves the FP32
// range; the FP64 form inherits the tensor value sweep's bound.
// Non-finite L_q: a cell whose parts are all -inf contributes 0 (as every
// one of its terms does); a +inf part gives a NaN term where the per-point
// form gives +inf (both non-finite, flagged by the finalize).
// UNI (FP64 form, every cell has the offsets ua_d): G_d and its factor
// depend on the target alone and are computed once per target, so one
// exponential per (cell, target) remains.  (The FP32 form measured slower
// with its factors split into cell and target parts: registers.)
template <int DIM, int TM, bool FP32, bool UNI>
__global__ void __launch_bounds__(DENSE_B_CTA, DENSE_B_PER_SM)
k_grad_dense_tensor(const double *__restrict__ x, const double *__restrict__ w, const double *__restrict__ Lq,
                    const double *__restrict__ tpack, const double *__restrict__ psi, EvalArgs a, int64_t ncells,
                    int64_t cslice, Spacing ua, double *__restrict__ gpart)
{
    constexpr int NQ = DIM == 3 ? TM * TM * TM : TM * TM;
    constexpr int TT = DENSE_B_TT;
    constexpr int QG = DENSE_B_QG;
    constexpr int NTH = DENSE_B_CTA;
    constexpr int GC = NTH / NQ < 64 ? NTH / NQ : 64;  // cells staged at a time: one point per thread
    constexpr int CR = 16;                             // cell record: W (NQ), C (DIM), k (DIM), reference
    static_assert(NQ + 2 * DIM + 1 <= CR, "cell record");
    static_assert(!(UNI && FP32), "per-target factors: FP64 form only");
    constexpr double H = TM == 2 ? 2.0 : 1.0;
    using R = typename std::conditional<FP32, float, double>::type;
    __shared__ double tab[16];
    __shared__ __align__(16) R crec[GC * CR];
    __shared__ double pb[GC * NQ];
    if (threadIdx.x < 16) tab[threadIdx.x] = c_exp2_tab[threadIdx.x];
    const int tid = threadIdx.x;
    const int lt = tid % DENSE_B_THREADS;
    const int grp = tid / DENSE_B_THREADS;
    const int64_t j0 = blockIdx.x * (int64_t)(DENSE_B_THREADS * TT);
    GradTargets<TT> T;
    grad_targets<DIM, FP32, NTH>(tpack, psi, a, j0, lt, T);
    double acc64[TT];
#pragma unroll
    for (int k = 0; k < TT; ++k) acc64[k] = 0.0;
    // UNI: the per-dimension factors and their exponents' sum, per target
    double rt[TT][DIM], st[TT];
    if constexpr (UNI) {
        __syncthreads();  // tab
#pragma unroll
        for (int k = 0; k < TT; ++k) {
            st[k] = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                const double G = T.B[k][d] * ua.a[d];
                rt[k][d] = exp2_16(H * G, tab);
                st[k] += G;
            }
        }
    }
    const int64_t ca = blockIdx.y * cslice;
    const int64_t cb = min(ncells, ca + cslice);
    const float c32 = (float)a.c32;
    for (int64_t c0 = ca; c0 < cb; c0 += GC) {
        const int cn = (int)min((int64_t)GC, cb - c0);
        const int cl = tid / NQ, qi = tid - cl * NQ;
        const bool act = cl < cn;
        const int64_t cq0 = (c0 + (act ? cl : 0)) * NQ;
        // the cell's centre and half spacing from its extreme points along each dimension
        double cen[DIM], ah[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const int stride = d == 0 ? 1 : (d == 1 ? TM : TM * TM);
            const double lo = x[cq0 * DIM + d], hi = x[(cq0 + (int64_t)(TM - 1) * stride) * DIM + d];
            cen[d] = 0.5 * (lo + hi);
            ah[d] = hi - cen[d];
        }
        __syncthreads();  // the previous cells' records are consumed
        double wq = 0.0;
        if (act) {
            // the part of point q's exponent that does not depend on the target
            const int64_t q = cq0 + qi;
            double part;
            if (FP32) {
                double dsq = 0.0;
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    const double dl = x[q * DIM + d] - cen[d];
                    dsq += dl * dl;
                }
                part = -LOG2E * Lq[q] + T.aref - a.c32 * dsq;
            } else {
                double xsq = 0.0;
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    const double xt = x[q * DIM + d] - a.o[d];
                    xsq += xt * xt;
                }
                part = -a.halfs * xsq - KAPPA * Lq[q];
            }
            pb[tid] = part;
            wq = w[q];
        }
        __syncthreads();
        if (act) {
            double ref = -CUDART_INF;
#pragma unroll
            for (int u = 0; u < NQ; ++u) ref = fmax(ref, pb[cl * NQ + u]);
            const bool none = ref == -CUDART_INF;  // every term of the cell is 0
            const double own = pb[tid];
            const double Wq = none ? 0.0 : (FP32 ? wq * exp2(own - ref) : wq * exp2_16(own - ref, tab));
            R *rec = crec + cl * CR;
            rec[qi] = (R)Wq;
            if (qi == 0) {
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    rec[NQ + d] = FP32 ? (R)(cen[d] - T.ob[d]) : (R)(cen[d] - a.o[d]);
                    rec[NQ + DIM + d] = FP32 ? (R)(-2.0 * a.c32 * ah[d]) : (R)ah[d];
                }
                rec[NQ + 2 * DIM] = (R)(none ? 0.0 : ref);
            }
        }
        __syncthreads();
        if constexpr (FP32) {
            float acc[TT];
#pragma unroll
            for (int k = 0; k < TT; ++k) acc[k] = 0.f;
            int n = 0;
            for (int cc = grp; cc < cn; cc += QG, ++n) {
                const float *rec = crec + cc * CR;
                float Wc[NQ], Cc[DIM], kd[DIM];
#pragma unroll
                for (int u = 0; u < NQ; ++u) Wc[u] = rec[u];
#pragma unroll
                for (int d = 0; d < DIM; ++d) { Cc[d] = rec[NQ + d]; kd[d] = rec[NQ + DIM + d]; }
                const float bref = rec[NQ + 2 * DIM];
#pragma unroll
                for (int k = 0; k < TT; ++k) {
                    float D2 = 0.f, sv = 0.f, r[DIM];
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        const float dc = Cc[d] - T.yt[k][d];
                        D2 = fmaf(dc, dc, D2);
                        const float v = kd[d] * dc;
                        sv += v;
                        r[d] = ex2_approx((float)H * v);
                    }
                    const float P = ex2_approx(fmaf(-c32, D2, T.alpha[k] + bref) - sv);
                    acc[k] = fmaf(P, cell_sum<DIM, TM, float>(Wc, r), acc[k]);
                }
                if ((n & 7) == 7) {
#pragma unroll
                    for (int k = 0; k < TT; ++k) { acc64[k] += (double)acc[k]; acc[k] = 0.f; }
                }
            }
#pragma unroll
            for (int k = 0; k < TT; ++k) acc64[k] += (double)acc[k];
        } else {
            for (int cc = grp; cc < cn; cc += QG) {
                const double *rec = crec + cc * CR;
                double Wc[NQ], Cm[DIM], ad[DIM];
#pragma unroll
                for (int u = 0; u < NQ; ++u) Wc[u] = rec[u];
#pragma unroll
                for (int d = 0; d < DIM; ++d) { Cm[d] = rec[NQ + d]; ad[d] = rec[NQ + DIM + d]; }
                const double Dref = rec[NQ + 2 * DIM];
#pragma unroll
                for (int k = 0; k < TT; ++k) {
                    double B0 = T.A[k], sg = 0.0, r[DIM];
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        B0 = fma(T.B[k][d], Cm[d], B0);
                        if constexpr (UNI) {
                            r[d] = rt[k][d];
                        } else {
                            const double G = T.B[k][d] * ad[d];
                            sg += G;
                            r[d] = exp2_16(H * G, tab);
                        }
                    }
                    if constexpr (UNI) sg = st[k];
                    const double P = exp2_16(B0 - sg + Dref, tab);
                    acc64[k] = fma(P, cell_sum<DIM, TM, double>(Wc, r), acc64[k]);
                }
            }
        }
    }
    // the groups' sums, added in group order by group 0
    __shared__ double gsum[(QG - 1) * TT * DENSE_B_THREADS];
    if (grp > 0) {
#pragma unroll
        for (int k = 0; k < TT; ++k) gsum[((grp - 1) * TT + k) * DENSE_B_THREADS + lt] = acc64[k];
    }
    __syncthreads();
    if (grp == 0) {
#pragma unroll
        for (int k = 0; k < TT; ++k) {
            for (int g = 1; g < QG; ++g) acc64[k] += gsum[((g - 1) * TT + k) * DENSE_B_THREADS + lt];
            const int64_t j = j0 + lt + k * DENSE_B_THREADS;
            if (j < a.nt) {
                double gv = acc64[k];
                if (!FP32) gv *= tpack[j * TPACK + 1 + DIM];  // nu_j (FP32 folds it into alpha)
                gpart[blockIdx.y * a.nt + j] = gv;
            }
        }
    }
}

template <int DIM, bool FP32>
__global__ void __launch_bounds__(DENSE_B_CTA, DENSE_B_PER_SM)
k_grad_dense(const double *__restrict__ x, const double *__restrict__ w, const double *__restrict__ Lq,
             const double *__restrict__ tpack, const double *__restrict__ psi, EvalArgs a, int64_t qslice,
             double *__restrict__ gpart)
{
    dense_grad_block<DIM, FP32, DENSE_B_QG>(x, w, Lq, tpack, psi, a, qslice, blockIdx.x, blockIdx.y, gpart);
}

// ---------------------------------------------------------------------------
// finalize: g_j = sum of partials - nu_j, plus the reductions the solver and
// the solver control need (SotSolver.cc:322-327, SotSolver.h:391-442).
// ---------------------------------------------------------------------------

constexpr int FIN_THREADS = 256;
constexpr int FIN_BLOCKS = 148;  // largest grid of k_finalize_grad
constexpr int NRED = 8;  // psinu, l1, linf, comp, l2sq, gp, nonfinite, unused

// Lanes per target of k_finalize_grad for nks slice partials: the smallest
// power of two >= nks, at most 8.
static int fin_parts(int nks)
{
    return nks <= 1 ? 1 : (nks <= 2 ? 2 : (nks <= 4 ? 4 : 8));
}

// Grid of k_finalize_grad for nt targets (FIN_THREADS / parts targets per CTA and pass).
static int fin_blocks(int64_t nt, int parts)
{
    const int64_t per = FIN_THREADS / parts;
    const int64_t g = (nt + per - 1) / per;
    return (int)std::max<int64_t>(1, std::min<int64_t>(FIN_BLOCKS, g));
}

// PARTS consecutive lanes own target j: lane u sums the slice partials
// k = u, u + PARTS, ... in order of k (each lane's loads in flight together),
// and xor exchanges add the lanes' sums in the fixed tree (s0 + s1) + (s2 +
// s3), ...  PARTS = 8, or any power of two PARTS >= nks, gives the sums of
// eight interleaved sums k mod 8 added in the tree ((s0 + s1) + (s2 + s3)) +
// ((s4 + s5) + (s6 + s7)) (the lanes past nks hold zeros).
template <int PARTS>
__global__ void __launch_bounds__(FIN_THREADS)
k_finalize_grad(int64_t nt, int nks, const double *__restrict__ gpart, const double *__restrict__ nu,
                const double *__restrict__ psi, const double *__restrict__ pdir, double tol, int sub_nu,
                double *__restrict__ grad, double *__restrict__ redpart)
{
    constexpr int FIN_PARTS = PARTS;
    constexpr int TPB = FIN_THREADS / FIN_PARTS;  // targets per CTA and pass
    const int u = threadIdx.x % FIN_PARTS;
    double psinu = 0.0, l1 = 0.0, linf = 0.0, comp = -CUDART_INF, l2 = 0.0, gp = 0.0, bad = 0.0;
    for (int64_t base = blockIdx.x * (int64_t)TPB; base < nt; base += (int64_t)gridDim.x * TPB) {
        const int64_t j = base + threadIdx.x / FIN_PARTS;
        const bool ok = j < nt;
        double acc = 0.0;
        if (ok) {
            int k = u;
            for (; k + 3 * FIN_PARTS < nks; k += 4 * FIN_PARTS) {
                const double v0 = gpart[(int64_t)k * nt + j];
                const double v1 = gpart[(int64_t)(k + FIN_PARTS) * nt + j];
                const double v2 = gpart[(int64_t)(k + 2 * FIN_PARTS) * nt + j];
                const double v3 = gpart[(int64_t)(k + 3 * FIN_PARTS) * nt + j];
                acc += v0;
                acc += v1;
                acc += v2;
                acc += v3;
            }
            for (; k < nks; k += FIN_PARTS) acc += gpart[(int64_t)k * nt + j];
        }
#pragma unroll
        for (int o = 1; o < FIN_PARTS; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (ok && u == 0) {
            const double s = acc;
            const double g = s - nu[j];
            grad[j] = sub_nu ? g : s;
            psinu += psi[j] * nu[j];
            const double ag = fabs(g);
            l1 += ag;
            linf = fmax(linf, ag);
            comp = fmax(comp, ag - nu[j] * tol);
            l2 += g * g;
            if (pdir) gp += g * pdir[j];
            if (!isfinite(g) || !isfinite(psi[j])) bad = 1.0;
        }
    }
    __shared__ double sh[NRED][FIN_THREADS / 32];
    psinu = warp_sum(psinu);
    l1 = warp_sum(l1);
    linf = warp_max(linf);
    comp = warp_max(comp);
    l2 = warp_sum(l2);
    gp = warp_sum(gp);
    bad = warp_max(bad);
    const int wi = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        sh[0][wi] = psinu; sh[1][wi] = l1; sh[2][wi] = linf; sh[3][wi] = comp;
        sh[4][wi] = l2; sh[5][wi] = gp; sh[6][wi] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r[7] = {0, 0, 0, -CUDART_INF, 0, 0, 0};
        for (int i = 0; i < FIN_THREADS / 32; ++i) {
            r[0] += sh[0][i]; r[1] += sh[1][i]; r[2] = fmax(r[2], sh[2][i]); r[3] = fmax(r[3], sh[3][i]);
            r[4] += sh[4][i]; r[5] += sh[5][i]; r[6] = fmax(r[6], sh[6][i]);
        }
        for (int k = 0; k < 7; ++k) redpart[blockIdx.x * NRED + k] = r[k];
    }
}

// k_finalize_grad with fin_parts(nks) lanes per target; returns its grid size.
static int launch_finalize_grad(int64_t nt, int nks, const double *gpart, const double *nu, const double *psi,
                                const double *pdir, double tol, int sub_nu, double *grad, double *redpart,
                                cudaStream_t st)
{
    const int parts = fin_parts(nks);
    const int fb = fin_blocks(nt, parts);
    auto go = [&](auto kern) {
        kern<<<fb, FIN_THREADS, 0, st>>>(nt, nks, gpart, nu, psi, pdir, tol, sub_nu, grad, redpart);
    };
    if (parts == 1) go(k_finalize_grad<1>);
    else if (parts == 2) go(k_finalize_grad<2>);
    else if (parts == 4) go(k_finalize_grad<4>);
    else go(k_finalize_grad<8>);
    return fb;
}

// One CTA of T threads: thread i sums value partials i, i + T, i + 2T, ...
// into four accumulators (partial i + kT into accumulator k mod 4, eight
// loads in flight), added in a fixed order, and the gradient blocks'
// reductions i, i + T, ...; then warp reductions, and warp 0 reduces the
// warps' results (a fixed tree throughout).  T = 256 for up to 2,048 value
// partials (the dense path), 1,024 above (one per source block).
template <int T>
__global__ void __launch_bounds__(T)
k_finalize_scalars(int nred, const double *__restrict__ redpart, int64_t nval, const double *__restrict__ valpart,
                   double *__restrict__ scal)
{
    constexpr int NW = T / 32;
    __shared__ double sh[11][NW];
    double va[4] = {0, 0, 0, 0}, ca[4] = {0, 0, 0, 0}, ska[4] = {0, 0, 0, 0}, npa[4] = {0, 0, 0, 0};
    const double4 *vp = reinterpret_cast<const double4 *>(valpart);
    int64_t b0 = threadIdx.x;
    for (; b0 + 7 * T < nval; b0 += 8 * T) {
        double4 t[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) t[u] = vp[b0 + u * T];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            va[u & 3] += t[u].x;
            ca[u & 3] += t[u].y;
            ska[u & 3] += t[u].z;
            npa[u & 3] += t[u].w;
        }
    }
#pragma unroll
    for (int u = 0; u < 7; ++u) {
        if (b0 + u * T < nval) {
            const double4 t = vp[b0 + u * T];
            va[u & 3] += t.x;
            ca[u & 3] += t.y;
            ska[u & 3] += t.z;
            npa[u & 3] += t.w;
        }
    }
    double v = (va[0] + va[1]) + (va[2] + va[3]), c = (ca[0] + ca[1]) + (ca[2] + ca[3]);
    double sk = (ska[0] + ska[1]) + (ska[2] + ska[3]), np = (npa[0] + npa[1]) + (npa[2] + npa[3]);
    double r[7] = {0, 0, 0, -CUDART_INF, 0, 0, 0};
    for (int b = threadIdx.x; b < nred; b += T) {
        const double *p = redpart + (int64_t)b * NRED;
        r[0] += p[0]; r[1] += p[1]; r[2] = fmax(r[2], p[2]); r[3] = fmax(r[3], p[3]);
        r[4] += p[4]; r[5] += p[5]; r[6] = fmax(r[6], p[6]);
    }
    v = warp_sum(v); c = warp_sum(c); sk = warp_sum(sk); np = warp_sum(np);
    r[0] = warp_sum(r[0]); r[1] = warp_sum(r[1]); r[2] = warp_max(r[2]); r[3] = warp_max(r[3]);
    r[4] = warp_sum(r[4]); r[5] = warp_sum(r[5]); r[6] = warp_max(r[6]);
    const int wi = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        sh[0][wi] = v; sh[1][wi] = c; sh[2][wi] = sk; sh[10][wi] = np;
#pragma unroll
        for (int k = 0; k < 7; ++k) sh[3 + k][wi] = r[k];
    }
    __syncthreads();
    if (wi == 0) {
        double t[11];
        // sums: 0 value, 1 C, 2 skipped, 3 psinu, 4 l1, 7 l2sq, 8 dot_gp, 10 pairs; maxima: 5 linf, 6 comp, 9 bad
#pragma unroll
        for (int k = 0; k < 11; ++k)
            t[k] = lane < NW ? sh[k][lane] : ((k == 5 || k == 6 || k == 9) ? -CUDART_INF : 0.0);
#pragma unroll
        for (int k = 0; k < 11; ++k) t[k] = (k == 5 || k == 6 || k == 9) ? warp_max(t[k]) : warp_sum(t[k]);
        if (lane == 0) {
            const double psinu = t[3];
            const double value = t[0] - psinu;
            scal[SC_VALUE] = value;
            scal[SC_VALSRC] = t[0];
            scal[SC_C] = t[1];
            scal[SC_SKIPPED] = t[2];
            scal[SC_PSINU] = psinu;
            scal[SC_L1] = t[4];
            scal[SC_LINF] = t[5];
            scal[SC_COMP] = t[6];
            scal[SC_L2SQ] = t[7];
            scal[SC_DOT_GP] = t[8];
            scal[SC_NONFINITE] = (t[9] != 0.0 || !isfinite(value)) ? 1.0 : 0.0;
            scal[SC_PAIRS] = t[10];
        }
    }
}

// k_finalize_scalars with its CTA size for nval value partials.
static void launch_finalize_scalars(cudaStream_t st, int nred, const double *redpart, int64_t nval,
                                    const double *valpart, double *scal)
{
    if (nval <= 2048) k_finalize_scalars<256><<<1, 256, 0, st>>>(nred, redpart, nval, valpart, scal);
    else k_finalize_scalars<1024><<<1, 1024, 0, st>>>(nred, redpart, nval, valpart, scal);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

static int grid_for(int64_t n, int threads, int cap = 148 * 8)
{
    int64_t g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (int)g;
}

void launch_target_prep_dense(sdot_ctx *c, const EvalArgs &a)
{
    if (c->dim == 2)
        k_target_prep<2><<<grid_for(a.nt, 256), 256, 0, c->stream>>>(a.nt, c->y.p, c->nu.p, c->psi.p, a, c->tpack.p);
    else
        k_target_prep<3><<<grid_for(a.nt, 256), 256, 0, c->stream>>>(a.nt, c->y.p, c->nu.p, c->psi.p, a, c->tpack.p);
}

void k_axpy_launch(cudaStream_t s, double *x, const double *x0, double a, const double *p, int64_t n)
{
    k_axpy<<<grid_for(n, 256), 256, 0, s>>>(x, x0, a, p, n);
}

sdot_status launch_gather(sdot_ctx *c, double *dst, const double *src, int64_t n)
{
    k_gather<<<grid_for(n, 256), 256, 0, c->stream>>>(dst, src, c->perm.p, n);
    c->klaunch[5] += 1;
    return cuda_error(c, cudaGetLastError(), "gather");
}

sdot_status launch_scatter(sdot_ctx *c, double *dst, const double *src, int64_t n)
{
    k_scatter<<<grid_for(n, 256), 256, 0, c->stream>>>(dst, src, c->perm.p, n);
    c->klaunch[5] += 1;
    return cuda_error(c, cudaGetLastError(), "scatter");
}

// largest double s with sqrt_rn(s) <= r (s* = NaN if r is NaN)
double sstar_of(double r)
{
    if (std::isnan(r)) return NAN;
    if (r < 0) return -1.0;
    if (r >= 1.3407807929942596e154) return DBL_MAX;
    double s = r * r;
    while (s > 0 && std::sqrt(s) > r) s = std::nextafter(s, 0.0);
    while (std::sqrt(std::nextafter(s, INFINITY)) <= r) s = std::nextafter(s, INFINITY);
    return s;
}

// SotSolver::compute_distance_threshold (SotSolver.cc:379-429), on the host
// with the same libm calls and operation order as the reference.
double host_threshold(sdot_ctx *c, double maxpsi, double minpsi)
{
    const sdot_solver_params &p = c->prm;
    if (p.threshold_type == SDOT_THRESH_INTEGRAL) {
        double absJ = std::fabs(c->global_functional);
        if (absJ < 1e-10) absJ = 1e-10;
        const double num = p.epsilon * c->C_global;
        const double den = p.tau * absJ;
        const double arg = num / den;
        const double r2 = 2.0 * maxpsi + 2.0 * p.epsilon * std::log(arg);
        const double r = std::sqrt(std::max(0.0, r2));
        return std::max(r, c->covering_radius);
    }
    if (p.threshold_type == SDOT_THRESH_GEOMETRIC) {
        double r0 = c->covering_radius;
        if (!(r0 > 0.0)) {
            double rr = 0.0;
            sdot_compute_covering_radius(c, &rr);
            r0 = rr;
        }
        const double range = maxpsi - minpsi;
        const double mind = c->min_target_density > 0.0 ? c->min_target_density : c->nu_min;
        double fv = std::fabs(c->global_functional);
        if (fv < 1e-10) fv = 1e-10;
        const double log_term = std::log(p.epsilon / (mind * p.tau * fv));
        double r2 = r0 * r0 + 2.0 * range + 2.0 * p.epsilon * log_term;
        if (r2 < r0 * r0) r2 = r0 * r0;
        return std::sqrt(r2);
    }
    const double numin = c->min_target_density > 0.0 ? c->min_target_density : c->nu_min;
    if (numin <= 0 || p.tau <= 0) return DBL_MAX;
    const double r2 = -2.0 * p.epsilon * std::log(p.tau / numin) + 2.0 * maxpsi;
    return std::sqrt(std::max(0.0, r2));
}

// Launch shape of the dense sweeps, shared by every dense evaluation path so
// that they sum in the same order: value-sweep point blocks (one quadrature
// point per thread) and, when those are too few to fill the GPU (fewer than
// four per SM), target slices of the value sweep (about twelve CTAs per SM in
// all, at least 64 targets per slice, at most 16 slices) merged per point;
// gradient target blocks, and q-slices of the gradient sweep (about eight
// CTAs per SM in all, at least 256 points per slice, at most 64 slices).
// With tm > 0 (cells whose points form a tm^dim tensor grid, at most 9
// points) the value sweep runs over cells (k_value_dense_tensor): ncb cell
// blocks x nvs target slices (about six CTAs per SM in all, at least 32
// targets per slice, at most 64 slices), always merged per point.
struct DenseShape {
    int64_t nval, tb;
    int nks;
    int nvs;          // target slices of the value sweep (1: unsliced)
    int64_t tslice;   // targets per value slice
    int tm;           // > 0: the cell-based tensor value sweep with tm points per dimension
    int64_t ncb;      // its cell blocks
};
// The tensor value sweep applies to the euclidean untruncated evaluation of
// cells whose points form a symmetric tensor grid of at most 9 points, with
// per-dimension factors that stay within 2^100 over the domain.
static int dense_tensor_m(const sdot_ctx *c, double s_scale)
{
    if (c->distance != 0 || c->tensor_m <= 0) return 0;
    const int tm = c->tensor_m;
    const int np = c->dim == 3 ? tm * tm * tm : tm * tm;
    if (np > 9 || c->qpc != np) return 0;
    const double span = (tm == 2 ? 2.0 : 1.0) * s_scale * 0.5 * c->diam * c->tensor_amax * (tm - 1) * c->dim / 16.0;
    return span <= 100.0 ? tm : 0;
}
static DenseShape dense_shape(int64_t nq, int64_t nt, int tm = 0, int64_t ncells = 0)
{
    DenseShape d{};
    const int64_t per = (int64_t)DENSE_A_THREADS * DENSE_A_QT;
    d.nval = (nq + per - 1) / per;
    d.nvs = 1;
    if (d.nval < 148 * 4) {
        const int64_t want = (148 * 12 + d.nval - 1) / d.nval;
        const int64_t maxs = std::max<int64_t>(1, nt / 64);
        d.nvs = (int)std::max<int64_t>(1, std::min<int64_t>(16, std::min(want, maxs)));
    }
    d.tslice = (nt + d.nvs - 1) / d.nvs;
    d.tb = (nt + DENSE_B_THREADS * DENSE_B_TT - 1) / (DENSE_B_THREADS * DENSE_B_TT);
    d.nks = dense_grad_slices(nq, nt);
    d.tm = tm;
    if (tm > 0) {
        d.ncb = (ncells + DENSE_A_THREADS - 1) / DENSE_A_THREADS;
        const int64_t want = (148 * 6 + d.ncb - 1) / d.ncb;
        const int64_t maxs = std::max<int64_t>(1, nt / 32);
        d.nvs = (int)std::max<int64_t>(1, std::min<int64_t>(64, std::min(want, maxs)));
        d.tslice = (nt + d.nvs - 1) / d.nvs;
    }
    return d;
}

template <int DIM>
static void launch_value_dense_tensor(const sdot_ctx *c, const DenseShape &ds, const double *tpack,
                                      const EvalArgs &a, double *ms, cudaStream_t st)
{
    const dim3 grid((unsigned)ds.ncb, (unsigned)ds.nvs);
    Spacing ua;
    for (int d = 0; d < 3; ++d) ua.a[d] = c->tensor_a[d];
    auto go = [&](auto kern) {
        kern<<<grid, DENSE_A_THREADS, 0, st>>>(c->x.p, tpack, a, c->ncells, ds.tslice, ua, ms);
    };
    const bool uni = c->tensor_uniform;
    if constexpr (DIM == 2) {
        if (ds.tm == 3) uni ? go(k_value_dense_tensor<2, 3, true>) : go(k_value_dense_tensor<2, 3, false>);
        else uni ? go(k_value_dense_tensor<2, 2, true>) : go(k_value_dense_tensor<2, 2, false>);
    } else {
        uni ? go(k_value_dense_tensor<3, 2, true>) : go(k_value_dense_tensor<3, 2, false>);
    }
}

// The tensor-cell gradient sweep runs on the tensor value sweep's cells; its
// FP32 form only where a cell's factors span at most 2^60 (their exponents
// vary by H log2(e) / eps |C - y| a_d (TM - 1) per dimension, |C - y| <= diam).
static bool dense_grad_tensor(const sdot_ctx *c, int tm, bool fp32, const EvalArgs &a)
{
    if (tm <= 0) return false;
    if (!fp32) return true;
    const double spread = (tm == 2 ? 2.0 : 1.0) * a.l2e_eps * c->diam * c->tensor_amax * (tm - 1) * c->dim;
    return spread <= 60.0;
}

template <int DIM>
static void launch_grad_dense(const sdot_ctx *c, const DenseShape &ds, bool fp32, const double *Lq,
                              const double *tpack, const double *psi, const EvalArgs &a, double *gpart,
                              cudaStream_t st)
{
    const dim3 g((unsigned)ds.tb, (unsigned)ds.nks);
    if (dense_grad_tensor(c, ds.tm, fp32, a)) {
        const int64_t cs = (c->ncells + ds.nks - 1) / ds.nks;
        Spacing ua;
        for (int d = 0; d < 3; ++d) ua.a[d] = c->tensor_a[d];
        auto go = [&](auto kern) {
            kern<<<g, DENSE_B_CTA, 0, st>>>(c->x.p, c->w.p, Lq, tpack, psi, a, c->ncells, cs, ua, gpart);
        };
        const bool uni = c->tensor_uniform;
        if constexpr (DIM == 2) {
            if (ds.tm == 3) {
                if (fp32) go(k_grad_dense_tensor<2, 3, true, false>);
                else uni ? go(k_grad_dense_tensor<2, 3, false, true>) : go(k_grad_dense_tensor<2, 3, false, false>);
            } else {
                if (fp32) go(k_grad_dense_tensor<2, 2, true, false>);
                else uni ? go(k_grad_dense_tensor<2, 2, false, true>) : go(k_grad_dense_tensor<2, 2, false, false>);
            }
        } else {
            if (fp32) go(k_grad_dense_tensor<3, 2, true, false>);
            else uni ? go(k_grad_dense_tensor<3, 2, false, true>) : go(k_grad_dense_tensor<3, 2, false, false>);
        }
        return;
    }
    const int64_t qslice = (a.nq + ds.nks - 1) / ds.nks;
    if (fp32) k_grad_dense<DIM, true><<<g, DENSE_B_CTA, 0, st>>>(c->x.p, c->w.p, Lq, tpack, psi, a, qslice, gpart);
    else k_grad_dense<DIM, false><<<g, DENSE_B_CTA, 0, st>>>(c->x.p, c->w.p, Lq, tpack, psi, a, qslice, gpart);
}

template <int DIM>
static sdot_status run_eval(sdot_ctx *c, const EvalArgs &a, bool dense, const double *pdir, double tol, bool partial)
{
    cudaStream_t st = c->stream;
    const int prec = c->precision;
    auto mark = [&](int i) {
        if (c->profiling) cudaEventRecord(c->pev[i], st);
    };
    mark(0);
    if (dense) k_target_prep<DIM><<<grid_for(a.nt, 256), 256, 0, st>>>(a.nt, c->y.p, c->nu.p, c->psi.p, a, c->tpack.p);
    mark(1);
    int64_t nval = 0;
    int nks = 1;
    if (c->distance == 1) {
        // spherical distance: its own sweeps over every (point, target) pair
        mark(7);
        sdot_status s = run_spherical(c, a, c->current_distance_threshold, &nval);
        if (s != SDOT_OK) return s;
        mark(2);
        mark(3);
        c->klaunch[2] += 1;
        c->klaunch[3] += 1;
    } else if (dense) {
        const DenseShape ds = dense_shape(a.nq, a.nt, dense_tensor_m(c, a.s), c->ncells);
        nval = ds.nval;
        if (ds.tm > 0) {
            const cudaError_t e = c->vpart.alloc((size_t)2 * ds.nvs * a.nq);
            if (e != cudaSuccess) return cuda_error(c, e, "dense value slices");
            launch_value_dense_tensor<DIM>(c, ds, c->tpack.p, a, c->vpart.p, st);
            k_value_dense_merge<DIM><<<(unsigned)nval, MERGE_THREADS, 0, st>>>(c->x.p, c->rho.p, c->jxw.p, c->vpart.p,
                                                                               ds.nvs, a, c->Lq.p, c->blkpart.p);
        } else if (ds.nvs > 1) {
            const cudaError_t e = c->vpart.alloc((size_t)2 * ds.nvs * a.nq);
            if (e != cudaSuccess) return cuda_error(c, e, "dense value slices");
            k_value_dense_slice<DIM><<<dim3((unsigned)nval, (unsigned)ds.nvs), DENSE_A_THREADS, 0, st>>>(
                c->x.p, c->tpack.p, a, ds.tslice, c->vpart.p);
            k_value_dense_merge<DIM><<<(unsigned)nval, MERGE_THREADS, 0, st>>>(c->x.p, c->rho.p, c->jxw.p, c->vpart.p,
                                                                               ds.nvs, a, c->Lq.p, c->blkpart.p);
        } else {
            k_value_dense<DIM><<<(unsigned)nval, DENSE_A_THREADS, 0, st>>>(c->x.p, c->rho.p, c->jxw.p, c->tpack.p, a,
                                                                           c->Lq.p, c->blkpart.p);
        }
        mark(2);
        // gradient: target blocks x point (or cell) slices
        nks = ds.nks;
        launch_grad_dense<DIM>(c, ds, prec != SDOT_PREC_FP64, c->Lq.p, c->tpack.p, c->psi.p, a, c->gpart.p, st);
    } else {
        nval = c->nsblk;
        k_target_prep_kd<DIM><<<grid_for(a.nt, 256), 256, 0, st>>>(a.nt, c->y.p, c->nu.p, c->psi.p, a, c->tpack.p);
        sdot_status s = run_trunc(c, a, c->current_distance_threshold);  // records pev 7, 2, 3
        if (s != SDOT_OK) return s;
    }
    if (dense) mark(3);
    const int fb = launch_finalize_grad(a.nt, nks, c->gpart.p, c->nu.p, c->psi.p, pdir, tol, partial ? 0 : 1, c->grad.p,
                                        c->redpart.p, st);
    launch_finalize_scalars(st, fb, c->redpart.p, nval, c->blkpart.p, c->scal.p);
    mark(4);
    c->klaunch[1] += 1;
    if (dense && c->distance == 0) {
        c->klaunch[2] += 1;
        c->klaunch[3] += 1;
    }
    c->klaunch[4] += 2;
    return cuda_error(c, cudaGetLastError(), "evaluate launch");
}

// Launch key of the untruncated evaluation's graph: every value its launches
// capture (arguments, sizes, buffer addresses).  Zero-filled before use, so
// that keys compare bytewise.
struct DenseGraphKey {
    EvalArgs a;
    const void *p[20];
    double tol;
    int64_t misc[4];
};

// Replays the context's graph when the key matches it; captures one on the
// second consecutive evaluation with the same key (the first one runs
// eagerly, so every buffer the launches use is allocated before the
// capture); anything else runs eagerly.  A capture that fails turns graphs
// off for the context and runs the evaluation eagerly.
template <class Body>
static sdot_status run_graphed(sdot_ctx *c, const DenseGraphKey &k, Body &&body)
{
    const unsigned char *kb = reinterpret_cast<const unsigned char *>(&k);
    const bool same = c->dg_key.size() == sizeof k && memcmp(c->dg_key.data(), kb, sizeof k) == 0;
    if (same && c->dg_exec) {
        const cudaError_t e = cudaGraphLaunch(c->dg_exec, c->stream);
        if (e != cudaSuccess) return cuda_error(c, e, "evaluation graph launch");
        for (int i = 0; i < 8; ++i) c->klaunch[i] += c->dg_launches[i];
        return SDOT_OK;
    }
    if (c->dg_exec) {
        cudaGraphExecDestroy(c->dg_exec);
        c->dg_exec = nullptr;
    }
    if (!same || !c->dg_armed) {
        c->dg_key.assign(kb, kb + sizeof k);
        c->dg_armed = true;
        return body();
    }
    int64_t before[8];
    memcpy(before, c->klaunch, sizeof before);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
    sdot_status s = SDOT_OK;
    if (e == cudaSuccess) {
        s = body();
        e = cudaStreamEndCapture(c->stream, &g);
        if (s == SDOT_OK && e == cudaSuccess && g) e = cudaGraphInstantiate(&c->dg_exec, g, 0);
        if (g) cudaGraphDestroy(g);
    }
    if (s != SDOT_OK || e != cudaSuccess || !c->dg_exec) {
        cudaGetLastError();
        if (c->dg_exec) cudaGraphExecDestroy(c->dg_exec);
        c->dg_exec = nullptr;
        c->graphs_off = true;
        memcpy(c->klaunch, before, sizeof before);
        return body();
    }
    for (int i = 0; i < 8; ++i) c->dg_launches[i] = c->klaunch[i] - before[i];
    e = cudaGraphLaunch(c->dg_exec, c->stream);
    return e == cudaSuccess ? SDOT_OK : cuda_error(c, e, "evaluation graph launch");
}

sdot_status evaluate_internal(sdot_ctx *c, const double *p_dir, double comp_tol, double *ms_out, bool partial)
{
    EvalPending pend;
    sdot_status s = evaluate_enqueue(c, p_dir, comp_tol, partial, pend);
    if (s != SDOT_OK) return s;
    const cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_error(c, e, "evaluate");
    return evaluate_complete(c, pend, ms_out);
}

sdot_status evaluate_enqueue(sdot_ctx *c, const double *p_dir, double comp_tol, bool partial, EvalPending &pend)
{
    if (c->dim == 0 || c->nq == 0) return set_error(c, SDOT_ESTATE, "source measure not set");
    if (c->nt == 0) return set_error(c, SDOT_ESTATE, "target measure not set");
    const sdot_solver_params &p = c->prm;
    if (c->distance == 1 && p.threshold_type != SDOT_THRESH_POINTWISE)
        return set_error(c, SDOT_EINVAL, "the spherical distance is supported with the pointwise threshold");
    // threshold (host, exact libm), from device max/min of psi
    double r = DBL_MAX;
    const bool may_truncate = (p.threshold_type != SDOT_THRESH_POINTWISE) ||
                              (p.tau > 0 && (c->min_target_density > 0.0 ? c->min_target_density
                                                                          : c->nu_min) > 0);
    cudaEventRecord(c->ev0, c->stream);
    double mm[3] = {0, 0, 0};
    auto launch_minmax = [&] {
        if (c->profiling) cudaEventRecord(c->pev[5], c->stream);
        k_minmax<<<1, 1024, 0, c->stream>>>(c->psi.p, c->nt, c->scal.p + SC_MAXPSI);
        if (c->profiling) cudaEventRecord(c->pev[6], c->stream);
        c->klaunch[0] += 1;
    };
    if (may_truncate) {
        launch_minmax();
        cudaError_t e = cudaMemcpyAsync(mm, c->scal.p + SC_MAXPSI, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) return cuda_error(c, e, "threshold readback");
        if (mm[2] != 0.0) return set_error(c, SDOT_ENONFINITE, "non-finite potential");
        c->scal_host[SC_MAXPSI] = mm[0];
        c->scal_host[SC_MINPSI] = mm[1];
        r = host_threshold(c, mm[0], mm[1]);
    }
    c->current_distance_threshold = r;
    const double sstar = sstar_of(r);
    const bool dense = !(r < c->diam * (1.0 + 1e-12)) || std::isinf(r) ? true : false;
    const bool dense_ok = dense && !std::isnan(r);

    EvalArgs a{};
    a.qpc = c->qpc;
    a.ql = c->ql;
    a.ngroups = c->ngroups;
    a.lse = p.use_log_sum_exp;
    a.nq = c->nq;
    a.ncells = c->ncells;
    a.nunits = c->ncells * a.ngroups;
    a.nt = c->nt;
    a.eps = p.epsilon;
    a.s = KAPPA / p.epsilon;
    a.halfs = 0.5 * a.s;
    for (int d = 0; d < 3; ++d) a.o[d] = c->origin[d];
    a.sstar = sstar;
    a.cull = std::isnan(r) ? 0.0 : std::min(r, 1e300);
    a.c32 = LOG2E / (2.0 * p.epsilon);
    a.l2e_eps = LOG2E / p.epsilon;

    if (!dense_ok && std::isnan(r)) {
        // NaN threshold: the reference's predicate d <= NaN rejects everything
        a.sstar = NAN;
    }
    // everything after the threshold, up to the copy of the scalars to the host
    // (an untruncated evaluation needs no ψ range: k_minmax runs only for the threshold)
    auto body = [&]() -> sdot_status {
        const sdot_status s = (c->dim == 2) ? run_eval<2>(c, a, dense_ok, p_dir, comp_tol, partial)
                                            : run_eval<3>(c, a, dense_ok, p_dir, comp_tol, partial);
        if (s != SDOT_OK) return s;
        const cudaError_t e = cudaMemcpyAsync(c->scal_host, c->scal.p, SC_COUNT * sizeof(double),
                                              cudaMemcpyDeviceToHost, c->stream);
        return e == cudaSuccess ? SDOT_OK : cuda_error(c, e, "evaluate");
    };
    // An untruncated euclidean evaluation has no host step between its
    // launches, so it runs as one CUDA graph once its launch key repeats.
    sdot_status s;
    if (!may_truncate && dense_ok && c->distance == 0 && !c->profiling && !c->graphs_off) {
        DenseGraphKey k;
        memset(&k, 0, sizeof k);
        k.a = a;
        const void *ptrs[] = {c->psi.p, c->y.p, c->nu.p, c->x.p, c->rho.p, c->jxw.p, c->w.p, c->tpack.p,
                              c->vpart.p, c->Lq.p, c->blkpart.p, c->gpart.p, c->grad.p, c->redpart.p,
                              c->scal.p, c->scal_host, p_dir};
        static_assert(sizeof(ptrs) <= sizeof(k.p), "key pointer slots");
        memcpy(k.p, ptrs, sizeof(ptrs));
        k.tol = comp_tol;
        k.misc[0] = c->dim;
        k.misc[1] = c->precision;
        k.misc[2] = partial ? 1 : 0;
        k.misc[3] = (int64_t)c->vpart.n;
        s = run_graphed(c, k, body);
    } else {
        s = body();
    }
    if (s != SDOT_OK) return s;
    cudaEventRecord(c->ev1, c->stream);
    pend.r = r;
    pend.dense = dense_ok;
    pend.ranged = may_truncate;
    return SDOT_OK;
}

sdot_status evaluate_complete(sdot_ctx *c, const EvalPending &pend, double *ms_out)
{
    const double r = pend.r;
    const bool dense_ok = pend.dense;
    if (ms_out) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        *ms_out = ms;
    }
    if (c->profiling) {
        float t = 0.f;
        if (pend.ranged) {
            cudaEventElapsedTime(&t, c->pev[5], c->pev[6]);
            c->kms[0] += t;
        }
        cudaEventElapsedTime(&t, c->pev[0], c->pev[1]);
        c->kms[1] += t;
        if (dense_ok) {
            cudaEventElapsedTime(&t, c->pev[1], c->pev[2]);
            c->kms[2] += t;
        } else {
            cudaEventElapsedTime(&t, c->pev[1], c->pev[7]);
            c->kms[6] += t;
            cudaEventElapsedTime(&t, c->pev[7], c->pev[2]);
            c->kms[2] += t;
        }
        cudaEventElapsedTime(&t, c->pev[2], c->pev[3]);
        c->kms[3] += t;
        cudaEventElapsedTime(&t, c->pev[3], c->pev[4]);
        c->kms[4] += t;
    }
    c->scal_host[SC_R] = r;
    if (!pend.ranged) {
        // no ψ range was computed (untruncated): the slots say so
        c->scal_host[SC_MAXPSI] = NAN;
        c->scal_host[SC_MINPSI] = NAN;
        c->scal_host[SC_PSIBAD] = 0.0;
    }
    c->global_functional = c->scal_host[SC_VALUE];
    c->C_global = c->scal_host[SC_C];
    if (c->scal_host[SC_NONFINITE] != 0.0) return set_error(c, SDOT_ENONFINITE, "non-finite value or gradient");
    return SDOT_OK;
}

}  // namespace sdot

// ---------------------------------------------------------------------------
// No-allocation dense evaluation (sdot_evaluate_device_noalloc).
//
// The scratch of one untruncated evaluation (gathered psi, gradient, packed
// targets, L_q, gradient partials per q-slice, value / reduction partials,
// scalars) lives in one file-scope device array of NOALLOC_BYTES instead of
// the context's lazily allocated evaluation buffers.  Its device address is
// looked up once per device with cudaGetSymbolAddress and cached for the
// life of the process; a cudaDeviceReset by the host application frees the
// module instance the cached address points into, so no-alloc calls must not
// follow one.  Every scratch word the evaluation reads is written earlier by
// the same evaluation on the same stream: nothing has to start at zero, and
// only the scalar slots the evaluation writes are copied back to the context.
// The array is shared by every context of the process on a device, so calls
// whose executions overlap corrupt each other.
// ---------------------------------------------------------------------------

namespace sdot {

constexpr size_t NOALLOC_BYTES = size_t(8) << 20;  // == SDOT_NOALLOC_SCRATCH_BYTES
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_BYTES / sizeof(double)];

static double *g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};
static std::mutex g_noalloc_mu;

// Scratch segments of an evaluation, each rounded up to 256 bytes.
struct NoallocLayout {
    int64_t psi, grad, tpack, Lq, gpart, blkpart, redpart, scal, vpart, total;  // offsets in doubles
    int64_t nval;
    int nks;
    int nvs;
    int64_t tslice;
    DenseShape ds;
};

static NoallocLayout noalloc_layout(const sdot_ctx *c)
{
    const int64_t nq = c->nq, nt = c->nt;
    auto up = [](int64_t n) { return (n + 31) / 32 * 32; };
    NoallocLayout L{};
    // the launch shape of the allocating dense path
    const DenseShape ds = dense_shape(nq, nt, dense_tensor_m(c, KAPPA / c->prm.epsilon), c->ncells);
    L.ds = ds;
    L.nval = ds.nval;
    L.nks = ds.nks;
    L.nvs = ds.nvs;
    L.tslice = ds.tslice;
    int64_t o = 0;
    L.psi = o;     o += up(nt);
    L.grad = o;    o += up(nt);
    L.tpack = o;   o += up(nt * TPACK);
    L.Lq = o;      o += up(nq);
    L.gpart = o;   o += up((int64_t)L.nks * nt);
    L.blkpart = o; o += up(4 * L.nval);
    L.redpart = o; o += up((int64_t)FIN_BLOCKS * NRED);
    L.scal = o;    o += up(SC_COUNT);
    L.vpart = o;   o += (L.nvs > 1 || ds.tm > 0) ? up((int64_t)2 * L.nvs * nq) : 0;
    L.total = o;
    return L;
}

static sdot_status noalloc_scratch(sdot_ctx *c, double **out)
{
    if (c->device < 0 || c->device >= NOALLOC_MAX_DEVICES)
        return set_error(c, SDOT_EINVAL, "no-alloc evaluation: device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[c->device]) {
        double *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_error(c, e, "no-alloc evaluation: cudaGetSymbolAddress of the scratch array");
        g_noalloc_ptr[c->device] = p;
    }
    *out = g_noalloc_ptr[c->device];
    return SDOT_OK;
}

template <int DIM>
static void noalloc_launch(sdot_ctx *c, const EvalArgs &a, double *S, const NoallocLayout &L)
{
    cudaStream_t st = c->stream;
    double *psi = S + L.psi, *grad = S + L.grad, *tpack = S + L.tpack, *Lq = S + L.Lq, *gpart = S + L.gpart;
    double *blkpart = S + L.blkpart, *redpart = S + L.redpart, *scal = S + L.scal;
    k_target_prep<DIM><<<grid_for(a.nt, 256), 256, 0, st>>>(a.nt, c->y.p, c->nu.p, psi, a, tpack);
    if (L.ds.tm > 0) {
        double *vpart = S + L.vpart;
        launch_value_dense_tensor<DIM>(c, L.ds, tpack, a, vpart, st);
        k_value_dense_merge<DIM><<<(unsigned)L.nval, MERGE_THREADS, 0, st>>>(c->x.p, c->rho.p, c->jxw.p, vpart, L.nvs,
                                                                             a, Lq, blkpart);
    } else if (L.nvs > 1) {
        double *vpart = S + L.vpart;
        k_value_dense_slice<DIM><<<dim3((unsigned)L.nval, (unsigned)L.nvs), DENSE_A_THREADS, 0, st>>>(
            c->x.p, tpack, a, L.tslice, vpart);
        k_value_dense_merge<DIM><<<(unsigned)L.nval, MERGE_THREADS, 0, st>>>(c->x.p, c->rho.p, c->jxw.p, vpart, L.nvs,
                                                                             a, Lq, blkpart);
    } else {
        k_value_dense<DIM><<<(unsigned)L.nval, DENSE_A_THREADS, 0, st>>>(c->x.p, c->rho.p, c->jxw.p, tpack, a, Lq,
                                                                          blkpart);
    }
    launch_grad_dense<DIM>(c, L.ds, c->precision != SDOT_PREC_FP64, Lq, tpack, psi, a, gpart, st);
    const int fb = launch_finalize_grad(a.nt, L.nks, gpart, c->nu.p, psi, nullptr, c->prm.tolerance, 1, grad, redpart,
                                        st);
    launch_finalize_scalars(st, fb, redpart, L.nval, blkpart, scal);
}

}  // namespace sdot

extern "C" sdot_status sdot_evaluate_device_noalloc(sdot_ctx *c, const double *psi_dev, double *grad_dev,
                                                    double *value)
{
    using namespace sdot;
    if (!c || !psi_dev || !grad_dev) return SDOT_EINVAL;
    if (c->dim == 0 || c->nq == 0) return set_error(c, SDOT_ESTATE, "source measure not set");
    if (c->nt == 0) return set_error(c, SDOT_ESTATE, "target measure not set");
    const sdot_solver_params &p = c->prm;
    if (p.threshold_type != SDOT_THRESH_POINTWISE || p.tau > 0)
        return set_error(c, SDOT_EINVAL,
                         "no-alloc evaluation covers untruncated problems only (pointwise threshold, tau <= 0)");
    if (c->distance != 0) return set_error(c, SDOT_EINVAL, "no-alloc evaluation covers the euclidean distance only");
    const NoallocLayout L = noalloc_layout(c);
    const size_t need = (size_t)L.total * sizeof(double);
    if (need > NOALLOC_BYTES)
        return set_error(c, SDOT_EINVAL,
                         "no-alloc evaluation needs " + std::to_string(need) + " bytes of scratch; the static limit is " +
                             std::to_string(NOALLOC_BYTES) + " bytes (use sdot_evaluate_device)");
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != c->device) {
        const cudaError_t e = cudaSetDevice(c->device);
        if (e != cudaSuccess) return cuda_error(c, e, "no-alloc evaluation: set device");
    }
    struct Restore {
        int dev;
        ~Restore() {
            if (dev >= 0) cudaSetDevice(dev);
        }
    } restore{prev != c->device ? prev : -1};
    double *S = nullptr;
    sdot_status s = noalloc_scratch(c, &S);
    if (s != SDOT_OK) return s;

    EvalArgs a{};
    a.qpc = c->qpc;
    a.ql = c->ql;
    a.ngroups = c->ngroups;
    a.lse = p.use_log_sum_exp;
    a.nq = c->nq;
    a.ncells = c->ncells;
    a.nunits = c->ncells * a.ngroups;
    a.nt = c->nt;
    a.eps = p.epsilon;
    a.s = KAPPA / p.epsilon;
    a.halfs = 0.5 * a.s;
    for (int d = 0; d < 3; ++d) a.o[d] = c->origin[d];
    a.sstar = sstar_of(DBL_MAX);
    a.cull = 1e300;
    a.c32 = LOG2E / (2.0 * p.epsilon);
    a.l2e_eps = LOG2E / p.epsilon;

    if ((s = launch_gather(c, S + L.psi, psi_dev, c->nt)) != SDOT_OK) return s;
    if (c->dim == 2) noalloc_launch<2>(c, a, S, L);
    else noalloc_launch<3>(c, a, S, L);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(c, e, "no-alloc evaluation launch");
    if ((s = launch_scatter(c, grad_dev, S + L.grad, c->nt)) != SDOT_OK) return s;
    // k_finalize_scalars writes slots SC_VALUE .. SC_VALSRC except the psi range,
    // the psi check and the threshold slots (the untruncated path needs none of
    // them); those are set on the host below, so nothing an earlier call left in
    // the shared array reaches the context.
    e = cudaMemcpyAsync(c->scal_host, S + L.scal, (SC_VALSRC + 1) * sizeof(double), cudaMemcpyDeviceToHost,
                        c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_error(c, e, "no-alloc evaluation");
    c->scal_host[SC_MAXPSI] = NAN;
    c->scal_host[SC_MINPSI] = NAN;
    c->scal_host[SC_PSIBAD] = 0.0;
    c->scal_host[SC_SSTAR] = a.sstar;
    for (int i = SC_VALSRC + 1; i < SC_COUNT; ++i) c->scal_host[i] = 0.0;
    c->klaunch[1] += 1;
    c->klaunch[2] += 1;
    c->klaunch[3] += 1;
    c->klaunch[4] += 2;
    c->current_distance_threshold = DBL_MAX;
    c->scal_host[SC_R] = DBL_MAX;
    c->global_functional = c->scal_host[SC_VALUE];
    c->C_global = c->scal_host[SC_C];
    c->last_pairs = (int64_t)((double)c->nq * (double)c->nt);
    if (value) *value = c->scal_host[SC_VALUE];
    if (c->scal_host[SC_NONFINITE] != 0.0) return set_error(c, SDOT_ENONFINITE, "non-finite value or gradient");
    return SDOT_OK;
}

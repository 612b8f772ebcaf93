// sdot_dense.cuh -- per-CTA bodies of the untruncated (dense) value and
// gradient sweeps, shared by the single-problem kernels (sdot_eval.cu) and
// the batched persistent kernels (sdot_batch.cu).
#pragma once

#include <float.h>

#include "sdot_device.cuh"

namespace sdot {

// ---------------------------------------------------------------------------
// value sweep, dense: thread <-> DENSE_A_QT quadrature points, all targets
// streamed through shared memory (broadcast reads).
// ---------------------------------------------------------------------------

constexpr int DA_CHUNK = 256;

// One CTA's work of the dense value sweep: quadrature points
// [blk * DENSE_A_THREADS * QT, +DENSE_A_THREADS * QT) of one source against
// all its targets; writes L_q and the block's (value, C, skipped, 0) to out4.
// Shared by the single-problem kernel and the batched one.
template <int DIM>
__device__ __forceinline__ void dense_value_block(const double *__restrict__ x, const double *__restrict__ rho,
                                                  const double *__restrict__ jxw, const double *__restrict__ tpack,
                                                  const EvalArgs &a, int64_t blk, double *__restrict__ Lq,
                                                  double *__restrict__ out4)
{
    constexpr int QT = DENSE_A_QT;
    constexpr int TS = DIM + 2;  // A, B(DIM), nu
    __shared__ double tab[16];
    __shared__ double stg[DA_CHUNK * TS];
    if (threadIdx.x < 16) tab[threadIdx.x] = c_exp2_tab[threadIdx.x];

    const int64_t qbase = blk * (DENSE_A_THREADS * QT) + threadIdx.x;
    double xt[QT][DIM], M[QT], S[QT], mx[QT];
#pragma unroll
    for (int k = 0; k < QT; ++k) {
        const int64_t q = qbase + (int64_t)k * DENSE_A_THREADS;
#pragma unroll
        for (int d = 0; d < DIM; ++d) xt[k][d] = (q < a.nq) ? x[q * DIM + d] - a.o[d] : 0.0;
        M[k] = -CUDART_INF;
        S[k] = 0.0;
        mx[k] = -CUDART_INF;
    }
    for (int64_t c0 = 0; c0 < a.nt; c0 += DA_CHUNK) {
        const int cn = (int)min((int64_t)DA_CHUNK, a.nt - c0);
        __syncthreads();
        for (int i = threadIdx.x; i < cn * TS; i += DENSE_A_THREADS) {
            const int t = i / TS, f = i - t * TS;
            stg[i] = tpack[(c0 + t) * TPACK + f];
        }
        __syncthreads();
#pragma unroll 2
        for (int t = 0; t < cn; ++t) {
            const double *tp = stg + t * TS;
            const double A = tp[0];
            double B[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) B[d] = tp[1 + d];
            const double nuj = tp[1 + DIM];
#pragma unroll
            for (int k = 0; k < QT; ++k) {
                double b = fma(B[0], xt[k][0], A);
#pragma unroll
                for (int d = 1; d < DIM; ++d) b = fma(B[d], xt[k][d], b);
                lse_update(b, nuj, M[k], S[k], mx[k], tab);
            }
        }
    }
    double tv = 0.0, tc = 0.0, ts = 0.0;
#pragma unroll
    for (int k = 0; k < QT; ++k) {
        const int64_t q = qbase + (int64_t)k * DENSE_A_THREADS;
        if (q < a.nq) {
            double xsq = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) xsq += xt[k][d] * xt[k][d];
            const double Cq = -a.halfs * xsq;
            const double Sref = (mx[k] == -CUDART_INF) ? 0.0 : S[k] * exp2_16(M[k] - mx[k], tab);
            double v, cv, L;
            int sk;
            value_epilogue(a, mx[k], Sref, Cq, rho[q], jxw[q], v, cv, L, sk);
            Lq[q] = L;
            tv += v;
            tc += cv;
            ts += sk;
        }
    }
    block_partials_at(tv, tc, ts, 0.0, out4);
}

// The same sweep over one slice of the targets [t0, t1), for problems too
// small to fill the GPU with one CTA per point block: per point it writes
// the slice's largest scaled exponent mx and the sum relative to it,
// ms[2 q] = mx, ms[2 q + 1] = sum_j nu_j 2^((b_qj - mx)/16); the merge
// (dense_value_merge) combines the slices in slice order and finishes.
template <int DIM>
__device__ __forceinline__ void dense_value_slice(const double *__restrict__ x, const double *__restrict__ tpack,
                                                  const EvalArgs &a, int64_t blk, int64_t t0, int64_t t1,
                                                  double *__restrict__ ms)
{
    constexpr int TS = DIM + 2;  // A, B(DIM), nu
    __shared__ double tab[16];
    __shared__ double stg[DA_CHUNK * TS];
    if (threadIdx.x < 16) tab[threadIdx.x] = c_exp2_tab[threadIdx.x];
    const int64_t q = blk * DENSE_A_THREADS + threadIdx.x;
    double xt[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) xt[d] = (q < a.nq) ? x[q * DIM + d] - a.o[d] : 0.0;
    double M = -CUDART_INF, S = 0.0, mx = -CUDART_INF;
    for (int64_t c0 = t0; c0 < t1; c0 += DA_CHUNK) {
        const int cn = (int)min((int64_t)DA_CHUNK, t1 - c0);
        __syncthreads();
        for (int i = threadIdx.x; i < cn * TS; i += DENSE_A_THREADS) {
            const int t = i / TS, f = i - t * TS;
            stg[i] = tpack[(c0 + t) * TPACK + f];
        }
        __syncthreads();
#pragma unroll 2
        for (int t = 0; t < cn; ++t) {
            const double *tp = stg + t * TS;
            double b = fma(tp[1], xt[0], tp[0]);
#pragma unroll
            for (int d = 1; d < DIM; ++d) b = fma(tp[1 + d], xt[d], b);
            lse_update(b, tp[1 + DIM], M, S, mx, tab);
        }
    }
    if (q < a.nq) {
        ms[2 * q] = mx;
        ms[2 * q + 1] = (mx == -CUDART_INF) ? 0.0 : S * exp2_16(M - mx, tab);
    }
}

// Merge of the target slices of point block blk (slice s of point q at
// ms[s * 2 nq + 2 q ..]) by DENSE_MERGE_SPLIT lanes per point: lane u takes
// the slices s = u, u + SPLIT, ... (their loads in flight together); the
// largest exponent over the slices, each lane's sums rescaled to it and
// added in order of s, the lanes' sums added by xor exchanges in a fixed
// tree; then the epilogue of dense_value_block (L_q, value, C, skipped) and
// the block's partials.  The CTA has DENSE_A_THREADS * SPLIT threads.
constexpr int DENSE_MERGE_SPLIT = 4;

template <int DIM>
__device__ __forceinline__ void dense_value_merge(const double *__restrict__ x, const double *__restrict__ rho,
                                                  const double *__restrict__ jxw, const double *__restrict__ ms,
                                                  int nslice, const EvalArgs &a, int64_t blk,
                                                  double *__restrict__ Lq, double *__restrict__ out4)
{
    constexpr int SP = DENSE_MERGE_SPLIT;
    __shared__ double tab[16];
    if (threadIdx.x < 16) tab[threadIdx.x] = c_exp2_tab[threadIdx.x];
    __syncthreads();
    const int u = threadIdx.x % SP;
    const int64_t q = blk * DENSE_A_THREADS + threadIdx.x / SP;
    const bool ok = q < a.nq;
    const double *mq = ms + 2 * (ok ? q : 0);
    const int64_t st = 2 * a.nq;
    double mx = -CUDART_INF;
    if (ok)
        for (int s = u; s < nslice; s += SP) mx = fmax(mx, mq[s * st]);
#pragma unroll
    for (int o = 1; o < SP; o <<= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    double S = 0.0;
    if (ok && mx > -CUDART_INF)
        for (int s = u; s < nslice; s += SP) {
            const double2 v = *reinterpret_cast<const double2 *>(mq + s * st);
            if (v.x > -CUDART_INF) S += v.y * exp2_16(v.x - mx, tab);
        }
#pragma unroll
    for (int o = 1; o < SP; o <<= 1) S += __shfl_xor_sync(0xffffffffu, S, o);
    double tv = 0.0, tc = 0.0, ts = 0.0;
    if (ok && u == 0) {
        double xsq = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const double xt = x[q * DIM + d] - a.o[d];
            xsq += xt * xt;
        }
        const double Cq = -a.halfs * xsq;
        double v, cv, L;
        int sk;
        value_epilogue(a, mx, S, Cq, rho[q], jxw[q], v, cv, L, sk);
        Lq[q] = L;
        tv = v;
        tc = cv;
        ts = sk;
    }
    block_partials_at(tv, tc, ts, 0.0, out4);
}

// ---------------------------------------------------------------------------
// gradient sweep, dense: thread <-> DENSE_B_TT targets, q-slices streamed
// through shared memory (broadcast reads); FP64 partial per (slice, target).
// ---------------------------------------------------------------------------

constexpr int DB_CHUNK = 256;

// Per-target data of one CTA of the gradient sweep: the TT targets j0 + lt +
// k * DENSE_B_THREADS of thread lane lt.  FP32: the CTA's target box centre
// ob and the reference aref = max_j (log2 nu_j + psi_j log2(e) / eps) (block
// reductions over the CTA's NTH threads), each target relative to ob (yt) and
// its exponent offset alpha = log2 nu_j + psi_j log2(e) / eps - aref; FP64:
// A_j and B_j of the packed target.
template <int TT>
struct GradTargets {
    double ob[3] = {0.0, 0.0, 0.0};
    double aref = 0.0;
    float yt[TT][3], alpha[TT];
    double A[TT], B[TT][3];
    bool has[TT];
};

template <int DIM, bool FP32, int NTH, int TT>
__device__ __forceinline__ void grad_targets(const double *__restrict__ tpack, const double *__restrict__ psi,
                                             const EvalArgs &a, int64_t j0, int lt, GradTargets<TT> &T)
{
    const int tid = threadIdx.x;
    if (FP32) {
        double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
        double amax = -DBL_MAX;
#pragma unroll
        for (int k = 0; k < TT; ++k) {
            const int64_t j = j0 + lt + k * DENSE_B_THREADS;
            if (j < a.nt) {
                const double *tp = tpack + j * TPACK;
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    lo[d] = fmin(lo[d], tp[2 + DIM + d]);
                    hi[d] = fmax(hi[d], tp[2 + DIM + d]);
                }
                const double al = log2(tp[1 + DIM]) + a.l2e_eps * psi[j];
                if (al > amax) amax = al;
            }
        }
        // block reductions (lo/hi/amax) through shared memory
        __shared__ double sred[7][NTH / 32];
        for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
                hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
            }
            amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
        }
        if ((tid & 31) == 0) {
#pragma unroll
            for (int d = 0; d < DIM; ++d) { sred[d][tid >> 5] = lo[d]; sred[3 + d][tid >> 5] = hi[d]; }
            sred[6][tid >> 5] = amax;
        }
        __syncthreads();
        for (int i = 0; i < NTH / 32; ++i) {
#pragma unroll
            for (int d = 0; d < DIM; ++d) { lo[d] = fmin(lo[d], sred[d][i]); hi[d] = fmax(hi[d], sred[3 + d][i]); }
            amax = fmax(amax, sred[6][i]);
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) T.ob[d] = 0.5 * (lo[d] + hi[d]);
        T.aref = (amax > -DBL_MAX && isfinite(amax)) ? amax : 0.0;
    }
#pragma unroll
    for (int k = 0; k < TT; ++k) {
        const int64_t j = j0 + lt + k * DENSE_B_THREADS;
        T.has[k] = j < a.nt;
        const double *tp = tpack + (T.has[k] ? j : 0) * TPACK;
        if (FP32) {
#pragma unroll
            for (int d = 0; d < 3; ++d) T.yt[k][d] = (d < DIM && T.has[k]) ? (float)(tp[2 + DIM + d] - T.ob[d]) : 0.f;
            T.alpha[k] = T.has[k] ? (float)(log2(tp[1 + DIM]) + a.l2e_eps * psi[j] - T.aref) : -INFINITY;
        } else {
            T.A[k] = tp[0];
#pragma unroll
            for (int d = 0; d < DIM; ++d) T.B[k][d] = tp[1 + d];
        }
    }
}

// One CTA's work of the dense gradient sweep: targets of block tblk against
// quadrature slice ks; writes gpart[ks * nt + j].  Shared by the
// single-problem kernel (QG = DENSE_B_QG) and the batched one (QG = 1).
// The CTA is QG groups of DENSE_B_THREADS threads: thread lt of every group
// holds the same TT targets, group g takes the staged points g, g + QG, ...,
// and the groups' sums are added in group order at the end, so a slice's
// partial does not depend on the scheduling.
template <int DIM, bool FP32, int QG = 1>
__device__ __forceinline__ void dense_grad_block(const double *__restrict__ x, const double *__restrict__ w,
                                                 const double *__restrict__ Lq, const double *__restrict__ tpack,
                                                 const double *__restrict__ psi, const EvalArgs &a, int64_t qslice,
                                                 int64_t tblk, int64_t ks, double *__restrict__ gpart)
{
    constexpr int TT = DENSE_B_TT;
    constexpr int TB = DENSE_B_THREADS * TT;
    constexpr int NTH = DENSE_B_THREADS * QG;          // threads of the CTA
    constexpr int CH = DB_CHUNK * (QG > 1 ? 2 : 1);    // points staged at a time
    __shared__ double tab[16];
    __shared__ __align__(16) double stgd[FP32 ? 1 : CH * (DIM + 2)];
    __shared__ __align__(16) float stgf[FP32 ? CH * 4 : 1];
    __shared__ float stgw[FP32 ? CH : 1];
    __shared__ double gsum[QG > 1 ? (QG - 1) * TT * DENSE_B_THREADS : 1];
    if (threadIdx.x < 16) tab[threadIdx.x] = c_exp2_tab[threadIdx.x];
    const int tid = threadIdx.x;
    const int lt = tid % DENSE_B_THREADS;  // target lane
    const int grp = tid / DENSE_B_THREADS; // point group
    const int64_t j0 = tblk * TB;
    const int64_t qa = ks * qslice;
    const int64_t qb = min(a.nq, qa + qslice);

    GradTargets<TT> T;
    grad_targets<DIM, FP32, NTH>(tpack, psi, a, j0, lt, T);
    const double *ob = T.ob;
    const double aref = T.aref;
    const auto &yt = T.yt;
    const auto &alpha = T.alpha;
    const auto &A = T.A;
    const auto &B = T.B;
    double acc64[TT];
#pragma unroll
    for (int k = 0; k < TT; ++k) acc64[k] = 0.0;
    const float c32 = (float)a.c32;
    for (int64_t c0 = qa; c0 < qb; c0 += CH) {
        const int cn = (int)min((int64_t)CH, qb - c0);
        __syncthreads();
        for (int i = tid; i < cn; i += NTH) {
            const int64_t q = c0 + i;
            double xt[3];
            double xsq = 0.0;
            if (FP32) {
#pragma unroll
                for (int d = 0; d < DIM; ++d) xt[d] = x[q * DIM + d] - ob[d];
                const double beta = -LOG2E * Lq[q] + aref;
                float4 v;
                v.x = (float)xt[0];
                v.y = (float)xt[1];
                v.z = DIM == 3 ? (float)xt[2] : (float)beta;
                v.w = DIM == 3 ? (float)beta : 0.f;
                reinterpret_cast<float4 *>(stgf)[i] = v;
                stgw[i] = (float)w[q];
            } else {
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    xt[d] = x[q * DIM + d] - a.o[d];
                    xsq += xt[d] * xt[d];
                    stgd[i * (DIM + 2) + d] = xt[d];
                }
                stgd[i * (DIM + 2) + DIM] = -a.halfs * xsq - KAPPA * Lq[q];
                stgd[i * (DIM + 2) + DIM + 1] = w[q];
            }
        }
        __syncthreads();
        if (FP32) {
            float acc[TT];
#pragma unroll
            for (int k = 0; k < TT; ++k) acc[k] = 0.f;
            int i = 0;
            for (int t = grp; t < cn; t += QG, ++i) {
                const float4 v = reinterpret_cast<const float4 *>(stgf)[t];
                const float beta = DIM == 3 ? v.w : v.z;
                const float wq = stgw[t];
#pragma unroll
                for (int k = 0; k < TT; ++k) {
                    const float d0 = v.x - yt[k][0], d1 = v.y - yt[k][1];
                    float d2 = d0 * d0;
                    d2 = fmaf(d1, d1, d2);
                    if (DIM == 3) {
                        const float dz = v.z - yt[k][2];
                        d2 = fmaf(dz, dz, d2);
                    }
                    const float e = fmaf(-c32, d2, alpha[k] + beta);
                    acc[k] = fmaf(wq, ex2_approx(e), acc[k]);
                }
                if ((i & 7) == 7) {
#pragma unroll
                    for (int k = 0; k < TT; ++k) { acc64[k] += (double)acc[k]; acc[k] = 0.f; }
                }
            }
#pragma unroll
            for (int k = 0; k < TT; ++k) acc64[k] += (double)acc[k];
        } else {
            for (int t = grp; t < cn; t += QG) {
                const double *v = stgd + t * (DIM + 2);
                const double D = v[DIM], wq = v[DIM + 1];
#pragma unroll
                for (int k = 0; k < TT; ++k) {
                    double u = fma(B[k][0], v[0], A[k] + D);
#pragma unroll
                    for (int d = 1; d < DIM; ++d) u = fma(B[k][d], v[d], u);
                    acc64[k] = fma(wq, exp2_16(u, tab), acc64[k]);
                }
            }
        }
    }
    if (QG > 1) {
        // the groups' sums, added in group order by group 0
        if (grp > 0) {
#pragma unroll
            for (int k = 0; k < TT; ++k) gsum[((grp - 1) * TT + k) * DENSE_B_THREADS + lt] = acc64[k];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < TT; ++k)
            for (int g = 1; g < QG; ++g) acc64[k] += gsum[((g - 1) * TT + k) * DENSE_B_THREADS + lt];
    }
#pragma unroll
    for (int k = 0; k < TT; ++k) {
        const int64_t j = j0 + lt + k * DENSE_B_THREADS;
        if (grp == 0 && j < a.nt) {
            double g = acc64[k];
            if (!FP32) g *= tpack[j * TPACK + 1 + DIM];  // nu_j (FP32 path folds it into alpha)
            gpart[ks * a.nt + j] = g;
        }
    }
}

}  // namespace sdot

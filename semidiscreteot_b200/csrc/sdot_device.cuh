// sdot_device.cuh -- device helpers shared by the evaluation, solver and
// Hessian kernels of libsdot_cuda (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "sdot_internal.h"

namespace sdot {

// 2^(k/16), k = 0..15, correctly rounded.  Kept in shared memory by every
// kernel that calls exp2_16: 16 doubles occupy all 32 banks, so any per-lane
// index pattern is conflict-free.
__device__ __constant__ double c_exp2_tab[16] = {
    0x1.0000000000000p+0, 0x1.0b5586cf9890fp+0, 0x1.172b83c7d517bp+0, 0x1.2387a6e756238p+0,
    0x1.306fe0a31b715p+0, 0x1.3dea64c123422p+0, 0x1.4bfdad5362a27p+0, 0x1.5ab07dd485429p+0,
    0x1.6a09e667f3bcdp+0, 0x1.7a11473eb0187p+0, 0x1.8ace5422aa0dbp+0, 0x1.9c49182a3f090p+0,
    0x1.ae89f995ad3adp+0, 0x1.c199bdd85529cp+0, 0x1.d5818dcfba487p+0, 0x1.ea4afa2a490dap+0};

// Lazy-rescale threshold of the online log-sum-exp, in units of 2^(1/16):
// the running shift M is only moved when a term would exceed 2^512, so the
// FP64 sum stays far from overflow and the rescale branch is rare.
constexpr double LSE_THR = 16.0 * 512.0;
constexpr double EXP2_CLAMP = -16.0 * 1000.0;

// FP64 2^(u/16) for u <= 16*1022, relative error <= 1.5e-13.
// Method: u = 16 e + k + f with n = rint(u) (k = n mod 16, e = n div 16,
// |f| <= 1/2); 2^(u/16) = 2^e * 2^(k/16) * exp(f ln2/16).  The last factor is
// the degree-5 Taylor polynomial of exp on |f ln2/16| <= 0.0217 (remainder
// < 1.5e-13); 2^(k/16) comes from a 16-entry table and 2^e is added to the
// exponent field.  Arguments below -16000 are clamped (result ~2^-1000, far
// below any sum it is added to).
__device__ __forceinline__ double exp2_16(double u, const double *tab)
{
    u = fmax(u, EXP2_CLAMP);
    const double magic = 6755399441055744.0;  // 1.5 * 2^52
    const double v = __dadd_rn(u, magic);
    const int n = __double2loint(v);
    const double f = __dsub_rn(u, __dsub_rn(v, magic));
    double p = fma(f, 0x1.5d87fe78a6731p-30, 0x1.3b2ab6fba4e77p-23);
    p = fma(f, p, 0x1.c6b08d704a0c0p-17);
    p = fma(f, p, 0x1.ebfbdff82c58fp-11);
    p = fma(f, p, 0x1.62e42fefa39efp-5);
    p = fma(f, p, 1.0);
    const double r = tab[n & 15] * p;
    const int hi = __double2hiint(r) + ((n >> 4) << 20);
    return __hiloint2double(hi, __double2loint(r));
}

// exp2_16 without the lower clamp, for arguments proven >= -16000 by the caller.
__device__ __forceinline__ double exp2_16_nc(double u, const double *tab)
{
    const double magic = 6755399441055744.0;  // 1.5 * 2^52
    const double v = __dadd_rn(u, magic);
    const int n = __double2loint(v);
    const double f = __dsub_rn(u, __dsub_rn(v, magic));
    double p = fma(f, 0x1.5d87fe78a6731p-30, 0x1.3b2ab6fba4e77p-23);
    p = fma(f, p, 0x1.c6b08d704a0c0p-17);
    p = fma(f, p, 0x1.ebfbdff82c58fp-11);
    p = fma(f, p, 0x1.62e42fefa39efp-5);
    p = fma(f, p, 1.0);
    const double r = tab[n & 15] * p;
    const int hi = __double2hiint(r) + ((n >> 4) << 20);
    return __hiloint2double(hi, __double2loint(r));
}

// Squared distance rounded exactly like the reference's
// (a-b).norm_square(): ((d0*d0) + d1*d1) + d2*d2, no contraction.
template <int DIM>
__device__ __forceinline__ double dist2_exact(const double *a, const double *b)
{
    double t = __dsub_rn(a[0], b[0]);
    double s = __dmul_rn(t, t);
    t = __dsub_rn(a[1], b[1]);
    s = __dadd_rn(s, __dmul_rn(t, t));
    if (DIM == 3) {
        t = __dsub_rn(a[2], b[2]);
        s = __dadd_rn(s, __dmul_rn(t, t));
    }
    return s;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// xor-butterfly sum: every lane ends with the same, order-fixed result.
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ int warp_sum_int(int v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float ex2_approx(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Exact floor(p / d) for p < 2^16, d <= 64 with m = ceil(2^32 / d).
__device__ __forceinline__ unsigned fast_div(unsigned p, unsigned m)
{
    return __umulhi(p, m);
}

struct EvalArgs {
    int qpc;          // quadrature points per cell
    int ql;           // quadrature points per warp unit (value sweep, trunc)
    int ngroups;      // units per cell
    int lse;          // use_log_sum_exp_trick
    int64_t nq, ncells, nunits, nt;
    double eps;
    double s;         // KAPPA / eps
    double halfs;     // s / 2
    double o[3];      // origin
    double sstar;     // candidate test d2 <= sstar
    double cull;      // block cull radius r (slightly enlarged)
    double c32;       // log2(e) / (2 eps) (FP32 gradient sweep)
    double l2e_eps;   // log2(e) / eps
};

// ---------------------------------------------------------------------------
// per-q epilogue of the value sweep (SotSolver.cc:843-866 + lambda :274-286)
// ---------------------------------------------------------------------------

// mx: max scaled exponent (without C_q); S: sum relative to mx.
__device__ __forceinline__ void value_epilogue(const EvalArgs &a, double mx, double S, double Cq,
                                               double rho, double jxw, double &val, double &cval,
                                               double &L, int &skipped)
{
    val = 0.0;
    cval = 0.0;
    L = CUDART_INF;
    skipped = 1;
    if (mx == -CUDART_INF) return;           // no candidates: cell skipped (:802)
    const double m_ref = (mx + Cq) * (1.0 / KAPPA);
    if (a.lse) {
        if (!(S > 0.0)) return;              // total_sum_exp <= 0 (:846)
        const double lt = m_ref + log(S);
        val = rho * a.eps * lt * jxw;
        cval = rho * jxw / S;
        L = lt;
    } else {
        const double total = S * exp(m_ref);  // sum of unshifted terms
        if (!(total > 0.0)) return;
        const double lt = log(total);
        val = rho * a.eps * lt * jxw;
        cval = rho * jxw / total;
        L = lt;
    }
    skipped = 0;
}

// One online-LSE update in scaled units (b relative to the unit's C_q).
__device__ __forceinline__ void lse_update(double b, double nu, double &M, double &S, double &mx,
                                           const double *tab)
{
    mx = fmax(mx, b);
    double u = b - M;
    if (u > LSE_THR) {
        S = S * exp2_16(M - b, tab);
        M = b;
        u = 0.0;
    }
    S = fma(nu, exp2_16(u, tab), S);
}

// Block-level ordered sum of (value, C, skipped, pairs) -> out4[0..3].
__device__ __forceinline__ void block_partials_at(double v, double c, double sk, double np, double *out4)
{
    __shared__ double sv[32], sc[32], ss[32], sp[32];
    v = warp_sum(v);
    c = warp_sum(c);
    sk = warp_sum(sk);
    np = warp_sum(np);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sv[w] = v; sc[w] = c; ss[w] = sk; sp[w] = np; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tv = 0.0, tc = 0.0, ts = 0.0, tp = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) { tv += sv[i]; tc += sc[i]; ts += ss[i]; tp += sp[i]; }
        out4[0] = tv;
        out4[1] = tc;
        out4[2] = ts;
        out4[3] = tp;
    }
}

// Block-level ordered sum of (value, C, skipped, pairs) -> part[blockIdx.x*4..].
__device__ __forceinline__ void block_partials(double v, double c, double sk, double np, double *part)
{
    block_partials_at(v, c, sk, np, part + (int64_t)blockIdx.x * 4);
}

}  // namespace sdot

// sdot_trunc.cu -- truncated evaluation (tau > 0): exact cell-centre candidate
// sets, one fused source-block kernel for both exponential sweeps, and an
// atomic-free reduction of the per-block gradient partials.
//
// Replaces find_nearest_target_points + local_assemble + the WorkStream
// copier (src/solvers/SotSolver.cc:553-570, 769-869, 307-311).
//
// Blocks.  Source cells and targets are ordered by k-d trees built at
// set_source / set_target; a source block is a leaf of <= 8 warp units
// (cell, q-group), a target block a leaf of <= 32 targets.  Each block has a
// bounding sphere (FP64 and a conservative FP32 copy).
//
// Per evaluation:
//   1. block-pair lists.  (b, t) is a pair iff dist(c_b, c_t) <= r + R_b + R_t
//      (FP32, conservatively enlarged).  The forward list (per b, t ascending)
//      and the inverse list (per t, b ascending) are built by count / scan /
//      fill kernels that evaluate the identical expression, so they hold the
//      same pairs.
//   2. k_fused (CTA <-> source block, warp <-> unit):
//      staging: the targets of the block's pairs, culled per target against
//        the block sphere (|y - c_b| <= r + R_b), compacted in order;
//      exact test: warp of cell K keeps j iff d2(y_j, c_K) <= s*, rounded like
//        the reference (this is the candidate set, bit-exact);
//      value sweep: lane <-> candidate, all q of the unit in registers, FP64
//        online log-sum-exp of b_qj = B0_Kj + G_Kj.delta_q + C'_q, where
//        B0_Kj = kappa (psi_j - d2/2)/eps, G_Kj = kappa (y_j - c_K)/eps,
//        delta_q = x_q - c_K, C'_q = -kappa |delta_q|^2 / (2 eps)
//        (kappa = 16/ln 2; the same expansion as |x_q - y_j|^2 about c_K);
//      gradient sweep: each warp over the same compacted candidates, lane <->
//        candidate, sum over the unit's q of
//        w_q nu_j 2^(E0_Kj + G'_Kj.delta_q + D_q) in FP32 ex2 (or FP64 exp2),
//        E0 and G' formed in FP64 per (cell, target) so every FP32 operand is
//        small, into the warp's partial row (FP32 rows in the hybrid mode,
//        FP64 rows in the FP64 mode); the rows are added in warp order in
//        FP64.  The block's partial for each target of each pair is written
//        to a slot of the pair in the inverse list order.
//   3. k_grad_reduce (warp <-> target block): sum of the partials over the
//      pairs in ascending source-block order, lane <-> target.  No atomics;
//      the summation order is fixed, results are bitwise reproducible.
#include <float.h>
#include <math.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "sdot_device.cuh"
#include "sdot_internal.h"

namespace sdot {

constexpr int FT_WARPS = 8;
constexpr int FT_MAXS = 1024;               // staged targets per chunk
// The 3D tensor-factored hybrid sweeps stage at most 624 targets per chunk so that
// their shared memory (75,312 B) lets 3 CTAs share an SM (24 warps instead of
// 16; registers capped at 80): measured 3.99 ms per trunc_3d evaluation against
// 4.19 ms with 1,024 targets and 2 CTAs, although more blocks need several chunks.
constexpr int FT_MAXS_TENSOR = 624;
__host__ __device__ constexpr bool fused_small(int dim, int tq, bool fp32b) { return dim == 3 && tq > 0 && fp32b; }
__host__ __device__ constexpr int fused_cap(int dim, int tq, bool fp32b) { return fused_small(dim, tq, fp32b) ? FT_MAXS_TENSOR : FT_MAXS; }
__host__ __device__ constexpr int fused_min_blocks(int dim, int tq, bool fp32b) { return fused_small(dim, tq, fp32b) ? 3 : 2; }
constexpr int FT_TS = 6;                    // doubles per staged target: y(3), nu, log2 nu, s*psi
constexpr int FT_MAXT = 96;                 // target blocks per chunk
constexpr int FT_MAXQ = 80;                 // quadrature points of one source block
constexpr int SUPER = 32;                   // blocks per super-block of the pair-list hierarchy
constexpr int FT_PREF = 192;                // forward entries of a block prefetched into smem

struct FusedArgs {
    const double *x, *rho, *jxw, *w, *cell_ctr;
    const double *tpk;           // per target: y(3), nu, log2 nu, s*psi, -, -
    const int64_t *sblk_cell;    // source block -> first cell (nsblk + 1)
    const double *sblk_sph;      // FP64 centre(3), radius
    const int64_t *tblk_off;     // target block -> first target (ntblk + 1)
    const int64_t *fwd_off;
    const int *fwd_t;
    const int64_t *fwd2inv;      // inverse position of each forward pair
    double *part;                // partials, 32 per pair, at inverse positions minus part_base (FP64 sweeps)
    float *part32;               // the same in FP32 (hybrid sweeps: their rows are FP32 already)
    double *Lq;                  // per q (written by the value sweep)
    double *valpart;             // per source block: value, C, skipped, pairs
    int do_a, do_b;
    int w_nonneg;                // all w_q >= 0: log2 w_q folded into the FP32 exponent
    int tlo, thi;                // gradient partials only for target blocks [tlo, thi)
    int64_t part_base;           // inverse position of the first pair of tlo
    double cullt;                // per-target cull radius addend (r, enlarged)
};

template <int CAP>
struct FTSmem {
    static constexpr int MAXS = CAP;
    double tab[16];
    double stg[FT_TS][CAP];    // staged targets, structure of arrays (conflict-free lane access)
    double qd[FT_MAXQ][4];        // delta_q (FP64) and C'_q
    double qn[FT_MAXQ];           // |delta_q|
    double qL[FT_MAXQ];           // L_q of the block
    __align__(16) float qb[FT_MAXQ][4];  // pass B: delta (3) as float, D_q (+ log2 w_q)
    float qw[FT_MAXQ];            // pass B: w_q
    float qtw[FT_MAXQ];           // pass B, tensor path: w_q 2^(D_q)
    double cellc[FT_WARPS][3];    // centre of each cell of the block
    float pvw[FT_WARPS][CAP];     // gradient partial of each unit (warp) per staged target (FP32 mode)
    unsigned short cand[FT_WARPS][CAP];
    short smap[FT_MAXT][TBLK_KD]; // (chunk target block, slot) -> staged position or -1
    int ctb[FT_MAXT];             // target blocks of the chunk
    int64_t cpos[FT_MAXT];        // their partial base index
    int ecnt[32];                 // survivors per examined forward entry (-1: none)
    int epre[32];                 // staged position of the first survivor of each accepted entry
    int eacc, etot;
    int wcount[FT_WARPS];
    int nstg;
    int ent_t[FT_PREF];            // forward entries of the block: target block,
    int ent_j0[FT_PREF];           // its first target
    unsigned char ent_sz[FT_PREF]; // and its size (prefetched once per block)
};

// Partial rows of the gradient sweep: FP32 in the hybrid mode (inside
// FTSmem), FP64 in the FP64 mode (appended after FTSmem in dynamic shared
// memory, so that the FP64 gradient keeps its precision through the sum of
// the warps' rows).
template <bool FP32B> struct PRow { using T = double; };
template <> struct PRow<true> { using T = float; };
__host__ __device__ constexpr size_t ft_rows64_bytes(int cap) { return sizeof(double) * FT_WARPS * cap; }

template <bool FP32B, class SM>
__device__ __forceinline__ typename PRow<FP32B>::T *partial_rows(SM &sm)
{
    if constexpr (FP32B) return &sm.pvw[0][0];
    else return reinterpret_cast<double *>(reinterpret_cast<unsigned char *>(&sm) + sizeof(SM));
}

// ---------------------------------------------------------------------------
// block-pair lists
// ---------------------------------------------------------------------------

// Rounded operation by operation (no contraction): the forward and inverse
// list kernels must reach bitwise identical decisions.
__device__ __forceinline__ bool pair_test(float4 s, float4 t, float cr)
{
    const float dx = __fsub_rn(s.x, t.x), dy = __fsub_rn(s.y, t.y), dz = __fsub_rn(s.z, t.z);
    const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    const float lim = __fadd_rn(__fadd_rn(cr, s.w), t.w);
    return d2 <= __fmul_rn(lim, lim);
}

// Super-block pairs: sp[si * nts + ti] = 1 iff source super-block si and
// target super-block ti may hold a pair (the same conservative test; a
// super-sphere contains its member spheres, so no block pair is lost).
__global__ void __launch_bounds__(256)
k_super_pairs(const float4 *__restrict__ ssph, int nss, const float4 *__restrict__ tsph, int nts, float cr,
              unsigned char *__restrict__ sp)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)nss * nts) return;
    const int si = (int)(i / nts), ti = (int)(i - (int64_t)si * nts);
    sp[i] = pair_test(ssph[si], tsph[ti], cr) ? 1 : 0;
}

// Warp <-> source super-block: its paired target super-blocks in ascending
// order (shit[si * nts + h]), their count, and the inverse map
// spidx[si * nts + ti] = h (or -1).
__global__ void __launch_bounds__(256)
k_super_compact(const unsigned char *__restrict__ sp, int nss, int nts, int *__restrict__ shit,
                int *__restrict__ scount, int *__restrict__ spidx)
{
    const int si = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (si >= nss) return;
    int h = 0;
    for (int t0 = 0; t0 < nts; t0 += 32) {
        const int ti = t0 + lane;
        const bool on = ti < nts && sp[(int64_t)si * nts + ti];
        const unsigned bal = __ballot_sync(0xffffffffu, on);
        const int pos = h + __popc(bal & ((1u << lane) - 1u));
        if (ti < nts) spidx[(int64_t)si * nts + ti] = on ? pos : -1;
        if (on) shit[(int64_t)si * nts + pos] = ti;
        h += __popc(bal);
    }
    if (lane == 0) scount[si] = h;
}

// Warp <-> source block b: for each paired target super-block h, the 32-bit
// mask of its target blocks t with pair_test(b, t), and the number of b's
// pairs before it; cnt[b] = total.  Pairs are ordered by t, so the forward
// position of (b, t) is fwd_off[b] + mpre[b, h] + popc(mask[b, h] below t).
__global__ void __launch_bounds__(256)
k_fwd_masks(const float4 *__restrict__ sph, int nsb, const float4 *__restrict__ tph, int ntb, int nts, int hmax,
            float cr, const int *__restrict__ shit, const int *__restrict__ scount, unsigned *__restrict__ mask,
            int *__restrict__ mpre, int64_t *__restrict__ cnt)
{
    const int b = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= nsb) return;
    const float4 me = sph[b];
    const int si = b / SUPER;
    const int nh = scount[si];
    int k = 0;
    for (int h = 0; h < nh; ++h) {
        const int t = shit[(int64_t)si * nts + h] * SUPER + lane;
        const bool hit = t < ntb && pair_test(me, tph[t], cr);
        const unsigned bal = __ballot_sync(0xffffffffu, hit);
        if (lane == 0) {
            mask[(int64_t)b * hmax + h] = bal;
            mpre[(int64_t)b * hmax + h] = k;
        }
        k += __popc(bal);
    }
    if (lane == 0) cnt[b] = k;
}

// Forward lists from the masks: fwd_t[fwd_off[b] ..] = paired t, ascending.
__global__ void __launch_bounds__(256)
k_fwd_fill(int nsb, int nts, int hmax, const int *__restrict__ shit, const int *__restrict__ scount,
           const unsigned *__restrict__ mask, const int64_t *__restrict__ fwd_off, int *__restrict__ fwd_t)
{
    const int b = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= nsb) return;
    const int si = b / SUPER;
    const int nh = scount[si];
    int64_t k = fwd_off[b];
    for (int h = 0; h < nh; ++h) {
        const unsigned bal = mask[(int64_t)b * hmax + h];
        if ((bal >> lane) & 1u) fwd_t[k + __popc(bal & ((1u << lane) - 1u))] = shit[(int64_t)si * nts + h] * SUPER + lane;
        k += __popc(bal);
    }
}

// Inverse lists by transposing the forward lists (the same pair set by
// construction).  Warp <-> source block b, lanes over its forward entries:
// count the pairs of each target block (integer atomics, exact totals).
__global__ void __launch_bounds__(256)
k_inv_count(int nsb, const int64_t *__restrict__ fwd_off, const int *__restrict__ fwd_t,
            unsigned long long *__restrict__ cnt)
{
    const int b = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= nsb) return;
    for (int64_t k = fwd_off[b] + lane; k < fwd_off[b + 1]; k += 32) atomicAdd(&cnt[fwd_t[k]], 1ull);
}

// Scatter each forward pair (b, t) into t's segment of the inverse list, in
// arrival order: tmp_b = b, tmp_k = forward position.  k_inv_order then
// fixes the order.
__global__ void __launch_bounds__(256)
k_inv_scatter(int nsb, const int64_t *__restrict__ fwd_off, const int *__restrict__ fwd_t,
              const int64_t *__restrict__ inv_off, unsigned long long *__restrict__ fill, int *__restrict__ tmp_b,
              int64_t *__restrict__ tmp_k)
{
    const int b = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= nsb) return;
    for (int64_t k = fwd_off[b] + lane; k < fwd_off[b + 1]; k += 32) {
        const int t = fwd_t[k];
        const int64_t pos = inv_off[t] + (int64_t)atomicAdd(&fill[t], 1ull);
        tmp_b[pos] = b;
        tmp_k[pos] = k;
    }
}

// CTA <-> target block t: order its segment by source block (distinct within
// a segment).  With at most 32 * INV_TILE source blocks: a bitmap of the
// segment's blocks in shared memory, an exclusive scan of its word
// popcounts, and rank(b) = prefix[b / 32] + popc(bits of the word below b).
// Otherwise, up to INV_TILE entries: bitonic sort of (b, entry); longer
// segments: the rank of each entry = the number of entries with a smaller b,
// counted against INV_TILE-entry tiles.  Every way, inv_b[off + rank] = b
// (ascending b, the order the gradient reduction sums in) and
// fwd2inv[k] = off + rank.
constexpr int INV_TILE = 2048;
constexpr int INV_PER = INV_TILE / 256;
__global__ void __launch_bounds__(256)
k_inv_order(int nsb, const int64_t *__restrict__ inv_off, const int *__restrict__ tmp_b,
            const int64_t *__restrict__ tmp_k, int *__restrict__ inv_b, int64_t *__restrict__ fwd2inv)
{
    __shared__ int sb[INV_TILE];
    __shared__ short si[INV_TILE];
    __shared__ unsigned bm[INV_TILE];
    __shared__ int pre[INV_TILE];
    __shared__ int wsum[8];
    const int t = blockIdx.x, tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    const int64_t off = inv_off[t];
    const int64_t L = inv_off[t + 1] - off;
    const int W = (nsb + 31) >> 5;
    if (W <= INV_TILE) {
        for (int i = tid; i < W; i += 256) bm[i] = 0u;
        __syncthreads();
        for (int64_t i = tid; i < L; i += 256) {
            const int b = tmp_b[off + i];
            atomicOr(&bm[b >> 5], 1u << (b & 31));
        }
        __syncthreads();
        int loc[INV_PER], run = 0;
#pragma unroll
        for (int u = 0; u < INV_PER; ++u) {
            const int w = tid * INV_PER + u;
            loc[u] = run;
            run += w < W ? __popc(bm[w]) : 0;
        }
        int x = run;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += v;
        }
        if (lane == 31) wsum[wp] = x;
        __syncthreads();
        int base = x - run;
        for (int w = 0; w < wp; ++w) base += wsum[w];
#pragma unroll
        for (int u = 0; u < INV_PER; ++u) {
            const int w = tid * INV_PER + u;
            if (w < W) pre[w] = base + loc[u];
        }
        __syncthreads();
        for (int64_t i = tid; i < L; i += 256) {
            const int b = tmp_b[off + i];
            const int r = pre[b >> 5] + __popc(bm[b >> 5] & ((1u << (b & 31)) - 1u));
            inv_b[off + r] = b;
            fwd2inv[tmp_k[off + i]] = off + r;
        }
        return;
    }
    if (L <= INV_TILE) {
        int n = 2;
        while (n < L) n <<= 1;
        for (int i = tid; i < n; i += 256) {
            sb[i] = i < L ? tmp_b[off + i] : 0x7fffffff;
            si[i] = (short)i;
        }
        __syncthreads();
        for (int k = 2; k <= n; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = tid; i < n; i += 256) {
                    const int p = i ^ j;
                    if (p > i) {
                        const int a = sb[i], b = sb[p];
                        if ((a > b) == ((i & k) == 0)) {
                            sb[i] = b;
                            sb[p] = a;
                            const short x = si[i];
                            si[i] = si[p];
                            si[p] = x;
                        }
                    }
                }
                __syncthreads();
            }
        }
        for (int i = tid; i < L; i += 256) {
            inv_b[off + i] = sb[i];
            fwd2inv[tmp_k[off + si[i]]] = off + i;
        }
        return;
    }
    for (int64_t i0 = 0; i0 < L; i0 += INV_TILE) {
        int mine[INV_PER], rank[INV_PER];
#pragma unroll
        for (int u = 0; u < INV_PER; ++u) {
            const int64_t i = i0 + tid + 256 * u;
            mine[u] = i < L ? tmp_b[off + i] : 0x7fffffff;
            rank[u] = 0;
        }
        for (int64_t j0 = 0; j0 < L; j0 += INV_TILE) {
            const int nj = (int)min((int64_t)INV_TILE, L - j0);
            __syncthreads();
            for (int j = tid; j < nj; j += 256) sb[j] = tmp_b[off + j0 + j];
            __syncthreads();
            for (int j = 0; j < nj; ++j) {
                const int v = sb[j];
#pragma unroll
                for (int u = 0; u < INV_PER; ++u) rank[u] += v < mine[u] ? 1 : 0;
            }
        }
#pragma unroll
        for (int u = 0; u < INV_PER; ++u) {
            const int64_t i = i0 + tid + 256 * u;
            if (i < L) {
                inv_b[off + rank[u]] = mine[u];
                fwd2inv[tmp_k[off + i]] = off + rank[u];
            }
        }
    }
}

// exclusive scan of n counts into off[0..n] (single CTA, order-fixed)
__global__ void __launch_bounds__(1024) k_scan(const int64_t *__restrict__ cnt, int64_t n, int64_t *__restrict__ off)
{
    // passes of 1,024 x SP counts: each thread loads SP consecutive counts at
    // once (the CTA is bound by load latency), the thread sums are scanned by
    // warp shuffles and warp 0, and a running carry crosses the passes
    // (integer sums: exact in any order)
    constexpr int SP = 8;
    __shared__ long long wsum[32];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    long long carry = 0;
    for (int64_t t0 = 0; t0 < n; t0 += 1024 * SP) {
        const int64_t base = t0 + (int64_t)tid * SP;
        long long v[SP], tsum = 0;
#pragma unroll
        for (int k = 0; k < SP; ++k) v[k] = base + k < n ? (long long)cnt[base + k] : 0;
#pragma unroll
        for (int k = 0; k < SP; ++k) tsum += v[k];
        long long x = tsum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        if (w == 0) {
            long long z = wsum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const long long y = __shfl_up_sync(0xffffffffu, z, o);
                if (lane >= o) z += y;
            }
            wsum[lane] = z;
        }
        __syncthreads();
        long long run = carry + (w > 0 ? wsum[w - 1] : 0) + x - tsum;
#pragma unroll
        for (int k = 0; k < SP; ++k) {
            if (base + k < n) off[base + k] = (int64_t)run;
            run += v[k];
        }
        carry += wsum[31];
        __syncthreads();  // wsum is rewritten by the next pass
    }
    if (tid == 0) off[n] = (int64_t)carry;
}

// ---------------------------------------------------------------------------
// fused value + gradient sweeps
// ---------------------------------------------------------------------------

// Stage the targets of the forward pairs [k0, k1) of block b, culled per
// target against the block sphere: each warp takes target blocks (lane <->
// target), counts its survivors with a ballot, and whole target blocks are
// accepted in list order while the staged total fits FT_MAXS.  Returns the
// number of forward entries consumed; staged order = (target block, slot).
template <int DIM, class SM>
__device__ int stage_chunk(SM &sm, const FusedArgs &f, int64_t kb, int64_t k0, int64_t k1, const double *bc,
                           double rcull2, bool for_b)
{
    constexpr int SUB = 4;                       // target blocks per warp per iteration
    constexpr int PER = FT_WARPS * SUB;          // entries examined per iteration
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    int total = 0, nb = 0;
    int64_t k = k0;
    while (k < k1 && nb < FT_MAXT) {
        unsigned bal[SUB];
        int tt[SUB];
        int64_t jj[SUB];
#pragma unroll
        for (int s = 0; s < SUB; ++s) {
            const int idx = s * FT_WARPS + wp;
            const int64_t e = k + idx;
            bal[s] = 0u;
            tt[s] = -1;
            jj[s] = 0;
            int cntv = -1;
            if (e < k1 && nb + idx < FT_MAXT) {
                int t, sz;
                int64_t j0;
                if (e - kb < FT_PREF) {
                    t = sm.ent_t[e - kb];
                    j0 = sm.ent_j0[e - kb];
                    sz = sm.ent_sz[e - kb];
                } else {
                    t = f.fwd_t[e];
                    j0 = f.tblk_off[t];
                    sz = (int)(f.tblk_off[t + 1] - j0);
                }
                tt[s] = t;
                jj[s] = j0;
                bool keep = false;
                if (lane < sz) {
                    const double *tp = f.tpk + (j0 + lane) * TPACK;
                    double d2 = 0.0;
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        const double q = tp[d] - bc[d];
                        d2 += q * q;
                    }
                    keep = d2 <= rcull2;
                }
                bal[s] = __ballot_sync(0xffffffffu, keep);
                cntv = __popc(bal[s]);
            }
            if (lane == 0) sm.ecnt[idx] = cntv;
        }
        __syncthreads();
        // accept entries in list order while they fit: warp 0 scans the PER
        // survivor counts (lane <-> entry), the prefix goes through smem
        if (wp == 0) {
            const int cv = sm.ecnt[lane];
            int incl = cv < 0 ? 0 : cv;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            const int excl = incl - (cv < 0 ? 0 : cv);
            const unsigned bad = __ballot_sync(0xffffffffu, cv < 0 || total + incl > SM::MAXS);
            const int na = bad ? __ffs(bad) - 1 : 32;
            sm.epre[lane] = total + excl;
            const int accsum = __shfl_sync(0xffffffffu, incl, na > 0 ? na - 1 : 0);
            if (lane == 0) {
                sm.eacc = na;
                sm.etot = total + (na > 0 ? accsum : 0);
            }
        }
        __syncthreads();
        const int nacc = sm.eacc;
        const int run = nacc > 0 ? sm.etot : total;
#pragma unroll
        for (int s = 0; s < SUB; ++s) {
            const int idx = s * FT_WARPS + wp;
            if (idx < nacc) {
                const int slot = nb + idx;
                const int64_t j0 = jj[s];
                const bool keep = (bal[s] >> lane) & 1u;
                short pos = -1;
                if (keep) {
                    pos = (short)(sm.epre[idx] + __popc(bal[s] & ((1u << lane) - 1u)));
                    const double *tp = f.tpk + (j0 + lane) * TPACK;
#pragma unroll
                    for (int d = 0; d < FT_TS; ++d) sm.stg[d][pos] = tp[d];
                }
                sm.smap[slot][lane] = pos;
                if (lane == 0) {
                    const int tb = tt[s];
                    sm.ctb[slot] = tb;
                    const int64_t ip = f.fwd2inv[k + idx];
                    sm.cpos[slot] = (for_b && ip >= 0 && tb >= f.tlo && tb < f.thi) ? (ip - f.part_base) * TBLK_KD
                                                                                    : (int64_t)-1;
                }
            }
        }
        total = run;
        nb += nacc;
        k += nacc;
        __syncthreads();
        if (nacc < PER) break;  // capacity reached, list exhausted or block limit
    }
    if (tid == 0) sm.nstg = total;
    __syncthreads();
    return nb;
}

// Exact squared distance from a staged target (SoA) to a cell centre.
template <int DIM, class SM>
__device__ __forceinline__ double stg_dist2(const SM &sm, int t, const double *c)
{
    const double y[3] = {sm.stg[0][t], sm.stg[1][t], DIM == 3 ? sm.stg[2][t] : 0.0};
    return dist2_exact<DIM>(y, c);
}

// Value-sweep pair loop of one unit over its compacted candidates.
// MODE 0: shift M = per-unit upper bound, exponents provably >= -16000 (no
//         clamp); MODE 1: same with the clamp; MODE 2: per-pair lazy rescale
//         (when the bound could sit more than 2^500 above the true maximum).
// NQ: quadrature points handled (== QL for full units: straight-line code
//     whose NQ exponential chains interleave).
template <int DIM, int QL, int NQ, int MODE, class SM>
__device__ __forceinline__ void value_pairs(const SM &sm, int wp, int lane, int ncand, int qoff, double cc0,
                                            double cc1, double cc2, const EvalArgs &a, double Munit, double *M,
                                            double *S, double *mx)
{
    for (int p = lane; p < ncand; p += 32) {
        const int ti = sm.cand[wp][p];
        const double g0 = sm.stg[0][ti] - cc0, g1 = sm.stg[1][ti] - cc1;
        const double g2 = DIM == 3 ? sm.stg[2][ti] - cc2 : 0.0;
        const double d2 = DIM == 3 ? g0 * g0 + g1 * g1 + g2 * g2 : g0 * g0 + g1 * g1;
        const double B0 = fma(-a.halfs, d2, sm.stg[5][ti]) - (MODE == 2 ? 0.0 : Munit);
        const double G0 = a.s * g0, G1 = a.s * g1, G2 = a.s * g2;
        const double nuj = sm.stg[3][ti];
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const double *dq = sm.qd[qoff + q];
            double bb = fma(G0, dq[0], B0);
            bb = fma(G1, dq[1], bb);
            if (DIM == 3) bb = fma(G2, dq[2], bb);
            if (MODE == 2) {
                lse_update(bb, nuj, M[q], S[q], mx[q], sm.tab);
            } else {
                mx[q] = fmax(mx[q], bb);
                S[q] = fma(nuj, MODE == 0 ? exp2_16_nc(bb, sm.tab) : exp2_16(bb, sm.tab), S[q]);
            }
        }
    }
}

// Units with fewer than QL quadrature points (the last q-group of a cell).
template <int DIM, int QL, int MODE, class SM>
__device__ __noinline__ void value_pairs_partial(const SM &sm, int wp, int lane, int ncand, int qoff, int nql,
                                                 double cc0, double cc1, double cc2, const EvalArgs &a, double Munit,
                                                 double *M, double *S, double *mx)
{
    for (int p = lane; p < ncand; p += 32) {
        const int ti = sm.cand[wp][p];
        const double g0 = sm.stg[0][ti] - cc0, g1 = sm.stg[1][ti] - cc1;
        const double g2 = DIM == 3 ? sm.stg[2][ti] - cc2 : 0.0;
        const double d2 = DIM == 3 ? g0 * g0 + g1 * g1 + g2 * g2 : g0 * g0 + g1 * g1;
        const double B0 = fma(-a.halfs, d2, sm.stg[5][ti]) - (MODE == 2 ? 0.0 : Munit);
        const double G0 = a.s * g0, G1 = a.s * g1, G2 = a.s * g2;
        const double nuj = sm.stg[3][ti];
#pragma unroll
        for (int q = 0; q < QL; ++q) {
            if (q < nql) {
                const double *dq = sm.qd[qoff + q];
                double bb = fma(G0, dq[0], B0);
                bb = fma(G1, dq[1], bb);
                if (DIM == 3) bb = fma(G2, dq[2], bb);
                if (MODE == 2) {
                    lse_update(bb, nuj, M[q], S[q], mx[q], sm.tab);
                } else {
                    mx[q] = fmax(mx[q], bb);
                    S[q] = fma(nuj, exp2_16(bb, sm.tab), S[q]);
                }
            }
        }
    }
}

// Exact candidate test of the staged targets for the warp's cell, in-order
// compaction into sm.cand[wp]; returns the count and (through bmax) the
// largest B0_Kj = kappa (psi_j - d2/2)/eps over the candidates.
template <int DIM, class SM>
__device__ __forceinline__ int compact_candidates(SM &sm, int wp, int lane, int nstg, const double *cc,
                                                  const EvalArgs &a, double &bmax)
{
    constexpr int U = 4;  // staged targets per lane in flight (independent distance chains)
    int ncand = 0;
    bmax = -CUDART_INF;
    for (int b0 = 0; b0 < nstg; b0 += 32 * U) {
        bool in[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int t = b0 + 32 * u + lane;
            in[u] = false;
            if (t < nstg) {
                const double d2 = stg_dist2<DIM>(sm, t, cc);
                in[u] = d2 <= a.sstar;
                if (in[u]) bmax = fmax(bmax, fma(-a.halfs, d2, sm.stg[5][t]));
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const unsigned bal = __ballot_sync(0xffffffffu, in[u]);
            if (in[u]) sm.cand[wp][ncand + __popc(bal & ((1u << lane) - 1u))] = (unsigned short)(b0 + 32 * u + lane);
            ncand += __popc(bal);
        }
    }
    bmax = warp_max(bmax);
    __syncwarp();
    return ncand;
}

// Gradient sweep of one unit over its compacted candidates: for each
// candidate target j (lane-strided) the unit's part of sum_q w_q nu_j
// e^{t_qj - L_q}, written to the warp's partial row (FP32).  E0 and G' are
// formed in FP64 per (cell, target) so that every FP32 operand is small.
template <int DIM, bool FP32B, class SM>
__device__ __forceinline__ void grad_pairs(SM &sm, const FusedArgs &f, int wp, int lane, int ncand, int qoff,
                                           int nql, const double *cc, double Lref, int64_t qblk0, const EvalArgs &a)
{
    const float sf = (float)(a.s * (1.0 / 16.0));
    for (int p = lane; p < ncand; p += 32) {
        const int ti = sm.cand[wp][p];
        const double g0 = sm.stg[0][ti] - cc[0], g1 = sm.stg[1][ti] - cc[1];
        const double g2 = DIM == 3 ? sm.stg[2][ti] - cc[2] : 0.0;
        const double d2 = DIM == 3 ? g0 * g0 + g1 * g1 + g2 * g2 : g0 * g0 + g1 * g1;
        double val;
        if (FP32B) {
            const float e0 = (float)(sm.stg[4][ti] + (fma(-a.halfs, d2, sm.stg[5][ti]) - KAPPA * Lref) * (1.0 / 16.0));
            const float G0 = sf * (float)g0, G1 = sf * (float)g1, G2 = sf * (float)g2;
            float acc0 = 0.f, acc1 = 0.f;
            if (f.w_nonneg) {
                int q = 0;
                for (; q + 1 < nql; q += 2) {
                    const float4 v0 = *reinterpret_cast<const float4 *>(sm.qb[qoff + q]);
                    const float4 v1 = *reinterpret_cast<const float4 *>(sm.qb[qoff + q + 1]);
                    float ea = fmaf(G0, v0.x, e0 + v0.w), eb = fmaf(G0, v1.x, e0 + v1.w);
                    ea = fmaf(G1, v0.y, ea);
                    eb = fmaf(G1, v1.y, eb);
                    if (DIM == 3) {
                        ea = fmaf(G2, v0.z, ea);
                        eb = fmaf(G2, v1.z, eb);
                    }
                    acc0 += ex2_approx(ea);
                    acc1 += ex2_approx(eb);
                }
                if (q < nql) {
                    const float4 v0 = *reinterpret_cast<const float4 *>(sm.qb[qoff + q]);
                    float ea = fmaf(G0, v0.x, e0 + v0.w);
                    ea = fmaf(G1, v0.y, ea);
                    if (DIM == 3) ea = fmaf(G2, v0.z, ea);
                    acc0 += ex2_approx(ea);
                }
            } else {
                for (int q = 0; q < nql; ++q) {
                    const float *qb = sm.qb[qoff + q];
                    float e = fmaf(G0, qb[0], e0 + qb[3]);
                    e = fmaf(G1, qb[1], e);
                    if (DIM == 3) e = fmaf(G2, qb[2], e);
                    acc0 = fmaf(sm.qw[qoff + q], ex2_approx(e), acc0);
                }
            }
            val = (double)(acc0 + acc1);
        } else {
            const double U0 = 16.0 * sm.stg[4][ti] + fma(-a.halfs, d2, sm.stg[5][ti]) - KAPPA * Lref;
            const double G0 = a.s * g0, G1 = a.s * g1, G2 = a.s * g2;
            double acc = 0.0;
            for (int q = 0; q < nql; ++q) {
                const double *dq = sm.qd[qoff + q];
                const double L = sm.qL[qoff + q];
                if (!isfinite(L)) continue;
                double u = fma(G0, dq[0], U0 + dq[3] - KAPPA * (L - Lref));
                u = fma(G1, dq[1], u);
                if (DIM == 3) u = fma(G2, dq[2], u);
                acc = fma(f.w[qblk0 + qoff + q], exp2_16(u, sm.tab), acc);
            }
            val = acc;
        }
        partial_rows<FP32B>(sm)[wp * SM::MAXS + ti] = (typename PRow<FP32B>::T)val;
    }
}

// Tensor-product points (TM per dimension, symmetric about the cell centre):
// delta_q = (s_0 a_0, s_1 a_1, s_2 a_2) with s_d in {-1, 0, +1}, so
// 2^(b_qj/16) = nu_j 2^(B0_Kj/16) prod_d 2^(s_d G_Kj,d a_d/16) and one
// candidate costs 1 + DIM exponentials and DIM reciprocals for its TM^DIM
// points.  Sums stay relative to Munit (LSE mode only).
template <int TM, int D>
__device__ __forceinline__ constexpr int tstride()
{
    return D == 0 ? 1 : (D == 1 ? TM : TM * TM);
}

// The per-q maximum exponent (the reference's m of the log-sum-exp, which
// C_global depends on) is taken exactly, as in value_pairs, but only over the
// candidates that can attain it: b_qj lies within s r |delta|max of B0_Kj, so
// a candidate with B0 below (running max B0) - 2 s r |delta|max is never a
// maximum; thr is that bound relative to Munit.
template <int DIM, int TM, int TS, class SM>
__device__ __forceinline__ void value_pairs_tensor(const SM &sm, int wp, int lane, int ncand, int qoff,
                                                   const double *cc, const EvalArgs &a, double Munit, double thr,
                                                   double *S, double *mx)
{
    constexpr int NQ = DIM == 3 ? TM * TM * TM : TM * TM;
    double ah[3];
    ah[0] = sm.qd[qoff + (TM - 1) * tstride<TM, 0>()][0];
    ah[1] = sm.qd[qoff + (TM - 1) * tstride<TM, 1>()][1];
    ah[2] = DIM == 3 ? sm.qd[qoff + (TM - 1) * tstride<TM, 2>()][2] : 0.0;
    for (int p = lane; p < ncand; p += 32) {
        const int ti = sm.cand[wp][p];
        const double g0 = sm.stg[0][ti] - cc[0], g1 = sm.stg[1][ti] - cc[1];
        const double g2 = DIM == 3 ? sm.stg[2][ti] - cc[2] : 0.0;
        const double d2 = DIM == 3 ? g0 * g0 + g1 * g1 + g2 * g2 : g0 * g0 + g1 * g1;
        const double B0 = fma(-a.halfs, d2, sm.stg[5][ti]) - Munit;
        const double G[3] = {a.s * g0, a.s * g1, a.s * g2};
        if (B0 >= thr) {
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                const double *dq = sm.qd[qoff + q];
                double bb = fma(G[0], dq[0], B0);
                bb = fma(G[1], dq[1], bb);
                if (DIM == 3) bb = fma(G[2], dq[2], bb);
                mx[q] = fmax(mx[q], bb);
            }
        }
        // per-dimension factors 2^(G_d delta_d): with TS, relative to the lowest
        // point (1, r, r^2 with the shift folded into P); otherwise 2^(-G a), (1), 2^(G a)
        double F[3][TM];
        double P;
        if constexpr (TS >= 1) {
            double sga = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                const double ga = G[d] * ah[d];
                sga += ga;
                const double r = exp2_16(TM == 2 ? 2.0 * ga : ga, sm.tab);
                F[d][0] = 1.0;
                F[d][1] = r;
                if (TM == 3) F[d][2] = r * r;
            }
            P = sm.stg[3][ti] * exp2_16(B0 - sga, sm.tab);
        } else {
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                const double xp = exp2_16(G[d] * ah[d], sm.tab);
                F[d][0] = __drcp_rn(xp);
                F[d][TM - 1] = xp;
                if (TM == 3) F[d][1] = 1.0;
            }
            P = sm.stg[3][ti] * exp2_16(B0, sm.tab);
        }
#pragma unroll
        for (int i0 = 0; i0 < TM; ++i0) {
            const double t0 = P * F[0][i0];
            if (DIM == 2) {
#pragma unroll
                for (int i1 = 0; i1 < TM; ++i1) S[i0 + TM * i1] = fma(t0, F[1][i1], S[i0 + TM * i1]);
            } else {
#pragma unroll
                for (int i1 = 0; i1 < TM; ++i1) {
                    const double t1 = t0 * F[1][i1];
#pragma unroll
                    for (int i2 = 0; i2 < TM; ++i2) {
                        const int q = i0 + TM * i1 + TM * TM * i2;
                        S[q] = fma(t1, F[2][i2], S[q]);
                    }
                }
            }
        }
    }
}

__device__ __forceinline__ float rcp_approx(float x)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// FP32 gradient sweep on tensor-product points: per candidate
// 2^(e0) sum_q W_q prod_d F_d[i_d], W_q = w_q 2^(D_q), summed dimension by
// dimension (Horner order), into the warp's partial row.
template <int DIM, int TM, int TS, class SM>
__device__ __forceinline__ void grad_pairs_tensor(SM &sm, int wp, int lane, int ncand, int qoff,
                                                  const double *cc, double Lref, const EvalArgs &a)
{
    constexpr int NQ = DIM == 3 ? TM * TM * TM : TM * TM;
    const float sf = (float)(a.s * (1.0 / 16.0));
    float ah[3];
    ah[0] = (float)sm.qd[qoff + (TM - 1) * tstride<TM, 0>()][0];
    ah[1] = (float)sm.qd[qoff + (TM - 1) * tstride<TM, 1>()][1];
    ah[2] = DIM == 3 ? (float)sm.qd[qoff + (TM - 1) * tstride<TM, 2>()][2] : 0.f;
    float W[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) W[q] = sm.qtw[qoff + q];
    for (int p = lane; p < ncand; p += 32) {
        const int ti = sm.cand[wp][p];
        const double g0 = sm.stg[0][ti] - cc[0], g1 = sm.stg[1][ti] - cc[1];
        const double g2 = DIM == 3 ? sm.stg[2][ti] - cc[2] : 0.0;
        const double d2 = DIM == 3 ? g0 * g0 + g1 * g1 + g2 * g2 : g0 * g0 + g1 * g1;
        float e0 = (float)(sm.stg[4][ti] + (fma(-a.halfs, d2, sm.stg[5][ti]) - KAPPA * Lref) * (1.0 / 16.0));
        const float gd[3] = {(float)g0, (float)g1, (float)g2};
        float F[3][TM];
        if constexpr (TS >= 1) {
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                const float ga = sf * gd[d] * ah[d];
                e0 -= ga;
                const float r = ex2_approx(TM == 2 ? 2.f * ga : ga);
                F[d][0] = 1.f;
                F[d][1] = r;
                if (TM == 3) F[d][2] = r * r;
            }
        } else {
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                const float xp = ex2_approx(sf * gd[d] * ah[d]);
                F[d][0] = rcp_approx(xp);
                F[d][TM - 1] = xp;
                if (TM == 3) F[d][1] = 1.f;
            }
        }
        float w = 0.f;
        if (DIM == 2) {
#pragma unroll
            for (int i0 = 0; i0 < TM; ++i0) {
                float u = 0.f;
#pragma unroll
                for (int i1 = 0; i1 < TM; ++i1) u = fmaf(W[i0 + TM * i1], F[1][i1], u);
                w = fmaf(u, F[0][i0], w);
            }
        } else {
#pragma unroll
            for (int i0 = 0; i0 < TM; ++i0) {
                float u = 0.f;
#pragma unroll
                for (int i1 = 0; i1 < TM; ++i1) {
                    float v = 0.f;
#pragma unroll
                    for (int i2 = 0; i2 < TM; ++i2) v = fmaf(W[i0 + TM * i1 + TM * TM * i2], F[2][i2], v);
                    u = fmaf(v, F[1][i1], u);
                }
                w = fmaf(u, F[0][i0], w);
            }
        }
        partial_rows<true>(sm)[wp * SM::MAXS + ti] = ex2_approx(e0) * w;
    }
}

// CTA sum of the warp partial rows (warp order) and the write of every slot
// of every pair of the chunk (zeros where a target was not staged).
template <bool FP32B, class SM>
__device__ __forceinline__ void write_partials(SM &sm, const FusedArgs &f, int nt, int nunit)
{
    const typename PRow<FP32B>::T *rows = partial_rows<FP32B>(sm);
    const int tid = threadIdx.x;
    for (int i = tid; i < nt * TBLK_KD; i += blockDim.x) {
        const int ti = i / TBLK_KD, sl = i - ti * TBLK_KD;
        const int64_t base = sm.cpos[ti];
        if (base < 0) continue;
        const short p = sm.smap[ti][sl];
        double v = 0.0;
        if (p >= 0)
            for (int w = 0; w < nunit; ++w) v += (double)rows[w * SM::MAXS + p];
        if constexpr (FP32B) f.part32[base + sl] = (float)v;
        else f.part[base + sl] = v;
    }
}

template <int DIM, int QL, bool FP32B, int MODE, int TQ, int TS>
__global__ void __launch_bounds__(FT_WARPS * 32, fused_min_blocks(DIM, TQ, FP32B))
k_fused(FusedArgs f, EvalArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using SMem = FTSmem<fused_cap(DIM, TQ, FP32B)>;
    SMem &sm = *reinterpret_cast<SMem *>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    const int b = blockIdx.x;
    if (tid < 16) sm.tab[tid] = c_exp2_tab[tid];
    const int64_t cb0 = f.sblk_cell[b], cb1 = f.sblk_cell[b + 1];
    const int ncell = (int)(cb1 - cb0);
    const int nunit = ncell * a.ngroups;
    const bool valid = wp < nunit;
    const int cl = valid ? wp / a.ngroups : 0;          // cell of this warp (block-local)
    const int grp = valid ? wp - cl * a.ngroups : 0;
    const int qoff = cl * a.qpc + grp * a.ql;           // block-local index of the unit's first q
    const int nql = valid ? min(a.ql, a.qpc - grp * a.ql) : 0;
    const int64_t qblk0 = cb0 * a.qpc;                  // first q of the block
    const int nqb = ncell * a.qpc;
    const double *bs = f.sblk_sph + (int64_t)b * 4;
    const double bc[3] = {bs[0], bs[1], bs[2]};
    const double rc = (f.cullt + bs[3]) * (1.0 + 1e-12) + 1e-300;
    const double rcull2 = rc * rc;
    const int64_t k0 = f.fwd_off[b], k1 = f.fwd_off[b + 1];
    for (int i = tid; i < ncell * 3; i += blockDim.x) {
        const int c = i / 3, d = i - c * 3;
        sm.cellc[c][d] = d < DIM ? f.cell_ctr[(cb0 + c) * DIM + d] : 0.0;
    }
    for (int i = tid; i < (int)min((int64_t)FT_PREF, k1 - k0); i += blockDim.x) {
        const int t = f.fwd_t[k0 + i];
        const int64_t j0 = f.tblk_off[t];
        sm.ent_t[i] = t;
        sm.ent_j0[i] = (int)j0;
        sm.ent_sz[i] = (unsigned char)(f.tblk_off[t + 1] - j0);
    }
    __syncthreads();
    for (int i = tid; i < nqb; i += blockDim.x) {
        const int c = i / a.qpc;
        double dsq = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double dl = d < DIM ? f.x[(qblk0 + i) * DIM + d] - sm.cellc[c][d] : 0.0;
            sm.qd[i][d] = dl;
            dsq += dl * dl;
        }
        sm.qd[i][3] = -a.halfs * dsq;
        sm.qn[i] = sqrt(dsq);
    }
    __syncthreads();
    const double cc[3] = {sm.cellc[cl][0], sm.cellc[cl][1], sm.cellc[cl][2]};
    int tail_off = -1;  // first entry (minus k0) of the value sweep's last chunk, still staged for the gradient sweep
    int tail_nt = 0;
    int ncand_single = 0;

    // ---------------- value sweep ----------------
    if (f.do_a) {
        // Shift of the online sums.  MODE 0/1: Munit = max_j B0_Kj + s r
        // max_q |delta_q| bounds every exponent of the unit from above
        // (|G_Kj| <= s r for a candidate), so no per-pair rescale is needed;
        // exponents are kept relative to Munit (mx too) and a chunk that raises
        // the bound rescales S once.  MODE 2 keeps a per-q lazy shift M[q].
        double M[MODE == 2 ? QL : 1], S[QL], mx[QL];
#pragma unroll
        for (int k = 0; k < QL; ++k) { S[k] = 0.0; mx[k] = -CUDART_INF; }
#pragma unroll
        for (int k = 0; k < (MODE == 2 ? QL : 1); ++k) M[k] = -CUDART_INF;
        double Munit = -CUDART_INF;
        double dqmax = 0.0;
        for (int q = 0; q < nql; ++q) dqmax = fmax(dqmax, sm.qn[qoff + q]);
        double npairs = 0.0;
        double bmax_run = -CUDART_INF;  // largest B0 of the candidates so far
        const double sr = a.s * a.cull;
        for (int64_t k = k0; k < k1;) {
            const int nt = stage_chunk<DIM>(sm, f, k0, k, k1, bc, rcull2, f.do_b != 0);
            const int nstg = sm.nstg;
            if (valid) {
                double bmax;
                const int ncand = compact_candidates<DIM>(sm, wp, lane, nstg, cc, a, bmax);
                ncand_single = ncand;
                npairs += (double)ncand * nql;
                if (MODE != 2 && bmax > -CUDART_INF) {
                    const double mnew = bmax + sr * dqmax;
                    if (mnew > Munit) {
                        if (Munit > -CUDART_INF) {
                            const double sc = exp2_16(Munit - mnew, sm.tab);
#pragma unroll
                            for (int q = 0; q < QL; ++q) {
                                S[q] *= sc;
                                mx[q] += Munit - mnew;
                            }
                        }
                        Munit = mnew;
                    }
                }
                if (bmax > bmax_run) bmax_run = bmax;
                if constexpr (TQ > 0)
                    value_pairs_tensor<DIM, TQ, TS>(sm, wp, lane, ncand, qoff, cc, a, Munit,
                                                    bmax_run - 2.0 * sr * dqmax - Munit, S, mx);
                else if (nql == QL)
                    value_pairs<DIM, QL, QL, MODE>(sm, wp, lane, ncand, qoff, cc[0], cc[1], cc[2], a, Munit, M, S, mx);
                else
                    value_pairs_partial<DIM, QL, MODE>(sm, wp, lane, ncand, qoff, nql, cc[0], cc[1], cc[2], a, Munit,
                                                       M, S, mx);
            }
            k += nt;
            if (k >= k1) {
                tail_off = (int)(k - nt - k0);  // kept staged (with each warp's candidates) for the gradient sweep
                tail_nt = nt;
            } else {
                __syncthreads();  // the next chunk overwrites the staged targets
            }
        }
        // merge the lanes of each q (max, sum); the lane that ends with q's
        // totals runs q's epilogue, so the QL epilogues proceed in parallel
        double my_mx = -CUDART_INF, my_S = 0.0;
        int my_q = lane;   // the q whose totals this lane holds
        bool epi = lane < nql;
        if constexpr (MODE != 2 && QL == 8) {
            // Transposed butterflies: the xor-16, -8 and -4 exchanges each
            // halve the q's a lane keeps (q = lane >> 2 after them), the xor-2
            // and -1 exchanges finish: 9 exchanges per reduction instead of 40.
            // Every lane's sums are relative to Munit, so they add directly and
            // one exponential per q rescales the total to its maximum.
            const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
            double m4[4], s4[4], m2[2], s2[2];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const double mk = b4 ? mx[4 + k] : mx[k], ms = b4 ? mx[k] : mx[4 + k];
                const double sk = b4 ? S[4 + k] : S[k], ss = b4 ? S[k] : S[4 + k];
                m4[k] = fmax(mk, __shfl_xor_sync(0xffffffffu, ms, 16));
                s4[k] = sk + __shfl_xor_sync(0xffffffffu, ss, 16);
            }
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const double mk = b3 ? m4[2 + k] : m4[k], ms = b3 ? m4[k] : m4[2 + k];
                const double sk = b3 ? s4[2 + k] : s4[k], ss = b3 ? s4[k] : s4[2 + k];
                m2[k] = fmax(mk, __shfl_xor_sync(0xffffffffu, ms, 8));
                s2[k] = sk + __shfl_xor_sync(0xffffffffu, ss, 8);
            }
            double m1 = fmax(b2 ? m2[1] : m2[0], __shfl_xor_sync(0xffffffffu, b2 ? m2[0] : m2[1], 4));
            double s1 = (b2 ? s2[1] : s2[0]) + __shfl_xor_sync(0xffffffffu, b2 ? s2[0] : s2[1], 4);
#pragma unroll
            for (int o = 2; o > 0; o >>= 1) {
                m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
                s1 += __shfl_xor_sync(0xffffffffu, s1, o);
            }
            my_q = lane >> 2;
            epi = (lane & 3) == 0 && my_q < nql;
            my_mx = m1;
            my_S = (Munit == -CUDART_INF || m1 == -CUDART_INF) ? 0.0 : s1 * exp2_16(-m1, sm.tab);
        } else {
#pragma unroll
            for (int q = 0; q < QL; ++q) {
                const double mxw = warp_max(mx[q]);
                // shift of this lane's sum: Munit (exponents relative to it: 0) or the lazy M[q]
                const double Ml = MODE == 2 ? M[MODE == 2 ? q : 0] : (Munit > -CUDART_INF ? 0.0 : -CUDART_INF);
                const double sl = (Ml == -CUDART_INF || mxw == -CUDART_INF) ? 0.0 : S[q] * exp2_16(Ml - mxw, sm.tab);
                const double Sw = warp_sum(sl);
                if (lane == q) {
                    my_mx = mxw;
                    my_S = Sw;
                }
            }
        }
        double tv = 0.0, tcv = 0.0, tsk = 0.0;
        if (valid && epi) {
            const int qi = qoff + my_q;
            const int64_t qg = qblk0 + qi;
            double v, cv, L;
            int sk;
            value_epilogue(a, MODE == 2 ? my_mx : my_mx + Munit, my_S, sm.qd[qi][3], f.rho[qg], f.jxw[qg], v, cv, L,
                           sk);
            f.Lq[qg] = L;
            sm.qL[qi] = L;
            tv = v;
            tcv = cv;
            tsk = sk;
        }
        block_partials(tv, tcv, tsk, lane == 0 ? npairs : 0.0, f.valpart);  // contains __syncthreads
    } else {
        for (int i = tid; i < nqb; i += blockDim.x) sm.qL[i] = f.Lq[qblk0 + i];
        __syncthreads();
    }
    if (!f.do_b) return;

    // ---------------- gradient sweep ----------------
    // per-unit reference L_Kref = min L over the unit's q; per-q FP32 data
    double Lref = CUDART_INF;
    if (valid) {
        double lv = lane < nql ? sm.qL[qoff + lane] : CUDART_INF;
        Lref = -warp_max(-lv);
        if (lane < nql) {
            const int i = qoff + lane;
            const double L = sm.qL[i];
            const double D = (!isfinite(Lref) || !isfinite(L)) ? -CUDART_INF
                                                                : (sm.qd[i][3] - KAPPA * (L - Lref)) * (1.0 / 16.0);
            const double wq = f.w[qblk0 + i];
            sm.qb[i][0] = (float)sm.qd[i][0];
            sm.qb[i][1] = (float)sm.qd[i][1];
            sm.qb[i][2] = (float)sm.qd[i][2];
            sm.qb[i][3] = (float)(f.w_nonneg ? D + log2(wq) : D);  // w_q folded in: p = 2^e directly
            sm.qw[i] = (float)wq;
            if (TQ > 0) sm.qtw[i] = (float)(wq * exp2(D));
        }
        __syncwarp();
    }
    // The value sweep's last chunk (the only one when everything fit) is still
    // staged with each warp's candidates: its gradient comes first, then the
    // earlier chunks are staged again (the same chunks: the greedy rule over
    // [k0, k0 + tail_off) ends where the value sweep's did).  Every pair's partial
    // is written once, so the order of the chunks does not change any sum.
    int64_t kend = k1;
    if (tail_off >= 0) {
        const int nt = tail_nt;
        const int nstg = sm.nstg;
        if (valid) {
            for (int t = lane; t < nstg; t += 32) partial_rows<FP32B>(sm)[wp * SMem::MAXS + t] = 0;
            __syncwarp();
            if (isfinite(Lref)) {
                if constexpr (TQ > 0 && FP32B) grad_pairs_tensor<DIM, TQ, TS>(sm, wp, lane, ncand_single, qoff, cc, Lref, a);
                else grad_pairs<DIM, FP32B>(sm, f, wp, lane, ncand_single, qoff, nql, cc, Lref, qblk0, a);
            }
        }
        if (tid < nt) {
            const int tb = sm.ctb[tid];
            const int64_t ip = f.fwd2inv[k0 + tail_off + tid];
            sm.cpos[tid] = (ip >= 0 && tb >= f.tlo && tb < f.thi) ? (ip - f.part_base) * TBLK_KD : (int64_t)-1;
        }
        __syncthreads();
        write_partials<FP32B>(sm, f, nt, nunit);
        if (tail_off == 0) return;
        kend = k0 + tail_off;
        __syncthreads();  // the earlier chunks overwrite the staged targets
    }
    for (int64_t k = k0; k < kend;) {
        const int nt = stage_chunk<DIM>(sm, f, k0, k, kend, bc, rcull2, true);
        const int nstg = sm.nstg;
        if (valid) {
            double bmax;
            const int ncand = compact_candidates<DIM>(sm, wp, lane, nstg, cc, a, bmax);
            for (int t = lane; t < nstg; t += 32) partial_rows<FP32B>(sm)[wp * SMem::MAXS + t] = 0;
            __syncwarp();
            if (isfinite(Lref)) {
                if constexpr (TQ > 0 && FP32B) grad_pairs_tensor<DIM, TQ, TS>(sm, wp, lane, ncand, qoff, cc, Lref, a);
                else grad_pairs<DIM, FP32B>(sm, f, wp, lane, ncand, qoff, nql, cc, Lref, qblk0, a);
            }
        }
        __syncthreads();
        write_partials<FP32B>(sm, f, nt, nunit);
        k += nt;
        __syncthreads();
    }
}

// gradient of target block t = sum of its pair partials in inverse order
// (ascending source block), lane <-> target.  CTA <-> target block: warp w
// sums rows w, w+8, ...; the 8 warp sums are added in warp order.
template <typename PT>
__global__ void __launch_bounds__(256)
k_grad_reduce(const int64_t *__restrict__ tblk_off, const int64_t *__restrict__ inv_off, int tlo, int thi,
              int64_t part_base, const PT *__restrict__ part, double *__restrict__ gacc)
{
    __shared__ double ws[8][32];
    const int t = tlo + blockIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t p0 = inv_off[t], p1 = inv_off[t + 1];
    double acc = 0.0;
    for (int64_t p = p0 + w; p < p1; p += 8) acc += (double)part[(p - part_base) * TBLK_KD + lane];
    ws[w][lane] = acc;
    __syncthreads();
    if (w == 0) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < 8; ++i) s += ws[i][lane];
        const int64_t j = tblk_off[t] + lane;
        if (j < tblk_off[t + 1]) gacc[j] = s;
    }
}

template <int DIM, int QL, bool FP32B, int MODE, int TQ, int TS>
static void launch_fused(sdot_ctx *c, const FusedArgs &f, const EvalArgs &a, size_t smem, int nb)
{
    cudaFuncSetAttribute(k_fused<DIM, QL, FP32B, MODE, TQ, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_fused<DIM, QL, FP32B, MODE, TQ, TS>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
    k_fused<DIM, QL, FP32B, MODE, TQ, TS><<<(unsigned)nb, FT_WARPS * 32, smem, c->stream>>>(f, a);
}

template <int DIM, int QL, int MODE, int TQ = 0, int TS = 0>
static void dispatch_fused_b(sdot_ctx *c, const FusedArgs &f, const EvalArgs &a, bool fp32b, int nb)
{
    if (fp32b) launch_fused<DIM, QL, true, MODE, TQ, TS>(c, f, a, sizeof(FTSmem<fused_cap(DIM, TQ, true)>), nb);
    else
        launch_fused<DIM, QL, false, MODE, TQ, TS>(c, f, a, sizeof(FTSmem<fused_cap(DIM, TQ, false)>) + ft_rows64_bytes(fused_cap(DIM, TQ, false)),
                                               nb);
}

template <int DIM, int MODE>
static void dispatch_fused_q(sdot_ctx *c, const FusedArgs &f, const EvalArgs &a, bool fp32b, int nb)
{
    // 2D: units of 4 (order 2) or 9 (order 3 and groups of 9); 3D: 8 or 9.
    if constexpr (DIM == 2) {
        if (a.ql <= 4) dispatch_fused_b<DIM, 4, MODE>(c, f, a, fp32b, nb);
        else dispatch_fused_b<DIM, 9, MODE>(c, f, a, fp32b, nb);
    } else {
        if (a.ql <= 8) dispatch_fused_b<DIM, 8, MODE>(c, f, a, fp32b, nb);
        else dispatch_fused_b<DIM, 9, MODE>(c, f, a, fp32b, nb);
    }
}

// MODE selection.  The shift Munit may exceed the true maximum exponent of a
// q by up to 2 s r |delta|max (units of 2^(1/16)); beyond 2^500 the lazy form
// is used.  Exponents u relative to Munit satisfy
// u >= -s (psi_max - psi_min + r^2/2 + 2 r |delta|max); when that is above
// -16000 the clamp of exp2 is provably inactive and dropped.
//
// Tensor form of the sweeps (tensor-product points with an instantiation):
// -1 none (per-point sweeps), 0 symmetric factors 2^(+-G a), 1 factors
// relative to the lowest point.
static int fused_tensor_mode(const sdot_ctx *c, const EvalArgs &a, double psi_range)
{
    const double gap = 2.0 * a.s * a.cull * c->delta_max;
    const double umin = -a.s * (psi_range + 0.5 * a.cull * a.cull + 2.0 * a.cull * c->delta_max);
    // tensor-product points: per-dimension factors 2^(+-G a/16) stay within
    // 2^300 (FP64 value sweep) and 2^40 (FP32 gradient sweep)
    const double fac = a.s * a.cull * c->tensor_amax / 16.0;
    const bool tensor = c->tensor_m > 0 && a.lse && a.ngroups == 1 && fac <= 40.0 && umin > -15000.0 &&
                        gap < 16.0 * 500.0;
    const bool shape = (c->dim == 3 && c->tensor_m == 2 && a.ql == 8) ||
                       (c->dim == 2 && c->tensor_m == 3 && a.ql == 9) || (c->dim == 2 && c->tensor_m == 2 && a.ql == 4);
    if (!tensor || !shape) return -1;
    // factors <= 2^8 per dimension: the relative form (no reciprocals, the lowest point's factor 1)
    return fac > 4.0 ? 0 : 1;
}

template <int DIM>
static void dispatch_fused(sdot_ctx *c, const FusedArgs &f, const EvalArgs &a, bool fp32b, int nb, double psi_range,
                           int tmode)
{
    const double gap = 2.0 * a.s * a.cull * c->delta_max;
    const double umin = -a.s * (psi_range + 0.5 * a.cull * a.cull + 2.0 * a.cull * c->delta_max);
    if (gap >= 16.0 * 500.0) {
        dispatch_fused_q<DIM, 2>(c, f, a, fp32b, nb);
        return;
    }
    if (tmode >= 0) {
        if constexpr (DIM == 3) {
            if (tmode == 1) dispatch_fused_b<3, 8, 0, 2, 1>(c, f, a, fp32b, nb);
            else dispatch_fused_b<3, 8, 0, 2, 0>(c, f, a, fp32b, nb);
        } else if (c->tensor_m == 3) {
            if (tmode == 1) dispatch_fused_b<2, 9, 0, 3, 1>(c, f, a, fp32b, nb);
            else dispatch_fused_b<2, 9, 0, 3, 0>(c, f, a, fp32b, nb);
        } else {
            if (tmode == 1) dispatch_fused_b<2, 4, 0, 2, 1>(c, f, a, fp32b, nb);
            else dispatch_fused_b<2, 4, 0, 2, 0>(c, f, a, fp32b, nb);
        }
        return;
    }
    if (umin > -15000.0) dispatch_fused_q<DIM, 0>(c, f, a, fp32b, nb);
    else dispatch_fused_q<DIM, 1>(c, f, a, fp32b, nb);
}

sdot_status run_trunc(sdot_ctx *c, const EvalArgs &a, double r)
{
    cudaStream_t st = c->stream;
    // 1. block-pair structure (conservative FP32 test)
    const float cr = (float)(std::min(r, 1e30) * (1.0 + 1e-6) + 1e-6 * c->coord_scale);
    const int nsb = (int)c->nsblk, ntb = (int)c->ntblk;
    const int nss = (nsb + SUPER - 1) / SUPER, nts = (ntb + SUPER - 1) / SUPER;
    cudaError_t e = c->fwd_cnt.alloc(nsb + 1);
    if (e == cudaSuccess) e = c->fwd_off.alloc(nsb + 1);
    if (e == cudaSuccess) e = c->superpair.alloc((size_t)nss * nts);
    if (e == cudaSuccess) e = c->shit.alloc((size_t)nss * nts);
    if (e == cudaSuccess) e = c->spidx.alloc((size_t)nss * nts);
    if (e == cudaSuccess) e = c->scount.alloc(nss + 1);
    if (e != cudaSuccess) return cuda_error(c, e, "pair list alloc");
    k_super_pairs<<<(unsigned)(((int64_t)nss * nts + 255) / 256), 256, 0, st>>>(c->ssup_sph32.p, nss, c->tsup_sph32.p,
                                                                             nts, cr, c->superpair.p);
    k_super_compact<<<(unsigned)(((int64_t)nss * 32 + 255) / 256), 256, 0, st>>>(c->superpair.p, nss, nts, c->shit.p,
                                                                              c->scount.p, c->spidx.p);
    // Row length of the per-block pair masks: the most target super-blocks any
    // source super-block pairs with.  Every count is at most nts, so when the
    // nts-wide rows are small (<= 128 MiB for both arrays) they are used as
    // they are and the counts are not read back (one host round trip fewer).
    int hmax = std::max(1, nts);
    if ((size_t)nsb * (size_t)nts * 2 * sizeof(int) > ((size_t)128 << 20)) {
        std::vector<int> sc((size_t)nss);
        e = cudaMemcpyAsync(sc.data(), c->scount.p, nss * sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_error(c, e, "pair list count");
        hmax = 1;
        for (int v : sc) hmax = std::max(hmax, v);
    }
    e = c->pmask.alloc((size_t)nsb * hmax);
    if (e == cudaSuccess) e = c->pmpre.alloc((size_t)nsb * hmax);
    if (e != cudaSuccess) return cuda_error(c, e, "pair mask alloc");
    const unsigned gw = (unsigned)(((int64_t)nsb * 32 + 255) / 256);
    k_fwd_masks<<<gw, 256, 0, st>>>(c->sblk_sph32.p, nsb, c->tblk_sph32.p, ntb, nts, hmax, cr, c->shit.p, c->scount.p,
                                    c->pmask.p, c->pmpre.p, c->fwd_cnt.p);
    k_scan<<<1, 1024, 0, st>>>(c->fwd_cnt.p, nsb, c->fwd_off.p);
    int64_t npairs = 0;
    e = cudaMemcpyAsync(&npairs, c->fwd_off.p + nsb, 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_error(c, e, "pair list count");
    e = c->fwd_t.alloc(npairs + 1);
    if (e == cudaSuccess) e = c->inv_b.alloc(npairs + 1);
    if (e == cudaSuccess) e = c->fwd2inv.alloc(npairs + 1);
    if (e == cudaSuccess) e = c->inv_tmpb.alloc(npairs + 1);
    if (e == cudaSuccess) e = c->inv_tmpk.alloc(npairs + 1);
    if (e == cudaSuccess) e = c->inv_cnt.alloc(ntb + 1);
    if (e == cudaSuccess) e = c->inv_off.alloc(ntb + 1);
    if (e != cudaSuccess) return cuda_error(c, e, "pair list alloc");
    k_fwd_fill<<<gw, 256, 0, st>>>(nsb, nts, hmax, c->shit.p, c->scount.p, c->pmask.p, c->fwd_off.p, c->fwd_t.p);
    unsigned long long *icnt = reinterpret_cast<unsigned long long *>(c->inv_cnt.p);
    e = cudaMemsetAsync(c->inv_cnt.p, 0, (ntb + 1) * sizeof(int64_t), st);
    if (e != cudaSuccess) return cuda_error(c, e, "pair list clear");
    k_inv_count<<<gw, 256, 0, st>>>(nsb, c->fwd_off.p, c->fwd_t.p, icnt);
    k_scan<<<1, 1024, 0, st>>>(c->inv_cnt.p, ntb, c->inv_off.p);
    e = cudaMemsetAsync(c->inv_cnt.p, 0, (ntb + 1) * sizeof(int64_t), st);
    if (e != cudaSuccess) return cuda_error(c, e, "pair list clear");
    k_inv_scatter<<<gw, 256, 0, st>>>(nsb, c->fwd_off.p, c->fwd_t.p, c->inv_off.p, icnt, c->inv_tmpb.p, c->inv_tmpk.p);
    k_inv_order<<<(unsigned)ntb, 256, 0, st>>>(nsb, c->inv_off.p, c->inv_tmpb.p, c->inv_tmpk.p, c->inv_b.p, c->fwd2inv.p);
    c->klaunch[6] += 9;
    if (c->profiling) cudaEventRecord(c->pev[7], st);
    // 2. partial buffer (inverse order): all pairs at once under the cap, else target-block groups
    // partials are FP32 in the hybrid mode (the sweeps' rows are FP32), FP64 otherwise
    const bool fp32b = c->precision != SDOT_PREC_FP64;
    const size_t pel = fp32b ? sizeof(float) : sizeof(double);
    const int64_t cap_pairs = std::max<int64_t>(1, (int64_t)(c->part_cap_bytes / (TBLK_KD * pel)));
    std::vector<std::pair<int, int>> groups;
    std::vector<int64_t> inv_host;
    int64_t part_pairs = npairs;
    if (npairs <= cap_pairs) {
        groups.push_back({0, ntb});
    } else {
        inv_host.resize((size_t)ntb + 1);
        e = cudaMemcpyAsync(inv_host.data(), c->inv_off.p, (ntb + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_error(c, e, "pair list copy");
        part_pairs = 0;
        int t0 = 0;
        while (t0 < ntb) {
            int t1 = t0 + 1;
            while (t1 < ntb && inv_host[t1 + 1] - inv_host[t0] <= cap_pairs) ++t1;
            groups.push_back({t0, t1});
            part_pairs = std::max(part_pairs, inv_host[t1] - inv_host[t0]);
            t0 = t1;
        }
    }
    e = c->part.alloc(((size_t)std::max<int64_t>(1, part_pairs) * TBLK_KD * pel + sizeof(double) - 1) / sizeof(double));
    if (e != cudaSuccess) return cuda_error(c, e, "partial buffer alloc");
    FusedArgs f{};
    f.x = c->x.p; f.rho = c->rho.p; f.jxw = c->jxw.p; f.w = c->w.p; f.cell_ctr = c->cell_ctr.p;
    f.tpk = c->tpack.p; f.sblk_cell = c->sblk_cell.p; f.sblk_sph = c->sblk_sph.p; f.tblk_off = c->tblk_off.p;
    f.fwd_off = c->fwd_off.p; f.fwd_t = c->fwd_t.p; f.fwd2inv = c->fwd2inv.p;
    f.part = c->part.p; f.part32 = reinterpret_cast<float *>(c->part.p); f.Lq = c->Lq.p; f.valpart = c->blkpart.p;
    f.cullt = std::isnan(r) ? 0.0 : std::min(r, 1e300);
    f.w_nonneg = c->w_nonneg ? 1 : 0;
    const double prange0 = c->scal_host[SC_MAXPSI] - c->scal_host[SC_MINPSI];
    const double prange = std::isfinite(prange0) ? prange0 : 1e300;
    const int tmode = fused_tensor_mode(c, a, prange);
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        f.do_a = gi == 0;
        f.do_b = 1;
        f.tlo = groups[gi].first;
        f.thi = groups[gi].second;
        f.part_base = groups.size() == 1 ? 0 : inv_host[f.tlo];
        if (c->dim == 2) dispatch_fused<2>(c, f, a, fp32b, nsb, prange, tmode);
        else dispatch_fused<3>(c, f, a, fp32b, nsb, prange, tmode);
        if (c->profiling && gi + 1 == groups.size()) cudaEventRecord(c->pev[2], st);
        const int nw = f.thi - f.tlo;
        if (fp32b)
            k_grad_reduce<float><<<(unsigned)nw, 256, 0, st>>>(c->tblk_off.p, c->inv_off.p, f.tlo, f.thi, f.part_base,
                                                               f.part32, c->gpart.p);
        else
            k_grad_reduce<double><<<(unsigned)nw, 256, 0, st>>>(c->tblk_off.p, c->inv_off.p, f.tlo, f.thi,
                                                                f.part_base, c->part.p, c->gpart.p);
        c->klaunch[2] += 1;
        c->klaunch[3] += 1;
    }
    if (c->profiling) cudaEventRecord(c->pev[3], st);
    return cuda_error(c, cudaGetLastError(), "truncated evaluation");
}

}  // namespace sdot

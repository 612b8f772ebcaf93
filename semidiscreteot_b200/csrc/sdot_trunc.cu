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
// Registers per thread follow from the CTAs an SM holds: the 3D tensor-factored
// value sweep runs three CTAs per SM (24 warps, 80 registers), the others two.
__host__ __device__ constexpr int value_min_blocks(int dim, int tq) { return dim == 3 && tq > 0 ? 3 : 2; }
constexpr int FT_TS = 6;                    // doubles per staged target: y(3), nu, log2 nu, s*psi
constexpr int FT_MAXT = 96;                 // target blocks per chunk
constexpr int FT_MAXQ = 80;                 // quadrature points of one source block
constexpr int SUPER = 32;                   // blocks per super-block of the pair-list hierarchy
constexpr int FT_PREF = 192;                // forward entries of a block prefetched into smem

struct FusedArgs {
    const double *x, *rho, *jxw, *cell_ctr;
    const double *tpk;           // per target: y(3), nu, log2 nu, s*psi, -, -
    const int64_t *sblk_cell;    // source block -> first cell (nsblk + 1)
    const double *sblk_sph;      // FP64 centre(3), radius
    const int64_t *tblk_off;     // target block -> first target (ntblk + 1)
    const int64_t *fwd_off;
    const int *fwd_t;
    unsigned *cmask;             // candidate masks: FT_WARPS per forward pair (cell-major within the pair)
    double *Lq;                  // per q (written by the value sweep)
    double *valpart;             // per source block: value, C, skipped, pairs
    double cullt;                // per-target cull radius addend (r, enlarged)
};

// Shared memory of the value sweep: 71 KB, so that three CTAs share an SM.
struct FTSmem {
    double tab[16];
    double stg[FT_TS][FT_MAXS];   // staged targets, structure of arrays (conflict-free lane access)
    double qd[FT_MAXQ][4];        // delta_q (FP64) and C'_q
    double qn[FT_MAXQ];           // |delta_q|
    double cellc[FT_WARPS][3];    // centre of each cell of the block
    unsigned short cand[FT_WARPS][FT_MAXS];
    unsigned cbits[FT_WARPS][FT_MAXS / 32];  // candidate bits of each unit by staged position
    unsigned ebal[FT_MAXT];       // surviving lanes of each entry of the chunk
    short epos[FT_MAXT];          // staged position of each entry's first survivor
    int ecnt[32];                 // survivors per examined forward entry (-1: none)
    int epre[32];                 // staged position of the first survivor of each accepted entry
    int eacc, etot;
    int nstg;
    int ent_j0[FT_PREF];           // forward entries of the block: first target of the target block
    unsigned char ent_sz[FT_PREF]; // and its size (prefetched once per block)
};

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
// (ascending b, the order the gradient gather sums in) and
// inv2fwd[off + rank] = k, the forward position of the same pair.
constexpr int INV_TILE = 2048;
constexpr int INV_PER = INV_TILE / 256;
__global__ void __launch_bounds__(256)
k_inv_order(int nsb, const int64_t *__restrict__ inv_off, const int *__restrict__ tmp_b,
            const int64_t *__restrict__ tmp_k, int *__restrict__ inv_b, int64_t *__restrict__ inv2fwd)
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
            inv2fwd[off + r] = tmp_k[off + i];
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
            inv2fwd[off + i] = tmp_k[off + si[i]];
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
                inv2fwd[off + rank[u]] = tmp_k[off + i];
            }
        }
    }
}

// exclusive scan of n counts into off[0..n] (single CTA, order-fixed)
__global__ void __launch_bounds__(1024) k_scan(const int64_t *__restrict__ cnt, int64_t n, int64_t *__restrict__ off)
{
    // coalesced tiles of 1,024 counts: warp-shuffle inclusive scans, the warp
    // totals scanned by warp 0, a running carry across tiles (integer sums:
    // exact in any order)
    __shared__ long long wsum[32];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    long long carry = 0;
    for (int64_t t0 = 0; t0 < n; t0 += 1024) {
        const int64_t i = t0 + tid;
        const long long v = i < n ? (long long)cnt[i] : 0;
        long long x = v;
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
        const long long before = w > 0 ? wsum[w - 1] : 0;
        if (i < n) off[i] = (int64_t)(carry + before + x - v);
        carry += wsum[31];
        __syncthreads();  // wsum is rewritten by the next tile
    }
    if (tid == 0) off[n] = (int64_t)carry;
}

// ---------------------------------------------------------------------------
// value sweep (CTA <-> source block)
// ---------------------------------------------------------------------------

// Stage the targets of the forward pairs [k0, k1) of block b, culled per
// target against the block sphere: each warp takes target blocks (lane <->
// target), counts its survivors with a ballot, and whole target blocks are
// accepted in list order while the staged total fits FT_MAXS.  Returns the
// number of forward entries consumed; staged order = (target block, slot).
// Per accepted entry e of the chunk: ebal[e] = its surviving lanes, epos[e] =
// the staged position of the first survivor.
template <int DIM>
__device__ int stage_chunk(FTSmem &sm, const FusedArgs &f, int64_t kb, int64_t k0, int64_t k1, const double *bc,
                           double rcull2)
{
    constexpr int SUB = 4;                       // target blocks per warp per iteration
    constexpr int PER = FT_WARPS * SUB;          // entries examined per iteration
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    int total = 0, nb = 0;
    int64_t k = k0;
    while (k < k1 && nb < FT_MAXT) {
        unsigned bal[SUB];
        int64_t jj[SUB];
#pragma unroll
        for (int s = 0; s < SUB; ++s) {
            const int idx = s * FT_WARPS + wp;
            const int64_t e = k + idx;
            bal[s] = 0u;
            jj[s] = 0;
            int cntv = -1;
            if (e < k1 && nb + idx < FT_MAXT) {
                int sz;
                int64_t j0;
                if (e - kb < FT_PREF) {
                    j0 = sm.ent_j0[e - kb];
                    sz = sm.ent_sz[e - kb];
                } else {
                    const int t = f.fwd_t[e];
                    j0 = f.tblk_off[t];
                    sz = (int)(f.tblk_off[t + 1] - j0);
                }
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
            const unsigned bad = __ballot_sync(0xffffffffu, cv < 0 || total + incl > FT_MAXS);
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
                const int64_t j0 = jj[s];
                if ((bal[s] >> lane) & 1u) {
                    const int pos = sm.epre[idx] + __popc(bal[s] & ((1u << lane) - 1u));
                    const double *tp = f.tpk + (j0 + lane) * TPACK;
#pragma unroll
                    for (int d = 0; d < FT_TS; ++d) sm.stg[d][pos] = tp[d];
                }
                if (lane == 0) {
                    sm.ebal[nb + idx] = bal[s];
                    sm.epos[nb + idx] = (short)sm.epre[idx];
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
template <int DIM>
__device__ __forceinline__ double stg_dist2(const FTSmem &sm, int t, const double *c)
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
template <int DIM, int QL, int NQ, int MODE>
__device__ __forceinline__ void value_pairs(const FTSmem &sm, int wp, int lane, int ncand, int qoff, double cc0,
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
template <int DIM, int QL, int MODE>
__device__ __noinline__ void value_pairs_partial(const FTSmem &sm, int wp, int lane, int ncand, int qoff, int nql,
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
// compaction into sm.cand[wp] and the candidate bits by staged position into
// sm.cbits[wp]; returns the count and (through bmax) the largest
// B0_Kj = kappa (psi_j - d2/2)/eps over the candidates.
template <int DIM>
__device__ __forceinline__ int compact_candidates(FTSmem &sm, int wp, int lane, int nstg, const double *cc,
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
            if (lane == 0 && b0 + 32 * u < nstg) sm.cbits[wp][(b0 >> 5) + u] = bal;
            ncand += __popc(bal);
        }
    }
    bmax = warp_max(bmax);
    __syncwarp();
    return ncand;
}

// Candidate masks of the chunk's entries for the warp's cell: bit l of
// cmask[(k + e) * FT_WARPS + cell] is set iff target l of the entry's target
// block is a candidate of the cell (staged, and passed the exact test).
__device__ __forceinline__ void write_masks(const FTSmem &sm, const FusedArgs &f, int wp, int lane, int cl,
                                            int64_t k, int nt)
{
    for (int e = 0; e < nt; ++e) {
        const unsigned eb = sm.ebal[e];
        bool c = false;
        if ((eb >> lane) & 1u) {
            const int pos = sm.epos[e] + __popc(eb & ((1u << lane) - 1u));
            c = (sm.cbits[wp][pos >> 5] >> (pos & 31)) & 1u;
        }
        const unsigned m = __ballot_sync(0xffffffffu, c);
        if (lane == 0) f.cmask[(k + e) * FT_WARPS + cl] = m;
    }
}

// Tensor-product points (TM per dimension, symmetric about the cell centre):
// delta_q = (s_0 a_0, s_1 a_1, s_2 a_2) with s_d in {-1, 0, +1}, so
// 2^(b_qj/16) = nu_j 2^(B0_Kj/16) prod_d 2^(s_d G_Kj,d a_d/16) and one
// candidate costs 1 + DIM exponentials and DIM reciprocals for its TM^DIM
// points.  Sums stay relative to Munit (LSE mode only).
template <int TM, int D>
__host__ __device__ __forceinline__ constexpr int tstride()
{
    return D == 0 ? 1 : (D == 1 ? TM : TM * TM);
}

// The per-q maximum exponent (the reference's m of the log-sum-exp, which
// C_global depends on) is taken exactly, as in value_pairs, but only over the
// candidates that can attain it: b_qj lies within s r |delta|max of B0_Kj, so
// a candidate with B0 below (running max B0) - 2 s r |delta|max is never a
// maximum; thr is that bound relative to Munit.
template <int DIM, int TM, bool TS>
__device__ __forceinline__ void value_pairs_tensor(const FTSmem &sm, int wp, int lane, int ncand, int qoff,
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
        if constexpr (TS) {
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

// Value sweep: per source block, stage its paired targets chunk by chunk,
// find each cell's candidates exactly (and record them as masks per block
// pair for the gradient gather), accumulate the per-point online
// log-sum-exp, and finish each point (L_q, value, C_global, skipped).
template <int DIM, int QL, int MODE, int TQ, bool TS>
__global__ void __launch_bounds__(FT_WARPS * 32, value_min_blocks(DIM, TQ))
k_value_trunc(FusedArgs f, EvalArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FTSmem &sm = *reinterpret_cast<FTSmem *>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    const int b = blockIdx.x;
    if (tid < 16) sm.tab[tid] = c_exp2_tab[tid];
    const int64_t cb0 = f.sblk_cell[b], cb1 = f.sblk_cell[b + 1];
    const int ncell = (int)(cb1 - cb0);
    const int nunit = ncell * a.ngroups;
    const bool valid = wp < nunit;
    const int cl = valid ? wp / a.ngroups : 0;          // cell of this warp (block-local)
    const int grp = valid ? wp - cl * a.ngroups : 0;
    const bool masks = valid && grp == 0;               // one warp per cell records the masks
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

    // Shift of the online sums.  MODE 0/1: Munit = max_j B0_Kj + s r
    // max_q |delta_q| bounds every exponent of the unit from above (|G_Kj| <=
    // s r for a candidate), so no per-pair rescale is needed; exponents are
    // kept relative to Munit (mx too) and a chunk that raises the bound
    // rescales S once.  MODE 2 keeps a per-q lazy shift M[q].
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
        const int nt = stage_chunk<DIM>(sm, f, k0, k, k1, bc, rcull2);
        const int nstg = sm.nstg;
        if (valid) {
            double bmax;
            const int ncand = compact_candidates<DIM>(sm, wp, lane, nstg, cc, a, bmax);
            if (masks) write_masks(sm, f, wp, lane, cl, k, nt);
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
                value_pairs_partial<DIM, QL, MODE>(sm, wp, lane, ncand, qoff, nql, cc[0], cc[1], cc[2], a, Munit, M,
                                                   S, mx);
        }
        k += nt;
        __syncthreads();  // the next chunk overwrites the staged targets
    }
    // merge the lanes of each q (warp max / sum); lane q keeps q's totals
    // and runs q's epilogue, so the QL epilogues proceed in parallel
    double my_mx = -CUDART_INF, my_S = 0.0;
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
    double tv = 0.0, tcv = 0.0, tsk = 0.0;
    if (valid && lane < nql) {
        const int qi = qoff + lane;
        const int64_t qg = qblk0 + qi;
        double v, cv, L;
        int sk;
        value_epilogue(a, MODE == 2 ? my_mx : my_mx + Munit, my_S, sm.qd[qi][3], f.rho[qg], f.jxw[qg], v, cv, L, sk);
        f.Lq[qg] = L;
        tv = v;
        tcv = cv;
        tsk = sk;
    }
    block_partials(tv, tcv, tsk, lane == 0 ? npairs : 0.0, f.valpart);
}

// ---------------------------------------------------------------------------
// gradient gather (CTA <-> target block)
// ---------------------------------------------------------------------------

// Per-cell (and per-point) data of the gradient from the value sweep's L_q.
// Each cell's reference L_K = min over its points of L_q keeps every FP32
// operand small: with delta_q = x_q - c_K and C'_q = -kappa |delta_q|^2/(2 eps),
//   w_q nu_j e^(t_qj - L_q) = 2^(e0_Kj + G'_Kj.delta_q + D_q) w_q,
//   e0_Kj = log2 nu_j + (kappa (psi_j - |y_j - c_K|^2/2)/eps - kappa L_K)/16,
//   G'_Kj = kappa (y_j - c_K)/(16 eps),  D_q = (C'_q - kappa (L_q - L_K))/16.
//   gcell[K] = {c_K, L_K};
//   FP32, tensor points: gten[16 K ..] = {a_0, a_1, a_2, -, W_q = w_q 2^D_q};
//   FP32 otherwise: gq (float4) = {delta_q, D_q + log2 w_q (w >= 0) or D_q}, gqw = w_q;
//   FP64: gq (double4) = {delta_q, C'_q - kappa (L_q - L_K)} (-inf for a
//         skipped point), gqw = w_q.
template <int DIM, int TM, bool FP32B>
__global__ void __launch_bounds__(256)
k_grad_prep(int64_t ncells, int qpc, const double *__restrict__ x, const double *__restrict__ cell_ctr,
            const double *__restrict__ Lq, const double *__restrict__ w, int w_nonneg, EvalArgs a,
            double4 *__restrict__ gcell, float *__restrict__ gten, void *__restrict__ gq, void *__restrict__ gqw)
{
    const int64_t K = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (K >= ncells) return;
    const double c[3] = {cell_ctr[K * DIM], cell_ctr[K * DIM + 1], DIM == 3 ? cell_ctr[K * DIM + 2] : 0.0};
    const int64_t q0 = K * qpc;
    double Lref = CUDART_INF;
    for (int q = 0; q < qpc; ++q) Lref = fmin(Lref, Lq[q0 + q]);
    gcell[K] = make_double4(c[0], c[1], c[2], Lref);
    for (int q = 0; q < qpc; ++q) {
        double dl[3], dsq = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            dl[d] = d < DIM ? x[(q0 + q) * DIM + d] - c[d] : 0.0;
            dsq += dl[d] * dl[d];
        }
        const double Cq = -a.halfs * dsq;
        const double L = Lq[q0 + q];
        const bool fin = isfinite(Lref) && isfinite(L);
        const double wq = w[q0 + q];
        if (FP32B) {
            const double D = fin ? (Cq - KAPPA * (L - Lref)) * (1.0 / 16.0) : -CUDART_INF;
            if (TM > 0) {
                gten[K * 16 + 4 + q] = (float)(wq * exp2(D));
            } else {
                reinterpret_cast<float4 *>(gq)[q0 + q] =
                    make_float4((float)dl[0], (float)dl[1], (float)dl[2], (float)(w_nonneg ? D + log2(wq) : D));
                reinterpret_cast<float *>(gqw)[q0 + q] = (float)wq;
            }
        } else {
            reinterpret_cast<double4 *>(gq)[q0 + q] =
                make_double4(dl[0], dl[1], dl[2], fin ? Cq - KAPPA * (L - Lref) : -CUDART_INF);
            reinterpret_cast<double *>(gqw)[q0 + q] = wq;
        }
        if (TM > 0) {
            // per-dimension offsets of the tensor grid: those of its last point along each axis
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                const int qa = (TM - 1) * (d == 0 ? 1 : (d == 1 ? TM : TM * TM));
                if (q == qa) gten[K * 16 + d] = (float)dl[d];
            }
        }
    }
}

struct GatherArgs {
    const double *tpk;            // per target (internal order): y(3), nu, log2 nu, s*psi
    const int64_t *tblk_off, *inv_off, *inv2fwd;
    const int *inv_b;
    const int64_t *sblk_cell;
    const unsigned *cmask;        // candidate masks per (forward pair, block-local cell)
    const double4 *gcell;
    const float *gten;
    const void *gq, *gqw;
    int qpc;
    int w_nonneg;
    double *gacc;                 // per target (internal order): sum_q w_q pi_qj
};

// One candidate (cell K, target j): sum over the cell's points of
// w_q nu_j e^(t_qj - L_q), with the expansion of k_grad_prep.
template <int DIM, int TM, bool TS, bool FP32B>
__device__ __forceinline__ double grad_term(const GatherArgs &g, const EvalArgs &a, int64_t K, const double4 cd,
                                            const double *y, double l2nu, double spsi, const double *tab)
{
    const double g0 = y[0] - cd.x, g1 = y[1] - cd.y, g2 = DIM == 3 ? y[2] - cd.z : 0.0;
    const double d2 = DIM == 3 ? g0 * g0 + g1 * g1 + g2 * g2 : g0 * g0 + g1 * g1;
    if constexpr (FP32B) {
        float e0 = (float)(l2nu + (fma(-a.halfs, d2, spsi) - KAPPA * cd.w) * (1.0 / 16.0));
        const float sf = (float)(a.s * (1.0 / 16.0));
        const float G[3] = {sf * (float)g0, sf * (float)g1, sf * (float)g2};
        if constexpr (TM > 0) {
            constexpr int NQ = DIM == 3 ? TM * TM * TM : TM * TM;
            const float *ct = g.gten + K * 16;
            const float4 ah = *reinterpret_cast<const float4 *>(ct);
            const float ahv[3] = {ah.x, ah.y, ah.z};
            float W[NQ];
#pragma unroll
            for (int q = 0; q < NQ; ++q) W[q] = ct[4 + q];
            float F[3][TM];
            if constexpr (TS) {
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    const float ga = G[d] * ahv[d];
                    e0 -= ga;
                    const float r = ex2_approx(TM == 2 ? 2.f * ga : ga);
                    F[d][0] = 1.f;
                    F[d][1] = r;
                    if (TM == 3) F[d][2] = r * r;
                }
            } else {
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    const float xp = ex2_approx(G[d] * ahv[d]);
                    F[d][0] = __frcp_rn(xp);
                    F[d][TM - 1] = xp;
                    if (TM == 3) F[d][1] = 1.f;
                }
            }
            float wsum = 0.f;
            if (DIM == 2) {
#pragma unroll
                for (int i0 = 0; i0 < TM; ++i0) {
                    float u = 0.f;
#pragma unroll
                    for (int i1 = 0; i1 < TM; ++i1) u = fmaf(W[i0 + TM * i1], F[1][i1], u);
                    wsum = fmaf(u, F[0][i0], wsum);
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
                    wsum = fmaf(u, F[0][i0], wsum);
                }
            }
            return (double)(ex2_approx(e0) * wsum);
        } else {
            const float4 *qb = reinterpret_cast<const float4 *>(g.gq) + K * g.qpc;
            const float *qw = reinterpret_cast<const float *>(g.gqw) + K * g.qpc;
            float acc0 = 0.f, acc1 = 0.f;
            if (g.w_nonneg) {
                int q = 0;
                for (; q + 1 < g.qpc; q += 2) {
                    const float4 v0 = qb[q], v1 = qb[q + 1];
                    float ea = fmaf(G[0], v0.x, e0 + v0.w), eb = fmaf(G[0], v1.x, e0 + v1.w);
                    ea = fmaf(G[1], v0.y, ea);
                    eb = fmaf(G[1], v1.y, eb);
                    if (DIM == 3) {
                        ea = fmaf(G[2], v0.z, ea);
                        eb = fmaf(G[2], v1.z, eb);
                    }
                    acc0 += ex2_approx(ea);
                    acc1 += ex2_approx(eb);
                }
                if (q < g.qpc) {
                    const float4 v0 = qb[q];
                    float ea = fmaf(G[0], v0.x, e0 + v0.w);
                    ea = fmaf(G[1], v0.y, ea);
                    if (DIM == 3) ea = fmaf(G[2], v0.z, ea);
                    acc0 += ex2_approx(ea);
                }
            } else {
                for (int q = 0; q < g.qpc; ++q) {
                    const float4 v = qb[q];
                    float e = fmaf(G[0], v.x, e0 + v.w);
                    e = fmaf(G[1], v.y, e);
                    if (DIM == 3) e = fmaf(G[2], v.z, e);
                    acc0 = fmaf(qw[q], ex2_approx(e), acc0);
                }
            }
            return (double)(acc0 + acc1);
        }
    } else {
        const double U0 = 16.0 * l2nu + fma(-a.halfs, d2, spsi) - KAPPA * cd.w;
        const double G0 = a.s * g0, G1 = a.s * g1, G2 = a.s * g2;
        const double4 *qd = reinterpret_cast<const double4 *>(g.gq) + K * g.qpc;
        const double *qw = reinterpret_cast<const double *>(g.gqw) + K * g.qpc;
        double acc = 0.0;
        for (int q = 0; q < g.qpc; ++q) {
            const double4 v = qd[q];
            if (v.w == -CUDART_INF) continue;   // skipped point
            double u = fma(G0, v.x, U0 + v.w);
            u = fma(G1, v.y, u);
            if (DIM == 3) u = fma(G2, v.z, u);
            acc = fma(qw[q], exp2_16(u, tab), acc);
        }
        return acc;
    }
}

// gacc[j] = sum over the candidates (K, j) of the cell's gradient term, for
// the targets j of target block t (lane <-> target).  Warp w takes an equal
// contiguous share of t's inverse list (ascending source block) and walks it
// in batches of 32 block pairs: lane i loads pair i's source block, cells and
// the value sweep's candidate masks of its cells (one 32-bit word per cell,
// the bits of t's targets), so neither the exact test nor the staging is
// repeated and the loads of a batch are issued together.  Scanning the
// masks, each lane queues its own candidate cells (GQ deep, in shared
// memory); a step computes one queued cell per lane, taken when every lane
// has one (or a queue is full), so the lanes stay busy although a mask word
// holds about a quarter of the block's targets.  Each lane adds its terms in
// queue order, i.e. in (pair, cell) order; the 8 warp sums are added in warp
// order: no atomics, the order is fixed.
constexpr int GQ = 16;
template <int DIM, int TM, bool TS, bool FP32B>
__global__ void __launch_bounds__(256)
k_grad_gather(GatherArgs g, EvalArgs a)
{
    __shared__ double ws[8][32];
    __shared__ double tab[16];
    __shared__ int queue[8][GQ][32];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (tid < 16) tab[tid] = c_exp2_tab[tid];
    __syncthreads();
    const int t = blockIdx.x;
    const int64_t j = g.tblk_off[t] + lane;
    const bool have = j < g.tblk_off[t + 1];
    double y[3] = {0.0, 0.0, 0.0}, l2nu = 0.0, spsi = 0.0;
    if (have) {
        const double *tp = g.tpk + j * TPACK;
        y[0] = tp[0];
        y[1] = tp[1];
        y[2] = DIM == 3 ? tp[2] : 0.0;
        l2nu = tp[4];
        spsi = tp[5];
    }
    int *qw = &queue[w][0][0];
    int head = 0, tail = 0;
    double acc = 0.0;
    auto step = [&]() {
        if (tail > head) {
            const int K = qw[(head % GQ) * 32 + lane];
            ++head;
            const double4 cd = g.gcell[K];
            if (cd.w < CUDART_INF) acc += grad_term<DIM, TM, TS, FP32B>(g, a, K, cd, y, l2nu, spsi, tab);
        }
    };
    const int64_t q0 = g.inv_off[t], L = g.inv_off[t + 1] - q0;
    const int64_t pa = q0 + (L * w) / 8, pb = q0 + (L * (w + 1)) / 8;
    for (int64_t p0 = pa; p0 < pb; p0 += 32) {
        const int64_t p = p0 + lane;
        int K0 = 0, nc = 0;
        uint4 m0 = make_uint4(0u, 0u, 0u, 0u), m1 = m0;
        if (p < pb) {
            const int b = g.inv_b[p];
            const int64_t k = g.inv2fwd[p];
            const int64_t c0 = g.sblk_cell[b];
            K0 = (int)c0;
            nc = (int)(g.sblk_cell[b + 1] - c0);
            const uint4 *mk = reinterpret_cast<const uint4 *>(g.cmask + k * FT_WARPS);
            m0 = mk[0];
            if (nc > 4) m1 = mk[1];
        }
        const int np = (int)min((int64_t)32, pb - p0);
        for (int i = 0; i < np; ++i) {
            const int K0i = __shfl_sync(0xffffffffu, K0, i), nci = __shfl_sync(0xffffffffu, nc, i);
            unsigned mw[8];
            mw[0] = __shfl_sync(0xffffffffu, m0.x, i);
            mw[1] = __shfl_sync(0xffffffffu, m0.y, i);
            mw[2] = __shfl_sync(0xffffffffu, m0.z, i);
            mw[3] = __shfl_sync(0xffffffffu, m0.w, i);
            mw[4] = __shfl_sync(0xffffffffu, m1.x, i);
            mw[5] = __shfl_sync(0xffffffffu, m1.y, i);
            mw[6] = __shfl_sync(0xffffffffu, m1.z, i);
            mw[7] = __shfl_sync(0xffffffffu, m1.w, i);
#pragma unroll
            for (int c = 0; c < FT_WARPS; ++c) {
                if (c < nci && ((mw[c] >> lane) & 1u)) {
                    qw[(tail % GQ) * 32 + lane] = K0i + c;
                    ++tail;
                }
                if (__all_sync(0xffffffffu, tail > head) || __any_sync(0xffffffffu, tail - head == GQ)) step();
            }
        }
    }
    while (__any_sync(0xffffffffu, tail > head)) step();
    ws[w][lane] = acc;
    __syncthreads();
    if (w == 0 && have) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < 8; ++i) s += ws[i][lane];
        g.gacc[j] = s;
    }
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------

template <int DIM, int QL, int MODE, int TQ, bool TS>
static void launch_value(sdot_ctx *c, const FusedArgs &f, const EvalArgs &a, int nb)
{
    const size_t smem = sizeof(FTSmem);
    cudaFuncSetAttribute(k_value_trunc<DIM, QL, MODE, TQ, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_value_trunc<DIM, QL, MODE, TQ, TS>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
    k_value_trunc<DIM, QL, MODE, TQ, TS><<<(unsigned)nb, FT_WARPS * 32, smem, c->stream>>>(f, a);
}

template <int DIM, int MODE>
static void dispatch_value_q(sdot_ctx *c, const FusedArgs &f, const EvalArgs &a, int nb)
{
    // 2D: units of 4 (order 2) or 9 (order 3 and groups of 9); 3D: 8 or 9.
    if constexpr (DIM == 2) {
        if (a.ql <= 4) launch_value<DIM, 4, MODE, 0, false>(c, f, a, nb);
        else launch_value<DIM, 9, MODE, 0, false>(c, f, a, nb);
    } else {
        if (a.ql <= 8) launch_value<DIM, 8, MODE, 0, false>(c, f, a, nb);
        else launch_value<DIM, 9, MODE, 0, false>(c, f, a, nb);
    }
}

// Variant of the sweeps for this evaluation.  The shift Munit may exceed the
// true maximum exponent of a q by up to 2 s r |delta|max (units of
// 2^(1/16)); beyond 2^500 the lazy form (MODE 2) is used.  Exponents u
// relative to Munit satisfy u >= -s (psi_max - psi_min + r^2/2 + 2 r
// |delta|max); when that is above -16000 the clamp of exp2 is provably
// inactive and dropped (MODE 0).  Tensor-product points: per-dimension
// factors 2^(+-G a/16) stay within 2^300 (FP64 value sweep) and 2^40 (FP32
// gradient); within 2^8 the relative form (no reciprocals) applies (ts).
struct SweepPlan {
    int mode;   // 0, 1, 2
    int tm;     // tensor points per dimension (0: not factored)
    bool ts;
};

static SweepPlan plan_sweeps(const sdot_ctx *c, const EvalArgs &a, double psi_range)
{
    SweepPlan p{0, 0, false};
    const double gap = 2.0 * a.s * a.cull * c->delta_max;
    const double umin = -a.s * (psi_range + 0.5 * a.cull * a.cull + 2.0 * a.cull * c->delta_max);
    const double fac = a.s * a.cull * c->tensor_amax / 16.0;
    if (gap >= 16.0 * 500.0) {
        p.mode = 2;
        return p;
    }
    p.mode = umin > -15000.0 ? 0 : 1;
    const bool tensor = c->tensor_m > 0 && a.lse && a.ngroups == 1 && fac <= 40.0 && umin > -15000.0;
    if (tensor && ((c->dim == 3 && c->tensor_m == 2 && a.ql == 8) ||
                   (c->dim == 2 && ((c->tensor_m == 3 && a.ql == 9) || (c->tensor_m == 2 && a.ql == 4))))) {
        p.mode = 0;
        p.tm = c->tensor_m;
        p.ts = fac <= 4.0;
    }
    return p;
}

template <int DIM>
static void dispatch_value(sdot_ctx *c, const FusedArgs &f, const EvalArgs &a, int nb, const SweepPlan &p)
{
    if (p.tm > 0) {
        if constexpr (DIM == 3) {
            if (p.ts) launch_value<3, 8, 0, 2, true>(c, f, a, nb);
            else launch_value<3, 8, 0, 2, false>(c, f, a, nb);
        } else {
            if (p.tm == 3) {
                if (p.ts) launch_value<2, 9, 0, 3, true>(c, f, a, nb);
                else launch_value<2, 9, 0, 3, false>(c, f, a, nb);
            } else {
                if (p.ts) launch_value<2, 4, 0, 2, true>(c, f, a, nb);
                else launch_value<2, 4, 0, 2, false>(c, f, a, nb);
            }
        }
        return;
    }
    if (p.mode == 2) dispatch_value_q<DIM, 2>(c, f, a, nb);
    else if (p.mode == 1) dispatch_value_q<DIM, 1>(c, f, a, nb);
    else dispatch_value_q<DIM, 0>(c, f, a, nb);
}

template <int DIM, int TM, bool TS, bool FP32B>
static void launch_gather(sdot_ctx *c, const GatherArgs &g, const EvalArgs &a, int ntb)
{
    const unsigned cg = (unsigned)((c->ncells + 255) / 256);
    k_grad_prep<DIM, TM, FP32B><<<cg, 256, 0, c->stream>>>(c->ncells, c->qpc, c->x.p, c->cell_ctr.p, c->Lq.p, c->w.p,
                                                           c->w_nonneg ? 1 : 0, a,
                                                           reinterpret_cast<double4 *>(c->gcell.p), c->gten.p,
                                                           c->gq.p, c->gqw.p);
    k_grad_gather<DIM, TM, TS, FP32B><<<(unsigned)ntb, 256, 0, c->stream>>>(g, a);
}

template <int DIM>
static void dispatch_gather(sdot_ctx *c, const GatherArgs &g, const EvalArgs &a, int ntb, const SweepPlan &p,
                            bool fp32b)
{
    if (fp32b && p.tm > 0) {
        if constexpr (DIM == 3) {
            if (p.ts) launch_gather<3, 2, true, true>(c, g, a, ntb);
            else launch_gather<3, 2, false, true>(c, g, a, ntb);
        } else {
            if (p.tm == 3) {
                if (p.ts) launch_gather<2, 3, true, true>(c, g, a, ntb);
                else launch_gather<2, 3, false, true>(c, g, a, ntb);
            } else {
                if (p.ts) launch_gather<2, 2, true, true>(c, g, a, ntb);
                else launch_gather<2, 2, false, true>(c, g, a, ntb);
            }
        }
        return;
    }
    if (fp32b) launch_gather<DIM, 0, false, true>(c, g, a, ntb);
    else launch_gather<DIM, 0, false, false>(c, g, a, ntb);
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
    std::vector<int> sc((size_t)nss);
    e = cudaMemcpyAsync(sc.data(), c->scount.p, nss * sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_error(c, e, "pair list count");
    int hmax = 1;
    for (int v : sc) hmax = std::max(hmax, v);
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
    if (e == cudaSuccess) e = c->inv2fwd.alloc(npairs + 1);
    if (e == cudaSuccess) e = c->inv_tmpb.alloc(npairs + 1);
    if (e == cudaSuccess) e = c->inv_tmpk.alloc(npairs + 1);
    if (e == cudaSuccess) e = c->inv_cnt.alloc(ntb + 1);
    if (e == cudaSuccess) e = c->inv_off.alloc(ntb + 1);
    if (e == cudaSuccess) e = c->cmask.alloc((size_t)(npairs + 1) * FT_WARPS);
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
    k_inv_order<<<(unsigned)ntb, 256, 0, st>>>(nsb, c->inv_off.p, c->inv_tmpb.p, c->inv_tmpk.p, c->inv_b.p,
                                               c->inv2fwd.p);
    c->klaunch[6] += 9;
    if (c->profiling) cudaEventRecord(c->pev[7], st);

    // 2. value sweep (L_q, value partials, candidate masks per block pair)
    const bool fp32b = c->precision != SDOT_PREC_FP64;
    const double prange = c->scal_host[SC_MAXPSI] - c->scal_host[SC_MINPSI];
    const SweepPlan plan = plan_sweeps(c, a, std::isfinite(prange) ? prange : 1e300);
    const bool gq_needed = !(fp32b && plan.tm > 0);
    e = c->gcell.alloc((size_t)c->ncells * 4);
    if (e == cudaSuccess) e = c->gten.alloc((size_t)c->ncells * 16);
    if (e == cudaSuccess && gq_needed) e = c->gq.alloc((size_t)c->nq * 4);
    if (e == cudaSuccess && gq_needed) e = c->gqw.alloc((size_t)c->nq);
    if (e != cudaSuccess) return cuda_error(c, e, "gradient gather buffers");
    FusedArgs f{};
    f.x = c->x.p; f.rho = c->rho.p; f.jxw = c->jxw.p; f.cell_ctr = c->cell_ctr.p;
    f.tpk = c->tpack.p; f.sblk_cell = c->sblk_cell.p; f.sblk_sph = c->sblk_sph.p; f.tblk_off = c->tblk_off.p;
    f.fwd_off = c->fwd_off.p; f.fwd_t = c->fwd_t.p; f.cmask = c->cmask.p;
    f.Lq = c->Lq.p; f.valpart = c->blkpart.p;
    f.cullt = std::isnan(r) ? 0.0 : std::min(r, 1e300);
    if (c->dim == 2) dispatch_value<2>(c, f, a, nsb, plan);
    else dispatch_value<3>(c, f, a, nsb, plan);
    if (c->profiling) cudaEventRecord(c->pev[2], st);

    // 3. gradient gather (per target block, no atomics, fixed order)
    GatherArgs g{};
    g.tpk = c->tpack.p; g.tblk_off = c->tblk_off.p; g.inv_off = c->inv_off.p; g.inv2fwd = c->inv2fwd.p;
    g.inv_b = c->inv_b.p; g.sblk_cell = c->sblk_cell.p; g.cmask = c->cmask.p;
    g.gcell = reinterpret_cast<const double4 *>(c->gcell.p); g.gten = c->gten.p;
    g.gq = gq_needed ? (const void *)c->gq.p : nullptr;
    g.gqw = gq_needed ? (const void *)c->gqw.p : nullptr;
    g.qpc = c->qpc;
    g.w_nonneg = c->w_nonneg ? 1 : 0;
    g.gacc = c->gpart.p;
    if (c->dim == 2) dispatch_gather<2>(c, g, a, ntb, plan, fp32b);
    else dispatch_gather<3>(c, g, a, ntb, plan, fp32b);
    c->klaunch[2] += 1;
    c->klaunch[3] += 2;
    if (c->profiling) cudaEventRecord(c->pev[3], st);
    return cuda_error(c, cudaGetLastError(), "truncated evaluation");
}

}  // namespace sdot

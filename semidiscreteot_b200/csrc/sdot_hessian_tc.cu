// sdot_hessian_tc.cu -- Hessian of the entropic dual on the tcgen05 tensor cores.
//
//     H = (1/eps) [ diag(sum_q w_q pi_q) - P_w^T P ],   P_w = diag(w) P,
//     pi_qj = nu_j exp(t_qj - L_q),  t_qj = (psi_j - |x_q - y_j|^2 / 2) / eps,
// the same matrix as the FP64 path in sdot_hessian.cu (SotSolver::compute_hessian,
// declared at include/SemiDiscreteOT/solvers/SotSolver.h:343-344).  Here the
// contraction S = P_w^T P runs on tcgen05.mma (kind::f16, BF16 operands, FP32
// accumulators in tensor memory):
//
//  * P is never stored.  A CTA owns a 128 x 256 tile of S (rows a, columns b)
//    and, for every stage of 64 quadrature points, regenerates the 128 rows
//    w_q pi_qa and the 256 rows pi_qb straight into 128B-swizzled K-major
//    shared memory, where one elected thread hands them to tcgen05.mma.
//  * BF16 hi+lo split: v = hi + lo with hi = bf16_rn(v) (nearest even), lo = bf16_rz(v - hi);
//    S ~ Ahi.Bhi + Ahi.Blo + Alo.Bhi (the lo.lo term, ~2^-18 relative, dropped).
//  * Exponents in FP32 with FP64-formed offsets: log2(w_q pi_qj) =
//    E_bj + G_bj . d_q + F_q, where b is the 64-point block of q, c_b its
//    bounding-box centre, d_q = x_q - c_b, and
//       E_bj = log2 nu_j + (log2 e / eps)(psi_j - |y_j - c_b|^2 / 2) - log2 e L_b,
//       G_bj = (log2 e / eps)(y_j - c_b),
//       F_q  = -(log2 e / eps)|d_q|^2 / 2 - log2 e (L_q - L_b) [+ log2 w_q],
//    L_b = min of L_q over the block.  E and G are computed in FP64 per
//    (stage, target) and rounded once, so every FP32 operand is O(1)-O(100)
//    and the exponent error stays ~1e-5 (relative error of pi ~ 1e-5).
//  * Tensor-core FP32 accumulation over all Q points would lose accuracy, so
//    the accumulator is double-buffered in TMEM (2 x 256 columns) and drained
//    into FP64 every `ch` stages; the drain of one chunk overlaps the MMAs of
//    the next.
//  * Upper triangle only: tile (ta, tb) exists iff it holds some b >= a;
//    entries with b > a are written to H[a][b] and mirrored to H[b][a], so H is
//    exactly symmetric.
//
// Targets are in the caller's order (no permutation pass); quadrature points in
// the library's internal order (the sum over q is order-free).  Every mbarrier
// wait is bounded (~1 s of SM clocks); a timeout sets an error flag, the CTA
// waits (bounded) for its MMAs in flight, frees its tensor memory and returns.
// No TMA and no cluster multicast are used.
#include <float.h>
#include <math.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "sdot_device.cuh"
#include "sdot_internal.h"

namespace sdot {

namespace htc {

constexpr int M = 128;               // rows a per tile (MMA M)
constexpr int N = 256;               // columns b per tile (MMA N)
constexpr int KQ = 64;               // quadrature points per stage (one 128-byte swizzle row of BF16)
constexpr int WARPS = 16;
constexpr int THREADS = WARPS * 32;
constexpr int RG = WARPS * 4;        // row groups (4 per warp, 8 lanes = 8 K-chunks each)
static_assert(M % RG == 0, "row split");

constexpr uint32_t A_BYTES = M * KQ * 2;                 // 16 KB
constexpr int QS_STRIDE = 44;                            // floats per K-chunk: dx[8] dy[8] dz[8] fb[8] fa[8] + pad
constexpr uint32_t RAW_BYTES = 32 + KQ * 16 + KQ * 4;    // per-stage inputs as loaded: block {c_b, L_b},
                                                         // points {d, F^B}, points F^A
constexpr int TMEM_COLS = 2 * N;                          // two FP32 accumulators
constexpr int SCR_PER_CTA = M * N;                        // FP64 drain scratch per CTA

// kind::f16 instruction descriptor: D F32 (bits 4-5 = 1), A BF16 (7-9 = 1),
// B BF16 (10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
                           ((uint32_t)(M >> 4) << 24);

// Waits of the stage loop give up after a limit of SM clocks set per context
// (sdot_set_hessian_wait_limit; default WAIT_LIMIT, about 1 s).  The error
// path's wait for the MMAs in flight always uses WAIT_LIMIT, so the tensor
// memory is released only after the last commit has landed.
constexpr long long WAIT_LIMIT = 2000000000ll;  // SM clocks (~1 s)

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Non-blocking test of the same phase (mbarrier.test_wait never suspends).
__device__ __forceinline__ bool mbar_test_nb(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the completion of the phase with the given parity.
// mbarrier.try_wait may suspend the thread in hardware until the phase
// completes (up to a system-dependent time), so with a bound below about
// 1e5 SM clocks the wait polls with the non-blocking test instead, which
// honours the bound to within one poll.
constexpr long long WAIT_POLL_BELOW = 100000;
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit)
{
    if (mbar_test_nb(bar, parity)) return true;
    const long long t0 = clock64();
    if (limit < WAIT_POLL_BELOW) {
        while (!mbar_test_nb(bar, parity))
            if (clock64() - t0 > limit) return false;
        return true;
    }
    while (!mbar_test(bar, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row atoms of
// 1024 bytes (SBO = 1024), descriptor version 1 (bits 46-47), layout type 2
// (SWIZZLE_128B, bits 61-63).  LBO is unused for this layout (set to 16 B).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void umma_bf16(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t accum)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
        "l"(ad), "l"(bd), "r"(IDESC), "r"(accum));
}

__device__ __forceinline__ void umma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Packed FP32 pairs (sm_100 f32x2 arithmetic).
typedef unsigned long long f2;
__device__ __forceinline__ f2 pack2(float a, float b)
{
    f2 r;
    asm("mov.b64 %0, {%1,%2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
// v0, v1 rounded to BF16 (round to nearest even), packed with v0 in the low half.
__device__ __forceinline__ uint32_t bf16x2_rn(float v0, float v1)
{
    uint32_t d;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(v1), "f"(v0));
    return d;
}
__device__ __forceinline__ void unpack2(f2 v, float &a, float &b) { asm("mov.b64 {%0,%1}, %2;" : "=f"(a), "=f"(b) : "l"(v)); }
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c)
{
    f2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ f2 add2(f2 a, f2 b)
{
    f2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b)
{
    f2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b)
{
    f2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// Shared-memory layout per CTA: NS operand stage buffers (Ahi, Alo, Bhi, Blo;
// 128B-swizzled, K-major), two buffers of per-row E/G (float [ROWS][8]:
// E,E,Gx,Gx,Gy,Gy,Gz,Gz) and of per-K-chunk point data (float [8][QS_STRIDE]),
// two raw input buffers, the mbarriers, 1 KB of alignment slack.
// PAIR: the CTA is one of an SM pair that
// runs M = 256 products together (tcgen05 cta_group::2): each CTA holds its
// 128 A rows and half of the 256 B rows of a stage, and its TMEM holds its
// 128 rows x 256 columns of the tile.
template <bool PAIR>
struct Lay {
    static constexpr int NB = PAIR ? N / 2 : N;          // B rows this CTA generates per stage
    static constexpr int ROWS = M + NB;
    static constexpr int RPT = ROWS / RG;
    static constexpr uint32_t B_BYTES = NB * KQ * 2;
    static constexpr uint32_t STAGE_BYTES = 2 * (A_BYTES + B_BYTES);
    static constexpr int NS = PAIR ? 3 : 2;                 // operand stage buffers (PAIR: 64 KB each)
    static constexpr uint32_t OFF_EG = NS * STAGE_BYTES;
    static constexpr uint32_t OFF_QS = OFF_EG + 2 * ROWS * 32;
    static constexpr uint32_t OFF_RAW = OFF_QS + 2 * 8 * QS_STRIDE * 4;
    static constexpr uint32_t OFF_BAR = OFF_RAW + 2 * RAW_BYTES;
    // mbarriers (8 bytes each) from OFF_BAR: NS stage buffers, 2 accumulators,
    // the TMEM address, and with PAIR NS more: the peer's half of each stage
    // buffer is in its shared memory (waited on by the pair's leader)
    static constexpr uint32_t BAR_ACC = 8 * NS;
    static constexpr uint32_t BAR_TSLOT = 8 * (NS + 2);
    static constexpr uint32_t BAR_FULL = 8 * (NS + 3);
    static constexpr uint32_t BAR_READY = BAR_FULL + 8 * NS;   // dual groups: a group's stage is written
    static constexpr uint32_t ABORT_FLAG = BAR_READY + 8 * NS; // dual groups: an int, set on any failed wait
    static constexpr uint32_t SMEM_BYTES = OFF_BAR + 128 + 1024;
    static constexpr int TILE_ROWS = PAIR ? 2 * M : M;     // rows a of a tile
    static_assert(ABORT_FLAG + 4 <= 128, "barrier region");
    static_assert(ROWS % RG == 0 && THREADS >= ROWS + 2 * KQ, "row split");
};
// M = 256 over the pair: M >> 4 = 16 at bits 24-28.
constexpr uint32_t IDESC2 = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | (16u << 24);

__device__ __forceinline__ void umma_bf16_pair(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t accum)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
        "l"(ad), "l"(bd), "r"(IDESC2), "r"(accum));
}

// Arrive on the mbarrier at the same offset in every CTA of the mask once the
// pair's products issued so far are complete.
__device__ __forceinline__ void umma_commit_pair(uint32_t bar, uint16_t mask)
{
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(bar),
                 "h"(mask)
                 : "memory");
}

__device__ __forceinline__ uint32_t cluster_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ void cluster_sync_all()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Arrive (release, cluster scope) on the mbarrier at offset bar of CTA cta of the cluster.
__device__ __forceinline__ void mbar_arrive_remote(uint32_t bar, uint32_t cta)
{
    asm volatile(
        "{\n\t.reg .b32 ra;\n\t"
        "mapa.shared::cluster.u32 ra, %0, %1;\n\t"
        "mbarrier.arrive.release.cluster.shared::cluster.b64 _, [ra];\n\t}" ::"r"(bar),
        "r"(cta)
        : "memory");
}

// Named barrier of one generation group (256 threads); returns the OR of v
// over the group, so that the group leaves its loop together.
__device__ __forceinline__ bool group_bar_or(int id, bool v)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.or.pred p, %2, 256, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(id)
        : "memory");
    return r != 0;
}
__device__ __forceinline__ void group_bar(int id) { asm volatile("bar.sync %0, 256;" ::"r"(id) : "memory"); }
__device__ __forceinline__ void mbar_arrive_local(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Bounded wait with acquire at cluster scope (the phase completed by a remote arrive).
__device__ __forceinline__ bool mbar_wait_cluster(uint32_t bar, uint32_t parity, long long limit)
{
    auto test = [&]() -> bool {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        return ok != 0;
    };
    if (test()) return true;
    const long long t0 = clock64();
    while (!test())
        if (clock64() - t0 > limit) return false;
    return true;
}

// 32 lanes x 16 consecutive 32-bit columns; the wait is in the same asm so the
// registers are never read before the load has landed.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

struct Args {
    const float4 *qa;       // per q: {dx, dy, dz, F^B}
    const float *qb;        // per q: F^A = F^B + log2 w_q
    const double4 *blk;     // per 64-point block: {c_b (3), log2 e * L_b}
    const double4 *tdat;    // per target (caller order, padded): {y - o (3), log2 nu + l2e_eps psi}
    const double *diag;     // per target: sum_q w_q pi_qj = g_j + nu_j
    const int2 *tiles;      // (ta, tb)
    int ntiles;
    int nst;                // stages per tile
    int ch;                 // stages per FP32 accumulation chunk
    int64_t n;
    double l2e_eps;         // log2(e) / eps
    double inv_eps;
    double *scratch;        // SCR_PER_CTA doubles per CTA
    void *H;
    int *err;
    long long wait_limit;   // SM clocks a stage-loop wait may take before the kernel aborts
    // factored generation (2 x 2 x 2 Gauss cells, one per 8-point chunk):
    const float4 *cd;       // per chunk: {dc (3), F_c^B}, {a (3), F_c^A}: cell centre - c_b, half spacing, max F
    const float2 *qw;       // per q: {2^(F^B - F_c^B), 2^(F^A - F_c^A)}
};

// FACT: the stage's 8-point chunks are 2 x 2 x 2 Gauss cells (x fastest,
// offsets +-a about the cell centre), so per (row, cell)
//   2^(E + F_q + G.d_q) = 2^(E + G.dc - G.a + F_c) * prod_d r_d^(i_d) * 2^(F_q - F_c),
//   r_d = 2^(2 G_d a_d), i_d the point's index bit along d, F_c = max_q F_q,
// one ex2 for the cell and one per dimension instead of one per point; the
// point factors 2^(F_q - F_c) <= 1 are formed once per point (k_htc_points).
// Every intermediate is a corner value 2^(E + G.d_q + F_c), within
// prod_d r_d^(+-1) of the cell's largest value, so none leaves FP32 where
// the per-point form would not.
// DG (dual groups, with PAIR): warps 0-7 and 8-15 generate alternate stages,
// each group synchronising on its own named barrier, and warp 16 issues the
// products in stage order once a stage's group has signalled it (and, in the
// pair's leader, once the peer's half has arrived); a group drains its half of
// the accumulator columns.  One group's barrier waits then overlap the other
// group's generation.
constexpr int DG_THREADS = THREADS + 32;
template <int DIM, typename OutT, bool FACT, bool PAIR, bool DG>
__global__ void __launch_bounds__(DG ? DG_THREADS : THREADS, 1) k_hessian_tc(const Args a)
{
    static_assert(!DG || PAIR, "dual groups run on SM pairs");
    using L = Lay<PAIR>;
    constexpr int RGX = DG ? RG / 2 : RG;          // row groups of one generating group
    constexpr int RPTX = L::ROWS / RGX;            // rows per thread per stage
    constexpr int ARPTX = M / RGX;                 // of which A rows
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw_s = smem_u32(smem_raw);
    uint8_t *sm = smem_raw + ((1024u - (raw_s & 1023u)) & 1023u);  // 1024-aligned shared address
    const uint32_t sm_s = smem_u32(sm);
    float *Eg = reinterpret_cast<float *>(sm + L::OFF_EG);
    float *qs = reinterpret_cast<float *>(sm + L::OFF_QS);
    const uint32_t bar0 = sm_s + L::OFF_BAR;   // mbarriers: see Lay
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + L::OFF_BAR + L::BAR_TSLOT);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t rank = PAIR ? cluster_rank() : 0u;
    if (tid == 0) {
        for (int i = 0; i < L::NS + 2; ++i) mbar_init(bar0 + 8 * i, 1);
        if constexpr (PAIR)
            for (int i = 0; i < L::NS; ++i) mbar_init(bar0 + L::BAR_FULL + 8 * i, 1);
        if constexpr (DG) {
            for (int i = 0; i < L::NS; ++i) mbar_init(bar0 + L::BAR_READY + 8 * i, 1);
            *reinterpret_cast<volatile int *>(sm + L::OFF_BAR + L::ABORT_FLAG) = 0;
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        if constexpr (PAIR) {
            asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                         "r"(TMEM_COLS)
                         : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
        } else {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                         "r"(TMEM_COLS)
                         : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        }
    }
    tc_fence_before();
    __syncthreads();
    if constexpr (PAIR) cluster_sync_all();   // both CTAs' barriers are initialised before any remote arrive
    tc_fence_after();
    const uint32_t tmem = *tslot;
    // tiles: one per CTA, or one per pair (PAIR: TILE_ROWS = 256 rows a, this CTA's half at 128 rank)
    const int t0 = PAIR ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
    const int tstride = PAIR ? (int)(gridDim.x >> 1) : (int)gridDim.x;
    const int64_t rhalf = PAIR ? (int64_t)M * rank : 0;

    // ---- staging of the per-stage inputs ----
    // The block and point data of stage g + 2 are copied by cp.async into
    // raw[g % 2] while stage g is generated; at the end of stage g every
    // thread turns one item of raw[(g + 1) % 2] (and its target row, held in
    // registers for the whole tile) into the FP32 operands of stage g + 1.
    uint8_t *raw = sm + L::OFF_RAW;
    const uint32_t rawb_s = sm_s + L::OFF_RAW;
    // staging items are indexed by tid, or with DG by the thread's index in its group
    const int sid = DG ? (tid & 255) : tid;
    double4 pt = make_double4(0, 0, 0, 0);   // target row sid (sid < L::ROWS) of the current tile
    auto load_target = [&](int2 tl) {
        if (sid < L::ROWS) {
            const int64_t j = sid < M ? (int64_t)tl.x * L::TILE_ROWS + rhalf + sid
                                      : (int64_t)tl.y * N + rhalf + (sid - M);
            pt = a.tdat[j];
        }
    };
    auto raw_copy = [&](int buf, int st) {   // 2 + 64 + 16 copies of 16 bytes (FACT: 2 + 16 + 32)
        const uint32_t d = rawb_s + buf * RAW_BYTES;
        if (sid < 2) cp_async16(d + sid * 16, reinterpret_cast<const uint8_t *>(a.blk + st) + sid * 16);
        else if constexpr (FACT) {
            // chunk data: 8 chunks x 2 float4; point factors: 64 float2 = 32 x 16 bytes
            if (sid < 2 + 16) cp_async16(d + 32 + (sid - 2) * 16, a.cd + (int64_t)st * 16 + (sid - 2));
            else if (sid < 2 + 16 + 32)
                cp_async16(d + 32 + 256 + (sid - 18) * 16, a.qw + (int64_t)st * KQ + (sid - 18) * 2);
        } else {
            if (sid < 2 + KQ) cp_async16(d + 32 + (sid - 2) * 16, a.qa + (int64_t)st * KQ + (sid - 2));
            else if (sid < 2 + KQ + KQ / 4) cp_async16(d + 32 + KQ * 16 + (sid - 2 - KQ) * 16, a.qb + (int64_t)st * KQ + (sid - 2 - KQ) * 4);
        }
        cp_async_commit();
    };
    // raw[buf] + pt -> Eg / qs [buf] for one staging item (rows, then points); with DG a
    // group's 256 threads take the rows and then, the first 128, the points
    auto stage_store = [&](int buf, int item) {
        const uint8_t *rb = raw + buf * RAW_BYTES;
        if (item < L::ROWS) {
            const double4 pb = *reinterpret_cast<const double4 *>(rb);
            const double dx = pt.x - pb.x, dy = pt.y - pb.y, dz = DIM == 3 ? pt.z - pb.z : 0.0;
            const float e = (float)(pt.w - 0.5 * a.l2e_eps * (dx * dx + dy * dy + dz * dz) - pb.w);
            const float gx = (float)(a.l2e_eps * dx), gy = (float)(a.l2e_eps * dy), gz = (float)(a.l2e_eps * dz);
            float4 *dst = reinterpret_cast<float4 *>(Eg + (buf * L::ROWS + item) * 8);
            dst[0] = make_float4(e, e, gx, gx);
            dst[1] = make_float4(gy, gy, gz, gz);
        } else if constexpr (FACT) {
            // chunk layout in qs: [0, 3) dc, 3 F_c^B, [4, 7) a, 7 F_c^A,
            // [8, 16) 2^(F^B - F_c^B), [16, 24) 2^(F^A - F_c^A)
            if (item < L::ROWS + KQ) {
                const int p = item - L::ROWS;
                const float2 wv = reinterpret_cast<const float2 *>(rb + 32 + 256)[p];
                float *d = qs + (buf * 8 + (p >> 3)) * QS_STRIDE + (p & 7);
                d[8] = wv.x;
                d[16] = wv.y;
            } else if (item < L::ROWS + 2 * KQ) {
                const int t = item - L::ROWS - KQ;       // 64 threads: chunk t >> 3, float t & 7
                qs[(buf * 8 + (t >> 3)) * QS_STRIDE + (t & 7)] = reinterpret_cast<const float *>(rb + 32)[t];
            }
        } else if (item < L::ROWS + KQ) {
            const int p = item - L::ROWS;            // point p of the stage: K-chunk p >> 3, slot p & 7
            const float4 pq = reinterpret_cast<const float4 *>(rb + 32)[p];
            float *d = qs + (buf * 8 + (p >> 3)) * QS_STRIDE + (p & 7);
            d[0] = pq.x;
            d[8] = pq.y;
            d[16] = pq.z;
            d[24] = pq.w;
        } else if (item < L::ROWS + 2 * KQ) {
            const int p = item - L::ROWS - KQ;
            qs[(buf * 8 + (p >> 3)) * QS_STRIDE + 32 + (p & 7)] = reinterpret_cast<const float *>(rb + 32 + KQ * 16)[p];
        }
    };

    // ---- generation of one stage's operands into shared memory ----
    // Per element: log2(w pi) = E + F + G.d in packed FP32 pairs, one ex2,
    // then v = hi + lo with hi rounded to BF16 and lo = v - hi (exact),
    // truncated to BF16 when packed.
    const int kc = lane & 7;                 // 16-byte chunk (8 points) of the 64-point stage
    const int rg = (DG ? (warp & 7) : warp) * 4 + (lane >> 3);   // row group (of the thread's generating group)
    auto generate = [&](int buf, int sb) {
        const float4 *qv = reinterpret_cast<const float4 *>(qs + (buf * 8 + kc) * QS_STRIDE);
        f2 dx[4], dy[4], dz[4], fa[4], fb[4];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const float4 x4 = qv[0 + h], y4 = qv[2 + h], b4 = qv[6 + h], a4 = qv[8 + h];
            dx[2 * h] = pack2(x4.x, x4.y);
            dx[2 * h + 1] = pack2(x4.z, x4.w);
            dy[2 * h] = pack2(y4.x, y4.y);
            dy[2 * h + 1] = pack2(y4.z, y4.w);
            fb[2 * h] = pack2(b4.x, b4.y);
            fb[2 * h + 1] = pack2(b4.z, b4.w);
            fa[2 * h] = pack2(a4.x, a4.y);
            fa[2 * h + 1] = pack2(a4.z, a4.w);
            if (DIM == 3) {
                const float4 z4 = qv[4 + h];
                dz[2 * h] = pack2(z4.x, z4.y);
                dz[2 * h + 1] = pack2(z4.z, z4.w);
            }
        }
        uint8_t *stage = sm + sb * L::STAGE_BYTES;
        // each row's E/G are loaded one row ahead, before the previous row's
        // stores, so that the rows' chains can overlap
        const float4 *eg0 = reinterpret_cast<const float4 *>(Eg + (buf * L::ROWS + rg) * 8);
        float4 e0 = eg0[0], e1 = eg0[1];
#pragma unroll
        for (int it = 0; it < RPTX; ++it) {
            const bool isA = it < ARPTX;
            const int r = rg + RGX * it;
            const f2 E = pack2(e0.x, e0.y), Gx = pack2(e0.z, e0.w), Gy = pack2(e1.x, e1.y), Gz = pack2(e1.z, e1.w);
            if (it + 1 < RPTX) {
                const float4 *egn = reinterpret_cast<const float4 *>(Eg + (buf * L::ROWS + r + RGX) * 8);
                e0 = egn[0];
                e1 = egn[1];
            }
            uint32_t hw[4], lw[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                f2 u = add2(E, isA ? fa[k] : fb[k]);
                u = fma2(Gx, dx[k], u);
                u = fma2(Gy, dy[k], u);
                if (DIM == 3) u = fma2(Gz, dz[k], u);
                float u0, u1;
                unpack2(u, u0, u1);
                const float v0 = ex2_approx(u0), v1 = ex2_approx(u1);
                // hi: both values rounded to BF16 (nearest even) and packed by one
                // cvt; widened back (shift / mask), lo = v - hi is exact
                const uint32_t hp = bf16x2_rn(v0, v1);
                const f2 lo = sub2(pack2(v0, v1), pack2(__uint_as_float(hp << 16), __uint_as_float(hp & 0xffff0000u)));
                float l0, l1;
                unpack2(lo, l0, l1);
                hw[k] = hp;
                lw[k] = __byte_perm(__float_as_uint(l0), __float_as_uint(l1), 0x7632);
            }
            const int rr = isA ? r : r - M;
            const uint32_t off = (uint32_t)(rr >> 3) * 1024u + (uint32_t)(rr & 7) * 128u + ((uint32_t)(kc ^ (rr & 7)) << 4);
            uint8_t *hi = stage + (isA ? 0u : 2u * A_BYTES);
            uint8_t *lo = hi + (isA ? A_BYTES : L::B_BYTES);
            *reinterpret_cast<uint4 *>(hi + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
            *reinterpret_cast<uint4 *>(lo + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
        }
    };

    // ---- factored generation (FACT): per (row, cell) one ex2 for the cell and
    // one per dimension; the 8 values by products with the point factors ----
    auto generate_fact = [&](int buf, int sb) {
        const float *qc = qs + (buf * 8 + kc) * QS_STRIDE;
        const float4 dc4 = *reinterpret_cast<const float4 *>(qc);
        const float4 a4 = *reinterpret_cast<const float4 *>(qc + 4);
        f2 wb[4], wa[4];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const float4 b4 = *reinterpret_cast<const float4 *>(qc + 8 + 4 * h);
            const float4 c4 = *reinterpret_cast<const float4 *>(qc + 16 + 4 * h);
            wb[2 * h] = pack2(b4.x, b4.y);
            wb[2 * h + 1] = pack2(b4.z, b4.w);
            wa[2 * h] = pack2(c4.x, c4.y);
            wa[2 * h + 1] = pack2(c4.z, c4.w);
        }
        uint8_t *stage = sm + sb * L::STAGE_BYTES;
        const float4 *eg0 = reinterpret_cast<const float4 *>(Eg + (buf * L::ROWS + rg) * 8);
        float4 e0 = eg0[0], e1 = eg0[1];
#pragma unroll
        for (int it = 0; it < RPTX; ++it) {
            const bool isA = it < ARPTX;
            const int r = rg + RGX * it;
            const float E = e0.x, Gx = e0.z, Gy = e1.x, Gz = e1.z;
            if (it + 1 < RPTX) {
                const float4 *egn = reinterpret_cast<const float4 *>(Eg + (buf * L::ROWS + r + RGX) * 8);
                e0 = egn[0];
                e1 = egn[1];
            }
            const float gx = Gx * a4.x, gy = Gy * a4.y, gz = Gz * a4.z;
            float ub = fmaf(Gx, dc4.x, E);
            ub = fmaf(Gy, dc4.y, ub);
            ub = fmaf(Gz, dc4.z, ub);
            ub = ub - (gx + gy + gz) + (isA ? a4.w : dc4.w);
            const float B = ex2_approx(ub);
            const float r0 = ex2_approx(gx + gx), r1 = ex2_approx(gy + gy), r2 = ex2_approx(gz + gz);
            // corners in point order (x fastest): c_q = B * prod_d r_d^(bit d of q)
            f2 cp[4];
            cp[0] = pack2(B, B * r0);
            cp[1] = mul2(cp[0], pack2(r1, r1));
            cp[2] = mul2(cp[0], pack2(r2, r2));
            cp[3] = mul2(cp[1], pack2(r2, r2));
            uint32_t hw[4], lw[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const f2 v = mul2(cp[k], isA ? wa[k] : wb[k]);
                float v0, v1;
                unpack2(v, v0, v1);
                const uint32_t hp = bf16x2_rn(v0, v1);
                const f2 lo = sub2(v, pack2(__uint_as_float(hp << 16), __uint_as_float(hp & 0xffff0000u)));
                float l0, l1;
                unpack2(lo, l0, l1);
                hw[k] = hp;
                lw[k] = __byte_perm(__float_as_uint(l0), __float_as_uint(l1), 0x7632);
            }
            const int rr = isA ? r : r - M;
            const uint32_t off = (uint32_t)(rr >> 3) * 1024u + (uint32_t)(rr & 7) * 128u + ((uint32_t)(kc ^ (rr & 7)) << 4);
            uint8_t *hi = stage + (isA ? 0u : 2u * A_BYTES);
            uint8_t *lo = hi + (isA ? A_BYTES : L::B_BYTES);
            *reinterpret_cast<uint4 *>(hi + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
            *reinterpret_cast<uint4 *>(lo + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
        }
    };

    // ---- drain of one accumulation chunk into FP64 (and the epilogue on a tile's last chunk) ----
    const int quad = warp & 3, cq = warp >> 2;   // TMEM lane quadrant, 64-column quarter
    const int row = quad * 32 + lane;
    double *scr = a.scratch + (size_t)blockIdx.x * SCR_PER_CTA;
    auto drain = [&](unsigned pc, int2 tl, bool first, bool last) -> bool {
        const bool ok = mbar_wait(bar0 + L::BAR_ACC + 8 * (pc & 1), (pc >> 1) & 1, a.wait_limit);
        tc_fence_after();
        // a warp reads its accumulator lanes only when every lane saw the
        // commit land (tcgen05.ld is warp-collective); otherwise the kernel is
        // aborting and the chunk is dropped
        if (!__all_sync(0xffffffffu, ok)) {
            tc_fence_before();
            return false;
        }
        const int64_t ga = (int64_t)tl.x * L::TILE_ROWS + rhalf + row;
        const uint32_t taddr = tmem + (pc & 1) * N + cq * 64 + ((uint32_t)(quad * 32) << 16);
#pragma unroll 1
        for (int c16 = 0; c16 < 4; ++c16) {
            float v[16];
            tmem_ld16(taddr + c16 * 16, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int col = cq * 64 + c16 * 16 + i;
                const size_t idx = (size_t)col * M + row;
                double s = (double)v[i];
                if (!last) {
                    // one thread owns each scratch entry, so a posted add (its result unused) keeps the chunk
                    // order and the rounding of a load + add + store without waiting for the load
                    if (first) scr[idx] = s;
                    else atomicAdd(&scr[idx], s);
                } else {
                    if (!first) s += scr[idx];
                    const int64_t gb = (int64_t)tl.y * N + col;
                    if (ga < a.n && gb < a.n && gb >= ga) {
                        const double h = ((gb == ga ? a.diag[ga] : 0.0) - s) * a.inv_eps;
                        OutT *H = reinterpret_cast<OutT *>(a.H);
                        H[ga * a.n + gb] = (OutT)h;
                        if (gb != ga) H[gb * a.n + ga] = (OutT)h;
                    }
                }
            }
        }
        tc_fence_before();
        return ok;
    };

    if constexpr (DG) {
        // ---- two generation groups (warps 0-7, 8-15) and the MMA warp (16) ----
        volatile int *abort_flag = reinterpret_cast<volatile int *>(sm + L::OFF_BAR + L::ABORT_FLAG);
        const int ntile_cta = t0 < a.ntiles ? (a.ntiles - 1 - t0) / tstride + 1 : 0;
        const int nch = (a.nst + a.ch - 1) / a.ch;            // accumulation chunks per tile
        const int64_t total = (int64_t)ntile_cta * a.nst;      // stages of this CTA
        const int64_t total_ch = (int64_t)ntile_cta * nch;    // chunks of this CTA
        auto tile_of = [&](int64_t gg) { return a.tiles[t0 + (int)(gg / a.nst) * tstride]; };
        if (warp == 2 * (WARPS / 2)) {
            if (lane == 0) {
                bool fail = false;
                unsigned nc[L::NS + 2] = {};   // commits issued (or, in the pair's second CTA, due) per mbarrier
                for (int64_t gg = 0; gg < total; ++gg) {
                    if (*abort_flag) {
                        fail = true;
                        break;
                    }
                    const int sb = (int)(gg % L::NS);
                    const int st = (int)(gg % a.nst);
                    const int64_t c = (gg / a.nst) * nch + st / a.ch;
                    const unsigned cb = (unsigned)(c & 1);
                    const bool first_in_chunk = (st % a.ch) == 0;
                    const bool last_in_chunk = (st % a.ch) == a.ch - 1 || st == a.nst - 1;
                    const uint32_t par = (uint32_t)((gg / L::NS) & 1);
                    // the stage's group has written and fenced it
                    if (!mbar_wait(bar0 + L::BAR_READY + 8 * sb, par, a.wait_limit)) {
                        fail = true;
                        break;
                    }
                    if (rank != 0) {
                        mbar_arrive_remote(bar0 + L::BAR_FULL + 8 * sb, 0);
                        ++nc[sb];
                        if (last_in_chunk) ++nc[L::NS + cb];
                        continue;
                    }
                    if (!mbar_wait_cluster(bar0 + L::BAR_FULL + 8 * sb, par, a.wait_limit)) {
                        fail = true;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sbase = sm_s + sb * L::STAGE_BYTES;
                    const uint32_t dcol = tmem + cb * N;
#pragma unroll
                    for (int kk = 0; kk < KQ / 16; ++kk) {
                        const uint64_t ah = sdesc(sbase + kk * 32), al = sdesc(sbase + A_BYTES + kk * 32);
                        const uint64_t bh = sdesc(sbase + 2 * A_BYTES + kk * 32);
                        const uint64_t bl = sdesc(sbase + 2 * A_BYTES + L::B_BYTES + kk * 32);
                        umma_bf16_pair(dcol, ah, bh, (first_in_chunk && kk == 0) ? 0u : 1u);
                        umma_bf16_pair(dcol, ah, bl, 1u);
                        umma_bf16_pair(dcol, al, bh, 1u);
                    }
                    umma_commit_pair(bar0 + 8 * sb, 3);
                    ++nc[sb];
                    if (last_in_chunk) {
                        umma_commit_pair(bar0 + L::BAR_ACC + 8 * cb, 3);
                        ++nc[L::NS + cb];
                    }
                }
                if (fail) *abort_flag = 1;
                // every commit issued (or due) lands before the tensor memory is released;
                // each mbarrier has at most one phase outstanding here
                for (int i = 0; i < L::NS + 2; ++i)
                    if (nc[i] > 0) mbar_wait(bar0 + 8 * i, (nc[i] - 1) & 1, WAIT_LIMIT);
            }
            __syncwarp();
        } else {
            const int grp = warp >> 3;           // stages grp, grp + 2, ...
            const int gbar = 1 + grp;            // the group's named barrier
            bool gbad = false;
            int64_t next_drain = 0;              // next chunk whose half of the columns this group drains
            auto drain_upto = [&](int64_t cend) {
                while (next_drain < cend) {
                    const int64_t c = next_drain++;
                    const int ci = (int)(c % nch);
                    if (!drain((unsigned)c, a.tiles[t0 + (int)(c / nch) * tstride], ci == 0, ci == nch - 1)) gbad = true;
                }
            };
            int64_t gg = grp;
            if (gg < total) {
                // the inputs of the group's first stage
                load_target(tile_of(gg));
                raw_copy(grp, (int)(gg % a.nst));
                cp_async_wait_all();
                group_bar(gbar);
                stage_store(grp, sid);
                if (sid < 2 * KQ) stage_store(grp, L::ROWS + sid);
                group_bar(gbar);
            }
            bool stop = false;
            for (; gg < total; gg += 2) {
                const int sb = (int)(gg % L::NS);
                const int st = (int)(gg % a.nst);
                const int64_t c = (gg / a.nst) * nch + st / a.ch;
                const bool more = gg + 2 < total;
                // raw[grp] was read by the stage_store of this stage: the inputs of stage gg + 2 go there
                if (more) raw_copy(grp, (int)((gg + 2) % a.nst));
                drain_upto(c);
                // the products that read this buffer NS stages ago must be complete
                if (gg >= L::NS && !mbar_wait(bar0 + 8 * sb, (uint32_t)(((gg / L::NS) - 1) & 1), a.wait_limit))
                    gbad = true;
                if constexpr (FACT) generate_fact(grp, sb);
                else generate(grp, sb);
                fence_async_smem();
                cp_async_wait_all();
                stop = group_bar_or(gbar, gbad || *abort_flag != 0);
                if (stop) break;
                if (sid == 0) mbar_arrive_local(bar0 + L::BAR_READY + 8 * sb);
                if (more) {
                    if ((gg + 2) / a.nst != gg / a.nst) load_target(tile_of(gg + 2));
                    stage_store(grp, sid);
                    if (sid < 2 * KQ) stage_store(grp, L::ROWS + sid);
                }
                group_bar(gbar);
            }
            if (!stop) stop = group_bar_or(gbar, gbad || *abort_flag != 0);
            if (!stop) drain_upto(total_ch);
            if ((stop || gbad) && sid == 0) *abort_flag = 1;
        }
        __syncthreads();
        if (tid == 0 && *abort_flag) atomicExch(a.err, 1);
    } else {
        int g = 0;               // global stage counter (stage-buffer phases)
        unsigned chunk = 0;      // global chunk counter (accumulator phases)
        int pend = -1;
        int2 pend_tl = make_int2(0, 0);
        bool pend_first = false, pend_last = false;
        bool bad = false;        // this thread saw a wait expire
        bool aborted = false;
        unsigned ncommit[L::NS + 2] = {};  // commits issued (or, in a pair's second CTA, due) per mbarrier (thread 0)

        if (t0 < a.ntiles) {
            // stage 0 into Eg/qs[0]; stage 1's inputs into raw[1]
            load_target(a.tiles[t0]);
            raw_copy(0, 0);
            cp_async_wait_all();
            __syncthreads();
            stage_store(0, tid);
            raw_copy(1, a.nst > 1 ? 1 : 0);
            cp_async_wait_all();
        }
        __syncthreads();

        // One block-wide barrier per stage: it publishes the stage's operands to
        // the MMA thread and orders the previous drain's TMEM reads before any MMA
        // that reuses that accumulator.
        for (int t = t0; t < a.ntiles && !aborted; t += tstride) {
            // tile coordinates of this and the next tile, loaded once per tile
            const int2 tl_cur = a.tiles[t];
            const int2 tl_nxt = t + tstride < a.ntiles ? a.tiles[t + tstride] : tl_cur;
            for (int st = 0; st < a.nst; ++st, ++g) {
                const int eb = g & 1;          // stage inputs and E/G, point data: double-buffered
                const int sb = g % L::NS;      // operand stage buffer
                const bool last_of_tile = st + 1 == a.nst;
                const bool has_next = !last_of_tile || t + tstride < a.ntiles;
                raw_copy(eb, (st + 2) % a.nst);     // inputs of stage g + 2 (its point block)
                // the MMAs that read this buffer NS stages ago must be complete
                if (g >= L::NS && !mbar_wait(bar0 + 8 * sb, ((g / L::NS) - 1) & 1, a.wait_limit)) bad = true;
                if constexpr (FACT) generate_fact(eb, sb);
                else generate(eb, sb);
                if (has_next) {
                    if (last_of_tile) load_target(tl_nxt);   // once per tile
                    stage_store(eb ^ 1, tid);
                }
                cp_async_wait_all();
                fence_async_smem();
                if (__syncthreads_or(bad)) { aborted = true; break; }
                const bool first_in_chunk = (st % a.ch) == 0;
                const bool last_in_chunk = (st % a.ch) == a.ch - 1 || st == a.nst - 1;
                const unsigned cb = chunk & 1;
                if (tid == 0) {
                    if constexpr (PAIR) {
                        if (rank != 0) {
                            // this CTA's half of stage g is written (and fenced for the async proxy)
                            mbar_arrive_remote(bar0 + L::BAR_FULL + 8 * sb, 0);
                            // the leader's commits arrive here too
                            ++ncommit[sb];
                            if (last_in_chunk) ++ncommit[L::NS + cb];
                        } else if (!mbar_wait_cluster(bar0 + L::BAR_FULL + 8 * sb, (g / L::NS) & 1, a.wait_limit)) {
                            bad = true;
                        } else {
                            tc_fence_after();
                            const uint32_t sbase = sm_s + sb * L::STAGE_BYTES;
                            const uint32_t dcol = tmem + cb * N;
    #pragma unroll
                            for (int kk = 0; kk < KQ / 16; ++kk) {
                                const uint64_t ah = sdesc(sbase + kk * 32), al = sdesc(sbase + A_BYTES + kk * 32);
                                const uint64_t bh = sdesc(sbase + 2 * A_BYTES + kk * 32);
                                const uint64_t bl = sdesc(sbase + 2 * A_BYTES + L::B_BYTES + kk * 32);
                                umma_bf16_pair(dcol, ah, bh, (first_in_chunk && kk == 0) ? 0u : 1u);
                                umma_bf16_pair(dcol, ah, bl, 1u);
                                umma_bf16_pair(dcol, al, bh, 1u);
                            }
                            umma_commit_pair(bar0 + 8 * sb, 3);
                            ++ncommit[sb];
                            if (last_in_chunk) {
                                umma_commit_pair(bar0 + L::BAR_ACC + 8 * cb, 3);
                                ++ncommit[L::NS + cb];
                            }
                        }
                    } else {
                        tc_fence_after();
                        const uint32_t sbase = sm_s + sb * L::STAGE_BYTES;
                        const uint32_t dcol = tmem + cb * N;
    #pragma unroll
                        for (int kk = 0; kk < KQ / 16; ++kk) {
                            const uint64_t ah = sdesc(sbase + kk * 32), al = sdesc(sbase + A_BYTES + kk * 32);
                            const uint64_t bh = sdesc(sbase + 2 * A_BYTES + kk * 32);
                            const uint64_t bl = sdesc(sbase + 2 * A_BYTES + L::B_BYTES + kk * 32);
                            umma_bf16(dcol, ah, bh, (first_in_chunk && kk == 0) ? 0u : 1u);
                            umma_bf16(dcol, ah, bl, 1u);
                            umma_bf16(dcol, al, bh, 1u);
                        }
                        umma_commit(bar0 + 8 * sb);
                        ++ncommit[sb];
                        if (last_in_chunk) {
                            umma_commit(bar0 + L::BAR_ACC + 8 * cb);
                            ++ncommit[L::NS + cb];
                        }
                    }
                }
                // drain the previous chunk while the tensor core works on this one
                if (first_in_chunk && pend >= 0) {
                    if (!drain((unsigned)pend, pend_tl, pend_first, pend_last)) bad = true;
                    pend = -1;
                }
                if (last_in_chunk) {
                    pend = (int)chunk;
                    pend_tl = tl_cur;
                    pend_first = st < a.ch;
                    pend_last = st == a.nst - 1;
                    ++chunk;
                }
            }
        }
        if (!aborted && pend >= 0) {
            if (!drain((unsigned)pend, pend_tl, pend_first, pend_last)) bad = true;
        }
        if (__syncthreads_or(bad)) aborted = true;
        if (aborted && tid == 0) {
            atomicExch(a.err, 1);
            // Let the MMAs in flight finish, and every commit arrive, before the
            // tensor memory is released and the CTA exits.  Each mbarrier has at
            // most one phase outstanding here (every earlier phase was waited for
            // successfully, or the loop would have stopped there), so waiting for
            // the phase of its last commit, in order, covers them all.
            for (int i = 0; i < L::NS + 2; ++i)
                if (ncommit[i] > 0) mbar_wait(bar0 + 8 * i, (ncommit[i] - 1) & 1, WAIT_LIMIT);
        }
    }
    tc_fence_before();
    __syncthreads();
    // PAIR: neither CTA frees its tensor memory or exits while the pair's
    // products or commits may still reach it
    if constexpr (PAIR) cluster_sync_all();
    tc_fence_after();
    if (warp == 0) {
        if constexpr (PAIR)
            asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
        else
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// Per-target data in the caller's order: tdat[perm[i]] = {y_i - o, log2 nu_i + l2e_eps psi_i},
// diag[perm[i]] = g_i + nu_i.  Padding rows (>= n) get log2 weight -inf (pi = 0).
template <int DIM>
__global__ void k_htc_targets(int64_t n, int64_t npad, const double *__restrict__ y, const double *__restrict__ nu,
                              const double *__restrict__ psi, const double *__restrict__ grad,
                              const int64_t *__restrict__ perm, double ox, double oy, double oz, double l2e_eps,
                              double4 *__restrict__ tdat, double *__restrict__ diag)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npad; i += (int64_t)gridDim.x * blockDim.x) {
        if (i < n) {
            const int64_t j = perm[i];
            const double lw = nu[i] > 0.0 ? log2(nu[i]) + l2e_eps * psi[i] : -CUDART_INF;
            tdat[j] = make_double4(y[i * DIM] - ox, y[i * DIM + 1] - oy, DIM == 3 ? y[i * DIM + 2] - oz : 0.0, lw);
            diag[j] = grad[i] + nu[i];
        } else {
            tdat[i] = make_double4(0.0, 0.0, 0.0, -CUDART_INF);
            diag[i] = 0.0;
        }
    }
}

// One warp per 64-point block: block centre, reference L_b, per-point offsets
// and the per-point exponent terms F^B, F^A.
template <int DIM>
__global__ void k_htc_points(int64_t nq, int nst, const double *__restrict__ x, const double *__restrict__ Lq,
                             const double *__restrict__ w, double ox, double oy, double oz, double l2e_eps,
                             float4 *__restrict__ qa, float *__restrict__ qb, double4 *__restrict__ blk,
                             float4 *__restrict__ cd, float2 *__restrict__ qw)
{
    const int lane = threadIdx.x & 31;
    const int b = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    if (b >= nst) return;
    const double o[3] = {ox, oy, oz};
    double xt[2][3];
    bool valid[2], fin[2];
    double Lv[2];
    double lo[3] = {CUDART_INF, CUDART_INF, CUDART_INF}, hi[3] = {-CUDART_INF, -CUDART_INF, -CUDART_INF};
    double lmin = CUDART_INF;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int64_t q = (int64_t)b * KQ + lane + 32 * h;
        valid[h] = q < nq;
        Lv[h] = valid[h] ? Lq[q] : CUDART_INF;
        fin[h] = valid[h] && isfinite(Lv[h]);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            xt[h][d] = (valid[h] && d < DIM) ? x[q * DIM + d] - o[d] : 0.0;
            if (valid[h]) {
                lo[d] = fmin(lo[d], xt[h][d]);
                hi[d] = fmax(hi[d], xt[h][d]);
            }
        }
        if (fin[h]) lmin = fmin(lmin, Lv[h]);
    }
#pragma unroll
    for (int o2 = 16; o2 > 0; o2 >>= 1) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o2));
            hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o2));
        }
        lmin = fmin(lmin, __shfl_xor_sync(0xffffffffu, lmin, o2));
    }
    double cb[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) cb[d] = (d < DIM && lo[d] <= hi[d]) ? 0.5 * (lo[d] + hi[d]) : 0.0;
    const double lref = isfinite(lmin) ? LOG2E * lmin : 0.0;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int64_t q = (int64_t)b * KQ + lane + 32 * h;
        float4 out = make_float4(0.f, 0.f, 0.f, -CUDART_INF_F);
        float fa = -CUDART_INF_F;
        if (fin[h]) {
            const double dx = xt[h][0] - cb[0], dy = xt[h][1] - cb[1], dz = xt[h][2] - cb[2];
            const double fb = -0.5 * l2e_eps * (dx * dx + dy * dy + dz * dz) - (LOG2E * Lv[h] - lref);
            const double wq = w[q];
            out = make_float4((float)dx, (float)dy, (float)dz, (float)fb);
            fa = wq > 0.0 ? (float)(fb + log2(wq)) : -CUDART_INF_F;
        }
        qa[q] = out;
        qb[q] = fa;
        if (cd) {
            // factored generation: per 8-point chunk (a 2 x 2 x 2 cell, all
            // points valid or none) its centre relative to c_b, its half
            // spacing per dimension and the largest F^B, F^A of its points,
            // rounded to FP32 first so that F_c + (F - F_c) is exact
            const double fbv = fin[h] ? (double)out.w : -CUDART_INF, fav = (double)fa;
            double clo[3], chi[3], mb = fbv, ma = fav;
#pragma unroll
            for (int d = 0; d < 3; ++d) clo[d] = chi[d] = xt[h][d];
#pragma unroll
            for (int o2 = 1; o2 < 8; o2 <<= 1) {
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    clo[d] = fmin(clo[d], __shfl_xor_sync(0xffffffffu, clo[d], o2));
                    chi[d] = fmax(chi[d], __shfl_xor_sync(0xffffffffu, chi[d], o2));
                }
                mb = fmax(mb, __shfl_xor_sync(0xffffffffu, mb, o2));
                ma = fmax(ma, __shfl_xor_sync(0xffffffffu, ma, o2));
            }
            const float mbf = (float)mb, maf = (float)ma;
            qw[q] = make_float2(fbv > -CUDART_INF ? (float)exp2(fbv - (double)mbf) : 0.f,
                                fav > -CUDART_INF ? (float)exp2(fav - (double)maf) : 0.f);
            if ((lane & 7) == 0) {
                const int64_t k = (int64_t)b * 8 + ((lane + 32 * h) >> 3);
                float4 m4 = make_float4(0.f, 0.f, 0.f, -CUDART_INF_F), s4 = m4;
                if (valid[h]) {
                    m4 = make_float4((float)(0.5 * (clo[0] + chi[0]) - cb[0]), (float)(0.5 * (clo[1] + chi[1]) - cb[1]),
                                     (float)(0.5 * (clo[2] + chi[2]) - cb[2]), mbf);
                    s4 = make_float4((float)(0.5 * (chi[0] - clo[0])), (float)(0.5 * (chi[1] - clo[1])),
                                     (float)(0.5 * (chi[2] - clo[2])), maf);
                }
                cd[2 * k] = m4;
                cd[2 * k + 1] = s4;
            }
        }
    }
    if (lane == 0) blk[b] = make_double4(cb[0], cb[1], cb[2], lref);
}

}  // namespace htc

// Tensor-core Hessian at the potential of the last evaluation (c->psi, c->Lq,
// c->grad must come from an untruncated evaluation).  H_dev: n x n row-major in
// the caller's target order, double or float.
int64_t hessian_tc_tiles(int64_t n)
{
    using namespace htc;
    const int64_t na = (n + M - 1) / M, nb = (n + N - 1) / N;
    int64_t k = 0;
    for (int64_t ta = 0; ta < na; ++ta) k += nb - (ta * M) / N;
    return k;
}

sdot_status hessian_tc(sdot_ctx *c, void *H_dev, bool out_f32, int chunk_stages, double *ms_out, int64_t tile_begin,
                       int64_t tile_end)
{
    using namespace htc;
    const int64_t n = c->nt;
    const int64_t na = (n + M - 1) / M, nb = (n + N - 1) / N;
    const int64_t nst = (c->nq + KQ - 1) / KQ;
    if (nst > INT32_MAX / 2) return set_error(c, SDOT_EINVAL, "too many quadrature points for the tensor-core Hessian");
    std::vector<int2> tiles;
    tiles.reserve((size_t)(na * nb));
    for (int64_t ta = 0; ta < na; ++ta)
        for (int64_t tb = (ta * M) / N; tb < nb; ++tb) tiles.push_back(make_int2((int)ta, (int)tb));
    const int64_t ntile1 = (int64_t)tiles.size();
    if (tile_end < 0 || tile_end > ntile1) tile_end = ntile1;
    if (tile_begin < 0) tile_begin = 0;
    if (tile_begin > tile_end) tile_begin = tile_end;
    // The whole matrix runs on SM pairs (256 x 256 tiles, M = 256 products
    // over two SMs) unless that is switched off; a range of the 128 x 256
    // tiles (sharding) runs on single SMs.
    const bool pair = c->hess_pair_mode > 0 && tile_begin == 0 && tile_end == ntile1;
    int64_t npad = std::max(na * M, nb * N);
    if (pair) {
        const int64_t n2 = (n + 2 * M - 1) / (2 * M);
        npad = std::max(npad, n2 * 2 * M);
        tiles.clear();
        for (int64_t ta = 0; ta < n2; ++ta)
            for (int64_t tb = ta; tb < n2; ++tb) tiles.push_back(make_int2((int)ta, (int)tb));
    } else {
        tiles = std::vector<int2>(tiles.begin() + tile_begin, tiles.begin() + tile_end);
    }
    if (tiles.empty()) {
        c->hess_tiles = 0;
        if (ms_out) *ms_out = 0.0;
        return SDOT_OK;
    }
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c->device);
    // PAIR: two CTAs (one cluster) per tile at a time, one CTA per SM
    const int grid = pair ? 2 * (int)std::min<int64_t>((int64_t)(dev_sms / 2), (int64_t)tiles.size())
                          : (int)std::min<int64_t>((int64_t)dev_sms, (int64_t)tiles.size());

    cudaError_t e = c->htc_tdat.alloc((size_t)npad * 4);
    if (e == cudaSuccess) e = c->htc_diag.alloc((size_t)npad);
    if (e == cudaSuccess) e = c->htc_blk.alloc((size_t)nst * 4);
    if (e == cudaSuccess) e = c->htc_qa.alloc((size_t)nst * KQ * 4);
    if (e == cudaSuccess) e = c->htc_qb.alloc((size_t)nst * KQ);
    if (e == cudaSuccess) e = c->htc_tiles.alloc(tiles.size() * 2);
    if (e == cudaSuccess) e = c->htc_scr.alloc((size_t)grid * SCR_PER_CTA);
    if (e == cudaSuccess) e = c->htc_err.alloc(1);
    // Factored generation: 2 x 2 x 2 Gauss cells (8-point chunks of the
    // 64-point stages), with the per-dimension factors r_d = 2^(2 G_d a_d)
    // within 2^(+-24) (|G_d| <= l2e_eps diam): a cell's corner values then stay
    // within 2^72 of its largest value, far inside FP32, and a value lost to
    // an underflowing point factor is below 2^-54 of that largest value.
    const bool fact = c->hess_factored && c->dim == 3 && c->tensor_m == 2 && c->qpc == 8 &&
                      2.0 * (LOG2E / c->prm.epsilon) * c->diam * c->tensor_amax <= 24.0;
    if (e == cudaSuccess && fact) e = c->htc_cd.alloc((size_t)nst * 16 * 4);
    if (e == cudaSuccess && fact) e = c->htc_qw.alloc((size_t)nst * KQ * 2);
    if (e != cudaSuccess) return cuda_error(c, e, "tensor-core Hessian buffers");
    float4 *cdp = fact ? reinterpret_cast<float4 *>(c->htc_cd.p) : nullptr;
    float2 *qwp = fact ? reinterpret_cast<float2 *>(c->htc_qw.p) : nullptr;
    e = cudaMemcpyAsync(c->htc_tiles.p, tiles.data(), tiles.size() * sizeof(int2), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->htc_err.p, 0, sizeof(int), c->stream);
    if (e != cudaSuccess) return cuda_error(c, e, "tensor-core Hessian setup");

    const double l2e_eps = LOG2E / c->prm.epsilon;
    const double *o = c->origin;
    double4 *tdat = reinterpret_cast<double4 *>(c->htc_tdat.p);
    double4 *blk = reinterpret_cast<double4 *>(c->htc_blk.p);
    float4 *qa = reinterpret_cast<float4 *>(c->htc_qa.p);
    const int tgrid = (int)std::min<int64_t>((npad + 255) / 256, 148 * 8);
    const int pgrid = (int)((nst * 32 + 255) / 256);
    cudaEventRecord(c->ev0, c->stream);
    if (c->dim == 2) {
        k_htc_targets<2><<<tgrid, 256, 0, c->stream>>>(n, npad, c->y.p, c->nu.p, c->psi.p, c->grad.p, c->perm.p, o[0],
                                                       o[1], o[2], l2e_eps, tdat, c->htc_diag.p);
        k_htc_points<2><<<pgrid, 256, 0, c->stream>>>(c->nq, (int)nst, c->x.p, c->Lq.p, c->w.p, o[0], o[1], o[2],
                                                      l2e_eps, qa, c->htc_qb.p, blk, nullptr, nullptr);
    } else {
        k_htc_targets<3><<<tgrid, 256, 0, c->stream>>>(n, npad, c->y.p, c->nu.p, c->psi.p, c->grad.p, c->perm.p, o[0],
                                                       o[1], o[2], l2e_eps, tdat, c->htc_diag.p);
        k_htc_points<3><<<pgrid, 256, 0, c->stream>>>(c->nq, (int)nst, c->x.p, c->Lq.p, c->w.p, o[0], o[1], o[2],
                                                      l2e_eps, qa, c->htc_qb.p, blk, cdp, qwp);
    }
    Args a{};
    a.qa = qa;
    a.qb = c->htc_qb.p;
    a.blk = blk;
    a.tdat = tdat;
    a.diag = c->htc_diag.p;
    a.tiles = reinterpret_cast<const int2 *>(c->htc_tiles.p);
    a.ntiles = (int)tiles.size();
    a.nst = (int)nst;
    a.ch = std::max(1, chunk_stages);
    a.n = n;
    a.l2e_eps = l2e_eps;
    a.inv_eps = 1.0 / c->prm.epsilon;
    a.scratch = c->htc_scr.p;
    a.H = H_dev;
    a.err = c->htc_err.p;
    a.wait_limit = c->hess_wait_limit > 0 ? c->hess_wait_limit : WAIT_LIMIT;
    a.cd = cdp;
    a.qw = qwp;
    void (*kern)(const Args) = nullptr;
    const bool dual = pair && c->hess_pair_mode == 2;
    if (dual) {
        if (c->dim == 2) kern = out_f32 ? k_hessian_tc<2, float, false, true, true> : k_hessian_tc<2, double, false, true, true>;
        else if (fact) kern = out_f32 ? k_hessian_tc<3, float, true, true, true> : k_hessian_tc<3, double, true, true, true>;
        else kern = out_f32 ? k_hessian_tc<3, float, false, true, true> : k_hessian_tc<3, double, false, true, true>;
    } else if (pair) {
        if (c->dim == 2) kern = out_f32 ? k_hessian_tc<2, float, false, true, false> : k_hessian_tc<2, double, false, true, false>;
        else if (fact) kern = out_f32 ? k_hessian_tc<3, float, true, true, false> : k_hessian_tc<3, double, true, true, false>;
        else kern = out_f32 ? k_hessian_tc<3, float, false, true, false> : k_hessian_tc<3, double, false, true, false>;
    } else {
        if (c->dim == 2) kern = out_f32 ? k_hessian_tc<2, float, false, false, false> : k_hessian_tc<2, double, false, false, false>;
        else if (fact) kern = out_f32 ? k_hessian_tc<3, float, true, false, false> : k_hessian_tc<3, double, true, false, false>;
        else kern = out_f32 ? k_hessian_tc<3, float, false, false, false> : k_hessian_tc<3, double, false, false, false>;
    }
    c->hess_last_factored = fact;
    c->hess_last_pair = pair ? (dual ? 2 : 1) : 0;
    const uint32_t smem = pair ? Lay<true>::SMEM_BYTES : Lay<false>::SMEM_BYTES;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_error(c, e, "tensor-core Hessian attribute");
    if (c->profiling) cudaEventRecord(c->pev[0], c->stream);
    if (pair) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)grid);
        cfg.blockDim = dim3(dual ? DG_THREADS : THREADS);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = c->stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        e = cudaLaunchKernelEx(&cfg, kern, a);
        if (e != cudaSuccess) return cuda_error(c, e, "tensor-core Hessian launch (SM pairs)");
    } else {
        kern<<<grid, THREADS, smem, c->stream>>>(a);
    }
    if (c->profiling) cudaEventRecord(c->pev[1], c->stream);
    cudaEventRecord(c->ev1, c->stream);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(c, e, "tensor-core Hessian launch");
    int herr = 0;
    e = cudaMemcpyAsync(&herr, c->htc_err.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_error(c, e, "tensor-core Hessian");
    if (c->profiling) {
        float kms = 0.f;
        cudaEventElapsedTime(&kms, c->pev[0], c->pev[1]);
        c->hess_kernel_ms = kms;
    }
    if (ms_out) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        *ms_out = ms;
    }
    c->hess_tiles = (int64_t)tiles.size();
    if (herr) return set_error(c, SDOT_ETIMEOUT, "tensor-core Hessian: a bounded mbarrier wait expired");
    return SDOT_OK;
}

}  // namespace sdot

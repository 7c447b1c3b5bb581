// g3x_lane16.cu -- lane-per-job sm_100a kernel for batched ksw_extend2 in int16x2
// (bwa/src/ksw.cu:303-401).
//
// The same row-synchronous lane-per-job design as the int32 lane kernel (g3x_lane.cu): each
// lane runs its job through the reference's row loop, all lanes start rows together, a row is
// walked in aligned 8-column blocks (first and last block masked to the band, the blocks
// between unmasked), and the row-end bookkeeping (ksw.cu:371-391) runs for all lanes together.
// What differs is the arithmetic of the unmasked blocks: the row buffer (ksw.cu:310) holds, for
// each 8-column block, four int16x2 words of H and four of E, word p holding columns p and p+4.
// One Blackwell DPX int16x2 instruction (__viaddmin_s16x2, __vimax3_s16x2, __viaddmax_s16x2)
// then does one step of the recurrence for two cells of the row, and the words need no
// unpacking or packing.  F runs through the block in its unrolled form,
// F(t) = max(F_in - t e_ins, V(t)), V(t+1) = max(V(t) - e_ins, T(t)): both halves compute the
// prefix V over their four columns at once, and the high half then takes in V(4) from the low.
// The first and last block of a row run the same arithmetic with per-half masks (block_edge),
// and the row end finds the next band eight columns at a time.
//
// Exactness of the 16-bit arithmetic: a job runs here only when every value of its DP fits
// (job_fits_int16): 0 <= h0, K * (h0 + max_score * min(qlen, tlen)) < 2^15 with K the smallest
// power of two >= 1 + max_score, and the gap penalties small enough that every difference stays
// above -2^15.  Then M = H ? H + S : 0 is min(H + S, K H) (equal when H > 0, <= 0 when H == 0,
// and every use clips it to 0 like the reference's 0).  The scheduler routes every other job
// to an int32 kernel.
#include <cuda_runtime.h>
#include "g3x_core.h"
#include "g3x_internal.h"
#include "g3x_stage.cuh"

namespace g3x {

namespace {

constexpr int kLB = 8;

// Blocks per lane: columns up to qcap + 16 (block loads reach (end-1)|7, the row-end scans
// column end <= qcap, the column-of-maximum scan one block further).
__host__ __device__ inline int pc_blocks(int qcap) { return (qcap + 7) / 8 + 2; }
__host__ __device__ inline int pc_nib_words(int len) { return (len + 7) / 8 + 2; }
__host__ __device__ inline size_t pc_warp_bytes(int qcap) {
    return (size_t)32 * pc_blocks(qcap) * 32 + (size_t)128 * pc_nib_words(qcap);
}

template <uint32_t SEL>
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "n"(SEL));
    return r;
}

// Scores of columns p and p+4 of a block as int16x2: byte p of lo and byte p of hi, each
// sign-extended to 16 bits.
template <int p>
__device__ __forceinline__ uint32_t pair_score(uint32_t lo, uint32_t hi) {
    constexpr uint32_t sel = (uint32_t)p | ((8u | p) << 4) | ((4u + p) << 8) | ((8u | (4u + p)) << 12);
    return prmt<sel>(lo, hi);
}

// The warp's row buffers: per lane and block, a uint4 of H pairs and a uint4 of E pairs.
struct Planes {
    uint4* H;
    uint4* E;
    uint32_t* H32;   // the same words, one at a time
    uint32_t* E32;
};

__device__ __forceinline__ int word_of(int c, int L) { return ((((c >> 3) << 5) + L) << 2) + (c & 3); }

__device__ __forceinline__ void set_col(uint32_t* P, int c, int L, int32_t v) {
    uint32_t& w = P[word_of(c, L)];
    w = (c & 4) ? ((w & 0x0000FFFFu) | ((uint32_t)v << 16)) : ((w & 0xFFFF0000u) | ((uint32_t)v & 0xFFFFu));
}

struct LaneJob {
    int job;                 // -1 = none
    int32_t qlen, tlen, w, h0;
    uint32_t t_off;
    int32_t trev;
    Commit K;
    int32_t beg, end;        // band of the next row before the clamps of ksw.cu:338-340
    uint32_t tx, tn, px, pn; // target chunk K.next >> 4 and the next one
};

struct RowState {
    int32_t beg, end, h1, f, m, mjb;
    uint32_t plo, phi;
    uint32_t hlast;          // high half: H of the last column done (int16x2 carry)
};

struct PairConst {
    uint32_t noe_del, ne_del, noe_ins, ne_ins;   // negated penalties in both halves
    uint32_t nt[4];          // (-p e_ins, -(p+4) e_ins)
    uint32_t cv[4];          // (-2^15, -(p+1) e_ins)
    uint32_t kmul;           // 2^k: M = min(H + S, H * 2^k)
};

// An unmasked block in int16x2.  Pair p = columns (p, p+4).  The H word written for column c
// is H(i, c-1): pairs 1..3 take the h pairs of 0..2, pair 0 takes (H(i, jb-1), h(3)).
__device__ __forceinline__ void block_mid(const Planes& P, const uint32_t* __restrict__ qn, int lane,
                                          int32_t jb, RowState& r, const PairConst& pc, int32_t e_ins8) {
    const int at = ((jb >> 3) << 5) + lane;
    const uint4 hq = P.H[at], eq = P.E[at];
    const uint32_t H2[4] = {hq.x, hq.y, hq.z, hq.w}, E2[4] = {eq.x, eq.y, eq.z, eq.w};
    const uint32_t qw = qn[(jb >> 3) * 32 + lane];
    const uint32_t sc_lo = __byte_perm(r.plo, r.phi, qw);
    const uint32_t sc_hi = __byte_perm(r.plo, r.phi, qw >> 16);
    const uint32_t S2[4] = {pair_score<0>(sc_lo, sc_hi), pair_score<1>(sc_lo, sc_hi),
                            pair_score<2>(sc_lo, sc_hi), pair_score<3>(sc_lo, sc_hi)};
    uint32_t M2[4], L2[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        M2[p] = __viaddmin_s16x2(H2[p], S2[p], H2[p] * pc.kmul);
        const uint32_t T2 = __viaddmax_s16x2(M2[p], pc.noe_ins, 0u);
        // per half: the prefix of V over its own four columns, started at 0
        L2[p] = p == 0 ? T2 : __viaddmax_s16x2(L2[p - 1], pc.ne_ins, T2);
    }
    // (V(p+1), V(p+5)): the high half takes in V(4) = low half of L2[3]
    const uint32_t v4 = prmt<0x1010>(L2[3], L2[3]);
    uint32_t Vf[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) Vf[p] = __viaddmax_s16x2(v4, pc.cv[p], L2[p]);
    const uint32_t fin2 = (uint32_t)r.f * 0x00010001u;
    uint32_t h2[4], oe[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const uint32_t vp = p == 0 ? prmt<0x1044>(L2[3], 0u) : Vf[p - 1];   // (V(p), V(p+4))
        const uint32_t F2 = __viaddmax_s16x2(fin2, pc.nt[p], vp);
        h2[p] = __vimax3_s16x2(M2[p], E2[p], F2);
        const uint32_t te = __viaddmax_s16x2(M2[p], pc.noe_del, 0u);
        oe[p] = __viaddmax_s16x2(E2[p], pc.ne_del, te);
    }
    P.H[at] = make_uint4(prmt<0x5432>(r.hlast, h2[3]), h2[0], h2[1], h2[2]);
    P.E[at] = make_uint4(oe[0], oe[1], oe[2], oe[3]);
    const uint32_t bm2 = __vimax3_s16x2(__vimax3_s16x2(h2[0], h2[1], h2[2]), h2[3], h2[3]);
    const int32_t blo = (int32_t)(bm2 & 0xFFFFu), bhi = (int32_t)(bm2 >> 16);
    const int32_t bm = blo > bhi ? blo : bhi;
    if (bm >= r.m) { r.m = bm; r.mjb = jb; }
    r.f = addmax_i32(r.f, -e_ins8, (int32_t)(Vf[3] >> 16));              // F(8)
    r.hlast = h2[3];
}

// Bit t set when column b+t (b a multiple of 8) has a non-zero H or E word.  Every half-word
// is reduced to 0 or 1 by an unsigned min, then the four pairs are summed with weights 1-8 (no
// carry: each half stays below 16), which leaves columns 0-3 in bits 0-3 and 4-7 in bits 16-19.
__device__ __forceinline__ uint32_t nonzero_cols(const Planes& P, int32_t b, int lane) {
    const int at = ((b >> 3) << 5) + lane;
    const uint4 hq = P.H[at], eq = P.E[at];
    const uint32_t one = 0x00010001u;
    const uint32_t z0 = __vimin3_u16x2(hq.x | eq.x, one, one), z1 = __vimin3_u16x2(hq.y | eq.y, one, one);
    const uint32_t z2 = __vimin3_u16x2(hq.z | eq.z, one, one), z3 = __vimin3_u16x2(hq.w | eq.w, one, one);
    const uint32_t s = z0 + 2u * z1 + 4u * z2 + 8u * z3;
    return (s & 0xFu) | ((s >> 12) & 0xF0u);
}

// The first or last block of a row in int16x2 (ksw.cu:346-370 for the columns of [r.beg, r.end)
// in it).  ge[o] holds, per pair word, 0xFFFF in each half whose column offset is >= o.
//  * Columns left of the band get H = 0, so their M <= 0 and their F contribution is 0; with
//    F_in = r.f (0 at a row's first column) the unrolled F of every band column is exact.
//  * The H word of the band's first column is H(i, beg-1), as the scalar loop writes it.
//  * Words right of column end keep their stale values (the band can regrow into them); the
//    row end then sets column end's words as the reference does (ksw.cu:371).
//  * The row maximum takes band columns only (every band H is >= 0, the rest are cleared).
// On return r.h1 = H of the last band column of the block and r.hlast holds it in its high half.
__device__ __forceinline__ void block_edge(const Planes& P, const uint32_t* __restrict__ qn, int lane,
                                           int32_t jb, RowState& r, const PairConst& pc, int32_t e_ins8,
                                           const uint4* __restrict__ ge) {
    const int at = ((jb >> 3) << 5) + lane;
    const uint4 hq = P.H[at], eq = P.E[at];
    const int lo = r.beg > jb ? r.beg - jb : 0;
    const int hi = r.end - jb < kLB ? r.end - jb : kLB;
    const uint4 ga = ge[lo], gh = ge[hi], gw = ge[hi + 1];
    const uint32_t A[4] = {ga.x, ga.y, ga.z, ga.w};
    const uint32_t V[4] = {ga.x & ~gh.x, ga.y & ~gh.y, ga.z & ~gh.z, ga.w & ~gh.w};
    const uint32_t W[4] = {~gw.x, ~gw.y, ~gw.z, ~gw.w};
    const uint32_t Hq[4] = {hq.x, hq.y, hq.z, hq.w}, E2[4] = {eq.x, eq.y, eq.z, eq.w};
    const uint32_t qw = qn[(jb >> 3) * 32 + lane];
    const uint32_t sc_lo = __byte_perm(r.plo, r.phi, qw);
    const uint32_t sc_hi = __byte_perm(r.plo, r.phi, qw >> 16);
    const uint32_t S2[4] = {pair_score<0>(sc_lo, sc_hi), pair_score<1>(sc_lo, sc_hi),
                            pair_score<2>(sc_lo, sc_hi), pair_score<3>(sc_lo, sc_hi)};
    uint32_t M2[4], L2[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const uint32_t H2 = Hq[p] & V[p];
        M2[p] = __viaddmin_s16x2(H2, S2[p], H2 * pc.kmul);
        const uint32_t T2 = __viaddmax_s16x2(M2[p], pc.noe_ins, 0u);
        L2[p] = p == 0 ? T2 : __viaddmax_s16x2(L2[p - 1], pc.ne_ins, T2);
    }
    const uint32_t v4 = prmt<0x1010>(L2[3], L2[3]);
    uint32_t Vf[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) Vf[p] = __viaddmax_s16x2(v4, pc.cv[p], L2[p]);
    const uint32_t fin2 = (uint32_t)r.f * 0x00010001u;
    const uint32_t hin2 = (r.hlast >> 16) * 0x00010001u;
    uint32_t h2[4], hw[4], nh[4], ne[4], hm[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const uint32_t vp = p == 0 ? prmt<0x1044>(L2[3], 0u) : Vf[p - 1];
        const uint32_t F2 = __viaddmax_s16x2(fin2, pc.nt[p], vp);
        h2[p] = __vimax3_s16x2(M2[p], E2[p], F2);
        const uint32_t te = __viaddmax_s16x2(M2[p], pc.noe_del, 0u);
        const uint32_t oe = __viaddmax_s16x2(E2[p], pc.ne_del, te);
        hw[p] = (h2[p] & A[p]) | (hin2 & ~A[p]);    // left of the band: H(i, beg-1)
        ne[p] = (oe & W[p]) | (E2[p] & ~W[p]);
        hm[p] = h2[p] & V[p];
    }
    nh[0] = prmt<0x5432>(r.hlast, hw[3]);
    nh[1] = hw[0]; nh[2] = hw[1]; nh[3] = hw[2];
#pragma unroll
    for (int p = 0; p < 4; ++p) nh[p] = (nh[p] & W[p]) | (Hq[p] & ~W[p]);
    P.H[at] = make_uint4(nh[0], nh[1], nh[2], nh[3]);
    P.E[at] = make_uint4(ne[0], ne[1], ne[2], ne[3]);
    const uint32_t bm2 = __vimax3_s16x2(__vimax3_s16x2(hm[0], hm[1], hm[2]), hm[3], hm[3]);
    const int32_t blo = (int32_t)(bm2 & 0xFFFFu), bhi = (int32_t)(bm2 >> 16);
    const int32_t bm = blo > bhi ? blo : bhi;
    if (bm >= r.m) { r.m = bm; r.mjb = jb; }
    r.f = addmax_i32(r.f, -e_ins8, (int32_t)(Vf[3] >> 16));              // F(8)
    const int t = hi - 1;
    const uint32_t wl = (t & 2) ? ((t & 1) ? h2[3] : h2[2]) : ((t & 1) ? h2[1] : h2[0]);
    r.h1 = (int32_t)((t & 4) ? (wl >> 16) : (wl & 0xFFFFu));
    r.hlast = (uint32_t)r.h1 << 16;
}

__device__ __forceinline__ JobConst job_const(const LaneJob& J, const ScoreParams& sp) {
    JobConst c;
    c.qlen = J.qlen; c.tlen = J.tlen; c.w = J.w; c.h0 = J.h0;
    c.o_del = sp.o_del; c.e_del = sp.e_del; c.o_ins = sp.o_ins; c.e_ins = sp.e_ins;
    c.oe_del = sp.oe_del; c.oe_ins = sp.oe_ins; c.zdrop = sp.zdrop;
    return c;
}

}  // namespace

size_t lane16_smem_per_warp(int qcap) { return pc_warp_bytes(qcap); }

__global__ void __launch_bounds__(128) lane16_kernel(LaunchDesc d, ScoreParams sp) {
    extern __shared__ __align__(16) char smem[];
    __shared__ uint2 pools[5];
    __shared__ uint4 ge[10];
    if (threadIdx.x < 10) {
        const int o = threadIdx.x;
        uint32_t g[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) g[p] = (p >= o ? 0x0000FFFFu : 0u) | (p + 4 >= o ? 0xFFFF0000u : 0u);
        ge[o] = make_uint4(g[0], g[1], g[2], g[3]);
    }
    if (threadIdx.x < 5) {
        uint32_t lo[5], hi[5];
        score_pools(sp, lo, hi);
#pragma unroll
        for (int t = 0; t < 5; ++t)
            if (threadIdx.x == t) pools[t] = make_uint2(lo[t], hi[t]);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int qcap = d.qmax, tcap = d.tmax;
    const int nbc = pc_blocks(qcap);
    char* base = smem + (size_t)warp * pc_warp_bytes(qcap);
    Planes P;
    P.H = reinterpret_cast<uint4*>(base);
    P.E = P.H + 32 * nbc;
    P.H32 = reinterpret_cast<uint32_t*>(P.H);
    P.E32 = reinterpret_cast<uint32_t*>(P.E);
    uint32_t* qn = reinterpret_cast<uint32_t*>(P.E + 32 * nbc);
    const int n = d.count ? *d.count : d.n;
    const int* order = d.order ? d.order + (d.order_off ? *d.order_off : 0) : nullptr;
    const int refill = d.warp_batch ? 32 : (d.refill > 0 ? d.refill : 1);
    PairConst pc;
    pc.noe_del = (uint32_t)(uint16_t)(-sp.oe_del) * 0x00010001u;
    pc.ne_del = (uint32_t)(uint16_t)(-sp.e_del) * 0x00010001u;
    pc.noe_ins = (uint32_t)(uint16_t)(-sp.oe_ins) * 0x00010001u;
    pc.ne_ins = (uint32_t)(uint16_t)(-sp.e_ins) * 0x00010001u;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        pc.nt[p] = (uint32_t)(uint16_t)(-p * sp.e_ins) | ((uint32_t)(uint16_t)(-(p + 4) * sp.e_ins) << 16);
        pc.cv[p] = 0x8000u | ((uint32_t)(uint16_t)(-(p + 1) * sp.e_ins) << 16);
    }
    pc.kmul = 1u << int16_shift(sp.max_sc);
    const int32_t e_ins8 = 8 * sp.e_ins;

    LaneJob J;
    J.job = -1;
    bool exhausted = false;
    unsigned long long busy = 0, idle = 0, waves = 0;
    for (;;) {
        // ---- refill wave: the warp stages one new job for every idle lane, together ----
        const unsigned idle_mask = __ballot_sync(0xFFFFFFFFu, J.job < 0);
        if (!exhausted && __popc(idle_mask) >= (idle_mask == 0xFFFFFFFFu ? 1 : refill)) {
            const int want = __popc(idle_mask);
            int first = 0;
            if (lane == 0) first = atomicAdd(d.queue, want);
            first = __shfl_sync(0xFFFFFFFFu, first, 0);
            if (first + want >= n) exhausted = true;
            ++waves;
            int my_job = -1;
            if ((idle_mask >> lane) & 1u) {
                const int slot = first + __popc(idle_mask & ((1u << lane) - 1u));
                if (slot < n) {
                    const int job = order ? order[slot] : slot;
                    const g3x_job_t jb = d.jobs[job];
                    JobConst c;
                    c.qlen = jb.qlen; c.tlen = jb.tlen; c.h0 = jb.h0;
                    c.o_del = sp.o_del; c.e_del = sp.e_del; c.o_ins = sp.o_ins; c.e_ins = sp.e_ins;
                    c.oe_del = sp.oe_del; c.oe_ins = sp.oe_ins; c.zdrop = sp.zdrop;
                    c.w = clamp_w(jb.w, c.qlen, sp.max_sc, sp.end_bonus, sp.o_del, sp.e_del, sp.o_ins, sp.e_ins);
                    if (c.qlen > qcap || c.tlen > tcap || !job_fits_int16(c, sp.max_sc)) {
                        d.out[job] = g3x_ext_t{0, 0, 0, 0, 0, 0};
                        d.status[job] = G3X_ERR_TOO_LONG;
                        if (d.cells) d.cells[job] = 0;
                    } else {
                        my_job = job;
                        J.job = job;
                        J.qlen = c.qlen; J.tlen = c.tlen; J.w = c.w; J.h0 = c.h0;
                        J.t_off = jb.t_off;
                        J.trev = (jb.flags & G3X_JOB_TREV) != 0;
                        commit_init(J.K, c);
                        J.beg = 0; J.end = c.qlen;
                        J.tx = J.tn = J.px = J.pn = 0;
                        if (c.tlen > 0) load16(d.codes, d.nmask, J.t_off, c.tlen, 0, J.trev, J.tx, J.tn);
                        if (c.tlen > 16) load16(d.codes, d.nmask, J.t_off, c.tlen, 1, J.trev, J.px, J.pn);
                        stage_own_query(d.codes, d.nmask, jb.q_off, c.qlen, (jb.flags & G3X_JOB_QREV) != 0,
                                        (c.qlen + 15) >> 4, qn, lane);
                    }
                }
            }
            // row -1 of every new job (ksw.cu:317-319), the whole warp on one job at a time:
            // H pairs from the closed form, E = 0
            unsigned m = __ballot_sync(0xFFFFFFFFu, my_job >= 0);
            while (m) {
                const int L = __ffs(m) - 1;
                m &= m - 1;
                const int qlen = __shfl_sync(0xFFFFFFFFu, J.qlen, L);
                JobConst c;
                c.qlen = qlen; c.h0 = __shfl_sync(0xFFFFFFFFu, J.h0, L); c.oe_ins = sp.oe_ins; c.e_ins = sp.e_ins;
                const int words = (((qlen + 1) >> 3) + 1) * 4;
                for (int k = lane; k < words; k += 32) {
                    const int b = k >> 2, p = k & 3;
                    const int32_t lo = init_h(8 * b + p, c), hi = init_h(8 * b + p + 4, c);
                    P.H32[((b << 5) + L) * 4 + p] = ((uint32_t)lo & 0xFFFFu) | ((uint32_t)hi << 16);
                    P.E32[((b << 5) + L) * 4 + p] = 0u;
                }
            }
            __syncwarp();
        }
        const bool active = J.job >= 0;
        if (!__any_sync(0xFFFFFFFFu, active)) {
            if (exhausted) break;
            continue;
        }
        const bool run = active && !J.K.stop;

        // ---- row begin (ksw.cu:335-345) ----
        RowState r;
        r.beg = 0; r.end = 0; r.h1 = 0; r.f = 0; r.m = 0; r.mjb = -1; r.plo = 0; r.phi = 0; r.hlast = 0;
        if (run) {
            const int32_t i = J.K.next;
            r.beg = J.beg > i - J.w ? J.beg : i - J.w;
            r.end = J.end < i + J.w + 1 ? J.end : i + J.w + 1;
            if (r.end > J.qlen) r.end = J.qlen;
            if (r.beg == 0) {
                const int32_t h = J.h0 - (sp.o_del + sp.e_del * (i + 1));
                r.h1 = h > 0 ? h : 0;
            }
            if ((i & 15) == 0 && i > 0) {
                J.tx = J.px; J.tn = J.pn;
                const int ch = (i >> 4) + 1;
                if ((ch << 4) < J.tlen) load16(d.codes, d.nmask, J.t_off, J.tlen, ch, J.trev, J.px, J.pn);
            }
            uint32_t code = (J.tx >> ((i & 15) << 1)) & 3u;
            if ((J.tn >> (i & 15)) & 1u) code = 4;
            const uint2 p = pools[code];
            r.plo = p.x;
            r.phi = p.y;
        }
        const bool nonempty = run && r.beg < r.end;
        const int32_t jb0 = r.beg & ~(kLB - 1);
        const int nblk = nonempty ? ((r.end - 1) >> 3) - (r.beg >> 3) + 1 : 0;
        const int kmax = __reduce_max_sync(0xFFFFFFFFu, (unsigned)nblk);
        busy += nblk;
        idle += kmax - nblk;

        // ---- masked first block, unmasked middle blocks in int16x2, masked last block ----
        r.hlast = (uint32_t)r.h1 << 16;
        if (nblk > 0) block_edge(P, qn, lane, jb0, r, pc, e_ins8, ge);
        for (int k = 1; k < kmax - 1; ++k)
            if (k < nblk - 1) block_mid(P, qn, lane, jb0 + k * kLB, r, pc, e_ins8);
        if (nblk > 1) block_edge(P, qn, lane, jb0 + (nblk - 1) * kLB, r, pc, e_ins8, ge);

        // ---- row end (ksw.cu:371-391) ----
        if (run) {
            const int32_t beg = r.beg, end = r.end;
            set_col(P.H32, end, lane, r.h1);
            set_col(P.E32, end, lane, 0);
            RowDone rd;
            rd.m = r.m;
            rd.mj = -1;
            if (r.m > 0) {
                // the last column of the winning block that reaches the maximum; H(i, c) is in
                // the H word of column c+1: columns mjb+1 .. mjb+7 of the block (pairs 1-3 low,
                // pairs 0-3 high) and column mjb+8, the first of the next block
                const int32_t mjb = r.mjb;
                const int32_t lo = mjb > beg ? mjb : beg;
                const int32_t hi = mjb + kLB < end ? mjb + kLB : end;
                const int at = ((mjb >> 3) << 5) + lane;
                const uint4 hq = P.H[at];
                const uint32_t nx = P.H[at + 32].x;
                const uint32_t hs[kLB] = {hq.y, hq.z, hq.w, hq.x >> 16, hq.y >> 16, hq.z >> 16, hq.w >> 16, nx};
#pragma unroll
                for (int t = 0; t < kLB; ++t) {
                    const int32_t c = mjb + t;
                    if (c >= lo && c < hi && (int32_t)(hs[t] & 0xFFFFu) == r.m) rd.mj = c;
                }
            }
            rd.gval = (nonempty ? end : beg) == J.qlen ? r.h1 : -1;
            rd.ncells = nonempty ? end - beg : 0;
            commit_row(J.K, job_const(J, sp), rd);
            if (!J.K.stop) {
                // ksw.cu:388-391, eight columns at a time: the first column of [beg, end) whose
                // H or E word is non-zero (beg itself when the band is empty) ...
                int32_t nb = beg < end ? end : beg;
                for (int32_t b = beg & ~(kLB - 1); b < end; b += kLB) {
                    uint32_t mk = nonzero_cols(P, b, lane);
                    if (b < beg) mk &= ~0u << (beg - b);
                    if (mk) {
                        const int32_t j = b + __ffs(mk) - 1;
                        nb = j < end ? j : end;
                        break;
                    }
                }
                // ... and the last column of [nb, end] whose word is non-zero (nb - 1 if none;
                // end itself when end < nb)
                int32_t last = end < nb ? end : nb - 1;
                if (end >= nb) {
                    for (int32_t b = end & ~(kLB - 1); b >= (nb & ~(kLB - 1)); b -= kLB) {
                        uint32_t mk = nonzero_cols(P, b, lane);
                        if (end - b < kLB - 1) mk &= (2u << (end - b)) - 1u;
                        if (b < nb) mk &= ~0u << (nb - b);
                        if (mk) {
                            last = b + 31 - __clz(mk);
                            break;
                        }
                    }
                }
                J.beg = nb;
                J.end = last + 2 < J.qlen ? last + 2 : J.qlen;
            }
        }
        if (active && J.K.stop) {
            const Commit& K = J.K;
            d.out[J.job] = g3x_ext_t{K.best, K.best_j + 1, K.best_i + 1, K.max_ie + 1, K.gscore, K.max_off};
            d.status[J.job] = G3X_OK;
            if (d.cells) d.cells[J.job] = (int32_t)K.cells;
            J.job = -1;
        }
        __syncwarp();
    }
    if (d.stats) {
        atomicAdd(d.stats + 0, busy);
        atomicAdd(d.stats + 1, idle);
        if (lane == 0) atomicAdd(d.stats + 2, waves);
    }
}

int launch_lane16(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream) {
    const size_t wb = pc_warp_bytes(d.qmax);
    size_t max_smem = 0;
    if (allow_max_smem(lane16_kernel, &max_smem) != cudaSuccess) return G3X_ERR_CUDA;
    if (wb > max_smem) return G3X_ERR_TOO_LONG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return G3X_ERR_CUDA;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int best_wpb = 1, best_warps = 0, best_blocks = 0;
    const int max_wpb = d.warps_per_block > 0 ? d.warps_per_block : 4;
    for (int wpb = 1; wpb <= max_wpb; wpb *= 2) {
        const size_t smem = (size_t)wpb * wb;
        if (smem > max_smem) break;
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lane16_kernel, 32 * wpb, smem);
        if (per_sm * wpb >= best_warps) { best_warps = per_sm * wpb; best_wpb = wpb; best_blocks = per_sm; }
    }
    const size_t smem = (size_t)best_wpb * wb;
    const int blocks = d.blocks > 0 ? d.blocks : sms * (best_blocks > 0 ? best_blocks : 1);
    lane16_kernel<<<blocks, 32 * best_wpb, smem, stream>>>(d, sp);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

}  // namespace g3x

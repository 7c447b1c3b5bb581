// g3x_lane16.cu -- lane-per-job-pair sm_100a kernel for batched ksw_extend2 in int16x2
// (bwa/src/ksw.cu:303-401).
//
// Each lane runs TWO jobs of the batch at once, one in each 16-bit half of its registers, with
// the Blackwell DPX int16x2 instructions: one __viaddmin_s16x2 / __vimax3_s16x2 /
// __viaddmax_s16x2 computes the same step of the recurrence for both jobs.  The two jobs are
// consecutive in the scheduler's order (similar query length, similar row count), start
// together and advance one row per step each, so they are always on the same row; each half
// keeps its own band [beg, end) (ksw.cu:338-340, 388-391), its own row bookkeeping
// (ksw.cu:371-386) and its own output.  A lane walks the union of the two bands in aligned
// blocks of eight columns: blocks inside both bands unmasked, the others with per-half masks
// that leave a half's state and row buffer untouched outside its band.  The warp is
// row-synchronous as in the int32 lane kernel.
//
// Exactness of the 16-bit arithmetic: a job runs here only when every value of its DP fits,
// i.e. 0 <= h0 and K * (h0 + max_score * min(qlen, tlen)) < 2^15, with K the smallest power
// of two >= 1 + max_score.  Then H, E, F < 2^15 / K, M = H ? H + S : 0 is written as
// min(H + S, K * H) (equal when H > 0, <= 0 when H == 0, and every use clips it to 0 like the
// reference's 0), and no sum or difference leaves the int16 range.  The scheduler routes every
// other job to an int32 kernel.
//
// Shared memory per lane: the two jobs' row buffers (ksw.cu:310) as a plane of H words
// (H_a | H_b << 16) and a plane of E words, lane-interleaved like the int32 lane kernel's
// (slot k of lane L is word ((k/4)*32 + L)*4 + k%4), and each job's query as 4-bit codes.
#include <cuda_runtime.h>
#include "g3x_core.h"
#include "g3x_internal.h"
#include "g3x_stage.cuh"

namespace g3x {

namespace {

constexpr int kLB = 8;

__host__ __device__ inline int pair_eh_words(int qcap) { return (qcap + 8 + kLB + 3) & ~3; }
__host__ __device__ inline int pair_nib_words(int len) { return (len + 7) / 8 + 2; }
__host__ __device__ inline size_t pair_warp_bytes(int qcap) {
    return (size_t)128 * (2 * pair_eh_words(qcap) + 2 * pair_nib_words(qcap));
}

__device__ __forceinline__ int ehw(int k, int L) { return (((k >> 2) * 32 + L) << 2) + (k & 3); }

// Scores of column byte t of both jobs as int16x2: byte t of a (job a) and byte t of b (job b),
// each sign-extended to 16 bits, in one prmt.
template <int t>
__device__ __forceinline__ uint32_t pair_score(uint32_t a, uint32_t b) {
    constexpr uint32_t sel = (uint32_t)t | ((8u | t) << 4) | ((4u + t) << 8) | ((8u | (4u + t)) << 12);
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "n"(sel));
    return r;
}

__device__ __forceinline__ int32_t half_of(uint32_t w, int x) {
    return x ? (int32_t)(int16_t)(w >> 16) : (int32_t)(int16_t)(w & 0xFFFFu);
}

struct HalfJob {
    int job;                 // -1 = none
    int32_t qlen, tlen, w, h0;
    uint32_t t_off;
    int32_t trev;
    Commit K;
    int32_t beg, end;        // band of the next row before the clamps of ksw.cu:338-340
    uint32_t tx, tn, px, pn; // target chunk K.next >> 4 and the next one
};

// Row state of both halves.
struct PairRow {
    int32_t beg[2], end[2];  // per half; halves without a row: beg = end = 0
    int32_t m[2], mjb[2];
    uint32_t H1, F;          // int16x2 running H(i, j-1) and F(i, j)
    uint32_t plo[2], phi[2]; // per half: this row's scores by query code
};

struct PairConst {
    uint32_t noe_del, ne_del, noe_ins, ne_ins;   // negated penalties in both halves
    int32_t kshift;
};

// Per-half mask of the halves whose band holds column col (a band may be empty, beg >= end).
__device__ __forceinline__ uint32_t pair_mask(const PairRow& r, int32_t col) {
    const bool va = col >= r.beg[0] && col < r.end[0];
    const bool vb = col >= r.beg[1] && col < r.end[1];
    return (va ? 0x0000FFFFu : 0u) | (vb ? 0xFFFF0000u : 0u);
}

template <bool kMasked>
__device__ __forceinline__ void pair_block(uint32_t* __restrict__ Hp, uint32_t* __restrict__ Ep,
                                           const uint32_t* __restrict__ qa, const uint32_t* __restrict__ qb,
                                           int lane, int32_t jb, PairRow& r, const PairConst& pc) {
    const int at = ehw(jb, lane);
    const uint4 h0 = *reinterpret_cast<const uint4*>(Hp + at);
    const uint4 h1 = *reinterpret_cast<const uint4*>(Hp + at + 128);
    const uint4 e0 = *reinterpret_cast<const uint4*>(Ep + at);
    const uint4 e1 = *reinterpret_cast<const uint4*>(Ep + at + 128);
    const uint32_t Hw[kLB] = {h0.x, h0.y, h0.z, h0.w, h1.x, h1.y, h1.z, h1.w};
    const uint32_t Ew[kLB] = {e0.x, e0.y, e0.z, e0.w, e1.x, e1.y, e1.z, e1.w};
    const uint32_t wa = qa[(jb >> 3) * 32 + lane], wb = qb[(jb >> 3) * 32 + lane];
    const uint32_t sa_lo = __byte_perm(r.plo[0], r.phi[0], wa), sa_hi = __byte_perm(r.plo[0], r.phi[0], wa >> 16);
    const uint32_t sb_lo = __byte_perm(r.plo[1], r.phi[1], wb), sb_hi = __byte_perm(r.plo[1], r.phi[1], wb >> 16);
    uint32_t oH[kLB], oE[kLB], hv[kLB];
    uint32_t H1 = r.H1, F = r.F;
#pragma unroll
    for (int t = 0; t < kLB; ++t) {
        uint32_t S;
        switch (t & 3) {
            case 0: S = pair_score<0>(t < 4 ? sa_lo : sa_hi, t < 4 ? sb_lo : sb_hi); break;
            case 1: S = pair_score<1>(t < 4 ? sa_lo : sa_hi, t < 4 ? sb_lo : sb_hi); break;
            case 2: S = pair_score<2>(t < 4 ? sa_lo : sa_hi, t < 4 ? sb_lo : sb_hi); break;
            default: S = pair_score<3>(t < 4 ? sa_lo : sa_hi, t < 4 ? sb_lo : sb_hi); break;
        }
        const uint32_t H = Hw[t], E = Ew[t];
        const uint32_t M = __viaddmin_s16x2(H, S, H << pc.kshift);
        const uint32_t h = __vimax3_s16x2(M, E, F);
        const uint32_t te = __viaddmax_s16x2(M, pc.noe_del, 0u);
        const uint32_t en = __viaddmax_s16x2(E, pc.ne_del, te);
        const uint32_t tf = __viaddmax_s16x2(M, pc.noe_ins, 0u);
        const uint32_t fn = __viaddmax_s16x2(F, pc.ne_ins, tf);
        if (kMasked) {
            const uint32_t m2 = pair_mask(r, jb + t);
            oH[t] = (H1 & m2) | (H & ~m2);
            oE[t] = (en & m2) | (E & ~m2);
            hv[t] = h | ~m2;                       // -1 in a half outside its band
            F = (fn & m2) | (F & ~m2);
            H1 = (h & m2) | (H1 & ~m2);
        } else {
            oH[t] = H1;
            oE[t] = en;
            hv[t] = h;
            F = fn;
            H1 = h;
        }
    }
    *reinterpret_cast<uint4*>(Hp + at) = make_uint4(oH[0], oH[1], oH[2], oH[3]);
    *reinterpret_cast<uint4*>(Hp + at + 128) = make_uint4(oH[4], oH[5], oH[6], oH[7]);
    *reinterpret_cast<uint4*>(Ep + at) = make_uint4(oE[0], oE[1], oE[2], oE[3]);
    *reinterpret_cast<uint4*>(Ep + at + 128) = make_uint4(oE[4], oE[5], oE[6], oE[7]);
    const uint32_t bm = __vimax3_s16x2(__vimax3_s16x2(hv[0], hv[1], hv[2]), __vimax3_s16x2(hv[3], hv[4], hv[5]),
                                       __vimax3_s16x2(hv[6], hv[7], hv[7]));
    const int32_t ba = (int32_t)(int16_t)(bm & 0xFFFFu), bb = (int32_t)(int16_t)(bm >> 16);
    if (ba >= r.m[0]) { r.m[0] = ba; r.mjb[0] = jb; }   // ties: the later block holds the later column
    if (bb >= r.m[1]) { r.m[1] = bb; r.mjb[1] = jb; }
    r.H1 = H1;
    r.F = F;
}

__device__ __forceinline__ JobConst half_const(const HalfJob& J, const ScoreParams& sp) {
    JobConst c;
    c.qlen = J.qlen; c.tlen = J.tlen; c.w = J.w; c.h0 = J.h0;
    c.o_del = sp.o_del; c.e_del = sp.e_del; c.o_ins = sp.o_ins; c.e_ins = sp.e_ins;
    c.oe_del = sp.oe_del; c.oe_ins = sp.oe_ins; c.zdrop = sp.zdrop;
    return c;
}

// Row begin of half X (ksw.cu:335-345); sets the half's band, first-column H and score pool.
template <int X>
__device__ __forceinline__ void half_begin(HalfJob& J, PairRow& r, const LaunchDesc& d, const ScoreParams& sp,
                                           const uint2* pools, int32_t& h1) {
    h1 = 0;
    r.beg[X] = r.end[X] = 0;
    r.plo[X] = r.phi[X] = 0;
    if (J.job < 0 || J.K.stop) return;
    const int32_t i = J.K.next;
    int32_t beg = J.beg > i - J.w ? J.beg : i - J.w;
    int32_t end = J.end < i + J.w + 1 ? J.end : i + J.w + 1;
    if (end > J.qlen) end = J.qlen;
    if (beg == 0) {
        const int32_t h = J.h0 - (sp.o_del + sp.e_del * (i + 1));
        h1 = h > 0 ? h : 0;
    }
    r.beg[X] = beg;
    r.end[X] = end;
    if ((i & 15) == 0 && i > 0) {
        J.tx = J.px; J.tn = J.pn;
        const int ch = (i >> 4) + 1;
        if ((ch << 4) < J.tlen) load16(d.codes, d.nmask, J.t_off, J.tlen, ch, J.trev, J.px, J.pn);
    }
    uint32_t code = (J.tx >> ((i & 15) << 1)) & 3u;
    if ((J.tn >> (i & 15)) & 1u) code = 4;
    const uint2 p = pools[code];
    r.plo[X] = p.x;
    r.phi[X] = p.y;
}

// Row end of half X (ksw.cu:371-391), then the job's output when it stops.
template <int X>
__device__ __forceinline__ void half_end(HalfJob& J, const PairRow& r, uint32_t* Hp, uint32_t* Ep, int lane,
                                         const LaunchDesc& d, const ScoreParams& sp) {
    if (J.job < 0) return;
    if (!J.K.stop) {
        const uint32_t keep = X ? 0x0000FFFFu : 0xFFFF0000u;
        const int32_t beg = r.beg[X], end = r.end[X];
        const bool nonempty = beg < end;
        const int32_t h1 = half_of(r.H1, X);
        {   // eh[end] = {h1, 0} (ksw.cu:371), in this half only
            const int at = ehw(end, lane);
            Hp[at] = (Hp[at] & keep) | ((uint32_t)(h1 & 0xFFFF) << (16 * X));
            Ep[at] = Ep[at] & keep;
        }
        RowDone rd;
        rd.m = r.m[X];
        rd.mj = -1;
        if (rd.m > 0) {
            const int32_t lo = r.mjb[X] > beg ? r.mjb[X] : beg;
            const int32_t hi = r.mjb[X] + kLB < end ? r.mjb[X] + kLB : end;
            for (int32_t c = hi - 1; c >= lo; --c)
                if (half_of(Hp[ehw(c + 1, lane)], X) == rd.m) { rd.mj = c; break; }
        }
        rd.gval = (nonempty ? end : beg) == J.qlen ? h1 : -1;
        rd.ncells = nonempty ? end - beg : 0;
        const JobConst c = half_const(J, sp);
        commit_row(J.K, c, rd);
        if (!J.K.stop) {
            int32_t j = beg;
            while (j < end && half_of(Hp[ehw(j, lane)], X) == 0 && half_of(Ep[ehw(j, lane)], X) == 0) ++j;
            const int32_t nb = j;
            j = end;
            while (j >= nb && half_of(Hp[ehw(j, lane)], X) == 0 && half_of(Ep[ehw(j, lane)], X) == 0) --j;
            J.beg = nb;
            J.end = j + 2 < J.qlen ? j + 2 : J.qlen;
        }
    }
    if (J.K.stop) {
        const Commit& K = J.K;
        d.out[J.job] = g3x_ext_t{K.best, K.best_j + 1, K.best_i + 1, K.max_ie + 1, K.gscore, K.max_off};
        d.status[J.job] = G3X_OK;
        if (d.cells) d.cells[J.job] = (int32_t)K.cells;
        J.job = -1;
    }
}

// Sets up half J for `job` (ksw.cu:305-333); false (status written) when the job does not
// belong to this kernel.
__device__ __forceinline__ bool half_stage(HalfJob& J, int job, const LaunchDesc& d, const ScoreParams& sp) {
    const g3x_job_t jb = d.jobs[job];
    JobConst c;
    c.qlen = jb.qlen; c.tlen = jb.tlen; c.h0 = jb.h0;
    c.o_del = sp.o_del; c.e_del = sp.e_del; c.o_ins = sp.o_ins; c.e_ins = sp.e_ins;
    c.oe_del = sp.oe_del; c.oe_ins = sp.oe_ins; c.zdrop = sp.zdrop;
    c.w = clamp_w(jb.w, c.qlen, sp.max_sc, sp.end_bonus, sp.o_del, sp.e_del, sp.o_ins, sp.e_ins);
    if (c.qlen > d.qmax || c.tlen > d.tmax || !job_fits_int16(c, sp.max_sc)) {
        d.out[job] = g3x_ext_t{0, 0, 0, 0, 0, 0};
        d.status[job] = G3X_ERR_TOO_LONG;
        if (d.cells) d.cells[job] = 0;
        J.job = -1;
        return false;
    }
    J.job = job;
    J.qlen = c.qlen; J.tlen = c.tlen; J.w = c.w; J.h0 = c.h0;
    J.t_off = jb.t_off;
    J.trev = (jb.flags & G3X_JOB_TREV) != 0;
    commit_init(J.K, c);
    J.beg = 0; J.end = c.qlen;
    J.tx = J.tn = J.px = J.pn = 0;
    if (c.tlen > 0) load16(d.codes, d.nmask, J.t_off, c.tlen, 0, J.trev, J.tx, J.tn);
    if (c.tlen > 16) load16(d.codes, d.nmask, J.t_off, c.tlen, 1, J.trev, J.px, J.pn);
    return true;
}

// The warp writes job `job`'s query codes into half plane q of lane L.
__device__ __forceinline__ void stage_query(uint32_t* q, int L, int job, int lane, const LaunchDesc& d) {
    const g3x_job_t jb = d.jobs[job];
    const int qlen = jb.qlen;
    const bool qrev = (jb.flags & G3X_JOB_QREV) != 0;
    for (int ch = lane; (ch << 4) < qlen; ch += 32) {
        uint32_t x, nb;
        load16(d.codes, d.nmask, jb.q_off, qlen, ch, qrev, x, nb);
        const uint64_t v = nibbles16(x, nb);
        q[(2 * ch) * 32 + L] = (uint32_t)v;
        q[(2 * ch + 1) * 32 + L] = (uint32_t)(v >> 32);
    }
}

}  // namespace

size_t lane16_smem_per_warp(int qcap) { return pair_warp_bytes(qcap); }

__global__ void __launch_bounds__(128) lane16_kernel(LaunchDesc d, ScoreParams sp) {
    extern __shared__ __align__(16) char smem[];
    __shared__ uint2 pools[5];
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
    const int qcap = d.qmax;
    uint32_t* base = reinterpret_cast<uint32_t*>(smem + (size_t)warp * pair_warp_bytes(qcap));
    uint32_t* Hp = base;
    uint32_t* Ep = Hp + 32 * pair_eh_words(qcap);
    uint32_t* qa = Ep + 32 * pair_eh_words(qcap);
    uint32_t* qb = qa + 32 * pair_nib_words(qcap);
    const int n = d.count ? *d.count : d.n;
    const int* order = d.order ? d.order + (d.order_off ? *d.order_off : 0) : nullptr;
    const int refill = d.warp_batch ? 32 : (d.refill > 0 ? d.refill : 1);
    PairConst pc;
    pc.noe_del = (uint32_t)(uint16_t)(-sp.oe_del) * 0x00010001u;
    pc.ne_del = (uint32_t)(uint16_t)(-sp.e_del) * 0x00010001u;
    pc.noe_ins = (uint32_t)(uint16_t)(-sp.oe_ins) * 0x00010001u;
    pc.ne_ins = (uint32_t)(uint16_t)(-sp.e_ins) * 0x00010001u;
    pc.kshift = int16_shift(sp.max_sc);

    HalfJob A, B;
    A.job = B.job = -1;
    bool exhausted = false;
    unsigned long long busy = 0, idle = 0, waves = 0;
    for (;;) {
        // ---- refill wave: every lane whose two jobs are done takes the next two jobs ----
        const unsigned idle_mask = __ballot_sync(0xFFFFFFFFu, A.job < 0 && B.job < 0);
        if (!exhausted && __popc(idle_mask) >= (idle_mask == 0xFFFFFFFFu ? 1 : refill)) {
            const int want = __popc(idle_mask);
            int first = 0;
            if (lane == 0) first = atomicAdd(d.queue, 2 * want);
            first = __shfl_sync(0xFFFFFFFFu, first, 0);
            if (first + 2 * want >= n) exhausted = true;
            ++waves;
            int ja = -1, jbj = -1;
            if ((idle_mask >> lane) & 1u) {
                const int slot = first + 2 * __popc(idle_mask & ((1u << lane) - 1u));
                if (slot < n && half_stage(A, order ? order[slot] : slot, d, sp)) ja = A.job;
                if (slot + 1 < n && half_stage(B, order ? order[slot + 1] : slot + 1, d, sp)) jbj = B.job;
            }
            unsigned m = __ballot_sync(0xFFFFFFFFu, ja >= 0 || jbj >= 0);
            while (m) {
                const int L = __ffs(m) - 1;
                m &= m - 1;
                const int job_a = __shfl_sync(0xFFFFFFFFu, ja, L);
                const int job_b = __shfl_sync(0xFFFFFFFFu, jbj, L);
                JobConst ca, cb;
                ca.qlen = cb.qlen = 0; ca.h0 = cb.h0 = 0;
                ca.oe_ins = cb.oe_ins = sp.oe_ins; ca.e_ins = cb.e_ins = sp.e_ins;
                if (job_a >= 0) { stage_query(qa, L, job_a, lane, d); ca.qlen = d.jobs[job_a].qlen; ca.h0 = d.jobs[job_a].h0; }
                if (job_b >= 0) { stage_query(qb, L, job_b, lane, d); cb.qlen = d.jobs[job_b].qlen; cb.h0 = d.jobs[job_b].h0; }
                const int top = (ca.qlen > cb.qlen ? ca.qlen : cb.qlen) + 1;
                for (int k = lane; k <= top; k += 32) {
                    const uint32_t va = job_a >= 0 ? (uint32_t)init_h(k, ca) & 0xFFFFu : 0u;
                    const uint32_t vb = job_b >= 0 ? (uint32_t)init_h(k, cb) & 0xFFFFu : 0u;
                    Hp[ehw(k, L)] = va | (vb << 16);
                    Ep[ehw(k, L)] = 0u;
                }
            }
            __syncwarp();
        }
        const bool active = A.job >= 0 || B.job >= 0;
        if (!__any_sync(0xFFFFFFFFu, active)) {
            if (exhausted) break;
            continue;
        }

        // ---- row begin for both halves ----
        PairRow r;
        int32_t ha, hb;
        half_begin<0>(A, r, d, sp, pools, ha);
        half_begin<1>(B, r, d, sp, pools, hb);
        r.H1 = ((uint32_t)ha & 0xFFFFu) | ((uint32_t)hb << 16);
        r.F = 0;
        r.m[0] = r.m[1] = 0;
        r.mjb[0] = r.mjb[1] = -1;
        const bool na = r.beg[0] < r.end[0], nb = r.beg[1] < r.end[1];
        // union of the two bands, and the blocks inside both
        int nh = 0, nf = 0, nt = 0;
        int32_t ub0 = 0, fb0 = 0, fb1 = 0;
        if (na || nb) {
            const int32_t ubeg = na && nb ? min(r.beg[0], r.beg[1]) : (na ? r.beg[0] : r.beg[1]);
            const int32_t uend = na && nb ? max(r.end[0], r.end[1]) : (na ? r.end[0] : r.end[1]);
            ub0 = ubeg & ~(kLB - 1);
            if (na && nb) {
                fb0 = (max(r.beg[0], r.beg[1]) + kLB - 1) & ~(kLB - 1);
                fb1 = min(r.end[0], r.end[1]) & ~(kLB - 1);
            }
            if (na && nb && fb1 > fb0) {
                nh = (fb0 - ub0) >> 3;
                nf = (fb1 - fb0) >> 3;
                nt = (uend - fb1 + kLB - 1) >> 3;
            } else {
                nh = (uend - ub0 + kLB - 1) >> 3;
                fb0 = fb1 = ub0 + nh * kLB;
            }
        }
        const int kh = __reduce_max_sync(0xFFFFFFFFu, (unsigned)nh);
        const int kf = __reduce_max_sync(0xFFFFFFFFu, (unsigned)nf);
        const int kt = __reduce_max_sync(0xFFFFFFFFu, (unsigned)nt);
        busy += nh + nf + nt;
        idle += (kh + kf + kt) - (nh + nf + nt);

        // ---- the union's blocks: masked head, unmasked middle, masked tail ----
        for (int k = 0; k < kh; ++k)
            if (k < nh) pair_block<true>(Hp, Ep, qa, qb, lane, ub0 + k * kLB, r, pc);
        for (int k = 0; k < kf; ++k)
            if (k < nf) pair_block<false>(Hp, Ep, qa, qb, lane, fb0 + k * kLB, r, pc);
        for (int k = 0; k < kt; ++k)
            if (k < nt) pair_block<true>(Hp, Ep, qa, qb, lane, fb1 + k * kLB, r, pc);

        // ---- row end for both halves ----
        half_end<0>(A, r, Hp, Ep, lane, d, sp);
        half_end<1>(B, r, Hp, Ep, lane, d, sp);
        __syncwarp();
    }
    if (d.stats) {
        atomicAdd(d.stats + 0, busy);
        atomicAdd(d.stats + 1, idle);
        if (lane == 0) atomicAdd(d.stats + 2, waves);
    }
}

int launch_lane16(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream) {
    const size_t wb = pair_warp_bytes(d.qmax);
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

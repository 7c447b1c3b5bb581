// g3x_lane.cu -- lane-per-job sm_100a kernel for batched ksw_extend2 (bwa/src/ksw.cu:303-401).
//
// Each lane of a warp runs one job through the reference's own row loop: rows in order, the
// reference's band [beg, end) per row (ksw.cu:338-340, 388-391) and the per-row bookkeeping of
// ksw.cu:371-386, so the semantics are the scalar loop's by construction.  The warp is
// row-synchronous: every lane starts its job's next row at the same time, walks it in aligned
// blocks of eight columns (the first and last block of a row masked to [beg, end), the blocks
// between them unmasked), and all lanes do the row-end bookkeeping together.  The 32 jobs of a
// warp are chosen by the scheduler to have rows of similar width, so few lanes wait.
//
// Per cell the lane keeps no bookkeeping besides its running H and F: the row maximum is taken
// per block (three-input maxima), and the column that reaches it (the last one, ksw.cu:364) is
// found at row end among the eight H values of the winning block, which the row buffer holds
// (eh[c+1].h = H(i, c), ksw.cu:350 and 371).  The next row's band is found as the reference
// finds it, by scanning the row buffer from both ends (ksw.cu:388-391); beg only grows and end
// regrows by at most two columns per row, so the scans take O(1) steps per row on average.
//
// Shared memory holds, per lane, the row buffer (ksw.cu:310) as 16-bit H | 16-bit E words
// (jobs with 0 <= h0 and H <= h0 + max_score * min(qlen, tlen) < 2^15) and the query as 4-bit
// codes, both lane-interleaved so that every access of the warp is free of bank conflicts
// whatever column each lane is at: row-buffer slot k of lane L is word ((k/4)*32 + L)*4 + k%4,
// so an aligned 8-column block is two 16-byte loads.  The target is read from the packed
// planes in global memory, sixteen codes at a time, one chunk ahead.  Idle lanes are refilled
// in waves at row boundaries: when at least `refill` lanes of the warp are idle, the whole warp
// stages one new job per idle lane together.
//
// Ring variant (kRing, for queries longer than the band): a row only touches columns
// [beg, end] inside [i-w, i+w+1], columns left of beg are never read again (beg never
// decreases), and a column right of every band so far still holds its row -1 value.  So the
// row buffer and the query codes live in rings of R >= 2w+16 columns (column c in slot
// c mod R): the valid columns a row reads or writes span at most 2w+2, so no two of them share
// a slot, and every column entering the band for the first time is given its row -1 value
// (ksw.cu:317-319) first.  Shared memory then no longer grows with the query.
#include <cuda_runtime.h>
#include "g3x_core.h"
#include "g3x_internal.h"
#include "g3x_stage.cuh"

namespace g3x {

namespace {

constexpr int kLB = 8;    // columns per lane-block

__host__ __device__ inline int lane_eh_words(int qcap) { return (qcap + 8 + kLB + 3) & ~3; }

// Word index of row-buffer slot k of lane L.
__device__ __forceinline__ int ehw(int k, int L) { return (((k >> 2) * 32 + L) << 2) + (k & 3); }
__host__ __device__ inline int lane_nib_words(int len) { return (len + 7) / 8 + 2; }

// Byte t of x, sign-extended (prmt with the sign-replicating selector for bytes 1-3).
template <int t>
__device__ __forceinline__ int32_t sbyte(uint32_t x) {
    constexpr uint32_t sel = (uint32_t)t | ((8u | t) << 4) | ((8u | t) << 8) | ((8u | t) << 12);
    uint32_t r;
    asm("prmt.b32 %0, %1, 0, %2;" : "=r"(r) : "r"(x), "n"(sel));
    return (int32_t)r;
}

struct LaneJob {
    int job;                 // job index, -1 = none
    int32_t hi, qc;          // ring: last column given its row -1 value, query chunks loaded
    int32_t qlen, tlen, w, h0;
    uint32_t t_off;
    int32_t trev;
    Commit K;                // K.next is the row to run next
    int32_t beg, end;        // that row's band before the clamps of ksw.cu:338-340
    uint32_t tx, tn, px, pn; // target codes / N bits of chunk K.next >> 4 and of the next chunk
};

// State of the row a lane is running.
struct RowState {
    int32_t beg, end, h1, f, m, mjb;
    uint32_t plo, phi;       // this row's scores by query code (byte permute pools)
};

// One aligned block of eight columns at jb (ksw.cu:346-370).  M = H(i-1,j-1) ? H(i-1,j-1) + S : 0
// is min(H + S, 256 H): equal when H > 0, and <= 0 when H == 0, which every use clips to 0
// exactly like the reference's 0.  Writes eh[col] = {H(i, col-1), E(i+1, col)}.  kMasked blocks
// leave columns outside [beg, end) untouched.
// The row-buffer words and query codes of the block at jb.
struct BlockIn {
    uint4 wa, wb;
    uint32_t qw;
};

// sb: the block's slot (its first column, or that column mod R for a ring).
__device__ __forceinline__ BlockIn load_block(const uint32_t* __restrict__ eh, const uint32_t* __restrict__ qn,
                                              int lane, int32_t sb) {
    const uint32_t* ep = eh + ehw(sb, lane);
    BlockIn b;
    b.wa = *reinterpret_cast<const uint4*>(ep);
    b.wb = *reinterpret_cast<const uint4*>(ep + 128);
    b.qw = qn[(sb >> 3) * 32 + lane];
    return b;
}

template <bool kMasked>
__device__ __forceinline__ void lane_block(uint32_t* __restrict__ eh, const BlockIn& in,
                                           int lane, int32_t jb, int32_t sb, RowState& r, const ScoreParams& sp) {
    uint32_t* ep = eh + ehw(sb, lane);
    const uint4 wa = in.wa, wb = in.wb;
    const uint32_t wv[kLB] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
    const uint32_t qw = in.qw;
    const uint32_t sc_lo = __byte_perm(r.plo, r.phi, qw);
    const uint32_t sc_hi = __byte_perm(r.plo, r.phi, qw >> 16);
    uint32_t ov[kLB];
    int32_t hv[kLB];
    int32_t h1 = r.h1, f = r.f;
#pragma unroll
    for (int t = 0; t < kLB; ++t) {
        const uint32_t w = wv[t];
        const int32_t hd = (int32_t)(w >> 16), ed = (int32_t)(w & 0xFFFFu);
        int32_t s;
        switch (t & 3) {
            case 0: s = sbyte<0>(t < 4 ? sc_lo : sc_hi); break;
            case 1: s = sbyte<1>(t < 4 ? sc_lo : sc_hi); break;
            case 2: s = sbyte<2>(t < 4 ? sc_lo : sc_hi); break;
            default: s = sbyte<3>(t < 4 ? sc_lo : sc_hi); break;
        }
        const int32_t M = addmin_i32(hd, s, hd * 256);
        const int32_t h = max3_i32(M, ed, f);
        const int32_t te = addmax_i32(M, -sp.oe_del, 0);
        const int32_t e2 = addmax_i32(ed, -sp.e_del, te);
        const uint32_t nw = __byte_perm((uint32_t)e2, (uint32_t)h1, 0x5410);
        const int32_t tf = addmax_i32(M, -sp.oe_ins, 0);
        const int32_t fn = addmax_i32(f, -sp.e_ins, tf);
        if (kMasked) {
            const int32_t col = jb + t;
            const bool valid = col >= r.beg && col < r.end;
            ov[t] = valid ? nw : w;
            hv[t] = valid ? h : -1;
            if (valid) { f = fn; h1 = h; }
        } else {
            ov[t] = nw;
            hv[t] = h;
            f = fn;
            h1 = h;
        }
    }
    *reinterpret_cast<uint4*>(ep) = make_uint4(ov[0], ov[1], ov[2], ov[3]);
    *reinterpret_cast<uint4*>(ep + 128) = make_uint4(ov[4], ov[5], ov[6], ov[7]);
    const int32_t bm = max3_i32(max3_i32(hv[0], hv[1], hv[2]), max3_i32(hv[3], hv[4], hv[5]),
                                hv[6] > hv[7] ? hv[6] : hv[7]);
    if (bm >= r.m) { r.m = bm; r.mjb = jb; }   // ties: the later block holds the later column
    r.h1 = h1;
    r.f = f;
}

// -t * e_ins for t = 0..8 (the F of cell t of a block, relative to the F entering it).
struct InsSteps {
    int32_t n[kLB + 1];
};

// An unmasked block, with F written out: F(t) = max(F_in - t e_ins, V(t)), V(0) = 0,
// V(t+1) = max(V(t) - e_ins, T(t)), T(t) = max(M(t) - oe_ins, 0) -- the recurrence
// F(t+1) = max(F(t) - e_ins, T(t)) of ksw.cu:368-370 unrolled.  V does not depend on F_in, so
// the only value a block hands to the next through a dependency chain is F_in itself (one
// operation per block instead of eight).
__device__ __forceinline__ void lane_block_mid(uint32_t* __restrict__ eh, const BlockIn& in, int lane,
                                               int32_t jb, int32_t sb, RowState& r, const ScoreParams& sp,
                                               const InsSteps& ins) {
    uint32_t* ep = eh + ehw(sb, lane);
    const uint32_t wv[kLB] = {in.wa.x, in.wa.y, in.wa.z, in.wa.w, in.wb.x, in.wb.y, in.wb.z, in.wb.w};
    const uint32_t sc_lo = __byte_perm(r.plo, r.phi, in.qw);
    const uint32_t sc_hi = __byte_perm(r.plo, r.phi, in.qw >> 16);
    int32_t M[kLB], ed[kLB], V[kLB + 1];
    uint32_t ov[kLB];
    int32_t hv[kLB];
    V[0] = 0;
#pragma unroll
    for (int t = 0; t < kLB; ++t) {
        const uint32_t w = wv[t];
        const int32_t hd = (int32_t)__umulhi(w, sp.k16);           // w >> 16 on the FMA pipe
        ed[t] = (int32_t)(w - (uint32_t)hd * sp.k16);               // w & 0xFFFF likewise
        int32_t s;
        switch (t & 3) {
            case 0: s = sbyte<0>(t < 4 ? sc_lo : sc_hi); break;
            case 1: s = sbyte<1>(t < 4 ? sc_lo : sc_hi); break;
            case 2: s = sbyte<2>(t < 4 ? sc_lo : sc_hi); break;
            default: s = sbyte<3>(t < 4 ? sc_lo : sc_hi); break;
        }
        M[t] = addmin_i32(hd, s, hd * (int32_t)sp.k8);
        const int32_t tf = addmax_i32(M[t], -sp.oe_ins, 0);
        V[t + 1] = addmax_i32(V[t], -sp.e_ins, tf);
    }
    const int32_t fin = r.f;
    int32_t h1 = r.h1;
#pragma unroll
    for (int t = 0; t < kLB; ++t) {
        const int32_t f = t == 0 ? fin : addmax_i32(fin, ins.n[t], V[t]);
        const int32_t h = max3_i32(M[t], ed[t], f);
        const int32_t te = addmax_i32(M[t], -sp.oe_del, 0);
        const int32_t e2 = addmax_i32(ed[t], -sp.e_del, te);
        ov[t] = (uint32_t)h1 * sp.k16 + (uint32_t)e2;              // {h1, e2}, both < 2^15
        hv[t] = h;
        h1 = h;
    }
    *reinterpret_cast<uint4*>(ep) = make_uint4(ov[0], ov[1], ov[2], ov[3]);
    *reinterpret_cast<uint4*>(ep + 128) = make_uint4(ov[4], ov[5], ov[6], ov[7]);
    const int32_t bm = max3_i32(max3_i32(hv[0], hv[1], hv[2]), max3_i32(hv[3], hv[4], hv[5]),
                                hv[6] > hv[7] ? hv[6] : hv[7]);
    if (bm >= r.m) { r.m = bm; r.mjb = jb; }
    r.h1 = h1;
    r.f = addmax_i32(fin, ins.n[kLB], V[kLB]);
}

__device__ __forceinline__ JobConst job_const(const LaneJob& J, const ScoreParams& sp) {
    JobConst c;
    c.qlen = J.qlen; c.tlen = J.tlen; c.w = J.w; c.h0 = J.h0;
    c.o_del = sp.o_del; c.e_del = sp.e_del; c.o_ins = sp.o_ins; c.e_ins = sp.e_ins;
    c.oe_del = sp.oe_del; c.oe_ins = sp.oe_ins; c.zdrop = sp.zdrop;
    return c;
}

}  // namespace

__host__ __device__ inline size_t lane_warp_bytes(int qcap) {
    return (size_t)128 * (lane_eh_words(qcap) + lane_nib_words(qcap));
}

// A ring of R columns: R row-buffer slots and R/8 query words per lane.
__host__ __device__ inline size_t ring_warp_bytes(int R) { return (size_t)128 * (R + R / 8); }

size_t lane_smem_per_warp(int qcap, int tcap) { (void)tcap; return lane_warp_bytes(qcap); }
size_t lane_ring_smem_per_warp(int ring) { return ring_warp_bytes(ring); }

__device__ __forceinline__ int32_t wrap_slot(int32_t s, int32_t R) { return s >= R ? s - R : s; }

template <bool kRing>
__global__ void __launch_bounds__(128) lane_kernel(LaunchDesc d, ScoreParams sp) {
    pdl_trigger();
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
    const int qcap = d.qmax, tcap = d.tmax;
    const int32_t R = kRing ? d.ring : 1;                        // ring columns (multiple of 16)
    uint32_t* base = reinterpret_cast<uint32_t*>(
        smem + (size_t)warp * (kRing ? ring_warp_bytes(R) : lane_warp_bytes(qcap)));
    uint32_t* eh = base;                                         // [slot*32 + lane]
    uint32_t* qn = eh + 32 * (kRing ? R : lane_eh_words(qcap));  // [word*32 + lane]
    const int n = d.count ? *d.count : d.n;
    const int* order = d.order ? d.order + (d.order_off ? *d.order_off : 0) : nullptr;
    const int refill = d.warp_batch ? 32 : (d.refill > 0 ? d.refill : 1);
    InsSteps ins;
#pragma unroll
    for (int t = 0; t <= kLB; ++t) ins.n[t] = -t * sp.e_ins;

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
            // Each idle lane takes the slot of its rank among the idle lanes and sets up its own
            // job state; then the whole warp decodes each new job into that lane's columns.
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
                    if (c.qlen > qcap || c.tlen > tcap || !job_fits_lane(c, sp.max_sc) ||
                        (kRing && 2 * c.w + 16 > R)) {
                        d.out[job] = g3x_ext_t{0, 0, 0, 0, 0, 0};
                        d.status[job] = G3X_ERR_TOO_LONG;
                        if (d.cells) d.cells[job] = 0;
                        if (d.rows) d.rows[job] = 0;
                    } else if (!job_in_planes(jb, d.n_bases)) {   // reaches past the planes: unread
                        d.out[job] = g3x_ext_t{0, 0, 0, 0, 0, 0};
                        d.status[job] = G3X_ERR_INVALID;
                        if (d.cells) d.cells[job] = 0;
                        if (d.rows) d.rows[job] = 0;
                    } else {
                        my_job = job;
                        J.job = job;
                        J.qlen = c.qlen; J.tlen = c.tlen; J.w = c.w; J.h0 = c.h0;
                        J.t_off = jb.t_off;
                        J.trev = (jb.flags & G3X_JOB_TREV) != 0;
                        commit_init(J.K, c);
                        J.beg = 0; J.end = c.qlen;
                        if (kRing) {   // staged below: columns 0 .. min(qlen + 1, R - 1), query chunks
                            J.hi = c.qlen + 1 < R - 1 ? c.qlen + 1 : R - 1;
                            const int32_t qc = (c.qlen + 15) >> 4;
                            J.qc = qc < (R >> 4) ? qc : (R >> 4);
                        }
                        J.tx = J.tn = J.px = J.pn = 0;
                        if (c.tlen > 0) load16(d.codes, d.nmask, J.t_off, c.tlen, 0, J.trev, J.tx, J.tn);
                        if (c.tlen > 16) load16(d.codes, d.nmask, J.t_off, c.tlen, 1, J.trev, J.px, J.pn);
                        const int32_t qch = (c.qlen + 15) >> 4;
                        stage_own_query(d.codes, d.nmask, jb.q_off, c.qlen, (jb.flags & G3X_JOB_QREV) != 0,
                                        kRing ? (qch < (R >> 4) ? qch : (R >> 4)) : qch, qn, lane);
                    }
                }
            }
            // row -1 of every new job (ksw.cu:317-319), the whole warp on one job at a time
            unsigned m = __ballot_sync(0xFFFFFFFFu, my_job >= 0);
            while (m) {
                const int L = __ffs(m) - 1;
                m &= m - 1;
                const int qlen = __shfl_sync(0xFFFFFFFFu, J.qlen, L);
                JobConst c;
                c.qlen = qlen; c.h0 = __shfl_sync(0xFFFFFFFFu, J.h0, L); c.oe_ins = sp.oe_ins; c.e_ins = sp.e_ins;
                const int top = kRing ? (qlen + 1 < R - 1 ? qlen + 1 : R - 1) : qlen + 1;
                for (int k = lane; k <= top; k += 32) eh[ehw(k, L)] = (uint32_t)init_h(k, c) << 16;
            }
            __syncwarp();
        }
        const bool active = J.job >= 0;
        if (!__any_sync(0xFFFFFFFFu, active)) {
            if (exhausted) break;
            continue;
        }
        // A job staged with tlen == 0 has no row: it finishes at once.
        const bool run = active && !J.K.stop;

        // ---- row begin (ksw.cu:335-345) ----
        RowState r;
        r.beg = 0; r.end = 0; r.h1 = 0; r.f = 0; r.m = 0; r.mjb = -1; r.plo = 0; r.phi = 0;
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
            if (kRing && r.beg < r.end) {
                // columns entering the band for the first time get their row -1 value
                if (J.hi < r.end - 1) {
                    JobConst c;
                    c.qlen = J.qlen; c.h0 = J.h0; c.oe_ins = sp.oe_ins; c.e_ins = sp.e_ins;
                    for (int32_t col = J.hi + 1; col < r.end; ++col)
                        eh[ehw(col % R, lane)] = (uint32_t)init_h(col, c) << 16;
                    J.hi = r.end - 1;
                }
                // query codes of the 16-column chunks up to the band's last block
                const int32_t need = (r.end - 1) >> 4;
                while (J.qc <= need) {
                    uint32_t x, nb;
                    const g3x_job_t jd = d.jobs[J.job];
                    load16(d.codes, d.nmask, jd.q_off, J.qlen, J.qc, (jd.flags & G3X_JOB_QREV) != 0, x, nb);
                    const uint64_t v = nibbles16(x, nb);
                    const int32_t wq = (2 * J.qc) % (kRing ? (R >> 3) : 1);
                    qn[wq * 32 + lane] = (uint32_t)v;
                    qn[(wq + 1) * 32 + lane] = (uint32_t)(v >> 32);
                    ++J.qc;
                }
            }
        }
        const bool nonempty = run && r.beg < r.end;
        const int32_t jb0 = r.beg & ~(kLB - 1);
        const int32_t sb0 = kRing ? jb0 % R : jb0;                     // slot of the first block
        const int nblk = nonempty ? ((r.end - 1) >> 3) - (r.beg >> 3) + 1 : 0;
        const int kmax = __reduce_max_sync(0xFFFFFFFFu, (unsigned)nblk);
        busy += nblk;
        idle += kmax - nblk;

        // ---- the row's blocks: masked first block, unmasked middle, masked last block ----
        // Each middle block's words are loaded one block ahead (blocks never overlap, so the
        // load may precede the previous block's store).
        // slots advance with the columns; a ring wraps at R
        auto slot_at = [&](int k) { return kRing ? wrap_slot(sb0 + k * kLB, R) : jb0 + k * kLB; };
        BlockIn next;
        if (nblk > 2) next = load_block(eh, qn, lane, slot_at(1));
        if (nblk > 0) lane_block<true>(eh, load_block(eh, qn, lane, sb0), lane, jb0, sb0, r, sp);
        for (int k = 1; k < kmax - 1; ++k) {
            if (k < nblk - 1) {
                const BlockIn cur = next;
                if (k + 1 < nblk - 1) next = load_block(eh, qn, lane, slot_at(k + 1));
                lane_block_mid(eh, cur, lane, jb0 + k * kLB, slot_at(k), r, sp, ins);
            }
        }
        if (nblk > 1) {
            const int32_t jl = jb0 + (nblk - 1) * kLB, sl = slot_at(nblk - 1);
            lane_block<true>(eh, load_block(eh, qn, lane, sl), lane, jl, sl, r, sp);
        }

        // ---- row end (ksw.cu:371-391) ----
        if (run) {
            const int32_t beg = r.beg, end = r.end;
            if (end >= 0) eh[ehw(kRing ? end % R : end, lane)] = (uint32_t)r.h1 << 16;
            RowDone rd;
            rd.m = r.m;
            rd.mj = -1;
            if (r.m > 0) {
                // the last column of the winning block that reaches the maximum; H(i, c) is
                // eh[c+1].h, so the block's eight H values are slots mjb+1 .. mjb+8
                const int32_t mjb = r.mjb;
                const int32_t lo = mjb > beg ? mjb : beg;
                const int32_t hi = mjb + kLB < end ? mjb + kLB : end;
                const int32_t ms = kRing ? mjb % R : mjb;
                const uint4 a = *reinterpret_cast<const uint4*>(eh + ehw(ms, lane));
                const uint4 b = *reinterpret_cast<const uint4*>(eh + ehw(ms + 4, lane));
                const int32_t m8 = kRing ? wrap_slot(ms + 8, R) : ms + 8;
                const uint32_t hs[kLB] = {a.y, a.z, a.w, b.x, b.y, b.z, b.w, eh[ehw(m8, lane)]};
#pragma unroll
                for (int t = 0; t < kLB; ++t) {
                    const int32_t c = mjb + t;
                    if (c >= lo && c < hi && (int32_t)(hs[t] >> 16) == r.m) rd.mj = c;
                }
            }
            rd.gval = (nonempty ? end : beg) == J.qlen ? r.h1 : -1;
            rd.ncells = nonempty ? end - beg : 0;
            const JobConst c = job_const(J, sp);
            commit_row(J.K, c, rd);
            if (!J.K.stop) {
                int32_t j = beg;
                if (kRing) {
                    int32_t s = beg % R;
                    while (j < end && eh[ehw(s, lane)] == 0u) { ++j; s = wrap_slot(s + 1, R); }
                } else {
                    while (j < end && eh[ehw(j, lane)] == 0u) ++j;
                }
                const int32_t nb = j;
                j = end;
                if (kRing) {
                    int32_t s = end % R;
                    while (j >= nb && eh[ehw(s, lane)] == 0u) { --j; s = s == 0 ? R - 1 : s - 1; }
                } else {
                    while (j >= nb && eh[ehw(j, lane)] == 0u) --j;
                }
                J.beg = nb;
                J.end = j + 2 < J.qlen ? j + 2 : J.qlen;
            }
        }
        if (active && J.K.stop) {
            const Commit& K = J.K;
            d.out[J.job] = g3x_ext_t{K.best, K.best_j + 1, K.best_i + 1, K.max_ie + 1, K.gscore, K.max_off};
            d.status[J.job] = G3X_OK;
            if (d.cells) d.cells[J.job] = (int32_t)K.cells;
            if (d.rows) d.rows[J.job] = K.next;
            J.job = -1;
        }
        __syncwarp();
    }
    if (d.stats) add_warp_stats(d.stats, busy, idle, waves, lane);
    pdl_chain_end();
}

template <bool kRing>
static int launch_lane_t(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream) {
    const size_t wb = kRing ? ring_warp_bytes(d.ring) : lane_warp_bytes(d.qmax);
    size_t max_smem = 0;
    if (allow_max_smem(lane_kernel<kRing>, &max_smem) != cudaSuccess) return G3X_ERR_CUDA;
    if (wb > max_smem) return G3X_ERR_TOO_LONG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return G3X_ERR_CUDA;
    sms = sm_count();
    // Warps per block: the choice among 1, 2 and 4 that keeps the most warps resident (shared
    // memory is allotted per block, so small blocks waste less of it).
    int best_wpb = 1, best_warps = 0, best_blocks = 0;
    const int max_wpb = d.warps_per_block > 0 ? d.warps_per_block : 4;
    for (int wpb = 1; wpb <= max_wpb; wpb *= 2) {
        const size_t smem = (size_t)wpb * wb;
        if (smem > max_smem) break;
        int per_sm = 0;
        per_sm = resident_blocks(lane_kernel<kRing>, 32 * wpb, smem);
        if (per_sm * wpb >= best_warps) { best_warps = per_sm * wpb; best_wpb = wpb; best_blocks = per_sm; }
    }
    const size_t smem = (size_t)best_wpb * wb;
    int blocks = d.blocks > 0 ? d.blocks : sms * (best_blocks > 0 ? best_blocks : 1);
    if (launch_class_kernel(lane_kernel<kRing>, blocks, 32 * best_wpb, smem, stream, d, sp) != cudaSuccess)
        return G3X_ERR_CUDA;
    return G3X_OK;
}

// The ring form when the launch names a ring (d.ring > 0, a multiple of 16, at least 64).
int launch_lane(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream) {
    if (d.ring > 0) {
        if (d.ring < 64 || d.ring % 16) return G3X_ERR_INVALID;
        return launch_lane_t<true>(d, sp, stream);
    }
    return launch_lane_t<false>(d, sp, stream);
}

}  // namespace g3x

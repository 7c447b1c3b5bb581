// g3x_lane2.cu -- lane-per-job sm_100a kernel with two rows of the job in flight per lane, for
// batched ksw_extend2 (bwa/src/ksw.cu:303-401).
//
// The int32 lane kernel (g3x_lane.cu) runs one row of its job at a time, so the F recurrence of
// that row is the only dependency chain a lane has, and with one or two warps per scheduler
// (shared memory per lane grows with the query) the SM waits on it.  Here each lane runs rows
// i ("A") and i+1 ("B") of its job together, B one or more 8-column blocks behind A: two
// independent chains in one instruction stream, with the same shared memory.
//
// B's band follows from A's row exactly as the reference derives it (ksw.cu:388-391):
//   * beg(i+1) = the first column of [beg_i, end_i) whose row-buffer word A left non-zero (end_i
//     if none), then max(., i+1-w).  It is known as soon as A has written a non-zero word, and
//     B does not start before.
//   * end(i+1) = min(last non-zero column of [beg(i+1), end_i] + 2, i+1+w+1, qlen).  B runs block
//     b (columns b..b+7) before A's row ends only when A has already written a non-zero word in a
//     block at or beyond b+8: then end(i+1) >= b+10 > every column of the block.  The rest of B's
//     row runs after A's row end, with end(i+1) exact.
// B reads the row-buffer words A wrote (or, beyond A's band, the stale words of earlier rows,
// ksw.cu:388-391 regrowth) only after A wrote them, and overwrites a block only after A is
// past it, so every word either row reads holds what it holds in the scalar loop.  When A's
// row ends the extension (m == 0 or z-drop, ksw.cu:376-386), B's partial row is discarded.
//
// A row's maximum and its last column (ksw.cu:362-364) come from per-block maxima of the key
// H * 8 + t (ties to the later column), so no row needs its words again after they are
// overwritten.  A's last non-zero column is read at A's row end from eh[end_i] and from the
// last block in which A wrote a non-zero word: B can only have overwritten blocks before it.
#include <cuda_runtime.h>
#include "g3x_core.h"
#include "g3x_internal.h"
#include "g3x_stage.cuh"

namespace g3x {

namespace {

constexpr int kLB = 8;

__host__ __device__ inline int eh_words(int qcap) { return (qcap + 8 + kLB + 3) & ~3; }
__host__ __device__ inline int nib_words(int len) { return (len + 7) / 8 + 2; }
__host__ __device__ inline size_t warp_bytes(int qcap) { return (size_t)128 * (eh_words(qcap) + nib_words(qcap)); }

__device__ __forceinline__ int ehw(int k, int L) { return (((k >> 2) * 32 + L) << 2) + (k & 3); }

template <int t>
__device__ __forceinline__ int32_t sbyte(uint32_t x) {
    constexpr uint32_t sel = (uint32_t)t | ((8u | t) << 4) | ((8u | t) << 8) | ((8u | t) << 12);
    uint32_t r;
    asm("prmt.b32 %0, %1, 0, %2;" : "=r"(r) : "r"(x), "n"(sel));
    return (int32_t)r;
}

__device__ __forceinline__ int32_t score_of(uint32_t lo, uint32_t hi, int t) {
    switch (t) {
        case 0: return sbyte<0>(lo);
        case 1: return sbyte<1>(lo);
        case 2: return sbyte<2>(lo);
        case 3: return sbyte<3>(lo);
        case 4: return sbyte<0>(hi);
        case 5: return sbyte<1>(hi);
        case 6: return sbyte<2>(hi);
        default: return sbyte<3>(hi);
    }
}

struct Job {
    int job;                 // -1 = none
    int32_t qlen, tlen, w, h0;
    uint32_t t_off;
    int32_t trev;
    Commit K;                // K.next: the next row to run (A of the next round)
    int32_t beg, end;        // band of that row before the clamps of ksw.cu:338-340
    uint32_t tx, tn, px, pn; // target chunk K.next >> 4 and the next one
};

// One row in flight.
struct Row {
    int32_t beg, end;        // band; B's end is a bound (min(i+w+2, qlen)) until A's row ends
    int32_t h1, f;           // H(i, j-1) and F(i, j) at the next column
    int32_t m, mj;           // row maximum so far and its last column
    uint32_t plo, phi;       // this row's scores by query code
    int32_t next, last;      // next block to run and the last one (start columns)
};

struct InsSteps {
    int32_t n[kLB + 1];      // -t * e_ins
};

// One aligned block at jb of row r, cells restricted to [r.beg, r.end) when kMasked.  Writes
// eh[col] = {H(i, col-1), E(i+1, col)} (ksw.cu:346-370; M = H ? H + S : 0 as min(H + S, 256 H)),
// updates the row maximum by the key H*8 + t, and returns the OR of the words it wrote.
template <bool kMasked>
__device__ __forceinline__ uint32_t row_block(uint32_t* __restrict__ eh, const uint32_t* __restrict__ qn,
                                              int lane, int32_t jb, Row& r, const ScoreParams& sp,
                                              const InsSteps& ins) {
    uint32_t* ep = eh + ehw(jb, lane);
    const uint4 wa = *reinterpret_cast<const uint4*>(ep);
    const uint4 wb = *reinterpret_cast<const uint4*>(ep + 128);
    const uint32_t wv[kLB] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
    const uint32_t qw = qn[(jb >> 3) * 32 + lane];
    const uint32_t sc_lo = __byte_perm(r.plo, r.phi, qw);
    const uint32_t sc_hi = __byte_perm(r.plo, r.phi, qw >> 16);
    uint32_t ov[kLB];
    int32_t key[kLB];
    uint32_t nz = 0;
    if (!kMasked) {
        // F written out: F(t) = max(F_in - t e_ins, V(t)), V(t+1) = max(V(t) - e_ins, T(t)), so
        // only F_in crosses from one block to the next
        int32_t M[kLB], ed[kLB], V[kLB + 1];
        V[0] = 0;
#pragma unroll
        for (int t = 0; t < kLB; ++t) {
            const int32_t hd = (int32_t)(wv[t] >> 16);
            ed[t] = (int32_t)(wv[t] & 0xFFFFu);
            const int32_t s = score_of(sc_lo, sc_hi, t);
            M[t] = addmin_i32(hd, s, hd * 256);
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
            ov[t] = __byte_perm((uint32_t)e2, (uint32_t)h1, 0x5410);
            key[t] = h * 8 + t;
            h1 = h;
        }
        r.h1 = h1;
        r.f = addmax_i32(fin, ins.n[kLB], V[kLB]);
        nz = (ov[0] | ov[1] | ov[2]) | (ov[3] | ov[4] | ov[5]) | (ov[6] | ov[7]);
    } else {
        int32_t h1 = r.h1, f = r.f;
#pragma unroll
        for (int t = 0; t < kLB; ++t) {
            const uint32_t w = wv[t];
            const int32_t hd = (int32_t)(w >> 16), ed = (int32_t)(w & 0xFFFFu);
            const int32_t s = score_of(sc_lo, sc_hi, t);
            const int32_t M = addmin_i32(hd, s, hd * 256);
            const int32_t h = max3_i32(M, ed, f);
            const int32_t te = addmax_i32(M, -sp.oe_del, 0);
            const int32_t e2 = addmax_i32(ed, -sp.e_del, te);
            const uint32_t nw = __byte_perm((uint32_t)e2, (uint32_t)h1, 0x5410);
            const int32_t tf = addmax_i32(M, -sp.oe_ins, 0);
            const int32_t fn = addmax_i32(f, -sp.e_ins, tf);
            const int32_t col = jb + t;
            const bool valid = col >= r.beg && col < r.end;
            ov[t] = valid ? nw : w;
            key[t] = valid ? h * 8 + t : -1;
            nz |= valid ? nw : 0u;
            if (valid) { f = fn; h1 = h; }
        }
        r.h1 = h1;
        r.f = f;
    }
    *reinterpret_cast<uint4*>(ep) = make_uint4(ov[0], ov[1], ov[2], ov[3]);
    *reinterpret_cast<uint4*>(ep + 128) = make_uint4(ov[4], ov[5], ov[6], ov[7]);
    const int32_t bk = max3_i32(max3_i32(key[0], key[1], key[2]), max3_i32(key[3], key[4], key[5]),
                                key[6] > key[7] ? key[6] : key[7]);
    if (bk >= 0 && (bk >> 3) >= r.m) { r.m = bk >> 3; r.mj = jb + (bk & 7); }   // ksw.cu:363-364
    return nz;
}

__device__ __forceinline__ JobConst job_const(const Job& J, const ScoreParams& sp) {
    JobConst c;
    c.qlen = J.qlen; c.tlen = J.tlen; c.w = J.w; c.h0 = J.h0;
    c.o_del = sp.o_del; c.e_del = sp.e_del; c.o_ins = sp.o_ins; c.e_ins = sp.e_ins;
    c.oe_del = sp.oe_del; c.oe_ins = sp.oe_ins; c.zdrop = sp.zdrop;
    return c;
}

// Row i's first-column H (ksw.cu:341-344) and score pool.
__device__ __forceinline__ void row_setup(Row& r, const Job& J, int32_t i, uint32_t code, const uint2* pools,
                                          const ScoreParams& sp) {
    r.h1 = 0;
    if (r.beg == 0) {
        const int32_t h = J.h0 - (sp.o_del + sp.e_del * (i + 1));
        r.h1 = h > 0 ? h : 0;
    }
    r.f = 0; r.m = 0; r.mj = -1;
    const uint2 p = pools[code];
    r.plo = p.x; r.phi = p.y;
    if (r.beg < r.end) {
        r.next = r.beg & ~(kLB - 1);
        r.last = (r.end - 1) & ~(kLB - 1);
    } else {
        r.next = 0;
        r.last = -kLB;
    }
}

}  // namespace

size_t lane2_smem_per_warp(int qcap) { return warp_bytes(qcap); }

__global__ void __launch_bounds__(128) lane2_kernel(LaunchDesc d, ScoreParams sp) {
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
    uint32_t* eh = reinterpret_cast<uint32_t*>(smem + (size_t)warp * warp_bytes(qcap));
    uint32_t* qn = eh + 32 * eh_words(qcap);
    const int n = d.count ? *d.count : d.n;
    const int* order = d.order ? d.order + (d.order_off ? *d.order_off : 0) : nullptr;
    const int refill = d.warp_batch ? 32 : (d.refill > 0 ? d.refill : 1);
    InsSteps ins;
#pragma unroll
    for (int t = 0; t <= kLB; ++t) ins.n[t] = -t * sp.e_ins;

    Job J;
    J.job = -1;
    bool exhausted = false;
    unsigned long long busy = 0, idle = 0, waves = 0;
    for (;;) {
        // ---- refill wave (as in the one-row lane kernel) ----
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
                    // the row-max key H * 8 + t needs H < 2^28, far above the 16-bit fields
                    if (c.qlen > qcap || c.tlen > tcap || !job_fits_lane(c, sp.max_sc)) {
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
                        J.tx = J.tn = J.px = J.pn = 0;
                        if (c.tlen > 0) load16(d.codes, d.nmask, J.t_off, c.tlen, 0, J.trev, J.tx, J.tn);
                        if (c.tlen > 16) load16(d.codes, d.nmask, J.t_off, c.tlen, 1, J.trev, J.px, J.pn);
                        stage_own_query(d.codes, d.nmask, jb.q_off, c.qlen, (jb.flags & G3X_JOB_QREV) != 0,
                                        (c.qlen + 15) >> 4, qn, lane);
                    }
                }
            }
            unsigned m = __ballot_sync(0xFFFFFFFFu, my_job >= 0);
            while (m) {
                const int L = __ffs(m) - 1;
                m &= m - 1;
                const int qlen = __shfl_sync(0xFFFFFFFFu, J.qlen, L);
                JobConst c;
                c.qlen = qlen; c.h0 = __shfl_sync(0xFFFFFFFFu, J.h0, L); c.oe_ins = sp.oe_ins; c.e_ins = sp.e_ins;
                for (int k = lane; k <= qlen + 1; k += 32) eh[ehw(k, L)] = (uint32_t)init_h(k, c) << 16;
            }
            __syncwarp();
        }
        const bool active = J.job >= 0;
        if (!__any_sync(0xFFFFFFFFu, active)) {
            if (exhausted) break;
            continue;
        }

        // ---- a round: rows i (A) and i+1 (B) ----
        const bool runA = active && !J.K.stop;
        const int32_t i = J.K.next;
        bool runB = runA && i + 1 < J.tlen;
        Row A, B;
        A.beg = A.end = B.beg = B.end = 0;
        uint32_t codeA = 0, codeB = 0;
        if (runA) {
            A.beg = J.beg > i - J.w ? J.beg : i - J.w;
            A.end = J.end < i + J.w + 1 ? J.end : i + J.w + 1;
            if (A.end > J.qlen) A.end = J.qlen;
            if ((i & 15) == 0 && i > 0) {          // i is even, so i and i+1 share a chunk
                J.tx = J.px; J.tn = J.pn;
                const int ch = (i >> 4) + 1;
                if ((ch << 4) < J.tlen) load16(d.codes, d.nmask, J.t_off, J.tlen, ch, J.trev, J.px, J.pn);
            }
            codeA = (J.tx >> ((i & 15) << 1)) & 3u;
            if ((J.tn >> (i & 15)) & 1u) codeA = 4;
            codeB = (J.tx >> (((i + 1) & 15) << 1)) & 3u;
            if ((J.tn >> ((i + 1) & 15)) & 1u) codeB = 4;
        }
        row_setup(A, J, i, codeA, pools, sp);
        if (!runA) { A.next = 0; A.last = -kLB; }
        // B's band: beg from A's first non-zero word (pending), end bounded by the fixed limits
        int32_t bbeg = -1;                      // first non-zero column of A's row, -1 = not yet
        int32_t lastnzblk = -kLB;               // last block in which A wrote a non-zero word
        bool b_started = false;
        B.next = 0; B.last = -kLB; B.m = 0; B.mj = -1; B.h1 = 0; B.f = 0; B.plo = B.phi = 0;
        const int32_t b_bound = runB ? min(i + 1 + J.w + 1, J.qlen) : 0;

        // ---- phase 1: A's blocks, B's blocks one or more behind.  A's first and last blocks are
        // masked steps every lane takes together; in between, the common step runs one unmasked
        // block of each row, two independent dependency chains in one instruction stream.
        const int nA = A.next <= A.last ? ((A.last - A.next) >> 3) + 1 : 0;
        auto a_after = [&](int32_t ja, uint32_t nza) {
            A.next += kLB;
            if (nza) {
                lastnzblk = ja;
                if (bbeg < 0) {
                    // the first non-zero word of A's row (ksw.cu:388) is in this block
                    int32_t c = ja > A.beg ? ja : A.beg;
                    while (eh[ehw(c, lane)] == 0u) ++c;
                    bbeg = c;
                }
            }
        };
        auto b_start = [&]() {
            if (runB && !b_started && bbeg >= 0) {
                B.beg = bbeg > i + 1 - J.w ? bbeg : i + 1 - J.w;
                B.end = b_bound;
                row_setup(B, J, i + 1, codeB, pools, sp);
                b_started = true;
            }
        };
        // B may run block B.next now: A has written a non-zero word at or beyond B.next + 8
        auto b_ready = [&]() { return b_started && B.next <= B.last && lastnzblk >= B.next + kLB; };
        auto b_full = [&]() { return B.next >= B.beg && B.next + kLB <= B.end; };
        if (nA > 0) {
            const int32_t ja = A.next;
            a_after(ja, row_block<true>(eh, qn, lane, ja, A, sp, ins));
        }
        const int kmid = (int)__reduce_max_sync(0xFFFFFFFFu, (unsigned)(nA > 2 ? nA - 2 : 0));
        for (int k = 0; k < kmid; ++k) {
            if (k < nA - 2) {
                b_start();
                const bool b_go = b_ready();
                const int32_t ja = A.next;
                uint32_t nza;
                if (b_go && b_full()) {
                    nza = row_block<false>(eh, qn, lane, ja, A, sp, ins);
                    row_block<false>(eh, qn, lane, B.next, B, sp, ins);
                } else if (b_go) {
                    nza = row_block<false>(eh, qn, lane, ja, A, sp, ins);
                    row_block<true>(eh, qn, lane, B.next, B, sp, ins);
                } else {
                    nza = row_block<false>(eh, qn, lane, ja, A, sp, ins);
                }
                if (b_go) B.next += kLB;
                a_after(ja, nza);
                busy += b_go ? 2 : 1;
                idle += b_go ? 0 : 1;
            } else {
                idle += 2;
            }
        }
        if (nA > 1) {
            b_start();
            const bool b_go = b_ready();
            const int32_t ja = A.next;
            const uint32_t nza = row_block<true>(eh, qn, lane, ja, A, sp, ins);
            if (b_go) {
                if (b_full()) row_block<false>(eh, qn, lane, B.next, B, sp, ins);
                else row_block<true>(eh, qn, lane, B.next, B, sp, ins);
                B.next += kLB;
            }
            a_after(ja, nza);
        }

        // ---- A's row end (ksw.cu:371-391) ----
        if (runA) {
            const bool nonempty = A.beg < A.end;
            eh[ehw(A.end, lane)] = (uint32_t)A.h1 << 16;
            RowDone rd;
            rd.m = A.m;
            rd.mj = A.m > 0 ? A.mj : -1;
            rd.gval = (nonempty ? A.end : A.beg) == J.qlen ? A.h1 : -1;
            rd.ncells = nonempty ? A.end - A.beg : 0;
            commit_row(J.K, job_const(J, sp), rd);
            if (J.K.stop) {
                runB = false;
            } else {
                const int32_t nb = bbeg >= 0 ? bbeg : A.end;
                // last non-zero word in [nb, end]: eh[end], else the last block with a
                // non-zero word (which B has not reached)
                int32_t j = A.end;
                if (eh[ehw(j, lane)] == 0u) {
                    j = nb - 1;
                    if (lastnzblk >= 0) {
                        int32_t c = lastnzblk + kLB - 1 < A.end - 1 ? lastnzblk + kLB - 1 : A.end - 1;
                        while (c >= nb && eh[ehw(c, lane)] == 0u) --c;
                        if (c >= nb) j = c;
                    }
                }
                const int32_t end1 = j + 2 < J.qlen ? j + 2 : J.qlen;
                if (runB) {
                    const int32_t bbeg1 = nb > i + 1 - J.w ? nb : i + 1 - J.w;
                    int32_t bend1 = end1 < i + 1 + J.w + 1 ? end1 : i + 1 + J.w + 1;
                    if (bend1 > J.qlen) bend1 = J.qlen;
                    if (!b_started) {
                        B.beg = bbeg1;
                        B.end = bend1;
                        row_setup(B, J, i + 1, codeB, pools, sp);
                        b_started = true;
                    } else {
                        B.end = bend1;              // beg was fixed when B started
                        B.last = B.beg < B.end ? (B.end - 1) & ~(kLB - 1) : B.next - kLB;
                    }
                } else {
                    J.beg = nb;
                    J.end = end1;
                }
            }
        }

        // ---- phase 2: the rest of B's row, its band now exact: the first remaining block and
        // the last masked, the ones between unmasked ----
        const int nB = runB && B.next <= B.last ? ((B.last - B.next) >> 3) + 1 : 0;
        if (nB > 0) {
            row_block<true>(eh, qn, lane, B.next, B, sp, ins);
            B.next += kLB;
        }
        const int kb = (int)__reduce_max_sync(0xFFFFFFFFu, (unsigned)(nB > 2 ? nB - 2 : 0));
        for (int k = 0; k < kb; ++k) {
            if (k < nB - 2) {
                row_block<false>(eh, qn, lane, B.next, B, sp, ins);
                B.next += kLB;
                ++busy;
            } else {
                ++idle;
            }
        }
        if (nB > 1) {
            row_block<true>(eh, qn, lane, B.next, B, sp, ins);
            B.next += kLB;
        }

        // ---- B's row end ----
        if (runB) {
            const bool nonempty = B.beg < B.end;
            eh[ehw(B.end, lane)] = (uint32_t)B.h1 << 16;
            RowDone rd;
            rd.m = B.m;
            rd.mj = B.m > 0 ? B.mj : -1;
            rd.gval = (nonempty ? B.end : B.beg) == J.qlen ? B.h1 : -1;
            rd.ncells = nonempty ? B.end - B.beg : 0;
            commit_row(J.K, job_const(J, sp), rd);
            if (!J.K.stop) {
                int32_t j = B.beg;
                while (j < B.end && eh[ehw(j, lane)] == 0u) ++j;
                const int32_t nb = j;
                j = B.end;
                while (j >= nb && eh[ehw(j, lane)] == 0u) --j;
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

int launch_lane2(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream) {
    const size_t wb = warp_bytes(d.qmax);
    size_t max_smem = 0;
    if (allow_max_smem(lane2_kernel, &max_smem) != cudaSuccess) return G3X_ERR_CUDA;
    if (wb > max_smem) return G3X_ERR_TOO_LONG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return G3X_ERR_CUDA;
    sms = sm_count();
    int best_wpb = 1, best_warps = 0, best_blocks = 0;
    const int max_wpb = d.warps_per_block > 0 ? d.warps_per_block : 4;
    for (int wpb = 1; wpb <= max_wpb; wpb *= 2) {
        const size_t smem = (size_t)wpb * wb;
        if (smem > max_smem) break;
        int per_sm = 0;
        per_sm = resident_blocks(lane2_kernel, 32 * wpb, smem);
        if (per_sm * wpb >= best_warps) { best_warps = per_sm * wpb; best_wpb = wpb; best_blocks = per_sm; }
    }
    const size_t smem = (size_t)best_wpb * wb;
    const int blocks = d.blocks > 0 ? d.blocks : sms * (best_blocks > 0 ? best_blocks : 1);
    if (launch_class_kernel(lane2_kernel, blocks, 32 * best_wpb, smem, stream, d, sp) != cudaSuccess)
        return G3X_ERR_CUDA;
    return G3X_OK;
}

}  // namespace g3x

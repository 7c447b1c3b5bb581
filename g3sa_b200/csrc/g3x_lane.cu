// g3x_lane.cu -- lane-per-job sm_100a kernel for batched ksw_extend2 (bwa/src/ksw.cu:303-401).
//
// Each lane of a warp runs one job through the reference's own row loop: rows in order, the
// reference's band [beg, end) per row (ksw.cu:338-340, 388-391), and the per-row bookkeeping
// of ksw.cu:371-386 -- so the semantics are the scalar loop's by construction.  A lane walks
// its current row in aligned blocks of eight columns; when it reaches the row's end it does
// the row bookkeeping and starts the next row (that step diverges from the lanes still inside
// their rows, and is short).  The 32 jobs of a warp are chosen by the scheduler to need
// similar work, so the lanes stay busy together.
//
// Shared memory holds each lane's job in a lane-interleaved layout, so that every access of
// the warp is free of bank conflicts whatever column each lane is at:
//   eh   : the row buffer (ksw.cu:310) as 16-bit H | 16-bit E words ("narrow" jobs only,
//          H <= h0 + max_score * min(qlen, tlen) < 2^15); slot k of lane L is word
//          ((k/4)*32 + L)*4 + k%4, so a lane's aligned 8-column block is two 16-byte loads
//   qnib : query codes, eight 4-bit codes per word; a byte permute of the row's score pool
//          turns four codes into four scores
//   tnib : target codes, eight 4-bit codes per word
// Idle lanes are refilled in waves: when at least `refill` lanes of the warp are idle, the
// whole warp stages one new job per idle lane together (all lanes decode each job).
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

struct LaneJob {
    int job;                 // job index, -1 = none
    int32_t qlen, tlen, w, h0;
    Commit K;
    int32_t i, beg, end, j;  // row, band, next column
    int32_t h1, f, key, fnz, lnz;
    uint32_t pool_lo, pool_hi;   // this row's scores by query code (byte permute pools)
};


__device__ __forceinline__ int32_t tcode_at(const uint32_t* tn, int lane, int i) {
    const uint32_t nib = (tn[(i >> 3) * 32 + lane] >> ((i & 7) << 2)) & 15u;
    return nib < 4u ? (int32_t)nib : 4;
}

// Begins row J.i: band clamps, first-column value, row score pool (ksw.cu:335-345).  `pools`
// holds, per target code t, the byte-permute pool of its scores (bytes 0-3: vs query codes
// 0-3, bytes 4-7: vs N), in shared memory so that t can index it.
__device__ __forceinline__ void begin_row(LaneJob& J, const ScoreParams& sp, const uint32_t* tn, int lane,
                                          const uint2* pools) {
    const int32_t i = J.i;
    if (J.beg < i - J.w) J.beg = i - J.w;
    if (J.end > i + J.w + 1) J.end = i + J.w + 1;
    if (J.end > J.qlen) J.end = J.qlen;
    if (J.beg == 0) {
        const int32_t h = J.h0 - (sp.o_del + sp.e_del * (i + 1));
        J.h1 = h > 0 ? h : 0;
    } else {
        J.h1 = 0;
    }
    J.j = J.beg;
    J.f = 0; J.key = -1; J.fnz = 0x7FFFFFFF; J.lnz = -1;
    const uint2 p = pools[tcode_at(tn, lane, i)];
    J.pool_lo = p.x;
    J.pool_hi = p.y;
}

}  // namespace

__host__ __device__ inline size_t lane_warp_bytes(int qcap, int tcap) {
    return (size_t)128 * (lane_eh_words(qcap) + lane_nib_words(qcap) + lane_nib_words(tcap));
}

size_t lane_smem_per_warp(int qcap, int tcap) { return lane_warp_bytes(qcap, tcap); }

__global__ void __launch_bounds__(128) lane_kernel(LaunchDesc d, ScoreParams sp) {
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
    uint32_t* base = reinterpret_cast<uint32_t*>(smem + (size_t)warp * lane_warp_bytes(qcap, tcap));
    uint32_t* eh = base;                                         // [slot*32 + lane]
    uint32_t* qn = eh + 32 * lane_eh_words(qcap);                // [word*32 + lane]
    uint32_t* tn = qn + 32 * lane_nib_words(qcap);
    const int n = d.count ? *d.count : d.n;
    const int* order = d.order ? d.order + (d.order_off ? *d.order_off : 0) : nullptr;
    const int refill = d.warp_batch ? 32 : (d.refill > 0 ? d.refill : 1);

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
                    if (c.qlen > qcap || c.tlen > tcap || !job_is_narrow(c, sp.max_sc)) {
                        d.out[job] = g3x_ext_t{0, 0, 0, 0, 0, 0};
                        d.status[job] = G3X_ERR_TOO_LONG;
                        if (d.cells) d.cells[job] = 0;
                    } else {
                        my_job = job;
                        J.job = job;
                        J.qlen = c.qlen; J.tlen = c.tlen; J.w = c.w; J.h0 = c.h0;
                        commit_init(J.K, c);
                        J.i = 0; J.beg = 0; J.end = c.qlen;
                        J.j = -1;                          // row 0 not begun
                    }
                }
            }
            unsigned m = __ballot_sync(0xFFFFFFFFu, my_job >= 0);
            while (m) {
                const int L = __ffs(m) - 1;
                m &= m - 1;
                const int job = __shfl_sync(0xFFFFFFFFu, my_job, L);
                const g3x_job_t jb = d.jobs[job];
                const int qlen = jb.qlen, tlen = jb.tlen;
                const bool qrev = (jb.flags & G3X_JOB_QREV) != 0, trev = (jb.flags & G3X_JOB_TREV) != 0;
                for (int ch = lane; (ch << 4) < qlen; ch += 32) {
                    uint32_t x, nb;
                    load16(d.codes, d.nmask, jb.q_off, qlen, ch, qrev, x, nb);
                    const uint64_t v = nibbles16(x, nb);
                    qn[(2 * ch) * 32 + L] = (uint32_t)v;
                    qn[(2 * ch + 1) * 32 + L] = (uint32_t)(v >> 32);
                }
                for (int ch = lane; (ch << 4) < tlen; ch += 32) {
                    uint32_t x, nb;
                    load16(d.codes, d.nmask, jb.t_off, tlen, ch, trev, x, nb);
                    const uint64_t v = nibbles16(x, nb);
                    tn[(2 * ch) * 32 + L] = (uint32_t)v;
                    tn[(2 * ch + 1) * 32 + L] = (uint32_t)(v >> 32);
                }
                JobConst c;
                c.qlen = qlen; c.h0 = jb.h0; c.oe_ins = sp.oe_ins; c.e_ins = sp.e_ins;
                for (int k = lane; k <= qlen + 1; k += 32) eh[ehw(k, L)] = (uint32_t)init_h(k, c) << 16;
            }
            __syncwarp();
        }
        const bool active = J.job >= 0;
        if (!__any_sync(0xFFFFFFFFu, active)) {
            if (exhausted) break;
            continue;
        }
        if (active) ++busy; else ++idle;
        // A freshly staged job begins its first row (a job with tlen == 0 has none).
        if (active && !J.K.stop && J.j < 0) begin_row(J, sp, tn, lane, pools);
        if (active && !J.K.stop) {
            // ---- one block of up to eight columns of the current row ----
            if (J.j < J.end) {
                const int32_t jb = J.j & ~(kLB - 1);
                const uint32_t qw = qn[(jb >> 3) * 32 + lane];
                // the block's eight slots, loaded up front (slots past the row are never used)
                uint32_t* ep = eh + ehw(jb, lane);
                const uint4 wa = *reinterpret_cast<const uint4*>(ep);
                const uint4 wb = *reinterpret_cast<const uint4*>(ep + 128);
                const uint32_t wv[kLB] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
                const uint32_t sc_lo = __byte_perm(J.pool_lo, J.pool_hi, qw & 0xFFFFu);
                const uint32_t sc_hi = __byte_perm(J.pool_lo, J.pool_hi, qw >> 16);
                int32_t h1 = J.h1, f = J.f, key = J.key, fnz = J.fnz, lnz = J.lnz;
                const int32_t lo = J.j, hi = J.end;
#pragma unroll
                for (int t = 0; t < kLB; ++t) {
                    const int32_t col = jb + t;
                    if (col >= lo && col < hi) {
                        const uint32_t w = wv[t];
                        const int32_t hd = (int32_t)(w >> 16), ed = (int32_t)(w & 0xFFFFu);
                        const uint32_t sw = t < 4 ? sc_lo : sc_hi;
                        const int32_t s = (int32_t)(int8_t)(sw >> (8 * (t & 3)));
                        const int32_t M = addmin_i32(hd, s, hd << 8);
                        const int32_t h = max3_i32(M, ed, f);
                        const int32_t te = addmax_i32(M, -sp.oe_del, 0);
                        const int32_t e2 = addmax_i32(ed, -sp.e_del, te);
                        const uint32_t nw = ((uint32_t)h1 << 16) | (uint32_t)e2;
                        ep[(t >> 2) * 128 + (t & 3)] = nw;
                        if (nw) { lnz = col; fnz = fnz < col ? fnz : col; }
                        const int32_t k2 = (h << 16) | col;
                        key = key > k2 ? key : k2;
                        const int32_t tf = addmax_i32(M, -sp.oe_ins, 0);
                        f = addmax_i32(f, -sp.e_ins, tf);
                        h1 = h;
                    }
                }
                J.h1 = h1; J.f = f; J.key = key; J.fnz = fnz; J.lnz = lnz;
                J.j = jb + kLB < hi ? jb + kLB : hi;
            }
            // ---- row end (ksw.cu:371-391) and the next row ----
            if (J.j >= J.end) {
                const int32_t beg = J.beg, end = J.end;
                const bool nonempty = beg < end;
                if (end >= 0) eh[ehw(end, lane)] = (uint32_t)J.h1 << 16;
                if (nonempty && J.h1 != 0) J.lnz = end;
                RowDone rd;
                rd.m = J.key < 0 ? 0 : (J.key >> 16);
                rd.mj = J.key < 0 ? -1 : (J.key & 0xFFFF);
                rd.gval = (nonempty ? end : beg) == J.qlen ? J.h1 : -1;
                rd.ncells = nonempty ? end - beg : 0;
                JobConst c;
                c.qlen = J.qlen; c.tlen = J.tlen; c.w = J.w; c.h0 = J.h0;
                c.o_del = sp.o_del; c.e_del = sp.e_del; c.o_ins = sp.o_ins; c.e_ins = sp.e_ins;
                c.oe_del = sp.oe_del; c.oe_ins = sp.oe_ins; c.zdrop = sp.zdrop;
                commit_row(J.K, c, rd);
                if (!J.K.stop) {
                    const int32_t nb = J.fnz < end ? J.fnz : end;
                    const int32_t L = J.lnz >= nb ? J.lnz : nb - 1;
                    J.beg = nb;
                    J.end = L + 2 < J.qlen ? L + 2 : J.qlen;
                    ++J.i;
                    begin_row(J, sp, tn, lane, pools);
                }
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

int launch_lane(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream) {
    const size_t wb = lane_warp_bytes(d.qmax, d.tmax);
    const size_t kMaxSmem = 227 * 1024;
    int wpb = d.warps_per_block > 0 ? d.warps_per_block : 4;
    while (wpb > 1 && (size_t)wpb * wb > kMaxSmem) --wpb;
    if (wb > kMaxSmem) return G3X_ERR_TOO_LONG;
    const size_t smem = (size_t)wpb * wb;
    if (cudaFuncSetAttribute(lane_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return G3X_ERR_CUDA;
    int blocks = d.blocks;
    if (blocks <= 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lane_kernel, 32 * wpb, smem);
        blocks = sms * (per_sm > 0 ? per_sm : 1);
    }
    lane_kernel<<<blocks, 32 * wpb, smem, stream>>>(d, sp);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

}  // namespace g3x

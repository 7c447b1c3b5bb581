// g3x_lane16.cu -- lane-per-job sm_100a kernel for batched ksw_extend2 in int16x2
// (bwa/src/ksw.cu:303-401).
//
// Each lane of a warp runs one job through the reference's row loop; the per-lane logic (row
// begin, the blocks of a row, the row end with its band trims) is in g3x_lane16.cuh, where the
// arithmetic and the band handling are described.  This file is the warp around it:
//  * refill waves: the warp takes a new job for every idle lane at once (one atomicAdd on the
//    class's job queue), and each new lane stages its query as 4-bit codes from the bit planes
//    and writes row -1 of its row buffer (ksw.cu:317-319);
//  * row-synchronous rows: all lanes begin a row together, walk it block by block (a lane with a
//    shorter row sits out the extra iterations), and end it together;
//  * a lane whose job ends writes the job's outputs and status and idles until the next wave.
// Jobs outside the int16 fit or the class's width get G3X_ERR_TOO_LONG (the scheduler never
// sends them here).
#include <cuda_runtime.h>
#include "g3x_core.h"
#include "g3x_internal.h"
#include "g3x_lane16.cuh"
#include "g3x_stage.cuh"

// Phase clocks (profiling builds only, -DG3X_PHASE_CLOCKS): each warp adds the SM clock cycles
// it spends in each phase of its row loop -- refill wave, row begin, the row's blocks, row end,
// output -- to g3x_phase_clocks[class][phase], the class taken as qcap / 32 (capped at 7); slot
// 5 counts warp rows and slot 6 the warp's block iterations.  A __syncwarp before each reading
// makes a phase's time the warp's.  The product library is built without it.
#ifdef G3X_PHASE_CLOCKS
__device__ unsigned long long g3x_phase_clocks[8][8];
extern "C" int g3x_phase_clocks_read(unsigned long long* h, int reset) {
    if (cudaMemcpyFromSymbol(h, g3x_phase_clocks, sizeof(g3x_phase_clocks)) != cudaSuccess) return G3X_ERR_CUDA;
    if (reset) {
        static const unsigned long long zero[8][8] = {};
        if (cudaMemcpyToSymbol(g3x_phase_clocks, zero, sizeof(zero)) != cudaSuccess) return G3X_ERR_CUDA;
    }
    return G3X_OK;
}
#define G3X_PHASE(k) do { __syncwarp(); const long long t1_ = clock64(); ph_[k] += t1_ - t0_; t0_ = t1_; } while (0)
#else
#define G3X_PHASE(k) do { } while (0)
#endif

namespace g3x {

size_t lane16_smem_per_warp(int qcap) { return l16::warp_bytes(qcap); }

template <bool kSym>
__global__ void __launch_bounds__(128) lane16_kernel(LaunchDesc d, ScoreParams sp) {
    pdl_trigger();
    using namespace l16;
    extern __shared__ __align__(16) char smem[];
    __shared__ uint2 pools[5];
    __shared__ uint4 ge[10];
    if (threadIdx.x < 10) {
        const int o = threadIdx.x;
        ge[o] = make_uint4(ge_word(o, 0), ge_word(o, 1), ge_word(o, 2), ge_word(o, 3));
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
    const int nbc = blocks_of(qcap);
    char* base = smem + (size_t)warp * warp_bytes(qcap);
    Planes P;
    P.H = reinterpret_cast<uint4*>(base);
    P.E = P.H + 32 * nbc;
    P.H32 = reinterpret_cast<uint32_t*>(P.H);
    P.E32 = reinterpret_cast<uint32_t*>(P.E);
    uint32_t* qn = reinterpret_cast<uint32_t*>(P.E + 32 * nbc);
    P.qn = qn;
    const int n = d.count ? *d.count : d.n;
    const int* order = d.order ? d.order + (d.order_off ? *d.order_off : 0) : nullptr;
    const int refill = d.warp_batch ? 32 : (d.refill > 0 ? d.refill : 1);
    const PairConst pc = pair_const(sp);

    LaneJob J;
    J.job = -1;
    bool exhausted = false;
    // occupancy counters (diagnostics): 32-bit sums per row, folded into the 64-bit totals at
    // every refill wave, every job end and every 16 rows of a running lane, so a lane's sums
    // span at most 16 rows of its job, or the rows of the warp between its job's end and the next
    // wave
    unsigned long long busy = 0, idle = 0, waves = 0;
    uint32_t busy32 = 0, kmax32 = 0;
#ifdef G3X_PHASE_CLOCKS
    unsigned long long ph_[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    long long t0_ = clock64();
#endif
    for (;;) {
#ifdef G3X_PHASE_CLOCKS
        t0_ = clock64();
#endif
        // ---- refill wave: the warp stages one new job for every idle lane, together ----
        const unsigned idle_mask = __ballot_sync(0xFFFFFFFFu, J.job < 0);
        if (!exhausted && __popc(idle_mask) >= (idle_mask == 0xFFFFFFFFu ? 1 : refill)) {
            const int want = __popc(idle_mask);
            int first = 0;
            if (lane == 0) first = atomicAdd(d.queue, want);
            first = __shfl_sync(0xFFFFFFFFu, first, 0);
            if (first + want >= n) exhausted = true;
            ++waves;
            busy += busy32; idle += kmax32 - busy32; busy32 = kmax32 = 0;
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
                        if (d.rows) d.rows[job] = 0;
                    } else if (!job_in_planes(jb, d.n_bases)) {   // reaches past the planes: unread
                        d.out[job] = g3x_ext_t{0, 0, 0, 0, 0, 0};
                        d.status[job] = G3X_ERR_INVALID;
                        if (d.cells) d.cells[job] = 0;
                        if (d.rows) d.rows[job] = 0;
                    } else {
                        J.job = job;
                        J.qlen = c.qlen; J.tlen = c.tlen; J.w = c.w; J.h0 = c.h0;
                        J.t_off = jb.t_off;
                        J.trev = (jb.flags & G3X_JOB_TREV) != 0;
                        commit_init(J.K, c);
                        J.beg = 0; J.end = c.qlen;
                        J.tx = J.tn = 0;
                        J.pv = J.pm = 0;
                        if (c.tlen > 0) load16(d.codes, d.nmask, J.t_off, c.tlen, 0, J.trev, J.tx, J.tn);
                        if (c.tlen > 16) load16_raw(d.codes, d.nmask, J.t_off, c.tlen, 1, J.trev, J.pv, J.pm);
                        stage_own_query(d.codes, d.nmask, jb.q_off, c.qlen, (jb.flags & G3X_JOB_QREV) != 0,
                                        (c.qlen + 15) >> 4, qn, lane);
                        // row -1 of the new job (ksw.cu:317-319), each new lane its own
                        init_row(P, lane, c.qlen, c.h0, sp, pc, ge);
                    }
                }
            }
            __syncwarp();
        }
        G3X_PHASE(0);
        const bool active = J.job >= 0;
        if (!__any_sync(0xFFFFFFFFu, active)) {
            if (exhausted) break;
            continue;
        }
        const bool run = active && !J.K.stop;

        // ---- row begin (ksw.cu:335-345) ----
        RowState r;                             // set by row_begin; read only by running lanes
        if (run) {
            const int32_t i = J.K.next;
            if ((i & 15) == 0 && i > 0) {       // the prefetched chunk, then the next one's words
                busy += busy32; idle += kmax32 - busy32; busy32 = kmax32 = 0;
                decode16(J.t_off, J.tlen, i >> 4, J.trev, J.pv, J.pm, J.tx, J.tn);
                const int ch = (i >> 4) + 1;
                if ((ch << 4) < J.tlen) load16_raw(d.codes, d.nmask, J.t_off, J.tlen, ch, J.trev, J.pv, J.pm);
            }
            row_begin(J, sp, pools, r);
        }
        G3X_PHASE(1);
        const bool nonempty = run && r.beg < r.end;
        const int nblk = run ? blocks_in_row(r) : 0;
        const int kmax = __reduce_max_sync(0xFFFFFFFFu, (unsigned)nblk);
        const bool any_single = __any_sync(0xFFFFFFFFu, nblk == 1);
        busy32 += nblk;
        kmax32 += kmax;

        // ---- the row's blocks: masked first block, middle blocks two at a time, masked last block ----
        uint32_t mF, mL;
        row_blocks<kSym>(P, lane, r, pc, ge, nblk, kmax, any_single, mF, mL);

        // ---- row end (ksw.cu:371-391) ----
        G3X_PHASE(2);
        if (run) row_end(J, P, lane, r, sp, nonempty, mF, mL);
        G3X_PHASE(3);
        if (active && J.K.stop) {
            const Commit& K = J.K;
            d.out[J.job] = g3x_ext_t{K.best, K.best_j + 1, K.best_i + 1, K.max_ie + 1, K.gscore, K.max_off};
            d.status[J.job] = G3X_OK;
            if (d.cells) d.cells[J.job] = (int32_t)K.cells;
            if (d.rows) d.rows[J.job] = K.next;
            J.job = -1;
            busy += busy32; idle += kmax32 - busy32; busy32 = kmax32 = 0;
        }
        __syncwarp();
#ifdef G3X_PHASE_CLOCKS
        G3X_PHASE(4);
        ph_[5] += 1;
        ph_[6] += kmax;
#endif
    }
#ifdef G3X_PHASE_CLOCKS
    if (lane == 0) {
        const int ci = qcap / 32 < 8 ? qcap / 32 : 7;
        for (int q = 0; q < 7; ++q) atomicAdd(&g3x_phase_clocks[ci][q], ph_[q]);
    }
#endif
    busy += busy32; idle += kmax32 - busy32;
    if (d.stats) add_warp_stats(d.stats, busy, idle, waves, lane);
    pdl_chain_end();
}

template <bool kSym>
static int launch_lane16_t(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream) {
    const size_t wb = l16::warp_bytes(d.qmax);
    size_t max_smem = 0;
    if (allow_max_smem(lane16_kernel<kSym>, &max_smem) != cudaSuccess) return G3X_ERR_CUDA;
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
        per_sm = resident_blocks(lane16_kernel<kSym>, 32 * wpb, smem);
        if (per_sm * wpb >= best_warps) { best_warps = per_sm * wpb; best_wpb = wpb; best_blocks = per_sm; }
    }
    const size_t smem = (size_t)best_wpb * wb;
    const int blocks = d.blocks > 0 ? d.blocks : sms * (best_blocks > 0 ? best_blocks : 1);
    if (launch_class_kernel(lane16_kernel<kSym>, blocks, 32 * best_wpb, smem, stream, d, sp) != cudaSuccess)
        return G3X_ERR_CUDA;
    return G3X_OK;
}

// Gap opening and extension costs that agree between deletions and insertions (oe_del == oe_ins,
// BWA's defaults) let the E step reuse the F step's max(M - oe, 0).
int launch_lane16(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream) {
    return sp.oe_del == sp.oe_ins ? launch_lane16_t<true>(d, sp, stream) : launch_lane16_t<false>(d, sp, stream);
}

}  // namespace g3x

// g3x_rowpar.cu -- row-parallel sm_100a kernels for batched ksw_extend2
// (bwa/src/ksw.cu:303-401).
//
// A job is run by a group of G lanes that computes the DP one target row at a time, in
// exactly the reference's row order, over exactly the reference's band [beg, end)
// (ksw.cu:338-340, 388-391).  A row is covered in tiles of S = G*C columns; lane r owns
// columns [t0 + r*C, t0 + r*C + C) of the tile starting at t0.
//
// Per row the cell recurrences split into column-independent work and one horizontal
// dependency.  M (the diagonal), E (vertical gaps) and the row buffer reads depend only on
// the previous row.  F (horizontal gaps) is the max-plus recurrence
//     F(j+1) = max(F(j) - e_ins, max(M(j) - oe_ins, 0)),   F(beg) = 0
// whose solution F(j+1) = max_{k<=j} (max(M(k)-oe_ins,0) - (j-k)*e_ins) is an exact
// integer prefix maximum with linear decay.  Each lane runs the recurrence over its own
// columns from F = 0, the group combines the lane results with a warp-shuffle scan
// (log2 G steps), and each lane then corrects its columns with the carried-in value.
// H = max(M, E, F) follows, and H(i, j-1) for a lane's first column comes from the
// previous lane by one shuffle.  The row maximum (ties: last column) is a shuffle
// max-reduction of (H << 16 | column) keys, and the next row's band comes from the first
// and last non-zero buffer entries (two more reductions), applied exactly as ksw.cu:388-391.
// The per-row bookkeeping (to-end score, max tracking, z-drop; ksw.cu:371-386) runs once per
// row, uniformly in the group.
//
// The warp holds 32/G groups and runs one loop for all of them: each iteration, every group
// with a job advances one row; a group whose job finished stages its next job first.
#include <cuda_runtime.h>
#include "g3x_core.h"
#include "g3x_internal.h"
#include "g3x_stage.cuh"

namespace g3x {

namespace {

constexpr int32_t kNeg = -0x3FFFFFFF;   // below every score; "no value" in max-scans

// Reductions over one group (aligned lanes gbase .. gbase+G-1; XOR partners stay inside).
template <int G>
__device__ __forceinline__ int32_t group_max(int32_t v, unsigned gmask) {
#pragma unroll
    for (int d = G / 2; d >= 1; d >>= 1) {
        const int32_t o = __shfl_xor_sync(gmask, v, d);
        v = v > o ? v : o;
    }
    return v;
}

template <int G>
__device__ __forceinline__ int32_t group_min(int32_t v, unsigned gmask) {
#pragma unroll
    for (int d = G / 2; d >= 1; d >>= 1) {
        const int32_t o = __shfl_xor_sync(gmask, v, d);
        v = v < o ? v : o;
    }
    return v;
}

// Loop-carried per-job state.  Only the per-job constants live here; the scoring constants
// are read from the kernel parameters (constant bank) when a row is computed.
struct RowJob {
    int job;             // job index, -1 = none
    int narrow;
    int32_t qlen, tlen, w, h0;
    Commit K;
    int32_t i;           // current row
    int32_t beg, end;    // band carried from the previous row (before this row's clamps)
    int32_t err;
};

__device__ __forceinline__ JobConst job_const(const RowJob& J, const ScoreParams& sp) {
    JobConst c;
    c.qlen = J.qlen; c.tlen = J.tlen; c.w = J.w; c.h0 = J.h0;
    c.o_del = sp.o_del; c.e_del = sp.e_del; c.o_ins = sp.o_ins; c.e_ins = sp.e_ins;
    c.oe_del = sp.oe_del; c.oe_ins = sp.oe_ins; c.zdrop = sp.zdrop;
    return c;
}

}  // namespace

// One row of one job.  All lanes of the group call it with identical (uniform) arguments;
// every shuffle names only the group's lanes, so groups of a warp may take different paths.
template <int G, int C, bool kNarrow>
__device__ __forceinline__ void dp_row(RowJob& J, const ScoreParams& sp, EhSlot32* __restrict__ eh,
                                       const int8_t* __restrict__ qp, const SmemTgt& tg, int qs,
                                       int r, int gbase, unsigned gmask) {
    const JobConst c = job_const(J, sp);
    const int32_t i = J.i;
    int32_t beg = J.beg, end = J.end;
    if (beg < i - c.w) beg = i - c.w;                     // ksw.cu:338-340
    if (end > i + c.w + 1) end = i + c.w + 1;
    if (end > c.qlen) end = c.qlen;
    int32_t h1 = 0;
    if (beg == 0) {                                        // ksw.cu:342-345
        h1 = c.h0 - (c.o_del + c.e_del * (i + 1));
        h1 = h1 > 0 ? h1 : 0;
    }
    const int8_t* __restrict__ prow = qp + tg.code(i) * qs;
    constexpr int S = G * C;
    int32_t fcarry = 0;                                    // F entering the tile
    int32_t key = -1, m = 0, mj = -1;                      // row max / last column reaching it
    int32_t fnz = 0x7FFFFFFF, lnz = -1;                    // first / last non-zero entry
    const int src_prev = gbase + ((r + G - 1) & (G - 1));
    for (int32_t t0 = beg; t0 < end; t0 += S) {            // uniform in the group
        const int32_t a = t0 + r * C;
        const int32_t tend = t0 + S < end ? t0 + S : end;
        int32_t Mv[C], Ev[C], Fv[C];
        int32_t f = 0;
#pragma unroll
        for (int k = 0; k < C; ++k) {                      // pass 1: M, E(i,j), lane-local F
            const int32_t col = a + k;
            if (col < tend) {
                const int2 v = *reinterpret_cast<const int2*>(eh + col);
                const int32_t s = prow[col];
                Mv[k] = addmin_i32(v.x, s, v.x << 8);
                Ev[k] = v.y;
                Fv[k] = f;
                const int32_t tf = addmax_i32(Mv[k], -c.oe_ins, 0);
                f = addmax_i32(f, -c.e_ins, tf);
            } else {
                Mv[k] = 0; Ev[k] = 0; Fv[k] = kNeg;
            }
        }
        // F leaving each lane's columns, scanned over the group: x = F entering column a + C.
        int32_t x = f;
#pragma unroll
        for (int d = 1; d < G; d <<= 1) {
            const int32_t y = __shfl_up_sync(gmask, x, d, G);
            if (r >= d) x = addmax_i32(y, -d * C * c.e_ins, x);
        }
        int32_t fin = __shfl_up_sync(gmask, x, 1, G);
        if (r == 0) fin = kNeg;
        fin = addmax_i32(fcarry, -r * C * c.e_ins, fin);   // F entering column a
        // pass 2a: H for every column of the lane
        int32_t dec = fin;
#pragma unroll
        for (int k = 0; k < C; ++k) {
            const int32_t F = dec > Fv[k] ? dec : Fv[k];
            Fv[k] = max3_i32(Mv[k], Ev[k], F);             // Fv now holds H(i, a+k)
            dec -= c.e_ins;
        }
        // H(i, a-1) from the previous lane; lane 0 takes the value carried into the tile
        const int32_t hlast_lane = Fv[C - 1];
        int32_t hprev = __shfl_sync(gmask, hlast_lane, src_prev);
        if (r == 0) hprev = h1;
        // pass 2b: E(i+1,j), row-buffer writes, row max, non-zero span
#pragma unroll
        for (int k = 0; k < C; ++k) {
            const int32_t col = a + k;
            if (col < tend) {
                const int32_t te = addmax_i32(Mv[k], -c.oe_del, 0);
                const int32_t e2 = addmax_i32(Ev[k], -c.e_del, te);
                *reinterpret_cast<int2*>(eh + col) = make_int2(hprev, e2);
                if ((hprev | e2) != 0) {
                    lnz = col;
                    fnz = fnz < col ? fnz : col;
                }
                const int32_t h = Fv[k];
                if (kNarrow) {
                    const int32_t k2 = (h << 16) | col;
                    key = key > k2 ? key : k2;
                } else {
                    if (h >= m) { m = h; mj = col; }
                }
                hprev = h;
            }
        }
        // carries into the next tile: F entering tend (used only when the tile was full) and
        // H at the tile's last column, held by the lane owning column tend - 1
        const int32_t xl = __shfl_sync(gmask, x, gbase + G - 1);
        fcarry = addmax_i32(fcarry, -S * c.e_ins, xl);
        h1 = __shfl_sync(gmask, hprev, gbase + (tend - 1 - t0) / C);
    }
    // Row end, ksw.cu:371-375.  h1 is H(i, end-1) for a non-empty row, the first-column value
    // otherwise; the loop variable j is end, or beg for an empty row.
    const bool nonempty = beg < end;
    if (r == 0 && end >= 0) *reinterpret_cast<int2*>(eh + end) = make_int2(h1, 0);
    const int32_t jfin = nonempty ? end : beg;
    RowDone d;
    if (kNarrow) {
        key = group_max<G>(key, gmask);
        d.m = key < 0 ? 0 : (key >> 16);
        d.mj = key < 0 ? -1 : (key & 0xFFFF);
    } else {
        // (m, mj) with ties on the larger column
        const int32_t mm = group_max<G>(m, gmask);
        const int32_t cand = m == mm ? mj : -1;
        d.m = mm;
        d.mj = group_max<G>(cand, gmask);
        if (mm == 0 && !nonempty) d.mj = -1;
    }
    d.gval = jfin == c.qlen ? h1 : -1;
    d.ncells = nonempty ? end - beg : 0;
    commit_row(J.K, c, d);
    if (J.K.stop) return;
    // next band, ksw.cu:388-391: first non-zero in [beg, end), last non-zero in [beg', end]
    fnz = group_min<G>(fnz, gmask);
    lnz = group_max<G>(lnz, gmask);
    if (h1 != 0 && nonempty) lnz = end;                    // eh[end] = {h1, 0}
    const int32_t nb = fnz < end ? fnz : end;
    const int32_t L = lnz >= nb ? lnz : nb - 1;
    J.beg = nb;
    J.end = L + 2 < c.qlen ? L + 2 : c.qlen;
    J.i = i + 1;
}

template <int G, int C>
__global__ void __launch_bounds__(128) rowpar_kernel(LaunchDesc d, ScoreParams sp) {
    pdl_trigger();
    extern __shared__ __align__(16) char smem[];
    const int lane = threadIdx.x & 31;
    const int r = lane & (G - 1);
    const int gbase = lane & ~(G - 1);
    const unsigned gmask = G == 32 ? 0xFFFFFFFFu : (((1u << G) - 1u) << gbase);
    const int groups_per_block = blockDim.x / G;
    const int gib = threadIdx.x / G;
    const int qs = qstride_of(d.qmax);
    char* gsm = smem + (size_t)gib * group_bytes(d.qmax, d.tmax);
    EhSlot32* eh = reinterpret_cast<EhSlot32*>(gsm);
    int8_t* qp = reinterpret_cast<int8_t*>(gsm + align16(eh_slots(d.qmax) * (int)sizeof(EhSlot32)));
    uint64_t* tgt = reinterpret_cast<uint64_t*>(reinterpret_cast<char*>(qp) + align16(5 * qs));
    const int n = d.count ? *d.count : d.n;
    const SmemTgt tg{tgt};

    const int* order = d.order ? d.order + (d.order_off ? *d.order_off : 0) : nullptr;
    RowJob J;
    J.job = -1;
    bool exhausted = false;
    int static_slot = blockIdx.x * groups_per_block + gib;
    const int gw = lane / G;                 // group index within the warp
    constexpr int kGroupsPerWarp = 32 / G;
    unsigned long long busy_rows = 0, idle_rows = 0, batches = 0;
    for (;;) {
        if (d.persistent && d.warp_batch) {
            // All groups of the warp take their next jobs together, once every group is done.
            if (!__any_sync(0xFFFFFFFFu, J.job >= 0)) {
                if (exhausted) break;
                int base = 0;
                if (lane == 0) base = atomicAdd(d.queue, kGroupsPerWarp);
                base = __shfl_sync(0xFFFFFFFFu, base, 0);
                if (base >= n) break;
                ++batches;
                const int slot = base + gw;
                if (base + kGroupsPerWarp >= n) exhausted = true;
                if (slot < n) {
                    const int job = order ? order[slot] : slot;
                    StagedJob sj;
                    uint32_t prof_lo[5], prof_hi[5];
                    score_pools(sp, prof_lo, prof_hi);
                    if (stage_job<G>(job, d, sp, prof_lo, prof_hi, eh, qp, tgt, qs, r, sj)) {
                        J.job = job; J.narrow = sj.narrow;
                        J.qlen = sj.c.qlen; J.tlen = sj.c.tlen; J.w = sj.c.w; J.h0 = sj.c.h0;
                        commit_init(J.K, sj.c);
                        J.i = 0;
                        J.beg = 0;
                        J.end = sj.c.qlen;
                        J.err = G3X_OK;
                    }
                }
            }
        } else if (J.job < 0 && !exhausted) {
            for (;;) {
                int slot;
                if (d.persistent) {
                    slot = 0;
                    if (r == 0) slot = atomicAdd(d.queue, 1);
                    slot = __shfl_sync(gmask, slot, 0, G);
                } else {
                    slot = static_slot;
                    static_slot = 0x7FFFFFFF;
                }
                if (slot >= n) { exhausted = true; break; }
                const int job = order ? order[slot] : slot;
                StagedJob sj;
                uint32_t prof_lo[5], prof_hi[5];
                score_pools(sp, prof_lo, prof_hi);
                if (stage_job<G>(job, d, sp, prof_lo, prof_hi, eh, qp, tgt, qs, r, sj)) {
                    J.job = job; J.narrow = sj.narrow;
                    J.qlen = sj.c.qlen; J.tlen = sj.c.tlen; J.w = sj.c.w; J.h0 = sj.c.h0;
                    commit_init(J.K, sj.c);
                    J.i = 0;
                    J.beg = 0;
                    J.end = sj.c.qlen;
                    J.err = G3X_OK;
                    break;
                }
            }
        }
        __syncwarp();
        const bool active = J.job >= 0;
        if (!__any_sync(0xFFFFFFFFu, active)) {
            if (d.persistent && d.warp_batch && !exhausted) continue;   // every job was rejected
            break;
        }
        if (active) ++busy_rows; else ++idle_rows;
        if (active) {
            if (!J.K.stop) {
                if (J.narrow) dp_row<G, C, true>(J, sp, eh, qp, tg, qs, r, gbase, gmask);
                else dp_row<G, C, false>(J, sp, eh, qp, tg, qs, r, gbase, gmask);
            }
            if (J.K.stop) {
                const Commit& K = J.K;
                if (r == 0) {
                    d.out[J.job] = g3x_ext_t{K.best, K.best_j + 1, K.best_i + 1, K.max_ie + 1, K.gscore, K.max_off};
                    d.status[J.job] = J.err;
                    if (d.cells) d.cells[J.job] = (int32_t)K.cells;
                    if (d.rows) d.rows[J.job] = K.next;
                }
                J.job = -1;
            }
        }
        __syncwarp();
    }
    if (d.stats && r == 0) {
        atomicAdd(d.stats + 0, busy_rows);
        atomicAdd(d.stats + 1, idle_rows);
        if (gw == 0) atomicAdd(d.stats + 2, batches);
    }
    pdl_chain_end();
}

template <int G, int C>
static int launch_rp(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream) {
    int wpb = d.warps_per_block > 0 ? d.warps_per_block : 1;
    const size_t gb = group_bytes(d.qmax, d.tmax);
    size_t max_smem = 0;
    if (allow_max_smem(rowpar_kernel<G, C>, &max_smem) != cudaSuccess) return G3X_ERR_CUDA;
    while (wpb > 1 && (size_t)(32 * wpb / G) * gb > max_smem) --wpb;
    const int threads = 32 * wpb;
    const int groups = threads / G;
    const size_t smem = groups * gb;
    if (smem > max_smem) return G3X_ERR_TOO_LONG;
    int blocks;
    if (d.persistent) {
        blocks = d.blocks;
        if (blocks <= 0) {
            int dev = 0, sms = 0, per_sm = 0;
            cudaGetDevice(&dev);
            sms = sm_count();
            per_sm = resident_blocks(rowpar_kernel<G, C>, threads, smem);
            blocks = sms * (per_sm > 0 ? per_sm : 1);
        }
    } else {
        blocks = (d.n + groups - 1) / groups;
        if (blocks == 0) return G3X_OK;
    }
    if (launch_class_kernel(rowpar_kernel<G, C>, blocks, threads, smem, stream, d, sp) != cudaSuccess)
        return G3X_ERR_CUDA;
    return G3X_OK;
}

// C is odd: lane r's columns start 2*C*r words apart in the 8-byte row-buffer slots, so the
// 16 lanes of a half-warp touch 16 distinct bank pairs on every cell load and store.
int launch_rowpar(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream) {
    switch (d.lanes * 100 + d.tile) {
        case 4 * 100 + 5: return launch_rp<4, 5>(d, sp, stream);
        case 4 * 100 + 9: return launch_rp<4, 9>(d, sp, stream);
        case 4 * 100 + 13: return launch_rp<4, 13>(d, sp, stream);
        case 8 * 100 + 5: return launch_rp<8, 5>(d, sp, stream);
        case 8 * 100 + 9: return launch_rp<8, 9>(d, sp, stream);
        case 8 * 100 + 13: return launch_rp<8, 13>(d, sp, stream);
        case 16 * 100 + 5: return launch_rp<16, 5>(d, sp, stream);
        case 16 * 100 + 9: return launch_rp<16, 9>(d, sp, stream);
        case 16 * 100 + 13: return launch_rp<16, 13>(d, sp, stream);
        case 32 * 100 + 5: return launch_rp<32, 5>(d, sp, stream);
        case 32 * 100 + 9: return launch_rp<32, 9>(d, sp, stream);
        case 32 * 100 + 13: return launch_rp<32, 13>(d, sp, stream);
        default: return G3X_ERR_INVALID;
    }
}

}  // namespace g3x

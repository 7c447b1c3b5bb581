// g3x_kernels.cu -- sm_100a kernels for batched ksw_extend2 (bwa/src/ksw.cu:303-401).
//
// Rolling anti-diagonal family.  A job is run by a group of G lanes (G = 8, 16 or 32) that
// sweeps anti-diagonals of the
// banded DP with the rolling-row protocol of g3x_core.h.  A warp holds 32/G groups and runs
// ONE step loop for all of them: every iteration each group with a job advances one step,
// and a group whose job finished stages its next job in the same iteration.  All warp
// collectives (progress shuffles, the row-end ballot, the commit broadcast) use the full
// warp with per-lane source lanes, so groups never split the warp's instruction stream
// except while one of them stages a job.
// The per-job shared-memory working set and its staging are in g3x_stage.cuh.
#include <cuda_runtime.h>
#include "g3x_core.h"
#include "g3x_internal.h"
#include "g3x_stage.cuh"

namespace g3x {

size_t group_smem_bytes(int qmax, int tmax) { return group_bytes(qmax, tmax); }

// Per-group job state of the rolling kernel, identical in every lane of the group.
struct GroupJob {
    int job;          // job index, -1 = none
    int narrow;
    JobConst c;
    Commit K;
    long long steps, limit;
};

template <int G>
__global__ void __launch_bounds__(256) extend_kernel(LaunchDesc d, ScoreParams sp) {
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
    const int pred = gbase + ((r + G - 1) & (G - 1));

    uint32_t prof_lo[5], prof_hi[5];
    score_pools(sp, prof_lo, prof_hi);

    GroupJob gj;
    gj.job = -1;
    Lane L;
    lane_init(L, 0, 0);
    int32_t err = G3X_OK;
    bool exhausted = false;
    int static_slot = blockIdx.x * groups_per_block + gib;   // non-persistent: one slot
    const SmemTgt tg{tgt};
    SmemEh buf{eh};

    for (;;) {
        // A group without a job stages its next one (divergent across groups, short).
        if (gj.job < 0 && !exhausted) {
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
                const int job = d.order ? d.order[slot] : slot;
                StagedJob sj;
                if (stage_job<G>(job, d, sp, prof_lo, prof_hi, eh, qp, tgt, qs, r, sj)) {
                    gj.job = job; gj.narrow = sj.narrow; gj.c = sj.c;
                    commit_init(gj.K, gj.c);
                    gj.steps = 0;
                    // Every step either advances a row or moves a lane between states; the
                    // oldest unfinished row always advances, so this bound is never reached
                    // by a correct run.  It turns a logic error into a per-job status.
                    gj.limit = d.step_limit > 0 ? d.step_limit
                                                : 8LL * ((long long)gj.c.tlen + 2) * ((long long)gj.c.qlen + 8) + 4096;
                    lane_init(L, r, gj.c.tlen);
                    err = G3X_OK;
                    break;
                }
            }
        }
        __syncwarp();
        const bool active = gj.job >= 0;
        if (!__any_sync(0xFFFFFFFFu, active)) break;

        const uint32_t pp = __shfl_sync(0xFFFFFFFFu, lane_prog(L), pred);
        const uint32_t pf = __shfl_sync(0xFFFFFFFFu, lane_fnz(L), pred);
        RowDone rd;
        rd.m = rd.mj = rd.gval = rd.ncells = 0;
        bool fin = false;
        if (active) {
            fin = gj.narrow ? lane_step<G, true>(L, gj.c, pp, pf, buf, qp, tg, qs, &rd)
                            : lane_step<G, false>(L, gj.c, pp, pf, buf, qp, tg, qs, &rd);
        }
        const unsigned b = __ballot_sync(0xFFFFFFFFu, fin);
        if (b) {
            const unsigned mine = G == 32 ? b : ((b >> gbase) & ((1u << G) - 1u));
            const int src = mine ? gbase + __ffs(mine) - 1 : lane;
            RowDone cd;
            cd.m = __shfl_sync(0xFFFFFFFFu, rd.m, src);
            cd.mj = __shfl_sync(0xFFFFFFFFu, rd.mj, src);
            cd.gval = __shfl_sync(0xFFFFFFFFu, rd.gval, src);
            cd.ncells = __shfl_sync(0xFFFFFFFFu, rd.ncells, src);
            if (mine) {
                if (__popc(mine) != 1) { err = G3X_ERR_INTERNAL; gj.K.stop = 1; }
                else commit_row(gj.K, gj.c, cd);
            }
        }
        if (active) {
            if (++gj.steps > gj.limit) { err = G3X_ERR_TIMEOUT; gj.K.stop = 1; }
            if (gj.K.stop) {
                const Commit& K = gj.K;
                if (r == 0) {
                    d.out[gj.job] = g3x_ext_t{K.best, K.best_j + 1, K.best_i + 1, K.max_ie + 1, K.gscore, K.max_off};
                    d.status[gj.job] = err;
                    if (d.cells) d.cells[gj.job] = (int32_t)K.cells;
                    if (d.rows) d.rows[gj.job] = K.next;
                }
                gj.job = -1;
            }
        }
        __syncwarp();
    }
}

template <int G>
static int launch_g(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream) {
    int wpb = d.warps_per_block > 0 ? d.warps_per_block : 1;
    const size_t gb = group_bytes(d.qmax, d.tmax);
    size_t max_smem = 0;
    if (allow_max_smem(extend_kernel<G>, &max_smem) != cudaSuccess) return G3X_ERR_CUDA;
    while (wpb > 1 && (size_t)(32 * wpb / G) * gb > max_smem) --wpb;   // fewer warps for long jobs
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
            per_sm = resident_blocks(extend_kernel<G>, threads, smem);
            blocks = sms * (per_sm > 0 ? per_sm : 1);
        }
    } else {
        blocks = (d.n + groups - 1) / groups;
        if (blocks == 0) return G3X_OK;
    }
    extend_kernel<G><<<blocks, threads, smem, stream>>>(d, sp);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

int launch_rolling(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream) {
    switch (d.lanes) {
        case 8: return launch_g<8>(d, sp, stream);
        case 16: return launch_g<16>(d, sp, stream);
        case 32: return launch_g<32>(d, sp, stream);
        default: return G3X_ERR_INVALID;
    }
}

int launch_extend(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream) {
    if (d.kernel == kKernelLane) return launch_lane(d, sp, stream);
    if (d.kernel == kKernelLane16) return launch_lane16(d, sp, stream);
    if (d.kernel == kKernelLane2) return launch_lane2(d, sp, stream);
    if (d.kernel == kKernelBand) return launch_band(d, sp, stream);
    return d.kernel == kKernelRowpar ? launch_rowpar(d, sp, stream) : launch_rolling(d, sp, stream);
}

}  // namespace g3x

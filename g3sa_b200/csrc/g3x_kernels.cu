// g3x_kernels.cu -- sm_100a kernels for batched ksw_extend2 (bwa/src/ksw.cu:303-401).
//
// A job is run by a group of G lanes (G = 8, 16 or 32) that sweeps anti-diagonals of the
// banded DP with the rolling-row protocol of g3x_core.h.  Per group, shared memory holds
// the job's working set:
//   eh   : the reference's H/E row buffer, qmax + 2 entries (ksw.cu:310)
//   qp   : the query profile, 5 rows of qstride int8 scores (ksw.cu:309, 312-315)
//   tgt  : the target codes, one byte per base
// Lanes exchange row progress with one warp shuffle per word per step; H/E values travel
// through the shared row buffer exactly as in the scalar loop.
#include <cuda_runtime.h>
#include "g3x_core.h"
#include "g3x_internal.h"

namespace g3x {

// int32 H/E slot of the shared row buffer.
struct EhSlot32 {
    int32_t h, e;
};

// The row buffer as lane_step sees it: one aligned block of four slots is read with two
// 16-byte shared loads; each computed cell is written back with one 8-byte store.
struct SmemEh {
    EhSlot32* p;
    __device__ __forceinline__ void load4(int jb, EhCell v[4]) const {
        const int4 a = *reinterpret_cast<const int4*>(p + jb);
        const int4 b = *reinterpret_cast<const int4*>(p + jb + 2);
        v[0] = EhCell{a.x, a.y}; v[1] = EhCell{a.z, a.w};
        v[2] = EhCell{b.x, b.y}; v[3] = EhCell{b.z, b.w};
    }
    __device__ __forceinline__ void store(int c, int32_t h, int32_t e) {
        *reinterpret_cast<int2*>(p + c) = make_int2(h, e);
    }
    __device__ __forceinline__ void note_read(int) const {}
};

__host__ __device__ constexpr int align16(int x) { return (x + 15) & ~15; }

// Slots: every block read (jb <= qmax-1, 4 slots) and the end write at qlen stay inside.
__host__ __device__ inline int eh_slots(int qmax) { return (qmax + 8) & ~3; }
// Query-profile row stride: a 4-byte read at any block start jb <= qmax-1 stays in the row.
__host__ __device__ inline int qstride_of(int qmax) { return (qmax + 4) & ~3; }

__host__ __device__ inline size_t group_bytes(int qmax, int tmax) {
    return (size_t)align16(eh_slots(qmax) * (int)sizeof(EhSlot32)) +
           (size_t)align16(5 * qstride_of(qmax)) + (size_t)align16(tmax + 1);
}

size_t group_smem_bytes(int qmax, int tmax) { return group_bytes(qmax, tmax); }

__device__ __forceinline__ int decode_base(const uint32_t* __restrict__ codes,
                                           const uint32_t* __restrict__ nmask, uint32_t off,
                                           int k, int len, bool rev) {
    uint32_t p = rev ? off + (uint32_t)(len - 1 - k) : off + (uint32_t)k;
    uint32_t c = (__ldg(codes + (p >> 4)) >> ((p & 15u) << 1)) & 3u;
    uint32_t nb = (__ldg(nmask + (p >> 5)) >> (p & 31u)) & 1u;
    return nb ? 4 : (int)c;
}

template <int G, bool kNarrow>
__device__ void run_dp(int job, const JobConst& c, const LaunchDesc& d, SmemEh buf,
                       const int8_t* qp, const uint8_t* tgt, int qs, int r, unsigned gmask) {
    Lane L;
    lane_init(L, r, c.tlen);
    Commit K;
    commit_init(K, c);
    const int pred = (r + G - 1) & (G - 1);
    // Every step either advances a row or moves a lane between states; the oldest
    // unfinished row always advances, so this bound is never reached by a correct run.  It
    // turns a logic error into a per-job status instead of a hang.
    const long long limit = 8LL * ((long long)c.tlen + 2) * ((long long)c.qlen + 8) + 4096;
    long long steps = 0;
    int32_t err = G3X_OK;
    while (!K.stop) {
        const uint32_t pp = __shfl_sync(gmask, lane_prog(L), pred, G);
        const uint32_t pf = __shfl_sync(gmask, lane_fnz(L), pred, G);
        RowDone rd;
        const bool fin = lane_step<G, kNarrow>(L, c, pp, pf, buf, qp, tgt, qs, &rd);
        const unsigned b = __ballot_sync(gmask, fin);
        if (b) {
            if (__popc(b) != 1) { err = G3X_ERR_INTERNAL; break; }
            const int src = (__ffs(b) - 1) & (G - 1);
            RowDone cd;
            cd.m = __shfl_sync(gmask, rd.m, src, G);
            cd.mj = __shfl_sync(gmask, rd.mj, src, G);
            cd.gval = __shfl_sync(gmask, rd.gval, src, G);
            cd.ncells = __shfl_sync(gmask, rd.ncells, src, G);
            commit_row(K, c, cd);
        }
        __syncwarp(gmask);
        if (++steps > limit) { err = G3X_ERR_TIMEOUT; break; }
    }
    if (r == 0) {
        d.out[job] = g3x_ext_t{K.best, K.best_j + 1, K.best_i + 1, K.max_ie + 1, K.gscore, K.max_off};
        d.status[job] = err;
        if (d.cells) d.cells[job] = (int32_t)K.cells;
    }
}

template <int G>
__device__ void run_job(int job, const LaunchDesc& d, const ScoreParams& sp, char* gsm,
                        int r, unsigned gmask) {
    const int qmax = d.qmax, tmax = d.tmax;
    const int qs = qstride_of(qmax);
    EhSlot32* eh = reinterpret_cast<EhSlot32*>(gsm);
    int8_t* qp = reinterpret_cast<int8_t*>(gsm + align16(eh_slots(qmax) * (int)sizeof(EhSlot32)));
    uint8_t* tgt = reinterpret_cast<uint8_t*>(gsm + align16(eh_slots(qmax) * (int)sizeof(EhSlot32)) +
                                              align16(5 * qs));

    const g3x_job_t jb = d.jobs[job];
    const int qlen = jb.qlen, tlen = jb.tlen;
    if (qlen > qmax || tlen > tmax || qlen > 65534) {
        if (r == 0) {
            d.out[job] = g3x_ext_t{0, 0, 0, 0, 0, 0};
            d.status[job] = G3X_ERR_TOO_LONG;
            if (d.cells) d.cells[job] = 0;
        }
        return;
    }
    JobConst c;
    c.qlen = qlen; c.tlen = tlen; c.h0 = jb.h0;
    c.o_del = sp.o_del; c.e_del = sp.e_del; c.o_ins = sp.o_ins; c.e_ins = sp.e_ins;
    c.oe_del = sp.o_del + sp.e_del; c.oe_ins = sp.o_ins + sp.e_ins; c.zdrop = sp.zdrop;
    c.w = clamp_w(jb.w, qlen, sp.max_sc, sp.end_bonus, sp.o_del, sp.e_del, sp.o_ins, sp.e_ins);

    // Stage the job: query profile, target codes, row buffer with row "-1".
    const bool qrev = (jb.flags & G3X_JOB_QREV) != 0, trev = (jb.flags & G3X_JOB_TREV) != 0;
    for (int k = r; k < qlen; k += G) {
        int code = decode_base(d.codes, d.nmask, jb.q_off, k, qlen, qrev);
#pragma unroll
        for (int a = 0; a < 5; ++a) qp[a * qs + k] = sp.mat[a * 5 + code];
    }
    for (int k = r; k < tlen; k += G) tgt[k] = (uint8_t)decode_base(d.codes, d.nmask, jb.t_off, k, tlen, trev);
    const int nslots = eh_slots(qlen);
    for (int k = r; k < nslots; k += G) {
        EhSlot32 v;
        v.h = k <= qlen + 1 ? init_h(k, c) : 0;
        v.e = 0;
        eh[k] = v;
    }
    __syncwarp(gmask);
    SmemEh buf{eh};
    if (job_is_narrow(c, sp.max_sc))
        run_dp<G, true>(job, c, d, buf, qp, tgt, qs, r, gmask);
    else
        run_dp<G, false>(job, c, d, buf, qp, tgt, qs, r, gmask);
    __syncwarp(gmask);
}

template <int G>
__global__ void __launch_bounds__(256) extend_kernel(LaunchDesc d, ScoreParams sp) {
    extern __shared__ __align__(16) char smem[];
    const int lane = threadIdx.x & 31;
    const int r = lane & (G - 1);
    const int gbase = lane & ~(G - 1);
    const unsigned gmask = G == 32 ? 0xFFFFFFFFu : (((1u << G) - 1u) << gbase);
    const int groups_per_block = blockDim.x / G;
    const int gib = threadIdx.x / G;
    char* gsm = smem + (size_t)gib * group_bytes(d.qmax, d.tmax);
    const int n = d.count ? *d.count : d.n;
    if (!d.persistent) {
        int slot = blockIdx.x * groups_per_block + gib;
        if (slot < n) run_job<G>(d.order ? d.order[slot] : slot, d, sp, gsm, r, gmask);
        return;
    }
    for (;;) {
        int slot = 0;
        if (r == 0) slot = atomicAdd(d.queue, 1);
        slot = __shfl_sync(gmask, slot, 0, G);
        if (slot >= n) break;
        run_job<G>(d.order ? d.order[slot] : slot, d, sp, gsm, r, gmask);
    }
}

template <int G>
static int launch_g(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream) {
    int wpb = d.warps_per_block > 0 ? d.warps_per_block : 1;
    const size_t gb = group_bytes(d.qmax, d.tmax);
    const size_t kMaxSmem = 227 * 1024;
    while (wpb > 1 && (size_t)(32 * wpb / G) * gb > kMaxSmem) --wpb;   // fewer warps for long jobs
    const int threads = 32 * wpb;
    const int groups = threads / G;
    const size_t smem = groups * gb;
    if (smem > kMaxSmem) return G3X_ERR_TOO_LONG;
    if (cudaFuncSetAttribute(extend_kernel<G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
        return G3X_ERR_CUDA;
    int blocks;
    if (d.persistent) {
        blocks = d.blocks;
        if (blocks <= 0) {
            int dev = 0, sms = 0, per_sm = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, extend_kernel<G>, threads, smem);
            blocks = sms * (per_sm > 0 ? per_sm : 1);
        }
    } else {
        blocks = (d.n + groups - 1) / groups;
        if (blocks == 0) return G3X_OK;
    }
    extend_kernel<G><<<blocks, threads, smem, stream>>>(d, sp);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

int launch_extend(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream) {
    switch (d.lanes) {
        case 8: return launch_g<8>(d, sp, stream);
        case 16: return launch_g<16>(d, sp, stream);
        case 32: return launch_g<32>(d, sp, stream);
        default: return G3X_ERR_INVALID;
    }
}

}  // namespace g3x

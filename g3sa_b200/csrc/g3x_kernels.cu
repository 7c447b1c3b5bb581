// g3x_kernels.cu -- sm_100a kernels for batched ksw_extend2 (bwa/src/ksw.cu:303-401).
//
// A job is run by a group of G lanes (G = 8, 16 or 32) that sweeps anti-diagonals of the
// banded DP with the rolling-row protocol of g3x_core.h.  A warp holds 32/G groups and runs
// ONE step loop for all of them: every iteration each group with a job advances one step,
// and a group whose job finished stages its next job in the same iteration.  All warp
// collectives (progress shuffles, the row-end ballot, the commit broadcast) use the full
// warp with per-lane source lanes, so groups never split the warp's instruction stream
// except while one of them stages a job.
//
// Per group, shared memory holds the job's working set:
//   eh   : the reference's H/E row buffer (ksw.cu:310), int32 pairs
//   qp   : the query profile, 5 rows of qstride int8 scores (ksw.cu:309, 312-315)
//   tgt  : the target codes, one nibble per base (0-3, >= 4 means N)
#include <cuda_runtime.h>
#include "g3x_core.h"
#include "g3x_internal.h"

namespace g3x {

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

// Target codes, 16 nibbles per 64-bit word.
struct SmemTgt {
    const uint64_t* p;
    __device__ __forceinline__ int32_t code(int32_t i) const {
        const uint32_t nib = (uint32_t)(p[i >> 4] >> ((i & 15) << 2)) & 15u;
        return nib < 4u ? (int32_t)nib : 4;
    }
};

__host__ __device__ constexpr int align16(int x) { return (x + 15) & ~15; }

// Slots: every block read (jb <= qmax-1, 4 slots), every 2-slot init store and the end write
// at qlen stay inside.
__host__ __device__ inline int eh_slots(int qmax) { return (qmax + 8) & ~3; }
// Query-profile row stride: 16-byte aligned rows; a 4-byte read at any block start
// jb <= qmax-1 and a 16-byte staging store at any 16-base chunk stay in the row.
__host__ __device__ inline int qstride_of(int qmax) { return (qmax + 16) & ~15; }
__host__ __device__ inline int tgt_bytes(int tmax) { return ((tmax + 15) >> 4) * 8 + 8; }

__host__ __device__ inline size_t group_bytes(int qmax, int tmax) {
    return (size_t)align16(eh_slots(qmax) * (int)sizeof(EhSlot32)) +
           (size_t)align16(5 * qstride_of(qmax)) + (size_t)align16(tgt_bytes(tmax));
}

size_t group_smem_bytes(int qmax, int tmax) { return group_bytes(qmax, tmax); }

// 16 bases of a sequence (bases 16*ch .. 16*ch+15, in the job's reading direction) as 16
// 2-bit fields (x) and 16 N bits (nb).  Only plane words that hold valid bases are read.
__device__ __forceinline__ void load16(const uint32_t* __restrict__ codes,
                                       const uint32_t* __restrict__ nmask, uint32_t off,
                                       int len, int ch, bool rev, uint32_t& x, uint32_t& nb) {
    const int k0 = ch << 4;
    const int nv = len - k0 < 16 ? len - k0 : 16;
    if (!rev) {
        const uint32_t p0 = off + (uint32_t)k0;
        const uint32_t w = p0 >> 4, sh = p0 & 15u;
        uint64_t v = __ldg(codes + w);
        if (sh + (uint32_t)nv > 16u) v |= (uint64_t)__ldg(codes + w + 1) << 32;
        x = (uint32_t)(v >> (sh << 1));
        const uint32_t nw = p0 >> 5, nsh = p0 & 31u;
        uint64_t m = __ldg(nmask + nw);
        if (nsh + (uint32_t)nv > 32u) m |= (uint64_t)__ldg(nmask + nw + 1) << 32;
        nb = (uint32_t)(m >> nsh) & 0xFFFFu;
    } else {
        const uint32_t ph = off + (uint32_t)(len - 1 - k0);   // plane position of base k0
        const uint32_t w = ph >> 4, sh = ph & 15u;
        uint64_t v = (uint64_t)__ldg(codes + w) << 32;
        if ((uint32_t)nv > sh + 1u) v |= __ldg(codes + w - 1);
        uint32_t y = (uint32_t)(v >> ((sh << 1) + 2));        // field 15 = position ph
        y = __brev(y);                                          // field order reversed...
        x = ((y >> 1) & 0x55555555u) | ((y & 0x55555555u) << 1);  // ...and each field's bits
        const uint32_t nw = ph >> 5, nsh = ph & 31u;
        uint64_t m = (uint64_t)__ldg(nmask + nw) << 32;
        if ((uint32_t)nv > nsh + 1u) m |= __ldg(nmask + nw - 1);
        nb = __brev((uint32_t)(m >> (nsh + 17)) & 0xFFFFu) >> 16;
    }
}

// 16 codes as 16 nibbles: the 2-bit code in bits 0-1, the N flag in bit 2.
__device__ __forceinline__ uint64_t nibbles16(uint32_t x, uint32_t nb) {
    uint64_t t = x;
    t = (t | (t << 16)) & 0x0000FFFF0000FFFFull;
    t = (t | (t << 8)) & 0x00FF00FF00FF00FFull;
    t = (t | (t << 4)) & 0x0F0F0F0F0F0F0F0Full;
    t = (t | (t << 2)) & 0x3333333333333333ull;
    uint64_t n = nb;
    n = (n | (n << 24)) & 0x000000FF000000FFull;
    n = (n | (n << 12)) & 0x000F000F000F000Full;
    n = (n | (n << 6)) & 0x0303030303030303ull;
    n = (n | (n << 3)) & 0x1111111111111111ull;
    return t | (n << 2);
}

// Per-group job state, identical in every lane of the group.
struct GroupJob {
    int job;          // job index, -1 = none
    int narrow;
    JobConst c;
    Commit K;
    long long steps, limit;
};

// Stages job `job` into the group's shared memory.  Returns false (after writing the job's
// status) when the job is rejected.
template <int G>
__device__ bool stage_job(int job, const LaunchDesc& d, const ScoreParams& sp,
                          const uint32_t (&prof_lo)[5], const uint32_t (&prof_hi)[5],
                          EhSlot32* eh, int8_t* qp, uint64_t* tgt, int qs, int r,
                          GroupJob& gj) {
    const g3x_job_t jb = d.jobs[job];
    const int qlen = jb.qlen, tlen = jb.tlen;
    if (qlen > d.qmax || tlen > d.tmax || qlen > 65534) {
        if (r == 0) {
            d.out[job] = g3x_ext_t{0, 0, 0, 0, 0, 0};
            d.status[job] = G3X_ERR_TOO_LONG;
            if (d.cells) d.cells[job] = 0;
        }
        return false;
    }
    JobConst& c = gj.c;
    c.qlen = qlen; c.tlen = tlen; c.h0 = jb.h0;
    c.o_del = sp.o_del; c.e_del = sp.e_del; c.o_ins = sp.o_ins; c.e_ins = sp.e_ins;
    c.oe_del = sp.o_del + sp.e_del; c.oe_ins = sp.o_ins + sp.e_ins; c.zdrop = sp.zdrop;
    c.w = clamp_w(jb.w, qlen, sp.max_sc, sp.end_bonus, sp.o_del, sp.e_del, sp.o_ins, sp.e_ins);
    const bool qrev = (jb.flags & G3X_JOB_QREV) != 0, trev = (jb.flags & G3X_JOB_TREV) != 0;
    // query profile, 16 bases per lane-iteration: one byte permute per 4 scores
    for (int ch = r; (ch << 4) < qlen; ch += G) {
        uint32_t x, nb;
        load16(d.codes, d.nmask, jb.q_off, qlen, ch, qrev, x, nb);
        const uint64_t sel = nibbles16(x, nb);
        const uint32_t s0 = (uint32_t)sel, s1 = (uint32_t)(sel >> 16), s2 = (uint32_t)(sel >> 32),
                       s3 = (uint32_t)(sel >> 48);
#pragma unroll
        for (int a = 0; a < 5; ++a) {
            uint4 v;
            v.x = __byte_perm(prof_lo[a], prof_hi[a], s0);
            v.y = __byte_perm(prof_lo[a], prof_hi[a], s1);
            v.z = __byte_perm(prof_lo[a], prof_hi[a], s2);
            v.w = __byte_perm(prof_lo[a], prof_hi[a], s3);
            *reinterpret_cast<uint4*>(qp + a * qs + (ch << 4)) = v;
        }
    }
    for (int ch = r; (ch << 4) < tlen; ch += G) {
        uint32_t x, nb;
        load16(d.codes, d.nmask, jb.t_off, tlen, ch, trev, x, nb);
        tgt[ch] = nibbles16(x, nb);
    }
    const int nslots = eh_slots(qlen);
    for (int k = r << 1; k < nslots; k += G << 1) {
        int4 v;
        v.x = k <= qlen + 1 ? init_h(k, c) : 0;
        v.y = 0;
        v.z = k + 1 <= qlen + 1 ? init_h(k + 1, c) : 0;
        v.w = 0;
        *reinterpret_cast<int4*>(eh + k) = v;
    }
    gj.narrow = job_is_narrow(c, sp.max_sc);
    commit_init(gj.K, c);
    gj.steps = 0;
    // Every step either advances a row or moves a lane between states; the oldest
    // unfinished row always advances, so this bound is never reached by a correct run.  It
    // turns a logic error into a per-job status instead of a hang.
    gj.limit = 8LL * ((long long)tlen + 2) * ((long long)qlen + 8) + 4096;
    gj.job = job;
    return true;
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
    const int qs = qstride_of(d.qmax);
    char* gsm = smem + (size_t)gib * group_bytes(d.qmax, d.tmax);
    EhSlot32* eh = reinterpret_cast<EhSlot32*>(gsm);
    int8_t* qp = reinterpret_cast<int8_t*>(gsm + align16(eh_slots(d.qmax) * (int)sizeof(EhSlot32)));
    uint64_t* tgt = reinterpret_cast<uint64_t*>(reinterpret_cast<char*>(qp) + align16(5 * qs));
    const int n = d.count ? *d.count : d.n;
    const int pred = gbase + ((r + G - 1) & (G - 1));

    // score rows as byte-permute pools: bytes 0-3 = codes 0-3, bytes 4-7 = N
    uint32_t prof_lo[5], prof_hi[5];
#pragma unroll
    for (int a = 0; a < 5; ++a) {
        prof_lo[a] = (uint32_t)(uint8_t)sp.mat[a * 5 + 0] | ((uint32_t)(uint8_t)sp.mat[a * 5 + 1] << 8) |
                     ((uint32_t)(uint8_t)sp.mat[a * 5 + 2] << 16) | ((uint32_t)(uint8_t)sp.mat[a * 5 + 3] << 24);
        prof_hi[a] = (uint32_t)(uint8_t)sp.mat[a * 5 + 4] * 0x01010101u;
    }

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
                if (stage_job<G>(job, d, sp, prof_lo, prof_hi, eh, qp, tgt, qs, r, gj)) {
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

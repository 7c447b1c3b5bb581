// g3x_stage.cuh -- per-job shared-memory working set and job staging, shared by the two
// extension kernel families (g3x_kernels.cu: rolling anti-diagonal; g3x_rowpar.cu:
// row-parallel).
//
// Per group of lanes, shared memory holds one job:
//   eh   : the reference's H/E row buffer (ksw.cu:310), int32 pairs, qmax + 8 slots
//   qp   : the query profile, 5 rows of qstride int8 scores (ksw.cu:309, 312-315)
//   tgt  : the target codes, one nibble per base (0-3, >= 4 means N)
// Staging decodes the 2-bit/N planes 16 bases per lane-iteration, builds four profile
// scores per byte permute, and writes row "-1" of the buffer (ksw.cu:317-319).
#pragma once
#include <cuda_runtime.h>
#include "g3x_core.h"
#include "g3x_internal.h"

namespace g3x {

struct EhSlot32 {
    int32_t h, e;
};

// The row buffer as the rolling kernel's lane_step sees it: one aligned block of four slots
// is read with two 16-byte shared loads; each computed cell is written back with one
// 8-byte store.
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

// Slots: every 4-slot block read (jb <= qmax-1), every 2-slot init store and the end write
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

// 16 bases of a sequence (bases 16*ch .. 16*ch+15, in the job's reading direction), in two
// steps: load16_raw reads the plane words that hold them (only words with valid bases), and
// decode16 turns those words into 16 2-bit fields (x) and 16 N bits (nb).  Split so that a
// prefetch issues its loads long before the decode needs their data.
__device__ __forceinline__ void load16_raw(const uint32_t* __restrict__ codes,
                                           const uint32_t* __restrict__ nmask, uint32_t off,
                                           int len, int ch, bool rev, uint64_t& v, uint64_t& m) {
    const int k0 = ch << 4;
    const int nv = len - k0 < 16 ? len - k0 : 16;
    if (!rev) {
        const uint32_t p0 = off + (uint32_t)k0;
        const uint32_t w = p0 >> 4, sh = p0 & 15u;
        v = __ldg(codes + w);
        if (sh + (uint32_t)nv > 16u) v |= (uint64_t)__ldg(codes + w + 1) << 32;
        const uint32_t nw = p0 >> 5, nsh = p0 & 31u;
        m = __ldg(nmask + nw);
        if (nsh + (uint32_t)nv > 32u) m |= (uint64_t)__ldg(nmask + nw + 1) << 32;
    } else {
        const uint32_t ph = off + (uint32_t)(len - 1 - k0);   // plane position of base k0
        const uint32_t w = ph >> 4, sh = ph & 15u;
        v = (uint64_t)__ldg(codes + w) << 32;
        if ((uint32_t)nv > sh + 1u) v |= __ldg(codes + w - 1);
        const uint32_t nw = ph >> 5, nsh = ph & 31u;
        m = (uint64_t)__ldg(nmask + nw) << 32;
        if ((uint32_t)nv > nsh + 1u) m |= __ldg(nmask + nw - 1);
    }
}

__device__ __forceinline__ void decode16(uint32_t off, int len, int ch, bool rev, uint64_t v, uint64_t m,
                                         uint32_t& x, uint32_t& nb) {
    const int k0 = ch << 4;
    if (!rev) {
        const uint32_t p0 = off + (uint32_t)k0;
        x = (uint32_t)(v >> ((p0 & 15u) << 1));
        nb = (uint32_t)(m >> (p0 & 31u)) & 0xFFFFu;
    } else {
        const uint32_t ph = off + (uint32_t)(len - 1 - k0);
        uint32_t y = (uint32_t)(v >> (((ph & 15u) << 1) + 2));  // field 15 = position ph
        y = __brev(y);                                          // field order reversed...
        x = ((y >> 1) & 0x55555555u) | ((y & 0x55555555u) << 1);  // ...and each field's bits
        nb = __brev((uint32_t)(m >> ((ph & 31u) + 17)) & 0xFFFFu) >> 16;
    }
}

__device__ __forceinline__ void load16(const uint32_t* __restrict__ codes,
                                       const uint32_t* __restrict__ nmask, uint32_t off,
                                       int len, int ch, bool rev, uint32_t& x, uint32_t& nb) {
    uint64_t v, m;
    load16_raw(codes, nmask, off, len, ch, rev, v, m);
    decode16(off, len, ch, rev, v, m, x, nb);
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

// Chunks 0 .. nch-1 of the calling lane's own query as 4-bit codes into its column of a
// lane-interleaved word array (chunk ch in words 2ch and 2ch+1, word k of lane L at
// qn[k * 32 + L]).  The lanes of a refill wave each stage their own job at the same time, four
// chunks in flight per lane, so a wave waits for about one global-memory latency per four
// chunks whatever the number of new jobs.
__device__ __forceinline__ void stage_own_query(const uint32_t* __restrict__ codes,
                                                const uint32_t* __restrict__ nmask, uint32_t q_off,
                                                int qlen, bool qrev, int nch, uint32_t* qn, int lane) {
    for (int c0 = 0; c0 < nch; c0 += 4) {
        uint32_t x[4], nb[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            x[u] = 0u; nb[u] = 0u;
            if (c0 + u < nch) load16(codes, nmask, q_off, qlen, c0 + u, qrev, x[u], nb[u]);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (c0 + u < nch) {
                const uint64_t v = nibbles16(x[u], nb[u]);
                qn[(2 * (c0 + u)) * 32 + lane] = (uint32_t)v;
                qn[(2 * (c0 + u) + 1) * 32 + lane] = (uint32_t)(v >> 32);
            }
        }
    }
}

// Score rows as byte-permute pools: bytes 0-3 = codes 0-3, bytes 4-7 = N.
__device__ __forceinline__ void score_pools(const ScoreParams& sp, uint32_t (&lo)[5],
                                            uint32_t (&hi)[5]) {
#pragma unroll
    for (int a = 0; a < 5; ++a) {
        lo[a] = (uint32_t)(uint8_t)sp.mat[a * 5 + 0] | ((uint32_t)(uint8_t)sp.mat[a * 5 + 1] << 8) |
                ((uint32_t)(uint8_t)sp.mat[a * 5 + 2] << 16) | ((uint32_t)(uint8_t)sp.mat[a * 5 + 3] << 24);
        hi[a] = (uint32_t)(uint8_t)sp.mat[a * 5 + 4] * 0x01010101u;
    }
}

struct StagedJob {
    JobConst c;
    int narrow;
};

// Stages job `job` into the group's shared memory.  Returns false (after writing the job's
// status) when the job is rejected.  The caller synchronizes the group before use.
template <int G>
__device__ bool stage_job(int job, const LaunchDesc& d, const ScoreParams& sp,
                          const uint32_t (&prof_lo)[5], const uint32_t (&prof_hi)[5],
                          EhSlot32* eh, int8_t* qp, uint64_t* tgt, int qs, int r,
                          StagedJob& sj) {
    const g3x_job_t jb = d.jobs[job];
    const int qlen = jb.qlen, tlen = jb.tlen;
    // M = H ? H + S : 0 is computed as min(H + S, 256 H), exact for H >= 0; the only H that can
    // be negative is eh[0].h = h0 (ksw.cu:317), and for h0 <= -max_score the two forms agree
    // too (both <= 0, which every use clips to 0).  Seed scores in between are rejected.
    const bool bad_h0 = jb.h0 < 0 && jb.h0 > -sp.max_sc;
    // a job reaching past the planes is refused before any of its bases is read
    const bool outside = !job_in_planes(jb, d.n_bases);
    if (qlen > d.qmax || tlen > d.tmax || qlen > 65534 || bad_h0 || outside) {
        if (r == 0) {
            d.out[job] = g3x_ext_t{0, 0, 0, 0, 0, 0};
            d.status[job] = bad_h0 || outside ? G3X_ERR_INVALID : G3X_ERR_TOO_LONG;
            if (d.cells) d.cells[job] = 0;
            if (d.rows) d.rows[job] = 0;
        }
        return false;
    }
    JobConst& c = sj.c;
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
    sj.narrow = job_is_narrow(c, sp.max_sc);
    return true;
}

// Programmatic dependent launch in the width-class kernels.  pdl_trigger, first thing in the
// kernel, lets the class kernel queued after this one on the stream start at once (its blocks
// take the SMs this kernel's blocks leave as they run out of jobs).  pdl_chain_end, last thing:
// one thread of block 0 waits for the kernel this one was launched after (no wait without a
// programmatic launch), so a kernel of the chain completes only after the kernels before it,
// and the work queued after the last class sees every class's outputs.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_chain_end() {
    if (blockIdx.x == 0 && threadIdx.x == 0) asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Occupancy counters of a lane-per-job warp: the lanes' busy and idle block steps summed over
// the warp first, so a warp adds to each counter once (every lane adding its own share put
// tens of thousands of same-address atomics at the end of each launch).
__device__ __forceinline__ void add_warp_stats(unsigned long long* stats, unsigned long long busy,
                                               unsigned long long idle, unsigned long long waves, int lane) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        busy += __shfl_xor_sync(0xFFFFFFFFu, busy, o);
        idle += __shfl_xor_sync(0xFFFFFFFFu, idle, o);
    }
    if (lane == 0) {
        atomicAdd(stats + 0, busy);
        atomicAdd(stats + 1, idle);
        atomicAdd(stats + 2, waves);
    }
}

}  // namespace g3x

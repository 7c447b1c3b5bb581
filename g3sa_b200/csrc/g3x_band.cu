// g3x_band.cu -- one-warp-per-job sm_100a kernel for batched ksw_extend2 on wide bands
// (bwa/src/ksw.cu:303-401), int32.
//
// A warp runs one job through the reference's row loop, one target row per step, with the
// row buffer eh[] (ksw.cu:310) held in registers over a window of W = 32 R columns that slides
// with the band: at row i, window index d holds column i - w + d, and lane L owns indices
// L*R .. L*R + R - 1.  The band of row i lies in columns [i - w, i + w + 1) (ksw.cu:338-340)
// and its end entry eh[end] (ksw.cu:371) at most one column further, so W >= 2w + 2 holds every
// entry a row reads or writes.  A column enters the window on the right only once, never
// written before (the reference writes eh[] at or left of its band end), so it enters with its
// row -1 value (ksw.cu:317-319); it leaves on the left once the band's left edge has passed it,
// never to be read again.  Every other entry keeps whatever the last row wrote there, so the
// stale entries the reference reads when its band regrows (ksw.cu:388-391) are exact.
//
// Because the window moves one column per row, the entry for column j, which row i reads at
// index d, is index d - 1 at row i + 1: each row writes its new entries one index down, and a
// lane's last index takes the next lane's first by one shuffle.  No shared memory holds the row.
//
// Per row: the cells' M = H(i-1,j-1) + S and E need only the previous row (pass 1, each lane
// over its R columns).  F is the max-plus recurrence F(j+1) = max(F(j) - e_ins,
// max(M(j) - oe_ins, 0)), F(beg) = 0, an exact prefix maximum with linear decay: each lane runs it
// over its own columns from 0, a five-step shuffle scan carries the lanes' results along the
// row, and pass 2 folds the carried value in (H = max(M, E, F)), writes the new entries
// (H(i, j-1) and E(i+1, j), ksw.cu:346-370), and forms the row's maximum and its non-zero span
// with one warp reduction each.  The row's bookkeeping (to-end score, max tracking, z-drop;
// ksw.cu:371-386) is the shared commit_row.
//
// The query is staged once per job as one code byte per base in shared memory (read when a
// column enters the window); the target code of each row comes from a 16-base chunk decoded
// from the bit planes, the next chunk's words loaded 16 rows ahead.
#include <cuda_runtime.h>
#include "g3x_core.h"
#include "g3x_internal.h"
#include "g3x_stage.cuh"

namespace g3x {

namespace {

// Byte-permute selector of a query code c (0-3, N 4-7): byte 0 takes byte c of the target's
// score pool, bytes 1-3 its sign, so the permute yields the score as an int32.
__device__ __forceinline__ uint32_t score_sel(uint32_t c) {
    const uint32_t s = c | 8u;
    return c | (s << 4) | (s << 8) | (s << 12);
}

// prmt.b32 in its default mode, where a selector nibble with bit 3 set replicates the sign of
// the byte it selects (__byte_perm ignores that bit).
__device__ __forceinline__ int32_t permute_score(uint32_t lo, uint32_t hi, uint32_t sel) {
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(lo), "r"(hi), "r"(sel));
    return (int32_t)r;
}

// Four 4-bit codes (one 16-bit group) as four bytes.
__device__ __forceinline__ uint32_t nib4_bytes(uint32_t v16) {
    uint32_t t = (v16 & 0xFFu) | ((v16 & 0xFF00u) << 8);
    return (t | (t << 4)) & 0x0F0F0F0Fu;
}

// Row -1 of the buffer at column j (0 outside [0, qlen + 1]).
__device__ __forceinline__ int32_t init_entry(int32_t j, const JobConst& c) {
    return j >= 0 && j <= c.qlen + 1 ? init_h(j, c) : 0;
}

// The job's band (2w' + 2 entries, w' the clamped width) fits the window, and its scores stay
// below 2^21 (the row maximum travels as score << 10 | window index in one 32-bit reduction):
// every H is at most h0 + qlen * max_score.
__device__ __forceinline__ bool band_fits(const JobConst& c, int32_t max_sc, int W) {
    return 2 * c.w + 2 <= W && (int64_t)c.qlen * max_sc + (c.h0 > 0 ? c.h0 : 0) < (1 << 21);
}

// Shared memory of one warp: the staged query, one byte per base.
__host__ __device__ inline size_t query_bytes(int qcap) { return (size_t)((qcap + 15) & ~15); }

__device__ __forceinline__ void refuse(const LaunchDesc& d, int job, int32_t status) {
    d.out[job] = g3x_ext_t{0, 0, 0, 0, 0, 0};
    d.status[job] = status;
    if (d.cells) d.cells[job] = 0;
    if (d.rows) d.rows[job] = 0;
}

}  // namespace

size_t band_smem_per_warp(int qcap) { return query_bytes(qcap); }

// kSym: oe_del == oe_ins (BWA's defaults), so E reuses F's max(M - oe, 0).
template <int R, bool kSym>
__global__ void __launch_bounds__(128) band_kernel(LaunchDesc d, ScoreParams sp) {
    pdl_trigger();
    constexpr int W = 32 * R;
    static_assert(W <= 1024, "window index must fit 10 bits");
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
    uint8_t* qc = reinterpret_cast<uint8_t*>(smem) + (size_t)warp * query_bytes(d.qmax);
    const int n = d.count ? *d.count : d.n;
    const int* order = d.order ? d.order + (d.order_off ? *d.order_off : 0) : nullptr;
    const int32_t e_ins = sp.e_ins, e_del = sp.e_del, oe_ins = sp.oe_ins, oe_del = sp.oe_del;
    unsigned long long busy = 0, idle = 0, jobs_run = 0;
    int static_slot = blockIdx.x * (blockDim.x >> 5) + warp;
    const int static_stride = gridDim.x * (blockDim.x >> 5);

    for (;;) {
        int slot;
        if (d.persistent) {
            slot = 0;
            if (lane == 0) slot = atomicAdd(d.queue, 1);
            slot = __shfl_sync(0xFFFFFFFFu, slot, 0);
        } else {
            slot = static_slot;
            static_slot += static_stride;
        }
        if (slot >= n) break;
        const int job = order ? order[slot] : slot;
        const g3x_job_t jb = d.jobs[job];
        JobConst c;
        c.qlen = jb.qlen; c.tlen = jb.tlen; c.h0 = jb.h0;
        c.o_del = sp.o_del; c.e_del = sp.e_del; c.o_ins = sp.o_ins; c.e_ins = sp.e_ins;
        c.oe_del = sp.oe_del; c.oe_ins = sp.oe_ins; c.zdrop = sp.zdrop;
        c.w = clamp_w(jb.w, c.qlen, sp.max_sc, sp.end_bonus, sp.o_del, sp.e_del, sp.o_ins, sp.e_ins);
        // the checks of stage_job (M = min(H + S, 256 H) needs h0 >= 0 or h0 <= -max_score),
        // and a band that fits the window
        const bool bad_h0 = jb.h0 < 0 && jb.h0 > -sp.max_sc;
        const bool outside = !job_in_planes(jb, d.n_bases);
        if (bad_h0 || outside || c.qlen > d.qmax || c.tlen > d.tmax || c.qlen > 65534 ||
            !band_fits(c, sp.max_sc, W)) {
            if (lane == 0) refuse(d, job, bad_h0 || outside ? G3X_ERR_INVALID : G3X_ERR_TOO_LONG);
            continue;
        }
        ++jobs_run;
        const bool qrev = (jb.flags & G3X_JOB_QREV) != 0, trev = (jb.flags & G3X_JOB_TREV) != 0;
        // ---- stage the query: one code byte per base (2-bit code | N << 2) ----
        __syncwarp();
        for (int ch = lane; (ch << 4) < c.qlen; ch += 32) {
            uint32_t x, nb;
            load16(d.codes, d.nmask, jb.q_off, c.qlen, ch, qrev, x, nb);
            const uint64_t nib = nibbles16(x, nb);
            *reinterpret_cast<uint4*>(qc + (ch << 4)) =
                make_uint4(nib4_bytes((uint32_t)nib & 0xFFFFu), nib4_bytes((uint32_t)(nib >> 16) & 0xFFFFu),
                           nib4_bytes((uint32_t)(nib >> 32) & 0xFFFFu), nib4_bytes((uint32_t)(nib >> 48)));
        }
        __syncwarp();
        // ---- row -1 over the window of row 0 (index d = column d - w) ----
        int32_t Hb[R], Eb[R];
        uint32_t S[R];
        {
            const int32_t j0 = -c.w + lane * R;
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int32_t j = j0 + k;
                Hb[k] = init_entry(j, c);
                Eb[k] = 0;
                S[k] = score_sel(j >= 0 && j < c.qlen ? qc[j] : 0u);
            }
        }
        // target chunks: codes of rows 16 ch .. 16 ch + 15, the next chunk's words prefetched
        uint32_t tx = 0, tn = 0;
        uint64_t pv = 0, pm = 0;
        if (c.tlen > 0) load16(d.codes, d.nmask, jb.t_off, c.tlen, 0, trev, tx, tn);
        if (c.tlen > 16) load16_raw(d.codes, d.nmask, jb.t_off, c.tlen, 1, trev, pv, pm);

        Commit K;
        commit_init(K, c);
        int32_t beg = 0, end = c.qlen;
        while (!K.stop) {
            const int32_t i = K.next;
            if ((i & 15) == 0 && i > 0) {
                decode16(jb.t_off, c.tlen, i >> 4, trev, pv, pm, tx, tn);
                const int ch = (i >> 4) + 1;
                if ((ch << 4) < c.tlen) load16_raw(d.codes, d.nmask, jb.t_off, c.tlen, ch, trev, pv, pm);
            }
            const int sh = i & 15;
            const uint32_t tcode = ((tn >> sh) & 1u) ? 4u : ((tx >> (2 * sh)) & 3u);
            const uint2 pl = pools[tcode];
            // ---- band of row i (ksw.cu:338-345) ----
            if (beg < i - c.w) beg = i - c.w;
            if (end > i + c.w + 1) end = i + c.w + 1;
            if (end > c.qlen) end = c.qlen;
            int32_t h1 = 0;
            if (beg == 0) {
                h1 = c.h0 - (c.o_del + c.e_del * (i + 1));
                h1 = h1 > 0 ? h1 : 0;
            }
            const bool nonempty = beg < end;
            const int32_t base = i - c.w;                 // column of window index 0
            const int32_t j0 = base + lane * R;           // this lane's first column
            const int32_t lo = beg - j0, hi = end - j0;   // this lane's cells: lo <= k < hi
            // Every entry left of beg is {0, 0}: the first row's are (columns < 0), the trim moves
            // beg only past entries found zero, and a zero entry left of beg stays zero (its M is at
            // most 0, its E and F are 0).  So the columns left of beg need no mask: they add
            // nothing to F and compute {0, 0} again.  Columns from end on keep their (stale)
            // entries, except the end entry itself (ksw.cu:371).
            // ---- pass 1: M and the F recurrence from 0 over each segment of kSeg columns (the
            // segments' chains are independent) ----
            constexpr int kSeg = R < 8 ? R : 8, kNs = R / kSeg;
            int32_t M[R];
            int32_t so[kNs];                               // F leaving each segment, from 0 at its start
            int32_t flast = 0;                             // F entering the last column, from 0 at its segment
#pragma unroll
            for (int q = 0; q < kNs; ++q) so[q] = 0;
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int32_t s = permute_score(pl.x, pl.y, S[k]);
                M[k] = addmin_i32(Hb[k], s, Hb[k] << 8);
                if (k == R - 1) flast = so[k / kSeg];
                so[k / kSeg] = addmax_i32(so[k / kSeg], -e_ins, addmax_i32(M[k], -oe_ins, 0));
            }
            int32_t f = so[0];                             // F leaving the lane, from 0 at its start
#pragma unroll
            for (int q = 1; q < kNs; ++q) f = addmax_i32(f, -kSeg * e_ins, so[q]);
            // ---- F along the row: F entering each lane's first column ----
            int32_t x = f;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
                if (lane >= o) x = addmax_i32(y, -o * R * e_ins, x);
            }
            int32_t fin = __shfl_up_sync(0xFFFFFFFFu, x, 1);
            if (lane == 0) fin = 0;
            int32_t sf[kNs];                               // F entering each segment
            sf[0] = fin;
#pragma unroll
            for (int q = 1; q < kNs; ++q) sf[q] = addmax_i32(sf[q - 1], -kSeg * e_ins, so[q - 1]);
            // H at this lane's last column, for the next lane's first entry H(i, j-1)
            const int32_t hl = max3_i32(M[R - 1], Eb[R - 1], addmax_i32(sf[kNs - 1], -(kSeg - 1) * e_ins, flast));
            int32_t hleft = __shfl_up_sync(0xFFFFFFFFu, hl, 1);
            if (lane == 0) hleft = 0;                      // left of the window: left of beg, so 0
            // ---- pass 2: H, the new entries (written one index down), row max, non-zero span ----
            // New entries: column beg (H(i, beg-1) = h1, E(i+1, beg)), columns beg+1 .. end-1
            // (H(i, j-1), E(i+1, j)), column end (H(i, end-1), 0); the later ones keep theirs.
            // For an empty row the end entry is never read again (the row ends the job).
            int32_t f2[kNs], hend = 0;
            int32_t lk[kNs];                               // row max of each segment as H * 32 + k (ties: larger k)
            uint32_t nz[kNs];                              // bit k: the new entry at k is non-zero
#pragma unroll
            for (int q = 0; q < kNs; ++q) { f2[q] = 0; lk[q] = -1; nz[q] = 0; }
            int32_t nh0 = 0, ne0 = 0;
            uint32_t s0 = 0;
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int q = k / kSeg;
                const int32_t F = addmax_i32(sf[q], -(k % kSeg) * e_ins, f2[q]);
                const int32_t ti = addmax_i32(M[k], -oe_ins, 0);
                f2[q] = addmax_i32(f2[q], -e_ins, ti);
                const int32_t H = max3_i32(M[k], Eb[k], F);
                const int32_t te = kSym ? ti : addmax_i32(M[k], -oe_del, 0);
                const int32_t En = addmax_i32(Eb[k], -e_del, te);
                const bool in = k < hi, at_end = k == hi;
                const int32_t nh = in ? (k == lo ? h1 : hleft) : (at_end ? hleft : Hb[k]);
                const int32_t ne = in ? En : (at_end ? 0 : Eb[k]);
                if (at_end) hend = hleft;
                nz[q] = in ? (min((uint32_t)(nh | ne), 1u) << k) | nz[q] : nz[q];
                lk[q] = in ? max(lk[q], H * 32 + k) : lk[q];
                hleft = H;
                if (k == 0) { nh0 = nh; ne0 = ne; s0 = S[0]; }
                else { Hb[k - 1] = nh; Eb[k - 1] = ne; S[k - 1] = S[k]; }
            }
            int32_t lkey = lk[0];
            uint32_t nzm = nz[0];
#pragma unroll
            for (int q = 1; q < kNs; ++q) { lkey = max(lkey, lk[q]); nzm |= nz[q]; }
            const uint32_t key = lkey < 0 ? 0u
                                 : (((uint32_t)lkey >> 5) << 10 | (uint32_t)(lane * R + (lkey & 31))) + 1u;
            uint32_t fnz = nzm ? (uint32_t)(j0 + __ffs(nzm) - 1) + 1u : 0xFFFFFFFFu;
            uint32_t lnz = nzm ? (uint32_t)(j0 + 31 - __clz(nzm)) + 1u : 0u;
            // ---- row end (ksw.cu:371-386) ----
            const uint32_t wkey = __reduce_max_sync(0xFFFFFFFFu, key);
            if (nonempty) hend = __shfl_sync(0xFFFFFFFFu, hend, (end - base) / R);
            else hend = h1;
            RowDone rd;
            rd.m = wkey ? (int32_t)((wkey - 1u) >> 10) : 0;
            rd.mj = wkey ? base + (int32_t)((wkey - 1u) & 1023u) : -1;
            rd.gval = (nonempty ? end : beg) == c.qlen ? hend : -1;
            rd.ncells = nonempty ? end - beg : 0;
            busy += rd.ncells;
            idle += W - rd.ncells;
            commit_row(K, c, rd);
            if (K.stop) break;
            // next band, ksw.cu:388-391: first non-zero entry in [beg, end), last in [beg', end]
            fnz = __reduce_min_sync(0xFFFFFFFFu, fnz);
            lnz = __reduce_max_sync(0xFFFFFFFFu, lnz);
            const int32_t f0 = fnz == 0xFFFFFFFFu ? 0x7FFFFFFF : (int32_t)fnz - 1;
            int32_t l0 = (int32_t)lnz - 1;
            if (hend != 0 && nonempty) l0 = end;           // eh[end] = {H(i, end-1), 0}
            const int32_t nb = f0 < end ? f0 : end;
            const int32_t L = l0 >= nb ? l0 : nb - 1;
            beg = nb;
            end = L + 2 < c.qlen ? L + 2 : c.qlen;
            // ---- slide the window one column: the last index takes the next lane's first ----
            const int32_t hn = __shfl_down_sync(0xFFFFFFFFu, nh0, 1);
            const int32_t en = __shfl_down_sync(0xFFFFFFFFu, ne0, 1);
            const uint32_t sn = __shfl_down_sync(0xFFFFFFFFu, s0, 1);
            if (lane < 31) {
                Hb[R - 1] = hn;
                Eb[R - 1] = en;
                S[R - 1] = sn;
            } else {                                       // column base + W enters
                const int32_t j = base + W;
                Hb[R - 1] = init_entry(j, c);
                Eb[R - 1] = 0;
                S[R - 1] = score_sel(j >= 0 && j < c.qlen ? qc[j] : 0u);
            }
        }
        if (lane == 0) {
            d.out[job] = g3x_ext_t{K.best, K.best_j + 1, K.best_i + 1, K.max_ie + 1, K.gscore, K.max_off};
            d.status[job] = G3X_OK;
            if (d.cells) d.cells[job] = (int32_t)K.cells;
            if (d.rows) d.rows[job] = K.next;
        }
    }
    if (d.stats && lane == 0) {
        atomicAdd(d.stats + 0, busy);
        atomicAdd(d.stats + 1, idle);
        atomicAdd(d.stats + 2, jobs_run);
    }
    pdl_chain_end();
}

template <int R, bool kSym>
static int launch_band_t(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream) {
    auto kern = band_kernel<R, kSym>;
    const size_t wb = band_smem_per_warp(d.qmax);
    size_t max_smem = 0;
    if (allow_max_smem(kern, &max_smem) != cudaSuccess) return G3X_ERR_CUDA;
    if (wb > max_smem) return G3X_ERR_TOO_LONG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return G3X_ERR_CUDA;
    sms = sm_count();
    // warps per block: the choice among 1, 2 and 4 that keeps the most warps resident (registers
    // are allotted per block, so small blocks of this register-heavy kernel waste fewer)
    int best_wpb = 1, best_warps = 0, best_blocks = 0;
    for (int wpb = 1; wpb <= 4; wpb *= 2) {
        if ((size_t)wpb * wb > max_smem) break;
        int per_sm = 0;
        per_sm = resident_blocks(kern, 32 * wpb, (size_t)wpb * wb);
        if (per_sm * wpb > best_warps) { best_warps = per_sm * wpb; best_wpb = wpb; best_blocks = per_sm; }
    }
    const size_t smem = (size_t)best_wpb * wb;
    int blocks = d.blocks > 0 ? d.blocks : sms * (best_blocks > 0 ? best_blocks : 1);
    if (!d.persistent) {
        const int need = (d.n + best_wpb - 1) / best_wpb;
        blocks = need < blocks ? need : blocks;
        if (blocks == 0) return G3X_OK;
    }
    if (launch_class_kernel(kern, blocks, 32 * best_wpb, smem, stream, d, sp) != cudaSuccess)
        return G3X_ERR_CUDA;
    return G3X_OK;
}

template <int R>
static int launch_band_r(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream) {
    return sp.oe_del == sp.oe_ins ? launch_band_t<R, true>(d, sp, stream) : launch_band_t<R, false>(d, sp, stream);
}

// d.tile is the window W (256, 512 or 1024 columns): jobs whose band 2w' + 2 exceeds it get
// G3X_ERR_TOO_LONG.
int launch_band(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream) {
    switch (d.tile) {
        case 256: return launch_band_r<8>(d, sp, stream);
        case 512: return launch_band_r<16>(d, sp, stream);
        case 1024: return launch_band_r<32>(d, sp, stream);
        default: return G3X_ERR_INVALID;
    }
}

}  // namespace g3x

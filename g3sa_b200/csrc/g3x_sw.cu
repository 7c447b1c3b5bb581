// g3x_sw.cu -- batched striped local Smith-Waterman with 16-bit cells, as ksw_align2 computes
// it (bwa/src/ksw.cu:271-292 over the profile of ksw_qinit, :18-64, and the pass of ksw_i16,
// :155-262; the reference stops ksw_align2 at its first statement, :276, and this is the
// function as written after it).
//
// Four lanes per job (a quad), eight jobs per warp.  ksw_i16 works on vectors of eight 16-bit
// cells; here a vector is the quad's four int16x2 words (lane p holds cells 2p and 2p+1), so
// each vector step of the reference is one DPX/SIMD instruction per lane:
//   adds, then max with E and F      -> __viaddmax_s16x2(H, S, max(E, F))
//   max of non-negative cells        -> __vimax_s16x2_relu
//   "subtract, 0 if not positive"    -> __viaddmax_s16x2_relu with the negated penalty
//   "any cell of F beats H - oe"      -> max(F, H - oe) != H - oe
//   the one-cell shift                -> one quad shuffle and a byte permute
// (only DPX forms: the SIMD-video intrinsics are instruction sequences on this architecture).
// The query profile is not stored: segment j's word of lane p is the score of the row's target
// base against query positions j + 2p*slen and j + (2p+1)*slen, one sign-extending byte
// permute (prmt) of the score row by a selector built once per job.  The job's H and E rows
// live in registers: segment j sits in slot MAXSEG - slen + j, so the last segment, which the
// next row shifts in, is always the last slot.
//
// Exactness: the reference's int16 arithmetic wraps; every cell here stays in [0, 32639]
// (H <= max(mat) * qlen <= 127 * 256, plus one score) for queries up to 256 bases, so the
// wrapping and non-wrapping forms agree, and "subtract, 0 if not positive" of a non-negative
// cell never wraps.  Longer queries get G3X_ERR_TOO_LONG.
//
// Jobs are sorted by segment count and target length (a device counting sort), so a warp's
// eight jobs have about the same work; each of three launches (8, 16, 32 segments) takes its
// class's range from a device counter.
#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include "g3x_core.h"
#include "g3x_internal.h"
#include "g3x_stage.cuh"

namespace g3x {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kQuads = 8;                 // jobs per warp
constexpr int kWarps = 4;                 // warps per block
constexpr int kRowBins = 16;              // log2 of the target length
constexpr int kSegBins = 32;              // segments 1..32
constexpr int kBins = kSegBins * kRowBins + 1;   // + the bin of rejected jobs (qlen 0 or > 256)
constexpr int kNoScore = 0x10000;         // minsc / endsc when the flag is absent (ksw.cu:176-177)

struct SwDesc {
    const g3x_job_t* jobs;
    const uint32_t* codes;
    const uint32_t* nmask;
    const int32_t* order;      // job indices, sorted
    const int32_t* range;      // [offset, count] of this launch's jobs in `order`
    int32_t* queue;            // this launch's slot counter (zeroed)
    g3x_swr_t* out;
    int32_t* status;
    uint32_t* sub;             // XSUBO: row maxima per job (imax << 16 | row), sub_stride each
    int32_t sub_stride;
    int32_t xtra, maxmat;
    uint32_t tab[10];          // per target base: score bytes (lo: codes 0-3, hi: N, then 0)
    uint32_t nedel, noedel, neins, noeins;   // -e_del, -(o_del+e_del), ... as int16x2
    int64_t n_bases;           // bases the planes hold: jobs reaching past them are refused
};

__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}

// The vector moved up one cell (cell 0 gets 0), ksw.cu:86-97.
__device__ __forceinline__ uint32_t shift_up(uint32_t w, int p) {
    const uint32_t up = __shfl_up_sync(kFull, w, 1, 4);
    return __byte_perm(p ? up : 0u, w, 0x5432);
}

// Selector nibbles for one word: cell codes c0, c1 (5 = past the query, score 0); the high byte
// of each half replicates the sign of its low byte.
__device__ __forceinline__ uint32_t sel_of(uint32_t c0, uint32_t c1) {
    return c0 | (c0 | 8u) << 4 | c1 << 8 | (c1 | 8u) << 12;
}

__device__ __forceinline__ int quad_max(int v) {
    v = max(v, __shfl_xor_sync(kFull, v, 1));
    return max(v, __shfl_xor_sync(kFull, v, 2));
}
__device__ __forceinline__ int quad_min(int v) {
    v = min(v, __shfl_xor_sync(kFull, v, 1));
    return min(v, __shfl_xor_sync(kFull, v, 2));
}

// Code of position `pos` of a sequence stored at plane position off (backwards when rev).
__device__ __forceinline__ uint32_t base_at(const uint32_t* __restrict__ codes, const uint32_t* __restrict__ nmask,
                                            uint32_t off, int len, int pos, bool rev) {
    const uint32_t a = off + (uint32_t)(rev ? len - 1 - pos : pos);
    if ((__ldg(nmask + (a >> 5)) >> (a & 31u)) & 1u) return 4u;
    return (__ldg(codes + (a >> 4)) >> ((a & 15u) << 1)) & 3u;
}

// Target rows of a pass: row i is base i of the job's target, or, in the second pass, base
// te - i for i <= te (the prefix 0..te reversed, ksw.cu:287).  16 bases per refill.
struct Rows {
    uint32_t off, roff;
    int len, rlen, flip;       // flip: rows 0..flip-1 come from the reversed prefix
    bool rev, rrev;
    int chunk, view;
    uint32_t x, nb;
    __device__ __forceinline__ uint32_t code(const uint32_t* codes, const uint32_t* nmask, int i) {
        const int v = i < flip ? 1 : 0;
        if (v != view || (i >> 4) != chunk) {
            view = v; chunk = i >> 4;
            if (v) load16(codes, nmask, roff, rlen, chunk, rrev, x, nb);
            else load16(codes, nmask, off, len, chunk, rev, x, nb);
        }
        return ((nb >> (i & 15)) & 1u) ? 4u : (x >> ((i & 15) << 1)) & 3u;
    }
};

struct PassOut {
    int score, te, qe;
};

// Slot cases 0..31 of the unrolled segment loops.  A loop enters at the warp's first used slot
// with one jump (a switch on a warp-uniform value) and falls through the rest.
#define G3X_SW_CASES(F) F(0) F(1) F(2) F(3) F(4) F(5) F(6) F(7) F(8) F(9) F(10) F(11) F(12) F(13) F(14) \
    F(15) F(16) F(17) F(18) F(19) F(20) F(21) F(22) F(23) F(24) F(25) F(26) F(27) F(28) F(29) F(30) F(31)

// The row loop of one pass over registers H, E (slot MAXSEG - slen + j = segment j).  UNI: every
// live quad of the warp has the same slot base, so no slot needs a per-quad guard; a quad that
// is not running computes on slots it never reads back.
template <int MAXSEG, bool UNI, bool SYM>
__device__ __forceinline__ void sw_rows(const SwDesc& d, bool live, int tlen, Rows& rows, int minsc, int endsc,
                                        uint32_t* sub, int& n_b, uint32_t (&H)[MAXSEG], uint32_t (&E)[MAXSEG],
                                        const uint32_t (&sel2)[MAXSEG / 2], int base, int base_min, uint32_t* hm,
                                        const uint32_t* tab, int lane, int& gmax, int& te) {
    const int p = lane & 3;
    const unsigned qmask = 0xFu << (lane & ~3);
    int last_row = -2, last_v = 0;
    bool run = live;
    for (int i = 0;; ++i) {
        run = run && i < tlen;
        if (!__any_sync(kFull, run)) break;
        uint32_t lo = 0u, hi = 0u;
        if (run) {
            const uint32_t t = rows.code(d.codes, d.nmask, i);
            lo = tab[2 * t]; hi = tab[2 * t + 1];
        }
        uint32_t hd = shift_up(H[MAXSEG - 1], p);
        uint32_t f = 0u, mx = 0u;
        // the row (ksw.cu:193-208): M = H(i-1, j-1) + S, H = max(M, E, F), E' and F' from H
        switch (base_min) {
#define G3X_SW_MAIN(S)                                                                               \
    case S:                                                                                          \
        if constexpr (S < MAXSEG) {                                                                  \
            if (UNI || S >= base) {                                                                  \
                const uint32_t sc = prmt(lo, hi, (S & 1) ? sel2[S >> 1] >> 16 : sel2[S >> 1]);         \
                const uint32_t h = __viaddmax_s16x2(hd, sc, __vimax_s16x2_relu(E[S], f));            \
                mx = __vimax_s16x2_relu(mx, h);                                                      \
                hd = H[S];                                                                           \
                H[S] = h;                                                                            \
                const uint32_t td = __viaddmax_s16x2_relu(h, d.noedel, 0u);                          \
                E[S] = __viaddmax_s16x2(E[S], d.nedel, td);                                          \
                f = __viaddmax_s16x2(f, d.neins, SYM ? td : __viaddmax_s16x2_relu(h, d.noeins, 0u)); \
            }                                                                                        \
        }
            G3X_SW_CASES(G3X_SW_MAIN)
#undef G3X_SW_MAIN
            default: break;
        }
        // lazy F (ksw.cu:209-220): at most 16 rounds of the F vector moved up one cell, then
        // H = max(H, F) segment by segment, E untouched, until a segment where no cell's F - e
        // beats its H - (o + e).  One ballot per segment gives every quad its stop; the warp
        // looks for the end every other segment (a stopped quad's steps change nothing).
        f = run ? f : 0u;
        // A quad that stops gets F = 0, which leaves its H unchanged and keeps it stopped; a quad
        // whose first segment is later (not UNI) waits with its F; the warp leaves when no quad
        // goes on.
        for (int round = 0; round < 16; ++round) {
            f = shift_up(f, p);
            switch (base_min) {
#define G3X_SW_LAZY(S)                                                                               \
    case S:                                                                                          \
        if constexpr (S < MAXSEG) {                                                                  \
            bool go;                                                                                 \
            const bool at = UNI || S >= base;                                                        \
            if (at) {                                                                                \
                const uint32_t h = __vimax_s16x2_relu(H[S], f);                                      \
                H[S] = h;                                                                            \
                f = __viaddmax_s16x2_relu(f, d.neins, 0u);                                           \
                const uint32_t hp = __viaddmax_s16x2_relu(h, d.noeins, 0u);                          \
                go = __vimax_s16x2_relu(f, hp) != hp;                                                \
            } else {                                                                                 \
                go = f != 0u;                                                                        \
            }                                                                                        \
            const unsigned bal = __ballot_sync(kFull, go);                                           \
            if (at && !(bal & qmask)) f = 0u;                                                        \
            if ((S & 1) && !bal) goto lazy_done;                                                     \
        }
                G3X_SW_CASES(G3X_SW_LAZY)
#undef G3X_SW_LAZY
                default: break;
            }
        }
    lazy_done:
        uint32_t m2 = __vimax_s16x2_relu(mx, __shfl_xor_sync(kFull, mx, 1));
        m2 = __vimax_s16x2_relu(m2, __shfl_xor_sync(kFull, m2, 2));
        const int im = max((int)(int16_t)(m2 & 0xFFFFu), (int)(int16_t)(m2 >> 16));
        if (run) {
            if (sub && im >= minsc && p == 0) {     // ksw.cu:223-232
                if (n_b == 0 || last_row + 1 != i) {
                    sub[n_b++] = (uint32_t)im << 16 | (uint32_t)i;
                    last_row = i; last_v = im;
                } else if (last_v < im) {
                    sub[n_b - 1] = (uint32_t)im << 16 | (uint32_t)i;
                    last_row = i; last_v = im;
                }
            }
            if (im > gmax) {                        // ksw.cu:233-238
                gmax = im; te = i;
                switch (base_min) {
#define G3X_SW_SNAP(S)                                                                               \
    case S:                                                                                          \
        if constexpr (S < MAXSEG) {                                                                  \
            if (UNI || S >= base) hm[S * 32 + lane] = H[S];                                          \
        }
                    G3X_SW_CASES(G3X_SW_SNAP)
#undef G3X_SW_SNAP
                    default: break;
                }
                if (gmax >= endsc) run = false;
            }
        }
    }
}

// One pass of ksw_i16 (ksw.cu:155-262) for the quad's job (live), query codes qcode(pos) for
// pos < qlen.  With `sub`, row maxima >= minsc go to the job's list (ksw.cu:223-232; lane p = 0
// keeps it) and *nb receives its length.
template <int MAXSEG, typename QCode>
__device__ __forceinline__ PassOut sw_pass(const SwDesc& d, bool live, int qlen, int tlen, QCode qcode, Rows rows,
                                           int minsc, int endsc, uint32_t* sub, int* nb, uint32_t* hm,
                                           const uint32_t* tab, int lane) {
    const int p = lane & 3;
    const int slen = live ? (qlen + 7) >> 3 : 0;
    const int base = MAXSEG - slen;
    const int base_min = (int)__reduce_min_sync(kFull, (unsigned)base);
    const bool uni = __all_sync(kFull, !live || base == base_min);
    uint32_t H[MAXSEG], E[MAXSEG], sel2[MAXSEG / 2];
#pragma unroll
    for (int s = 0; s < MAXSEG; s += 2) {
        uint32_t v = 0;
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int j = s + u - base;
            uint32_t c0 = 5u, c1 = 5u;
            if (live && j >= 0) {
                const int p0 = j + 2 * p * slen, p1 = p0 + slen;
                if (p0 < qlen) c0 = qcode(p0);
                if (p1 < qlen) c1 = qcode(p1);
            }
            v |= sel_of(c0, c1) << (16 * u);
        }
        sel2[s >> 1] = v;
        H[s] = H[s + 1] = 0u;
        E[s] = E[s + 1] = 0u;
    }
    int gmax = 0, te = -1, n_b = 0;
    // SYM: equal insertion and deletion costs, so E and F share H - (o + e)
    if (d.noedel == d.noeins) {
        if (uni) sw_rows<MAXSEG, true, true>(d, live, tlen, rows, minsc, endsc, sub, n_b, H, E, sel2, base, base_min, hm, tab, lane, gmax, te);
        else sw_rows<MAXSEG, false, true>(d, live, tlen, rows, minsc, endsc, sub, n_b, H, E, sel2, base, base_min, hm, tab, lane, gmax, te);
    } else {
        if (uni) sw_rows<MAXSEG, true, false>(d, live, tlen, rows, minsc, endsc, sub, n_b, H, E, sel2, base, base_min, hm, tab, lane, gmax, te);
        else sw_rows<MAXSEG, false, false>(d, live, tlen, rows, minsc, endsc, sub, n_b, H, E, sel2, base, base_min, hm, tab, lane, gmax, te);
    }
    __syncwarp();
    // end on the query: the smallest position holding the best row's largest cell, cells read
    // as uint16 (ksw.cu:244-248); with no best row the cells are all 0 and it is position 0
    const bool has = live && te >= 0;      // quad-uniform; every lane takes part in the shuffles
    int best = 0;
#pragma unroll
    for (int s = 0; s < MAXSEG; ++s)
        if (has && s >= base) {
            const uint32_t v = hm[s * 32 + lane];
            best = max(best, (int)max(v & 0xFFFFu, v >> 16));
        }
    best = quad_max(best);
    int pos = 0x7FFFFFFF;
#pragma unroll
    for (int s = 0; s < MAXSEG; ++s)
        if (has && s >= base) {
            const uint32_t v = hm[s * 32 + lane];
            const int j = s - base;
            if ((int)(v & 0xFFFFu) == best) pos = min(pos, j + 2 * p * slen);
            if ((int)(v >> 16) == best) pos = min(pos, j + (2 * p + 1) * slen);
        }
    pos = quad_min(pos);
    const int qe = has ? pos : 0;
    if (nb) *nb = n_b;
    return PassOut{gmax, te, qe};
}

template <int MAXSEG>
__global__ void __launch_bounds__(128) sw_kernel(SwDesc d) {
    constexpr int QMAX = 8 * MAXSEG;
    __shared__ __align__(16) uint8_t qcodes[kWarps][kQuads][QMAX];
    __shared__ uint32_t snap[kWarps][MAXSEG * 32];
    __shared__ uint32_t tab[10];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, quad = lane >> 2, p = lane & 3;
    if (threadIdx.x < 10) tab[threadIdx.x] = d.tab[threadIdx.x];
    __syncthreads();
    uint8_t* qc = qcodes[warp][quad];
    uint32_t* hm = snap[warp];
    const int off = d.range[0], cnt = d.range[1];
    const bool subo = (d.xtra & G3X_KSW_XSUBO) != 0;
    const int minsc = subo ? d.xtra & 0xFFFF : kNoScore;
    const int endsc = (d.xtra & G3X_KSW_XSTOP) ? d.xtra & 0xFFFF : kNoScore;
    for (;;) {
        int first = 0;
        if (lane == 0) first = atomicAdd(d.queue, kQuads);
        first = __shfl_sync(kFull, first, 0);
        if (first >= cnt) break;
        const int slot = first + quad;
        const int job = slot < cnt ? d.order[off + slot] : -1;
        int qlen = 0, tlen = 0;
        bool live = false;
        g3x_job_t jb;
        if (job >= 0) {
            jb = d.jobs[job];
            qlen = jb.qlen; tlen = jb.tlen;
            int st = G3X_OK;
            if (qlen < 1) st = G3X_ERR_INVALID;     // the reference reads before its buffers
            else if (!job_in_planes(jb, d.n_bases)) st = G3X_ERR_INVALID;   // past the planes: unread
            else if (qlen > QMAX || (subo && tlen > d.sub_stride)) st = G3X_ERR_TOO_LONG;
            if (st != G3X_OK) {
                if (p == 0) {
                    d.out[job] = g3x_swr_t{0, -1, -1, -1, -1, -1, -1};
                    d.status[job] = st;
                }
            } else {
                live = true;
                const bool qrev = (jb.flags & G3X_JOB_QREV) != 0;
                for (int pos = p; pos < qlen; pos += 4) qc[pos] = (uint8_t)base_at(d.codes, d.nmask, jb.q_off, qlen, pos, qrev);
            }
        }
        __syncwarp();
        const bool trev = live && (jb.flags & G3X_JOB_TREV) != 0;
        Rows rows;
        rows.off = live ? jb.t_off : 0u; rows.len = tlen; rows.rev = trev;
        rows.roff = 0u; rows.rlen = 0; rows.rrev = false; rows.flip = 0;
        rows.chunk = -1; rows.view = -1; rows.x = 0u; rows.nb = 0u;
        uint32_t* sub = subo && live ? d.sub + (int64_t)job * d.sub_stride : nullptr;
        int n_b = 0;
        const PassOut r = sw_pass<MAXSEG>(d, live, qlen, tlen, [&](int pos) { return (uint32_t)qc[pos]; }, rows,
                                          minsc, endsc, sub, &n_b, hm, tab, lane);
        g3x_swr_t o{r.score, r.te, r.qe, -1, -1, -1, -1};
        // second best: list entries more than ceil(score / max(mat)) rows from te (ksw.cu:249-256)
        if (live && p == 0 && n_b > 0) {
            const int c = (r.score + d.maxmat - 1) / d.maxmat, low = r.te - c, high = r.te + c;
            for (int k = 0; k < n_b; ++k) {
                const uint32_t v = sub[k];
                const int e = (int)(v & 0xFFFFu), sc = (int)(v >> 16);
                if ((e < low || e > high) && sc > o.score2) { o.score2 = sc; o.te2 = e; }
            }
        }
        // start positions (ksw.cu:286-291): the query prefix 0..qe and the target with its prefix
        // 0..te reversed, stopping at the first score; kept when it finds the same score
        const bool two = live && (d.xtra & G3X_KSW_XSTART) && !(subo && r.score < (d.xtra & 0xFFFF));
        if (__any_sync(kFull, two)) {
            const int lq = r.qe + 1, lt = r.te + 1;
            Rows rows2 = rows;
            rows2.chunk = -1; rows2.view = -1;
            rows2.flip = two ? lt : 0;
            rows2.rlen = lt;
            if (!trev) { rows2.roff = rows.off; rows2.rrev = true; }
            else { rows2.roff = rows.off + (uint32_t)(tlen - lt); rows2.rrev = false; }
            const int qe1 = r.qe;
            const PassOut rr = sw_pass<MAXSEG>(d, two, lq, tlen, [&](int pos) { return (uint32_t)qc[qe1 - pos]; },
                                               rows2, kNoScore, r.score, nullptr, nullptr, hm, tab, lane);
            if (two && rr.score == r.score) { o.tb = r.te - rr.te; o.qb = r.qe - rr.qe; }
        }
        if (live && p == 0) {
            d.out[job] = o;
            d.status[job] = G3X_OK;
        }
        __syncwarp();
    }
}

// Sort bins: segment count descending, then target length descending (log2); the last bin
// holds the jobs the kernels reject.
__global__ void sw_bin_kernel(const g3x_job_t* __restrict__ jobs, int n, int32_t* __restrict__ bin,
                              int32_t* __restrict__ hist) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const g3x_job_t jb = jobs[k];
    int b = kBins - 1;
    if (jb.qlen >= 1 && jb.qlen <= 8 * kSegBins) {
        const int slen = (jb.qlen + 7) >> 3;
        const int rb = 31 - __clz((int)jb.tlen | 1);
        b = (kSegBins - slen) * kRowBins + (kRowBins - 1 - min(rb, kRowBins - 1));
    }
    bin[k] = b;
    const unsigned peers = __match_any_sync(__activemask(), b);
    if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(hist + b, __popc(peers));
}

// Exclusive scan of the bins (one block) and the three launches' ranges: 17-32 segments, 9-16,
// and 1-8 together with the rejected bin.
__global__ void sw_scan_kernel(const int32_t* __restrict__ hist, int32_t* __restrict__ cursor,
                               int32_t* __restrict__ range, int n) {
    __shared__ int32_t part[1024];
    const int t = threadIdx.x;
    part[t] = t < kBins ? hist[t] : 0;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const int v = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    if (t < kBins) cursor[t] = t ? part[t - 1] : 0;
    __syncthreads();
    if (t == 0) {
        const int b16 = (kSegBins - 16) * kRowBins, b8 = (kSegBins - 8) * kRowBins;
        const int c16 = part[b16 - 1], c8 = part[b8 - 1];
        range[0] = 0;   range[1] = c16;
        range[2] = c16; range[3] = c8 - c16;
        range[4] = c8;  range[5] = n - c8;
    }
}

__global__ void sw_scatter_kernel(const int32_t* __restrict__ bin, int n, int32_t* __restrict__ cursor,
                                  int32_t* __restrict__ order) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int b = bin[k];
    const unsigned peers = __match_any_sync(__activemask(), b);
    const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
    int at = 0;
    if (lane == leader) at = atomicAdd(cursor + b, __popc(peers));
    at = __shfl_sync(peers, at, leader) + __popc(peers & ((1u << lane) - 1u));
    order[at] = k;
}

uint32_t pack16(int v) { return (uint32_t)(uint16_t)(int16_t)v * 0x10001u; }

template <int MAXSEG>
int launch_class(const SwDesc& d0, const int32_t* range, int32_t* queue, int sms, cudaStream_t st) {
    SwDesc d = d0;
    d.range = range;
    d.queue = queue;
    const int per_sm = resident_blocks(sw_kernel<MAXSEG>, 32 * kWarps, 0);
    sw_kernel<MAXSEG><<<sms * std::max(per_sm, 1), 32 * kWarps, 0, st>>>(d);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

}  // namespace
}  // namespace g3x

extern "C" int g3x_ksw_align2_batch(g3x_ctx* ctx, const g3x_score_t* score, const g3x_job_t* d_jobs, int32_t n,
                                    const uint32_t* d_codes, const uint32_t* d_nmask, int64_t n_bases, int32_t xtra,
                                    int32_t max_tlen,
                                    g3x_swr_t* d_out, int32_t* d_status, void* stream) {
    using namespace g3x;
    if (!ctx || !score || n < 0 || max_tlen < 0) return G3X_ERR_INVALID;
    // the reference fills an 8-bit profile for KSW_XBYTE and then reads it as 16-bit cells
    if (xtra & G3X_KSW_XBYTE) return G3X_ERR_INVALID;
    if (n == 0) return G3X_OK;
    if (!d_jobs || !d_codes || !d_nmask || !d_out || !d_status) return G3X_ERR_INVALID;
    if (n_bases < 1 || n_bases > 0x100000000ll) return G3X_ERR_INVALID;
    ScoreParams sp;
    int rc = score_params(score, &sp);
    if (rc) return rc;
    if (sp.oe_del > 32767 || sp.oe_ins > 32767) return G3X_ERR_SCORE;
    const bool subo = (xtra & G3X_KSW_XSUBO) != 0;
    if (subo && sp.max_sc < 1) return G3X_ERR_SCORE;   // ceil(score / max(mat)) of ksw.cu:250
    const int dev = ctx_device(ctx);
    if (cudaSetDevice(dev) != cudaSuccess) return G3X_ERR_CUDA;
    SwScratch& s = ctx_sw(ctx);
    const int64_t need = (int64_t)2 * n + 2 * kBins + 8 + 4;
    const int64_t sub_need = subo ? (int64_t)n * std::max(max_tlen, 1) : 0;
    if (s.cap < need || s.sub_cap < sub_need) {
        const int64_t cap = std::max(need, s.cap), sub_cap = std::max(sub_need, s.sub_cap);
        cudaFree(s.buf); cudaFree(s.sub);
        s.buf = nullptr; s.sub = nullptr; s.cap = 0; s.sub_cap = 0;
        if (cudaMalloc(&s.buf, (size_t)cap * sizeof(int32_t)) != cudaSuccess ||
            (sub_cap && cudaMalloc(&s.sub, (size_t)sub_cap * sizeof(uint32_t)) != cudaSuccess)) {
            cudaFree(s.buf); s.buf = nullptr; cudaGetLastError();
            return G3X_ERR_NOMEM;
        }
        s.cap = cap; s.sub_cap = sub_cap;
    }
    int32_t* bin = s.buf;
    int32_t* order = bin + n;
    int32_t* hist = order + n;
    int32_t* cursor = hist + kBins;
    int32_t* range = cursor + kBins;      // 6 used, 8 kept
    int32_t* queue = range + 8;           // 3 used, 4 kept
    const cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemsetAsync(hist, 0, sizeof(int32_t) * kBins, st) != cudaSuccess ||
        cudaMemsetAsync(queue, 0, sizeof(int32_t) * 4, st) != cudaSuccess)
        return G3X_ERR_CUDA;
    const int tb = 256, nb = (n + tb - 1) / tb;
    sw_bin_kernel<<<nb, tb, 0, st>>>(d_jobs, n, bin, hist);
    sw_scan_kernel<<<1, 1024, 0, st>>>(hist, cursor, range, n);
    sw_scatter_kernel<<<nb, tb, 0, st>>>(bin, n, cursor, order);
    if (cudaPeekAtLastError() != cudaSuccess) return G3X_ERR_CUDA;
    SwDesc d;
    memset(&d, 0, sizeof(d));
    d.jobs = d_jobs; d.codes = d_codes; d.nmask = d_nmask; d.order = order;
    d.out = d_out; d.status = d_status;
    d.sub = subo ? s.sub : nullptr;
    d.sub_stride = subo ? std::max(max_tlen, 1) : 0;
    d.xtra = xtra; d.maxmat = sp.max_sc; d.n_bases = n_bases;
    for (int a = 0; a < 5; ++a) {
        uint32_t lo = 0;
        for (int c = 0; c < 4; ++c) lo |= (uint32_t)(uint8_t)sp.mat[a * 5 + c] << (8 * c);
        d.tab[2 * a] = lo;
        d.tab[2 * a + 1] = (uint32_t)(uint8_t)sp.mat[a * 5 + 4];   // byte 5 (past the query) = 0
    }
    d.nedel = pack16(-sp.e_del); d.noedel = pack16(-sp.oe_del);
    d.neins = pack16(-sp.e_ins); d.noeins = pack16(-sp.oe_ins);
    int sms = 0;
    sms = sm_count();
    if ((rc = launch_class<32>(d, range, queue, sms, st))) return rc;
    if ((rc = launch_class<16>(d, range + 2, queue + 1, sms, st))) return rc;
    return launch_class<8>(d, range + 4, queue + 2, sms, st);
}

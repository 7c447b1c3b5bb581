// g3x_global.cu -- banded global alignment with backtrack (ksw_global2, bwa/src/ksw.cu:706-809)
// for batches of alignments on the GPU.
//
// One job per lane.  The jobs are first ordered by decreasing row count and row width (the
// scheduler's counting sort); a warp takes 32 consecutive ones and runs their target rows
// together (row i of every job in the same step); in a row each lane walks its own band
// [max(i-w, 0), min(i+w+1, qlen)) column by column (the reference's scalar recurrence, in int32
// with -2^30 outside the band, ksw.cu:548; see Ring for the int16 form of short batches).  The
// band has a fixed width and never trims, so the
// row buffer of H(i-1, j-1) and E(i, j) (ksw.cu:299-301) is a ring of R >= 2w+3 columns per lane
// in shared memory: a row reads columns [beg, end) and writes column end, and a column enters
// the ring either from the first row's fill (columns 0..w) or from the row end that precedes its
// first read.  Each cell's direction byte (ksw.cu:753-776: h from M, E or F in bits 0-1, E and F
// continuing in bits 2 and 4-5) goes to global scratch, laid out [row][band column][lane] per
// warp so that the 32 lanes of a step write one 32-byte sector.  The backtrack then walks each
// lane's bytes from the last cell (ksw.cu:783-806) and writes the CIGAR, merging runs as
// push_cigar does (ksw.cu:694-704); on request NM and the MD string follow, as the traceback
// stage computes them (bwa/src/aux.cu:2831-2860).
#include <cuda_runtime.h>
#include <algorithm>
#include "g3x_core.h"
#include "g3x_internal.h"
#include "g3x_stage.cuh"

namespace g3x {

namespace {

constexpr int32_t kNegInf = -0x40000000;

struct GlobalDesc {
    const g3x_job_t* jobs;
    const uint32_t* codes;
    const uint32_t* nmask;
    int32_t* score;
    uint32_t* cigar;
    int32_t* n_cigar;
    int32_t* status;
    uint8_t* z;            // direction bytes: per warp slot zwarp bytes
    int64_t zwarp;
    int32_t* queue;
    const int32_t* order;  // queue slot -> job, jobs alike in row count and width together
    int32_t* nm;           // optional: NM per job
    char* md;              // optional: MD string per job, md_stride bytes each
    int32_t n, qmax, tmax, wmax, ncol, ring, stride, md_stride;
    int64_t n_bases;       // bases the planes hold: jobs reaching past them are refused
};

// Appends the decimal digits of v (>= 0) to buf[l ...] while they fit below cap.
__device__ __forceinline__ bool put_uint(char* buf, int& l, int cap, int v) {
    char tmp[12];
    int k = 0;
    do { tmp[k++] = (char)('0' + v % 10); v /= 10; } while (v);
    if (l + k >= cap) return false;
    while (k) buf[l++] = tmp[--k];
    return true;
}

__device__ __forceinline__ int32_t sbyte0(uint32_t x) { return (int32_t)(int8_t)(x & 0xFFu); }

// The ring's H and E: int32 pairs with the reference's -2^30 outside the band, or, for batches
// whose every value fits (compact_fits), int16 pairs in one word with -2^14 outside the band.
// Every value outside the band is that constant plus a sum of scores and penalties, the same sum
// in both forms, and every value inside stays above -2^13 while every value outside stays below
// it: each comparison goes the same way in both, and a score from outside the band maps back to
// the reference's -2^30 plus the same sum.
template <bool C16> struct Ring;
template <> struct Ring<false> {
    static constexpr int32_t kNeg = kNegInf;
    static constexpr int kSlotBytes = 8;
    int2* p;
    __device__ __forceinline__ int2 ld(int k) const { return p[k]; }
    __device__ __forceinline__ void st(int k, int32_t h, int32_t e) const { p[k] = make_int2(h, e); }
};
template <> struct Ring<true> {
    static constexpr int32_t kNeg = -0x4000;
    static constexpr int kSlotBytes = 4;
    uint32_t* p;
    __device__ __forceinline__ int2 ld(int k) const {
        const uint32_t v = p[k];
        return make_int2((int32_t)(int16_t)(v & 0xFFFFu), (int32_t)v >> 16);
    }
    __device__ __forceinline__ void st(int k, int32_t h, int32_t e) const {
        p[k] = (uint32_t)(uint16_t)h | ((uint32_t)e << 16);
    }
};

template <bool C16>
__global__ void __launch_bounds__(64) global_kernel(GlobalDesc d, ScoreParams sp) {
    extern __shared__ __align__(16) char smem[];
    using RingT = Ring<C16>;
    constexpr int32_t kNeg = RingT::kNeg;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nq = (d.qmax + 7) / 8 + 1;                       // query words (8 codes each)
    uint32_t* qn = reinterpret_cast<uint32_t*>(
        smem + (size_t)warp * ((size_t)nq * 128 + (size_t)d.ring * 32 * RingT::kSlotBytes));
    RingT he;                                                   // ring slot s of lane L: index s*32 + L
    he.p = reinterpret_cast<decltype(he.p)>(qn + nq * 32);
    const int wslot = blockIdx.x * (blockDim.x >> 5) + warp;
    uint8_t* z = d.z + (int64_t)wslot * d.zwarp;
    uint32_t lo[5], hi[5];
    score_pools(sp, lo, hi);
    const int32_t oe_del = sp.o_del + sp.e_del, oe_ins = sp.o_ins + sp.e_ins;
    const int R = d.ring;

    for (;;) {
        int first = 0;
        if (lane == 0) first = atomicAdd(d.queue, 32);
        first = __shfl_sync(0xFFFFFFFFu, first, 0);
        if (first >= d.n) break;
        const int job = first + lane < d.n ? d.order[first + lane] : d.n;
        int32_t qlen = 0, tlen = 0, w = 0;
        uint32_t t_off = 0, flags = 0;
        bool trev = false, live = false;
        if (job < d.n) {
            const g3x_job_t jb = d.jobs[job];
            qlen = jb.qlen; tlen = jb.tlen; w = jb.w; flags = jb.flags;
            t_off = jb.t_off; trev = (jb.flags & G3X_JOB_TREV) != 0;
            const bool outside = !job_in_planes(jb, d.n_bases);   // refused before any base is read
            if (qlen > d.qmax || tlen > d.tmax || w < 0 || w > d.wmax || outside) {
                d.score[job] = 0; d.n_cigar[job] = 0; d.status[job] = outside ? G3X_ERR_INVALID : G3X_ERR_TOO_LONG;
                if (d.nm) { d.nm[job] = 0; d.md[(int64_t)job * d.md_stride] = 0; }
            } else {
                live = true;
                stage_own_query(d.codes, d.nmask, jb.q_off, qlen, (jb.flags & G3X_JOB_QREV) != 0,
                                (qlen + 15) >> 4, qn, lane);
                // the first row (ksw.cu:721-724): columns 0..min(w, qlen)
                const int top = qlen < w ? qlen : w;
                for (int j = 0; j <= top; ++j)
                    he.st((j % R) * 32 + lane, j == 0 ? 0 : -(oe_ins + sp.e_ins * (j - 1)), kNeg);
            }
        }
        __syncwarp();
        const int rows = __reduce_max_sync(0xFFFFFFFFu, (unsigned)(live ? tlen : 0));
        uint32_t tx = 0, tn = 0;
        for (int i = 0; i < rows; ++i) {
            const bool run = live && i < tlen;
            int beg = 0, end = 0;
            uint32_t plo = 0, phi = 0;
            int32_t h1 = kNeg, f = kNeg;
            if (run) {
                beg = i > w ? i - w : 0;
                end = i + w + 1 < qlen ? i + w + 1 : qlen;
                h1 = beg == 0 ? -(sp.o_del + sp.e_del * (i + 1)) : kNeg;
                if ((i & 15) == 0) load16(d.codes, d.nmask, t_off, tlen, i >> 4, trev, tx, tn);
                uint32_t code = (tx >> ((i & 15) << 1)) & 3u;
                if ((tn >> (i & 15)) & 1u) code = 4;
                plo = lo[code]; phi = hi[code];
            }
            const int width = run && end > beg ? end - beg : 0;   // rows past qlen + w have no cells
            const int wmax = __reduce_max_sync(0xFFFFFFFFu, (unsigned)width);
            uint8_t* zrow = z + (int64_t)i * d.ncol * 32 + lane;
            int s = run ? beg % R : 0;
            uint32_t qw = 0;
            for (int t = 0; t < wmax; ++t) {
                if (t < width) {
                    const int j = beg + t;
                    if (t == 0 || (j & 7) == 0) qw = qn[(j >> 3) * 32 + lane];
                    const int32_t sc = sbyte0(__byte_perm(plo, phi, (qw >> ((j & 7) << 2)) & 0xFu));
                    int2 c = he.ld(s * 32 + lane);
                    const int32_t m = c.x + sc;
                    int32_t e = c.y;
                    c.x = h1;
                    uint32_t dir = m >= e ? 0u : 1u;
                    int32_t h = m >= e ? m : e;
                    if (h < f) { dir = 2u; h = f; }
                    h1 = h;
                    int32_t tt = m - oe_del;
                    e -= sp.e_del;
                    if (e > tt) dir |= 1u << 2; else e = tt;
                    c.y = e;
                    he.st(s * 32 + lane, c.x, c.y);
                    tt = m - oe_ins;
                    f -= sp.e_ins;
                    if (f > tt) dir |= 2u << 4; else f = tt;
                    zrow[(int64_t)t * 32] = (uint8_t)dir;
                    s = s + 1 == R ? 0 : s + 1;
                }
            }
            if (run) he.st((end % R) * 32 + lane, h1, kNeg);   // ksw.cu:779
            __syncwarp();
        }
        // score and backtrack (ksw.cu:781-806)
        if (live) {
            // H of column qlen: written by the last row's end when its band reaches qlen, else
            // still the first row's value
            const int32_t init = qlen == 0 ? 0 : (qlen <= w ? -(oe_ins + sp.e_ins * (qlen - 1)) : kNeg);
            const int32_t score = tlen > 0 && tlen + w >= qlen ? he.ld((qlen % R) * 32 + lane).x : init;
            const bool finite = score > kNeg / 2;
            d.score[job] = finite ? score : kNegInf + (score - kNeg);
            uint32_t* cg = d.cigar + (int64_t)job * d.stride;
            int n = 0;
            bool full = false;
            auto push = [&](int op, int len) {
                if (n > 0 && (int)(cg[n - 1] & 0xFu) == op) cg[n - 1] += (uint32_t)len << 4;
                else if (n < d.stride) cg[n++] = (uint32_t)len << 4 | (uint32_t)op;
                else full = true;
            };
            bool bad = false;
            if (finite) {
                int i = tlen - 1, k = (i + w + 1 < qlen ? i + w + 1 : qlen) - 1, which = 0;
                while (i >= 0 && k >= 0 && !full) {
                    const int bi = i > w ? i - w : 0;
                    if (k - bi < 0 || k - bi >= d.ncol) { bad = true; break; }   // never on a path with a finite score
                    which = (z[((int64_t)i * d.ncol + (k - bi)) * 32 + lane] >> (which << 1)) & 3;
                    if (which == 0) { push(0, 1); --i; --k; }
                    else if (which == 1) { push(2, 1); --i; }
                    else { push(1, 1); --k; }
                }
                if (!bad && i >= 0) push(2, i + 1);
                if (!bad && k >= 0) push(1, k + 1);
                for (int a = 0; a < n >> 1; ++a) {
                    const uint32_t t = cg[a]; cg[a] = cg[n - 1 - a]; cg[n - 1 - a] = t;
                }
            }
            d.n_cigar[job] = full || bad ? 0 : n;
            int32_t stj = full ? G3X_ERR_TOO_LONG : bad ? G3X_ERR_INTERNAL : G3X_OK;
            if (d.nm && stj == G3X_OK) {
                // NM and MD along the CIGAR (aux.cu:2831-2860): the query from its codes in shared
                // memory, the target from the planes 16 codes at a time
                const char* alpha = (flags & 4u) ? "TGCAN" : "ACGTN";
                char* md = d.md + (int64_t)job * d.md_stride;
                int x = 0, y = 0, u = 0, n_mm = 0, n_gap = 0, l = 0, cy = -1;
                uint32_t ty = 0, tyn = 0;
                bool ok = true;
                auto qcode = [&](int p) -> uint32_t {
                    const uint32_t nib = (qn[(p >> 3) * 32 + lane] >> ((p & 7) << 2)) & 0xFu;
                    return (nib & 4u) ? 4u : nib;
                };
                auto tcode = [&](int p) -> uint32_t {
                    if ((p >> 4) != cy) { cy = p >> 4; load16(d.codes, d.nmask, t_off, tlen, cy, trev, ty, tyn); }
                    return ((tyn >> (p & 15)) & 1u) ? 4u : (ty >> ((p & 15) << 1)) & 3u;
                };
                for (int k = 0; k < n && ok; ++k) {
                    const int op = (int)(cg[k] & 0xFu), len = (int)(cg[k] >> 4);
                    if (op == 0) {
                        for (int i = 0; i < len && ok; ++i) {
                            const uint32_t tc = tcode(y + i);
                            if (qcode(x + i) != tc) {
                                ok = put_uint(md, l, d.md_stride - 1, u);
                                if (ok && l + 1 < d.md_stride) md[l++] = alpha[tc]; else ok = false;
                                ++n_mm; u = 0;
                            } else ++u;
                        }
                        x += len; y += len;
                    } else if (op == 2) {
                        if (k > 0 && k < n - 1) {
                            ok = put_uint(md, l, d.md_stride - 1, u);
                            if (ok && l + 1 < d.md_stride) md[l++] = '^'; else ok = false;
                            for (int i = 0; i < len && ok; ++i) {
                                if (l + 1 < d.md_stride) md[l++] = alpha[tcode(y + i)]; else ok = false;
                            }
                            u = 0; n_gap += len;
                        }
                        y += len;
                    } else if (op == 1) {
                        x += len; n_gap += len;
                    }
                }
                ok = ok && put_uint(md, l, d.md_stride - 1, u);
                md[ok ? l : 0] = 0;
                d.nm[job] = ok ? n_mm + n_gap : 0;
                if (!ok) stj = G3X_ERR_TOO_LONG;
            } else if (d.nm) {
                d.nm[job] = 0;
                d.md[(int64_t)job * d.md_stride] = 0;
            }
            d.status[job] = stj;
        }
        __syncwarp();
    }
}

}  // namespace

}  // namespace g3x

extern "C" int g3x_ksw_global2_batch(g3x_ctx* ctx, const g3x_score_t* score, const g3x_job_t* d_jobs, int32_t n,
                                     const uint32_t* d_codes, const uint32_t* d_nmask, int64_t n_bases, int32_t max_qlen,
                                     int32_t max_tlen, int32_t max_w, int32_t* d_score, uint32_t* d_cigar,
                                     int32_t cigar_stride, int32_t* d_n_cigar, int32_t* d_nm, char* d_md,
                                     int32_t md_stride, int32_t* d_status, void* stream) {
    using namespace g3x;
    if (!ctx || !score || n < 0 || max_qlen < 0 || max_tlen < 0 || max_w < 0 || cigar_stride <= 0)
        return G3X_ERR_INVALID;
    if ((d_nm != nullptr) != (d_md != nullptr) || (d_nm && md_stride < 2)) return G3X_ERR_INVALID;
    if (n == 0) return G3X_OK;
    if (n_bases < 1 || n_bases > 0x100000000ll) return G3X_ERR_INVALID;
    if (!d_jobs || !d_codes || !d_nmask || !d_score || !d_cigar || !d_n_cigar || !d_status) return G3X_ERR_INVALID;
    ScoreParams sp;
    int rc = score_params(score, &sp);
    if (rc) return rc;
    const int dev = ctx_device(ctx);
    if (cudaSetDevice(dev) != cudaSuccess) return G3X_ERR_CUDA;
    GlobalDesc d;
    d.jobs = d_jobs; d.codes = d_codes; d.nmask = d_nmask; d.score = d_score; d.cigar = d_cigar;
    d.n_cigar = d_n_cigar; d.status = d_status; d.n = n;
    d.nm = d_nm; d.md = d_md; d.md_stride = md_stride; d.n_bases = n_bases;
    d.qmax = std::max(max_qlen, 1); d.tmax = std::max(max_tlen, 1); d.wmax = max_w;
    d.ncol = std::max(1, std::min(d.qmax, 2 * max_w + 1));
    d.ring = ((2 * max_w + 3) + 3) & ~3;
    d.stride = cigar_stride;
    // int16 ring when every value of the batch fits: |inside-band values| <= bound <= 8000
    int max_abs = 0;
    for (int k = 0; k < 25; ++k) max_abs = std::max(max_abs, std::abs((int)sp.mat[k]));
    const int64_t bound = 2 * (int64_t)std::max(sp.o_del, sp.o_ins) +
                          (int64_t)std::max(sp.e_del, sp.e_ins) * (d.qmax + d.tmax + 2) +
                          (int64_t)max_abs * (std::min(d.qmax, d.tmax) + 1);
    const bool c16 = bound <= 8000;
    auto kern = c16 ? global_kernel<true> : global_kernel<false>;
    const int nq = (d.qmax + 7) / 8 + 1;
    const size_t warp_smem = (size_t)nq * 128 + (size_t)d.ring * 32 * (c16 ? 4 : 8);
    size_t max_smem = 0;
    if (allow_max_smem(kern, &max_smem) != cudaSuccess) return G3X_ERR_CUDA;
    if (warp_smem > max_smem) return G3X_ERR_TOO_LONG;
    const int wpb = 2 * warp_smem <= max_smem ? 2 : 1;
    int sms = 0, per_sm = 0;
    sms = sm_count();
    per_sm = resident_blocks(kern, 32 * wpb, wpb * warp_smem);
    int blocks = sms * std::max(per_sm, 1);
    // direction bytes: tmax rows x ncol columns x 32 lanes per resident warp, at most 8 GiB
    d.zwarp = (int64_t)d.tmax * d.ncol * 32;
    const int64_t cap = (int64_t)8 << 30;
    while (blocks > 1 && (int64_t)blocks * wpb * d.zwarp > cap) blocks = blocks / 2;
    const int64_t need = (int64_t)blocks * wpb * d.zwarp;
    GlobalScratch& gs = ctx_global(ctx);
    if (gs.bytes < need || !gs.queue) {
        cudaFree(gs.z); cudaFree(gs.queue);
        gs.z = nullptr; gs.queue = nullptr; gs.bytes = 0;
        if (cudaMalloc(&gs.z, (size_t)need) != cudaSuccess || cudaMalloc(&gs.queue, sizeof(int32_t)) != cudaSuccess) {
            cudaFree(gs.z); gs.z = nullptr; cudaGetLastError();
            return G3X_ERR_NOMEM;
        }
        gs.bytes = need;
    }
    d.z = gs.z;
    d.queue = gs.queue;
    const cudaStream_t st = (cudaStream_t)stream;
    if ((rc = cost_order(ctx, d_jobs, n, sp, st, &d.order))) return rc;
    if (cudaMemsetAsync(gs.queue, 0, sizeof(int32_t), st) != cudaSuccess) return G3X_ERR_CUDA;
    kern<<<blocks, 32 * wpb, wpb * warp_smem, st>>>(d, sp);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

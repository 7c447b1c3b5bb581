// g3x_produce.cu -- the extension stage's inputs built on the GPU from the reference's own data:
// the packed reference (bwa's pac, two bits per base, bwa/src/bntseq.cu:4-5), the reads as u8
// codes (d_seq with d_seq_offset), and the per-seed extension records that ExtendingPairGenerate
// (bwa/src/aux.cu:2101-2189) writes for localExtending.
//
//   g3x_pac_to_planes      : the forward strand and its reverse complement (what
//                            bns_get_seq_gpu returns for positions >= l_pac, bntseq.cu:39-60) as
//                            2*l_pac bases of the code planes;
//   g3x_pack_codes_device  : u8 codes into the planes (g3x_pack_codes on device buffers);
//   g3x_pair_generate      : per seed record, its chain's reference window (aux.cu:2134-2156,
//                            with the contig clipping of bns_fetch_seq_gpu, bntseq.cu:62-80), as
//                            one g3x_seed_t for g3x_extend_seeds, and the window's contig id.
//
// One thread per 32 bases of the planes (one N-plane word, two code words): every word has a
// single writer, and the first and last words keep the bits outside the written range.
#include <cuda_runtime.h>
#include "g3x_internal.h"

namespace g3x {

constexpr int kTracebackBandCap = 500;   // GLOBALSW_BANDWITH_CUTOFF, bwa/src/aux.cuh:428

namespace {

// bwa's pac order: base k in byte k >> 2, bits ((~k) & 3) << 1
__device__ __forceinline__ uint32_t pac_base(const uint8_t* __restrict__ pac, int64_t k) {
    return (pac[k >> 2] >> ((~k & 3) << 1)) & 3u;
}

// Writes bases [base, base + len) of the planes; value(p) gives the code (0-3) and N bit of
// base base + p.
template <typename F>
__device__ __forceinline__ void write_word32(uint32_t* __restrict__ codes, uint32_t* __restrict__ nmask,
                                             int64_t base, int64_t len, int64_t word, F value) {
    const int64_t b0 = word << 5;
    uint32_t c[2] = {codes[2 * word], codes[2 * word + 1]};
    uint32_t nm = nmask[word];
#pragma unroll 4
    for (int t = 0; t < 32; ++t) {
        const int64_t p = b0 + t - base;
        if (p < 0 || p >= len) continue;
        uint32_t code, nbit;
        value(p, code, nbit);
        const int sh = (t & 15) << 1;
        c[t >> 4] = (c[t >> 4] & ~(3u << sh)) | (code << sh);
        nm = (nm & ~(1u << t)) | (nbit << t);
    }
    codes[2 * word] = c[0];
    codes[2 * word + 1] = c[1];
    nmask[word] = nm;
}

__global__ void pac_planes_kernel(const uint8_t* __restrict__ pac, int64_t l_pac, uint32_t* __restrict__ codes,
                                  uint32_t* __restrict__ nmask, int64_t base, int64_t words) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= words) return;
    write_word32(codes, nmask, base, 2 * l_pac, (base >> 5) + w, [&](int64_t p, uint32_t& code, uint32_t& nb) {
        code = p < l_pac ? pac_base(pac, p) : 3u - pac_base(pac, 2 * l_pac - 1 - p);
        nb = 0u;
    });
}

__global__ void pack_u8_kernel(const uint8_t* __restrict__ seq, int64_t len, uint32_t* __restrict__ codes,
                               uint32_t* __restrict__ nmask, int64_t base, int64_t words) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= words) return;
    write_word32(codes, nmask, base, len, (base >> 5) + w, [&](int64_t p, uint32_t& code, uint32_t& nb) {
        const uint32_t c = seq[p];
        code = c & 3u;
        nb = c > 3 ? 1u : 0u;
    });
}

// cal_max_gap, aux.cu:168-175
__device__ __forceinline__ int gap_of(const g3x_opt_t& o, int qlen) {
    const int l_del = (int)((double)(qlen * o.a - o.score.o_del) / o.score.e_del + 1.);
    const int l_ins = (int)((double)(qlen * o.a - o.score.o_ins) / o.score.e_ins + 1.);
    int l = l_del > l_ins ? l_del : l_ins;
    l = l > 1 ? l : 1;
    return l < o.w << 1 ? l : o.w << 1;
}

__global__ void pair_kernel(g3x_opt_t opt, int64_t l_pac, int64_t ref_off, const g3x_ann_t* __restrict__ anns,
                            int n_seqs, const g3x_read_t* __restrict__ reads, int n_reads,
                            const g3x_chain_t* __restrict__ chains, int n_chains,
                            const g3x_cseed_t* __restrict__ seeds, int n_seeds,
                            const g3x_seedrec_t* __restrict__ recs, int n_recs, g3x_seed_t* __restrict__ out,
                            int32_t* __restrict__ rid_out, int32_t* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_recs) return;
    const g3x_seedrec_t rc = recs[i];
    g3x_seed_t q = {};
    rid_out[i] = -1;
    status[i] = G3X_ERR_INVALID;
    out[i] = q;                                       // no jobs unless the record is valid
    if (rc.read < 0 || rc.read >= n_reads || rc.chain < 0 || rc.chain >= n_chains) return;
    const g3x_read_t rd = reads[rc.read];
    const g3x_chain_t ch = chains[rc.chain];
    if (ch.n <= 0 || ch.seed_beg < 0 || ch.seed_beg + (int64_t)ch.n > n_seeds || rc.seed < 0 || rc.seed >= ch.n)
        return;
    const g3x_cseed_t* cs = seeds + ch.seed_beg;
    // the chain's span (aux.cu:2134-2150)
    int64_t r0 = l_pac << 1, r1 = 0;
    for (int k = 0; k < ch.n; ++k) {
        const g3x_cseed_t t = cs[k];
        const int tail = rd.l_query - t.qbeg - t.len;
        const int64_t b = t.rbeg - (t.qbeg + gap_of(opt, t.qbeg));
        const int64_t e = t.rbeg + t.len + (tail + gap_of(opt, tail));
        r0 = b < r0 ? b : r0;
        r1 = e > r1 ? e : r1;
    }
    r0 = r0 > 0 ? r0 : 0;
    r1 = r1 < (l_pac << 1) ? r1 : (l_pac << 1);
    if (r0 < l_pac && l_pac < r1) {               // one strand: the first seed's (aux.cu:2151-2154)
        if (cs[0].rbeg < l_pac) r1 = l_pac; else r0 = l_pac;
    }
    // bns_fetch_seq_gpu: the first seed's contig, on its strand (bntseq.cu:68-79)
    const int64_t mid = cs[0].rbeg;
    if (mid < 0 || mid >= (l_pac << 1)) return;
    const bool rev = mid >= l_pac;
    const int64_t pf = rev ? (l_pac << 1) - 1 - mid : mid;
    int lo = 0, hi = n_seqs;
    while (lo < hi) {
        const int m = (lo + hi) >> 1;
        if (anns[m].offset <= pf) lo = m + 1; else hi = m;
    }
    const int rid = lo > 0 ? lo - 1 : 0;
    int64_t fb = anns[rid].offset, fe = fb + anns[rid].len;
    if (rev) { const int64_t t = fb; fb = (l_pac << 1) - fe; fe = (l_pac << 1) - t; }
    if (r1 < r0) { const int64_t t = r0; r0 = r1; r1 = t; }
    r0 = r0 > fb ? r0 : fb;
    r1 = r1 < fe ? r1 : fe;
    const g3x_cseed_t s = cs[rc.seed];
    q.read_off = (uint32_t)rd.read_off;
    q.win_off = (uint32_t)(ref_off + r0);
    q.l_query = rd.l_query;
    q.qbeg = s.qbeg;
    q.len = s.len;
    q.rbeg = s.rbeg;
    q.rmax0 = r0;
    q.rmax1 = r1;
    out[i] = q;
    rid_out[i] = rid;
    status[i] = G3X_OK;
}

// Band width of the traceback stage's pair (aux.cu:506-513, infer_bw).
__device__ int infer_bw(int l1, int l2, int score, int a, int q, int r) {
    if (l1 == l2 && l1 * a - score < (q + r - a) << 1) return 0;
    const int w = (int)((double)((l1 < l2 ? l1 : l2) * a - score - q) / r + 2.);
    const int d = l1 > l2 ? l1 - l2 : l2 - l1;
    return w < d ? d : w;
}

// FINALIZEALN_preprocessing2_kernel (aux.cu:2698-2745) and the band cap of traceback_baseline
// (aux.cu:2810-2812) for one alignment record: the region's query and reference slices as a
// ksw_global2 job.
__global__ void tb_pair_kernel(g3x_opt_t opt, int64_t l_pac, int64_t ref_off, const g3x_read_t* __restrict__ reads,
                               int n_reads, const g3x_alnreg_t* __restrict__ regs, int n_regs,
                               const g3x_alnrec_t* __restrict__ recs, int n_recs, g3x_job_t* __restrict__ jobs,
                               int32_t* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_recs) return;
    const g3x_alnrec_t rc = recs[i];
    g3x_job_t jb = {};
    jobs[i] = jb;                                     // an empty job unless the record is valid
    status[i] = G3X_ERR_INVALID;
    if (rc.read < 0 || rc.read >= n_reads || rc.reg < 0 || rc.reg >= n_regs) return;
    const g3x_read_t rd = reads[rc.read];
    const g3x_alnreg_t g = regs[rc.reg];
    const int lq = g.qe - g.qb;
    if (lq < 0 || g.qb < 0 || rd.read_off + g.qb + (int64_t)lq > 0xFFFFFFFFLL) return;
    // the reference slice as bns_get_seq_gpu returns it (bntseq.cu:39-60)
    int64_t beg = g.rb, end = g.re, rlen = 0;
    if (end < beg) { const int64_t t = beg; beg = end; end = t; }
    if (end > l_pac << 1) end = l_pac << 1;
    if (beg < 0) beg = 0;
    if (beg >= l_pac || end <= l_pac) rlen = end - beg;
    if (rlen < 0) return;           // [rb, re) wholly outside [0, 2 l_pac): no slice (invalid)
    if (lq > 65535 || rlen > 65535) { status[i] = G3X_ERR_TOO_LONG; return; }
    // the band (aux.cu:2711-2737), stored as uint16 (aux.cu:2745), at most 500 (aux.cu:2812)
    int w = 0;
    if ((int64_t)lq != g.re - g.rb) {
        const g3x_score_t& sc = opt.score;
        const int l2 = (int)(g.re - g.rb);
        const int wd = infer_bw(lq, l2, g.score, opt.a, sc.o_del, sc.e_del);
        const int wi = infer_bw(lq, l2, g.score, opt.a, sc.o_ins, sc.e_ins);
        w = wd > wi ? wd : wi;
        const int half = ((lq + 1) >> 1) * opt.a;
        const int max_ins = (int)((double)(half - sc.o_ins) / sc.e_ins + 1.);
        const int max_del = (int)((double)(half - sc.o_del) / sc.e_del + 1.);
        int max_gap = max_ins > max_del ? max_ins : max_del;
        max_gap = max_gap > 1 ? max_gap : 1;
        const int dl = (int)rlen > lq ? (int)rlen - lq : lq - (int)rlen;
        const int hi = (max_gap + dl + 1) >> 1;
        w = w < hi ? w : hi;
        w = w > dl + 3 ? w : dl + 3;
    }
    w = (uint16_t)w;
    jb.q_off = (uint32_t)(rd.read_off + g.qb);
    jb.t_off = (uint32_t)(ref_off + beg);
    jb.qlen = (uint16_t)lq;
    jb.tlen = (uint16_t)rlen;
    jb.w = w < kTracebackBandCap ? w : kTracebackBandCap;
    jb.flags = g.rb >= l_pac ? G3X_JOB_MDRC : 0u;
    jobs[i] = jb;
    status[i] = G3X_OK;
}

}  // namespace

}  // namespace g3x

extern "C" {

int g3x_traceback_pairs(const g3x_opt_t* opt, const g3x_refinfo_t* ref, const g3x_read_t* d_reads, int32_t n_reads,
                        const g3x_alnreg_t* d_regs, int32_t n_regs, const g3x_alnrec_t* d_recs, int32_t n_recs,
                        g3x_job_t* d_jobs, int32_t* d_status, void* stream) {
    if (!opt || !ref || n_recs < 0 || n_reads < 0 || n_regs < 0) return G3X_ERR_INVALID;
    if (n_recs == 0) return G3X_OK;
    if (!d_reads || !d_regs || !d_recs || !d_jobs || !d_status || ref->l_pac <= 0 || ref->ref_off < 0 ||
        ref->ref_off + 2 * ref->l_pac > 0xFFFFFFFFLL)
        return G3X_ERR_INVALID;
    g3x::ScoreParams sp;
    const int rc = g3x::score_params(&opt->score, &sp);
    if (rc) return rc;
    const int tb = 128;
    g3x::tb_pair_kernel<<<(n_recs + tb - 1) / tb, tb, 0, (cudaStream_t)stream>>>(
        *opt, ref->l_pac, ref->ref_off, d_reads, n_reads, d_regs, n_regs, d_recs, n_recs, d_jobs, d_status);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

int g3x_pac_to_planes(const uint8_t* d_pac, int64_t l_pac, uint32_t* d_codes, uint32_t* d_nmask,
                      int64_t base, void* stream) {
    if (l_pac <= 0 || base < 0 || !d_pac || !d_codes || !d_nmask) return G3X_ERR_INVALID;
    const int64_t words = ((base + 2 * l_pac + 31) >> 5) - (base >> 5);
    const int tb = 256;
    g3x::pac_planes_kernel<<<(unsigned)((words + tb - 1) / tb), tb, 0, (cudaStream_t)stream>>>(
        d_pac, l_pac, d_codes, d_nmask, base, words);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

int g3x_pack_codes_device(const uint8_t* d_seq, int64_t len, uint32_t* d_codes, uint32_t* d_nmask,
                          int64_t base, void* stream) {
    if (len < 0 || base < 0 || (len && (!d_seq || !d_codes || !d_nmask))) return G3X_ERR_INVALID;
    if (len == 0) return G3X_OK;
    const int64_t words = ((base + len + 31) >> 5) - (base >> 5);
    const int tb = 256;
    g3x::pack_u8_kernel<<<(unsigned)((words + tb - 1) / tb), tb, 0, (cudaStream_t)stream>>>(
        d_seq, len, d_codes, d_nmask, base, words);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

int g3x_pair_generate(const g3x_opt_t* opt, const g3x_refinfo_t* ref, const g3x_read_t* d_reads, int32_t n_reads,
                      const g3x_chain_t* d_chains, int32_t n_chains, const g3x_cseed_t* d_seeds, int32_t n_seeds,
                      const g3x_seedrec_t* d_recs, int32_t n_recs, g3x_seed_t* d_out, int32_t* d_rid,
                      int32_t* d_status, void* stream) {
    if (!opt || !ref || n_recs < 0 || n_reads < 0 || n_chains < 0 || n_seeds < 0) return G3X_ERR_INVALID;
    if (n_recs == 0) return G3X_OK;
    if (!d_reads || !d_chains || !d_seeds || !d_recs || !d_out || !d_rid || !d_status || ref->l_pac <= 0 ||
        ref->n_seqs <= 0 || !ref->d_anns || ref->ref_off < 0 || ref->ref_off + 2 * ref->l_pac > 0xFFFFFFFFLL)
        return G3X_ERR_INVALID;
    g3x::ScoreParams sp;
    const int rc = g3x::score_params(&opt->score, &sp);
    if (rc) return rc;
    const int tb = 128;
    g3x::pair_kernel<<<(n_recs + tb - 1) / tb, tb, 0, (cudaStream_t)stream>>>(
        *opt, ref->l_pac, ref->ref_off, ref->d_anns, ref->n_seqs, d_reads, n_reads, d_chains, n_chains, d_seeds,
        n_seeds, d_recs, n_recs, d_out, d_rid, d_status);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

}  // extern "C"

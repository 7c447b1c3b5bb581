// g3x_seedflt.cu -- the seed filter of long reads (mem_flt_chained_seeds, bwa/src/aux.cu:145-162,
// as CHAINFILTERING_flt_chained_seeds_kernel runs it per read, aux.cu:1991-2030) with the window
// score of mem_seed_sw (aux.cu:117-143).
//
// Three steps on the stream: one thread per read turns every seed that mem_seed_sw would align
// into a g3x_ksw_align2_batch job over the planes (the seed +-50 bases on the read and on the
// reference, clipped as bns_fetch_seq_gpu clips, bntseq.cu:62-87); one batch aligns them all;
// one thread per read then keeps, chain by chain and in place, the seeds the reference keeps.
// mem_seed_sw asks ksw_align2 for start positions (KSW_XSTART) but reads only the score, which
// the first pass alone decides, so the batch runs without the start-position pass.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <algorithm>
#include "g3x_core.h"
#include "g3x_internal.h"

namespace g3x {
namespace {

constexpr int kShortExt = 50;    // MEM_SHORT_EXT, bwa/src/aux.cuh:396
constexpr int kShortLen = 200;   // MEM_SHORT_LEN, bwa/src/aux.cuh:397

// The read's chains and seeds lie inside their arrays.
__device__ bool read_ok(const g3x_read_t& rd, const g3x_chain_t* __restrict__ chains, int n_chains, int n_seeds) {
    if (rd.n_chains < 0 || rd.chain_beg < 0 || (int64_t)rd.chain_beg + rd.n_chains > n_chains || rd.l_query < 0)
        return false;
    for (int c = 0; c < rd.n_chains; ++c) {
        const g3x_chain_t ch = chains[rd.chain_beg + c];
        if (ch.n < 0 || ch.seed_beg < 0 || (int64_t)ch.seed_beg + ch.n > n_seeds) return false;
    }
    return true;
}

// Contig of forward position pf: the last one whose offset is <= pf (bns_pos2rid_gpu).
__device__ int contig_of(const g3x_ann_t* __restrict__ anns, int n_seqs, int64_t pf) {
    int lo = 0, hi = n_seqs;
    while (lo < hi) {
        const int m = (lo + hi) >> 1;
        if (anns[m].offset <= pf) lo = m + 1; else hi = m;
    }
    return lo > 0 ? lo - 1 : 0;
}

// Per read: flag 1 (the filter runs; min_hsp set), 0 (left alone: min_l > 0.05 l_query,
// aux.cu:147-149) or -1 (records outside their arrays); a job per seed to align (jobs are
// zeroed beforehand, so a seed without a job keeps qlen 0).
__global__ void sfl_jobs_kernel(g3x_opt_t opt, int32_t min_chain_weight, int64_t l_pac, int64_t ref_off,
                                const g3x_ann_t* __restrict__ anns, int n_seqs, const g3x_read_t* __restrict__ reads,
                                int n_reads, const g3x_chain_t* __restrict__ chains, int n_chains,
                                const g3x_cseed_t* __restrict__ seeds, int n_seeds, g3x_job_t* __restrict__ jobs,
                                int32_t* __restrict__ flag, int32_t* __restrict__ min_hsp) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_reads) return;
    const g3x_read_t rd = reads[r];
    if (!read_ok(rd, chains, n_chains, n_seeds)) { flag[r] = -1; return; }
    const int lq = rd.l_query;
    // float arithmetic where the reference's is float: 1.1f * w, 5.5f * logf(l), 0.05f * l
    const double min_l = min_chain_weight ? (double)(1.1f * (float)min_chain_weight) : (double)(5.5f * logf((float)lq));
    min_hsp[r] = (int)(opt.a * min_l + .499);
    if (min_l > (double)(0.05f * (float)lq)) { flag[r] = 0; return; }
    flag[r] = 1;
    for (int c = 0; c < rd.n_chains; ++c) {
        const g3x_chain_t ch = chains[rd.chain_beg + c];
        for (int j = 0; j < ch.n; ++j) {
            const g3x_cseed_t s = seeds[ch.seed_beg + j];
            if (s.len >= kShortLen) continue;                       // aux.cu:124
            int qb = s.qbeg, qe = s.qbeg + s.len;
            int64_t rb = s.rbeg, re = s.rbeg + s.len;
            const int64_t mid = (rb + re) >> 1;
            qb = max(qb - kShortExt, 0);
            qe = min(qe + kShortExt, lq);
            rb = rb - kShortExt > 0 ? rb - kShortExt : 0;
            re = re + kShortExt < (l_pac << 1) ? re + kShortExt : (l_pac << 1);
            if (rb < l_pac && l_pac < re) {                         // aux.cu:133-136
                if (mid < l_pac) re = l_pac; else rb = l_pac;
            }
            if (qe - qb >= kShortLen || re - rb >= kShortLen) continue;   // aux.cu:137
            if (mid < 0 || mid >= (l_pac << 1) || qb > qe) continue;     // outside the reference: no window
            // bns_fetch_seq_gpu: the contig of the middle, on its strand (bntseq.cu:68-79)
            const bool rev = mid >= l_pac;
            const int rid = contig_of(anns, n_seqs, rev ? (l_pac << 1) - 1 - mid : mid);
            int64_t fb = anns[rid].offset, fe = fb + anns[rid].len;
            if (rev) { const int64_t t = fb; fb = (l_pac << 1) - fe; fe = (l_pac << 1) - t; }
            rb = rb > fb ? rb : fb;
            re = re < fe ? re : fe;
            g3x_job_t jb = {};
            jb.q_off = (uint32_t)(rd.read_off + qb);
            jb.t_off = (uint32_t)(ref_off + rb);
            jb.qlen = (uint16_t)(qe - qb);
            jb.tlen = (uint16_t)(re > rb ? re - rb : 0);
            jobs[ch.seed_beg + j] = jb;
        }
    }
}

// Per read: the window scores (or -1 for a seed without a job), then each chain keeps, in order
// and in place, the seeds with score -1 (scored len * a) or at least min_hsp (aux.cu:150-160).
__global__ void sfl_keep_kernel(int32_t a, const g3x_read_t* __restrict__ reads, int n_reads,
                                g3x_chain_t* __restrict__ chains, g3x_cseed_t* __restrict__ seeds,
                                const g3x_swr_t* __restrict__ sw, const int32_t* __restrict__ sw_status,
                                const int32_t* __restrict__ flag, const int32_t* __restrict__ min_hsp,
                                int32_t* __restrict__ sw_score, int32_t* __restrict__ status) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_reads) return;
    const int fl = flag[r];
    if (fl < 0) { status[r] = G3X_ERR_INVALID; return; }
    const g3x_read_t rd = reads[r];
    for (int c = 0; c < rd.n_chains; ++c) {
        g3x_chain_t* ch = chains + rd.chain_beg + c;
        const int n = ch->n;
        if (fl == 0) {
            if (sw_score)
                for (int j = 0; j < n; ++j) sw_score[ch->seed_beg + j] = -2;
            continue;
        }
        int k = 0;
        for (int j = 0; j < n; ++j) {
            const int idx = ch->seed_beg + j;
            g3x_cseed_t s = seeds[idx];                 // read before slot k <= j is written
            const int sc = sw_status[idx] == G3X_OK ? sw[idx].score : -1;
            if (sw_score) sw_score[idx] = sc;
            if (sc < 0 || sc >= min_hsp[r]) {
                s.score = sc < 0 ? s.len * a : sc;
                seeds[ch->seed_beg + k++] = s;
            }
        }
        ch->n = k;
    }
    status[r] = G3X_OK;
}

}  // namespace
}  // namespace g3x

extern "C" int g3x_flt_chained_seeds(g3x_ctx* ctx, const g3x_opt_t* opt, int32_t min_chain_weight,
                                     const g3x_refinfo_t* ref, const g3x_read_t* d_reads, int32_t n_reads,
                                     g3x_chain_t* d_chains, int32_t n_chains, g3x_cseed_t* d_seeds, int32_t n_seeds,
                                     const uint32_t* d_codes, const uint32_t* d_nmask, int64_t n_bases,
                                     int32_t* d_sw_score, int32_t* d_status, void* stream) {
    using namespace g3x;
    if (!ctx || !opt || !ref || n_reads < 0 || n_chains < 0 || n_seeds < 0 || min_chain_weight < 0)
        return G3X_ERR_INVALID;
    if (n_reads == 0) return G3X_OK;
    if (!d_reads || !d_status || (n_chains && !d_chains) || (n_seeds && (!d_seeds || !d_codes || !d_nmask)) ||
        ref->l_pac <= 0 || ref->n_seqs <= 0 || !ref->d_anns || ref->ref_off < 0 ||
        ref->ref_off + 2 * ref->l_pac > 0xFFFFFFFFLL || (n_seeds && (n_bases < 1 || n_bases > 0x100000000ll)))
        return G3X_ERR_INVALID;
    ScoreParams sp;
    int rc = score_params(&opt->score, &sp);
    if (rc) return rc;
    const int dev = ctx_device(ctx);
    if (cudaSetDevice(dev) != cudaSuccess) return G3X_ERR_CUDA;
    SwScratch& s = ctx_sw(ctx);
    const int64_t ns = std::max<int64_t>(n_seeds, 1);
    const int64_t need = ns * (int64_t)(sizeof(g3x_job_t) + sizeof(g3x_swr_t) + sizeof(int32_t)) +
                         (int64_t)n_reads * 2 * (int64_t)sizeof(int32_t) + 256;
    if (s.flt_cap < need) {
        cudaFree(s.flt);
        s.flt = nullptr; s.flt_cap = 0;
        if (cudaMalloc(&s.flt, (size_t)need) != cudaSuccess) { cudaGetLastError(); return G3X_ERR_NOMEM; }
        s.flt_cap = need;
    }
    g3x_job_t* jobs = reinterpret_cast<g3x_job_t*>(s.flt);
    g3x_swr_t* sw = reinterpret_cast<g3x_swr_t*>(jobs + ns);
    int32_t* sw_st = reinterpret_cast<int32_t*>(sw + ns);
    int32_t* flag = sw_st + ns;
    int32_t* min_hsp = flag + n_reads;
    const cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemsetAsync(jobs, 0, (size_t)ns * sizeof(g3x_job_t), st) != cudaSuccess) return G3X_ERR_CUDA;
    const int tb = 128, nb = (n_reads + tb - 1) / tb;
    sfl_jobs_kernel<<<nb, tb, 0, st>>>(*opt, min_chain_weight, ref->l_pac, ref->ref_off, ref->d_anns, ref->n_seqs,
                                        d_reads, n_reads, d_chains, n_chains, d_seeds, n_seeds, jobs, flag, min_hsp);
    if (cudaPeekAtLastError() != cudaSuccess) return G3X_ERR_CUDA;
    if (n_seeds > 0 &&
        (rc = g3x_ksw_align2_batch(ctx, &opt->score, jobs, n_seeds, d_codes, d_nmask, n_bases, 0, 0, sw, sw_st,
                                   stream)))
        return rc;
    sfl_keep_kernel<<<nb, tb, 0, st>>>(opt->a, d_reads, n_reads, d_chains, d_seeds, sw, sw_st, flag, min_hsp,
                                        d_sw_score, d_status);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

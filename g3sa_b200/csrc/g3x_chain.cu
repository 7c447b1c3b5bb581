// g3x_chain.cu -- mem_chain2aln (bwa/src/aux.cu:178-315) for batches of reads on the GPU.
//
// The reference runs one read's chains, and within a chain its seeds, one after the other:
// whether a seed is extended depends on the regions its read already has.  But a seed's
// extension itself depends only on the seed, its chain's reference window and the read, not
// on any other seed.  So every seed of the batch is extended at once, and the order-dependent
// decisions are replayed afterwards on the results:
//   prep     : one thread per read: each chain's reference window (aux.cu:186-205 and the
//              contig clipping of bns_fetch_seq_gpu, bwa/src/bntseq.cu:62-80), its seeds'
//              processing order (keys score << 32 | index, aux.cu:207-210), and a seed-level
//              record per seed;
//   extend   : all seeds through g3x_extend_seeds (left and right extension with band retry,
//              aux.cu:253-309), i.e. one batch through the context's width classes;
//   resolve  : one thread per read: the seeds in order with the containment test and its
//              overlap rescue (aux.cu:214-245) against the read's regions so far; a seed that
//              passes takes its extension result and gives a region with its seed coverage
//              (aux.cu:247-256, 303-314).
// The results of the seeds the reference skips are computed and discarded: more DP cells
// than the reference's (the price of one batch instead of one batch per region of the most
// prolific read), the same regions.
#include <cuda_runtime.h>
#include <algorithm>
#include "g3x_internal.h"

namespace g3x {

namespace {

struct ReadState {
    int32_t chain;     // chain being walked (absolute index); end of the read's chains = done
    int32_t k;         // next position in that chain's order, counting down; -1 = chain done
    int32_t nreg;      // regions so far
    int32_t status;
};

// cal_max_gap, aux.cu:168-175 (the same double arithmetic)
__device__ __forceinline__ int max_gap(const g3x_opt_t& o, int qlen) {
    const int l_del = (int)((double)(qlen * o.a - o.score.o_del) / o.score.e_del + 1.);
    const int l_ins = (int)((double)(qlen * o.a - o.score.o_ins) / o.score.e_ins + 1.);
    int l = l_del > l_ins ? l_del : l_ins;
    l = l > 1 ? l : 1;
    return l < o.w << 1 ? l : o.w << 1;
}

// Contig of forward position pos_f: the last one whose offset is <= pos_f.
__device__ int pos2rid(const g3x_ann_t* anns, int n_seqs, int64_t pos_f) {
    int lo = 0, hi = n_seqs;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (anns[mid].offset <= pos_f) lo = mid + 1; else hi = mid;
    }
    return lo > 0 ? lo - 1 : 0;
}

// In-place ascending heap sort of a chain's keys (distinct, so the order is unique).
__device__ void sort_keys(uint64_t* a, int n) {
    auto sift = [&](int i, int m) {
        for (;;) {
            int c = 2 * i + 1;
            if (c >= m) return;
            if (c + 1 < m && a[c + 1] > a[c]) ++c;
            if (a[i] >= a[c]) return;
            const uint64_t t = a[i]; a[i] = a[c]; a[c] = t;
            i = c;
        }
    };
    for (int i = n / 2 - 1; i >= 0; --i) sift(i, n);
    for (int m = n - 1; m > 0; --m) {
        const uint64_t t = a[0]; a[0] = a[m]; a[m] = t;
        sift(0, m);
    }
}

__global__ void prep_kernel(const g3x_read_t* __restrict__ reads, int n_reads,
                            const g3x_chain_t* __restrict__ chains, int n_chains,
                            const g3x_cseed_t* __restrict__ seeds, int n_seeds, g3x_opt_t opt,
                            int64_t l_pac, const g3x_ann_t* __restrict__ anns, int n_seqs,
                            int64_t ref_off, int64_t* __restrict__ win, uint64_t* __restrict__ srt,
                            g3x_seed_t* __restrict__ xseeds, ReadState* __restrict__ state,
                            int32_t* __restrict__ maxlen) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_reads) return;
    const g3x_read_t rd = reads[r];
    ReadState st;
    st.chain = rd.chain_beg; st.k = -1; st.nreg = 0; st.status = G3X_OK;
    // the records must index inside their arrays, and the read's seeds must be one range
    bool ok = rd.n_chains >= 0 && rd.chain_beg >= 0 && rd.chain_beg + (int64_t)rd.n_chains <= n_chains &&
              rd.l_query >= 0 && rd.read_off >= 0 && rd.read_off + rd.l_query <= 0xFFFFFFFFLL;
    for (int c = 0; ok && c < rd.n_chains; ++c) {
        const g3x_chain_t ch = chains[rd.chain_beg + c];
        ok = ch.n >= 0 && ch.seed_beg >= 0 && ch.seed_beg + (int64_t)ch.n <= n_seeds &&
             (c == 0 || ch.seed_beg == chains[rd.chain_beg + c - 1].seed_beg + chains[rd.chain_beg + c - 1].n);
        for (int i = 0; ok && i < ch.n; ++i) {
            const g3x_cseed_t s = seeds[ch.seed_beg + i];
            ok = s.qbeg >= 0 && s.len >= 0 && s.qbeg + s.len <= rd.l_query && s.rbeg >= 0 &&
                 s.rbeg + s.len <= (l_pac << 1);
        }
    }
    if (!ok) {   // its seeds keep the all-zero records, which make no jobs
        st.status = G3X_ERR_INVALID;
        st.chain = rd.chain_beg + (rd.n_chains > 0 ? rd.n_chains : 0);
        state[r] = st;
        return;
    }
    for (int c = 0; c < rd.n_chains; ++c) {
        const int ci = rd.chain_beg + c;
        const g3x_chain_t ch = chains[ci];
        if (ch.n == 0) continue;
        const g3x_cseed_t* cs = seeds + ch.seed_beg;
        int64_t r0 = l_pac << 1, r1 = 0;
        for (int i = 0; i < ch.n; ++i) {
            const g3x_cseed_t t = cs[i];
            const int tail = rd.l_query - t.qbeg - t.len;
            const int64_t b = t.rbeg - (t.qbeg + max_gap(opt, t.qbeg));
            const int64_t e = t.rbeg + t.len + (tail + max_gap(opt, tail));
            r0 = b < r0 ? b : r0;
            r1 = e > r1 ? e : r1;
        }
        r0 = r0 > 0 ? r0 : 0;
        r1 = r1 < (l_pac << 1) ? r1 : (l_pac << 1);
        if (r0 < l_pac && l_pac < r1) {          // one strand: the first seed's (aux.cu:200-203)
            if (cs[0].rbeg < l_pac) r1 = l_pac; else r0 = l_pac;
        }
        // the first seed's contig, on its strand (bntseq.cu:68-79)
        const int64_t mid = cs[0].rbeg;
        const bool rev = mid >= l_pac;
        const int rid = pos2rid(anns, n_seqs, rev ? (l_pac << 1) - 1 - mid : mid);
        int64_t fb = anns[rid].offset, fe = fb + anns[rid].len;
        if (rev) { const int64_t t = fb; fb = (l_pac << 1) - fe; fe = (l_pac << 1) - t; }
        if (r1 < r0) { const int64_t t = r0; r0 = r1; r1 = t; }
        r0 = r0 > fb ? r0 : fb;
        r1 = r1 < fe ? r1 : fe;
        win[2 * ci] = r0;
        win[2 * ci + 1] = r1;
        // the extension jobs' length bounds: the read, and the window (either side's target
        // lies inside it)
        atomicMax(maxlen + 1, (int32_t)(r1 - r0 < 0x7FFFFFFF ? (r1 > r0 ? r1 - r0 : 0) : 0x7FFFFFFF));
        uint64_t* key = srt + ch.seed_beg;
        for (int i = 0; i < ch.n; ++i) key[i] = (uint64_t)cs[i].score << 32 | (uint64_t)i;
        sort_keys(key, ch.n);
        for (int i = 0; i < ch.n; ++i) {                    // every seed's extension record
            g3x_seed_t q;
            q.read_off = (uint32_t)rd.read_off;
            q.win_off = (uint32_t)(ref_off + r0);
            q.l_query = rd.l_query;
            q.qbeg = cs[i].qbeg;
            q.len = cs[i].len;
            q.pad_ = 0;
            q.rbeg = cs[i].rbeg;
            q.rmax0 = r0;
            q.rmax1 = r1;
            xseeds[ch.seed_beg + i] = q;
        }
    }
    if (rd.n_chains > 0) st.k = chains[rd.chain_beg].n - 1;
    atomicMax(maxlen, rd.l_query);
    state[r] = st;
}

// Is seed s (almost) inside region p (aux.cu:217-231).
__device__ bool around(const g3x_opt_t& opt, int l_query, const g3x_cseed_t& s, const g3x_alnreg_t& p) {
    if (s.rbeg < p.rb || s.rbeg + s.len > p.re || s.qbeg < p.qb || s.qbeg + s.len > p.qe) return false;
    if (s.len - p.seedlen0 > .1 * l_query) return false;
    int qd = s.qbeg - p.qb;
    int64_t rd = s.rbeg - p.rb;
    int gap = max_gap(opt, (int)(qd < rd ? qd : rd));
    int w = gap < p.w ? gap : p.w;
    if (qd - rd < w && rd - qd < w) return true;
    qd = p.qe - (s.qbeg + s.len);
    rd = p.re - (s.rbeg + s.len);
    gap = max_gap(opt, (int)(qd < rd ? qd : rd));
    w = gap < p.w ? gap : p.w;
    return qd - rd < w && rd - qd < w;
}

__global__ void resolve_kernel(const g3x_read_t* __restrict__ reads, int n_reads,
                               const g3x_chain_t* __restrict__ chains, const g3x_cseed_t* __restrict__ seeds,
                               g3x_opt_t opt, uint64_t* __restrict__ srt, ReadState* __restrict__ state,
                               const g3x_reg_t* __restrict__ xregs, const int32_t* __restrict__ xstatus,
                               g3x_alnreg_t* __restrict__ regs) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_reads) return;
    ReadState st = state[r];
    const g3x_read_t rd = reads[r];
    const int end = rd.chain_beg + rd.n_chains;
    if (st.status != G3X_OK || st.chain >= end) return;
    g3x_alnreg_t* av = regs + chains[rd.chain_beg].seed_beg;
    for (int ci = rd.chain_beg; ci < end; ++ci) {
        const g3x_chain_t ch = chains[ci];
        const g3x_cseed_t* cs = seeds + ch.seed_beg;
        uint64_t* key = srt + ch.seed_beg;
        for (int k = ch.n - 1; k >= 0; --k) {
            const int si = (int)(uint32_t)key[k];
            const g3x_cseed_t s = cs[si];
            int i = 0;
            while (i < st.nreg && !around(opt, rd.l_query, s, av[i])) ++i;
            if (i < st.nreg) {
                // extended anyway only when an earlier seed of the chain, at least 95% as
                // long, overlaps it by a quarter on another diagonal (aux.cu:234-244)
                int j;
                for (j = k + 1; j < ch.n; ++j) {
                    if (key[j] == 0) continue;
                    const g3x_cseed_t t = cs[(uint32_t)key[j]];
                    if (t.len < s.len * .95) continue;
                    if (s.qbeg <= t.qbeg && s.qbeg + s.len - t.qbeg >= s.len >> 2 &&
                        t.qbeg - s.qbeg != t.rbeg - s.rbeg) break;
                    if (t.qbeg <= s.qbeg && t.qbeg + t.len - s.qbeg >= s.len >> 2 &&
                        s.qbeg - t.qbeg != s.rbeg - t.rbeg) break;
                }
                if (j == ch.n) { key[k] = 0; continue; }
            }
            const int64_t xi = (int64_t)ch.seed_beg + si;
            if (xstatus[xi] != G3X_OK) {                // an extension beyond the job limits
                st.status = xstatus[xi];
                state[r] = st;
                return;
            }
            const g3x_reg_t x = xregs[xi];
            g3x_alnreg_t a;
            a.rb = x.rb; a.re = x.re; a.qb = x.qb; a.qe = x.qe;
            a.rid = ch.rid; a.score = x.score; a.truesc = x.truesc; a.w = x.w;
            a.seedcov = 0;
            for (int t = 0; t < ch.n; ++t) {            // aux.cu:303-307
                const g3x_cseed_t u = cs[t];
                if (u.qbeg >= a.qb && u.qbeg + u.len <= a.qe && u.rbeg >= a.rb && u.rbeg + u.len <= a.re)
                    a.seedcov += u.len;
            }
            a.seedlen0 = s.len;
            a.frac_rep = ch.frac_rep;
            a.pad_ = 0;
            av[st.nreg++] = a;
        }
    }
    st.chain = end;
    state[r] = st;
}

__global__ void finish_kernel(const ReadState* __restrict__ state, int n_reads, int32_t* __restrict__ nregs,
                              int32_t* __restrict__ status) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_reads) return;
    nregs[r] = state[r].nreg;
    status[r] = state[r].status;
}

}  // namespace

void free_chain_scratch(ChainScratch& w) {
    cudaFree(w.win); cudaFree(w.srt); cudaFree(w.state); cudaFree(w.xseeds); cudaFree(w.xregs);
    cudaFree(w.xstatus); cudaFree(w.maxlen);
    cudaFreeHost(w.h_maxlen);
    w = ChainScratch();
}

static int alloc_chain_scratch(ChainScratch& w, int64_t reads, int64_t chains, int64_t seeds) {
    if (w.maxlen && reads <= w.reads && chains <= w.chains && seeds <= w.seeds) return G3X_OK;
    const int64_t R = std::max(reads, w.reads), C = std::max(chains, w.chains), S = std::max(seeds, w.seeds);
    free_chain_scratch(w);
    bool ok = cudaMalloc(&w.win, std::max<int64_t>(C, 1) * 2 * sizeof(int64_t)) == cudaSuccess &&
              cudaMalloc(&w.srt, std::max<int64_t>(S, 1) * sizeof(uint64_t)) == cudaSuccess &&
              cudaMalloc(&w.state, std::max<int64_t>(R, 1) * 16) == cudaSuccess &&
              cudaMalloc(&w.xseeds, std::max<int64_t>(S, 1) * sizeof(g3x_seed_t)) == cudaSuccess &&
              cudaMalloc(&w.xregs, std::max<int64_t>(S, 1) * sizeof(g3x_reg_t)) == cudaSuccess &&
              cudaMalloc(&w.xstatus, std::max<int64_t>(S, 1) * sizeof(int32_t)) == cudaSuccess &&
              cudaMalloc(&w.maxlen, 2 * sizeof(int32_t)) == cudaSuccess &&
              cudaMallocHost(&w.h_maxlen, 2 * sizeof(int32_t)) == cudaSuccess;
    if (!ok) { free_chain_scratch(w); cudaGetLastError(); return G3X_ERR_NOMEM; }
    w.reads = R; w.chains = C; w.seeds = S;
    return G3X_OK;
}

}  // namespace g3x

extern "C" int g3x_chain2aln(g3x_ctx* ctx, const g3x_opt_t* opt, const g3x_refinfo_t* ref,
                             const g3x_read_t* d_reads, int32_t n_reads, const g3x_chain_t* d_chains,
                             int32_t n_chains, const g3x_cseed_t* d_seeds, int32_t n_seeds,
                             const uint32_t* d_codes, const uint32_t* d_nmask, g3x_alnreg_t* d_regs,
                             int32_t* d_nregs, int32_t* d_status, const g3x_batch_opts_t* opts,
                             void* stream) {
    using namespace g3x;
    if (!ctx || !opt || !ref || !opts || n_reads < 0 || n_chains < 0 || n_seeds < 0) return G3X_ERR_INVALID;
    if (n_reads == 0) return G3X_OK;
    if (!d_reads || !d_codes || !d_nmask || !d_nregs || !d_status || ref->l_pac <= 0 ||
        ref->n_seqs <= 0 || !ref->d_anns || ref->ref_off < 0 || ref->ref_off + 2 * ref->l_pac > 0xFFFFFFFFLL ||
        (n_chains > 0 && !d_chains) || (n_seeds > 0 && (!d_seeds || !d_regs)))
        return G3X_ERR_INVALID;
    ScoreParams sp;
    int rc = score_params(&opt->score, &sp);
    if (rc) return rc;
    if (cudaSetDevice(ctx_device(ctx)) != cudaSuccess) return G3X_ERR_CUDA;
    ChainScratch& w = ctx_chain(ctx);
    if ((rc = alloc_chain_scratch(w, n_reads, n_chains, n_seeds))) return rc;
    const cudaStream_t st = (cudaStream_t)stream;
    const int tb = 128, nb = (n_reads + tb - 1) / tb;
    ReadState* state = static_cast<ReadState*>(w.state);
    // all-zero seed records (an empty read and seed: no extension jobs) for every seed that no
    // valid read's chain sets
    if (cudaMemsetAsync(w.maxlen, 0, 2 * sizeof(int32_t), st) != cudaSuccess ||
        (n_seeds > 0 && cudaMemsetAsync(w.xseeds, 0, sizeof(g3x_seed_t) * (size_t)n_seeds, st) != cudaSuccess))
        return G3X_ERR_CUDA;
    prep_kernel<<<nb, tb, 0, st>>>(d_reads, n_reads, d_chains, n_chains, d_seeds, n_seeds, *opt, ref->l_pac,
                                   ref->d_anns, ref->n_seqs, ref->ref_off, w.win, w.srt, w.xseeds, state,
                                   w.maxlen);
    if (cudaPeekAtLastError() != cudaSuccess ||
        cudaMemcpyAsync(w.h_maxlen, w.maxlen, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return G3X_ERR_CUDA;
    if (n_seeds > 0) {
        // every seed extended in one batch: the caller's schedule and kernel choice, with length
        // bounds from the batch itself
        g3x_batch_opts_t xo = *opts;
        xo.max_qlen = std::max<int32_t>(w.h_maxlen[0], 1);
        xo.max_tlen = std::max<int32_t>(w.h_maxlen[1], 1);
        xo.d_cells = nullptr;
        xo.d_rows = nullptr;
        if ((rc = g3x_extend_seeds(ctx, opt, w.xseeds, n_seeds, d_codes, d_nmask, w.xregs, w.xstatus, &xo,
                                   stream)))
            return rc;
        resolve_kernel<<<nb, tb, 0, st>>>(d_reads, n_reads, d_chains, d_seeds, *opt, w.srt, state, w.xregs,
                                          w.xstatus, d_regs);
        if (cudaPeekAtLastError() != cudaSuccess) return G3X_ERR_CUDA;
    }
    finish_kernel<<<nb, tb, 0, st>>>(state, n_reads, d_nregs, d_status);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

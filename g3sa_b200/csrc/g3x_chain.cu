// g3x_chain.cu -- mem_chain2aln (bwa/src/aux.cu:178-315) for batches of reads on the GPU.
//
// The reference runs one read's chains, and within a chain its seeds, one after the other:
// whether a seed is extended depends on the regions its read already has.  Here reads run
// side by side and seeds in waves:
//   prep    : one thread per read: each chain's reference window (aux.cu:186-205 and the
//             contig clipping of bns_fetch_seq_gpu, bwa/src/bntseq.cu:62-80) and its seeds'
//             processing order (keys score << 32 | index, aux.cu:207-210);
//   decide  : one thread per read: walks the read's seeds in order from where the last wave
//             stopped, skipping every seed the containment test rejects (aux.cu:214-245),
//             and queues the first seed to extend;
//   extend  : the queued seeds through g3x_extend_seeds (left and right extension with band
//             retry, aux.cu:253-309), i.e. the context's width classes;
//   commit  : one thread per queued seed: the region with its seed coverage (aux.cu:247-256,
//             303-314) appended to its read's regions, which the next decide reads.
// The host reads each wave's size back; the waves end when no read queues a seed.
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
                            int64_t* __restrict__ win, uint64_t* __restrict__ srt,
                            ReadState* __restrict__ state, int32_t* __restrict__ maxlen) {
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
    if (!ok) {
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

__global__ void decide_kernel(const g3x_read_t* __restrict__ reads, int n_reads,
                              const g3x_chain_t* __restrict__ chains, const g3x_cseed_t* __restrict__ seeds,
                              g3x_opt_t opt, int64_t ref_off, const int64_t* __restrict__ win,
                              uint64_t* __restrict__ srt, ReadState* __restrict__ state,
                              const g3x_alnreg_t* __restrict__ regs, g3x_seed_t* __restrict__ wseeds,
                              int32_t* __restrict__ wsrc, int32_t* __restrict__ count) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_reads) return;
    ReadState st = state[r];
    const g3x_read_t rd = reads[r];
    const int end = rd.chain_beg + rd.n_chains;
    if (st.status != G3X_OK || st.chain >= end) return;
    const g3x_alnreg_t* av = regs + chains[rd.chain_beg].seed_beg;
    for (;;) {
        while (st.k < 0) {
            if (++st.chain >= end) { state[r] = st; return; }
            st.k = chains[st.chain].n - 1;
        }
        const g3x_chain_t ch = chains[st.chain];
        const g3x_cseed_t* cs = seeds + ch.seed_beg;
        uint64_t* key = srt + ch.seed_beg;
        const int k = st.k--;
        const g3x_cseed_t s = cs[(uint32_t)key[k]];
        int i = 0;
        while (i < st.nreg && !around(opt, rd.l_query, s, av[i])) ++i;
        if (i < st.nreg) {
            // extended anyway only when an earlier seed of the chain, at least 95% as long,
            // overlaps it by a quarter on another diagonal (aux.cu:234-244)
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
        const int64_t r0 = win[2 * st.chain], r1 = win[2 * st.chain + 1];
        g3x_seed_t q;
        q.read_off = (uint32_t)rd.read_off;
        q.win_off = (uint32_t)(ref_off + r0);
        q.l_query = rd.l_query;
        q.qbeg = s.qbeg;
        q.len = s.len;
        q.pad_ = 0;
        q.rbeg = s.rbeg;
        q.rmax0 = r0;
        q.rmax1 = r1;
        const int at = atomicAdd(count, 1);
        wseeds[at] = q;
        wsrc[3 * at] = r;
        wsrc[3 * at + 1] = st.chain;
        wsrc[3 * at + 2] = ch.seed_beg + (int32_t)(uint32_t)key[k];
        state[r] = st;
        return;
    }
}

__global__ void commit_kernel(const g3x_read_t* __restrict__ reads, const g3x_chain_t* __restrict__ chains,
                              const g3x_cseed_t* __restrict__ seeds, const int32_t* __restrict__ wsrc,
                              const g3x_reg_t* __restrict__ wregs, const int32_t* __restrict__ wstatus,
                              const int32_t* __restrict__ count, ReadState* __restrict__ state,
                              g3x_alnreg_t* __restrict__ regs) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= *count) return;
    const int r = wsrc[3 * e], ci = wsrc[3 * e + 1], si = wsrc[3 * e + 2];
    ReadState st = state[r];
    if (wstatus[e] != G3X_OK) {
        st.status = wstatus[e];
        state[r] = st;
        return;
    }
    const g3x_reg_t x = wregs[e];
    const g3x_chain_t ch = chains[ci];
    g3x_alnreg_t a;
    a.rb = x.rb; a.re = x.re; a.qb = x.qb; a.qe = x.qe;
    a.rid = ch.rid; a.score = x.score; a.truesc = x.truesc; a.w = x.w;
    a.seedcov = 0;
    for (int i = 0; i < ch.n; ++i) {                // aux.cu:303-307
        const g3x_cseed_t t = seeds[ch.seed_beg + i];
        if (t.qbeg >= a.qb && t.qbeg + t.len <= a.qe && t.rbeg >= a.rb && t.rbeg + t.len <= a.re)
            a.seedcov += t.len;
    }
    a.seedlen0 = seeds[si].len;
    a.frac_rep = ch.frac_rep;
    a.pad_ = 0;
    regs[chains[reads[r].chain_beg].seed_beg + st.nreg] = a;
    ++st.nreg;
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
    cudaFree(w.win); cudaFree(w.srt); cudaFree(w.state); cudaFree(w.wseeds); cudaFree(w.wsrc);
    cudaFree(w.wregs); cudaFree(w.wstatus); cudaFree(w.count); cudaFree(w.maxlen);
    cudaFreeHost(w.h_count);
    w = ChainScratch();
}

static int alloc_chain_scratch(ChainScratch& w, int64_t reads, int64_t chains, int64_t seeds) {
    if (w.count && reads <= w.reads && chains <= w.chains && seeds <= w.seeds) return G3X_OK;
    const int64_t R = std::max(reads, w.reads), C = std::max(chains, w.chains), S = std::max(seeds, w.seeds);
    free_chain_scratch(w);
    bool ok = cudaMalloc(&w.win, std::max<int64_t>(C, 1) * 2 * sizeof(int64_t)) == cudaSuccess &&
              cudaMalloc(&w.srt, std::max<int64_t>(S, 1) * sizeof(uint64_t)) == cudaSuccess &&
              cudaMalloc(&w.state, std::max<int64_t>(R, 1) * 16) == cudaSuccess &&
              cudaMalloc(&w.wseeds, std::max<int64_t>(R, 1) * sizeof(g3x_seed_t)) == cudaSuccess &&
              cudaMalloc(&w.wsrc, std::max<int64_t>(R, 1) * 3 * sizeof(int32_t)) == cudaSuccess &&
              cudaMalloc(&w.wregs, std::max<int64_t>(R, 1) * sizeof(g3x_reg_t)) == cudaSuccess &&
              cudaMalloc(&w.wstatus, std::max<int64_t>(R, 1) * sizeof(int32_t)) == cudaSuccess &&
              cudaMalloc(&w.count, sizeof(int32_t)) == cudaSuccess &&
              cudaMalloc(&w.maxlen, 2 * sizeof(int32_t)) == cudaSuccess &&
              cudaMallocHost(&w.h_count, 2 * sizeof(int32_t)) == cudaSuccess;
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
    if (cudaMemsetAsync(w.maxlen, 0, 2 * sizeof(int32_t), st) != cudaSuccess) return G3X_ERR_CUDA;
    prep_kernel<<<nb, tb, 0, st>>>(d_reads, n_reads, d_chains, n_chains, d_seeds, n_seeds, *opt, ref->l_pac,
                                   ref->d_anns, ref->n_seqs, w.win, w.srt, state, w.maxlen);
    if (cudaPeekAtLastError() != cudaSuccess ||
        cudaMemcpyAsync(w.h_count, w.maxlen, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return G3X_ERR_CUDA;
    // the extension waves' options: the caller's schedule and kernel choice, with length
    // bounds from the batch itself
    g3x_batch_opts_t xo = *opts;
    xo.max_qlen = std::max<int32_t>(w.h_count[0], 1);
    xo.max_tlen = std::max<int32_t>(w.h_count[1], 1);
    xo.d_cells = nullptr;
    // every wave extends at least one seed and every seed is visited once
    for (int64_t wave = 0; wave <= n_seeds; ++wave) {
        if (cudaMemsetAsync(w.count, 0, sizeof(int32_t), st) != cudaSuccess) return G3X_ERR_CUDA;
        decide_kernel<<<nb, tb, 0, st>>>(d_reads, n_reads, d_chains, d_seeds, *opt, ref->ref_off, w.win,
                                         w.srt, state, d_regs, w.wseeds, w.wsrc, w.count);
        if (cudaMemcpyAsync(w.h_count, w.count, sizeof(int32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return G3X_ERR_CUDA;
        const int32_t cnt = *w.h_count;
        if (cnt == 0) break;
        if ((rc = g3x_extend_seeds(ctx, opt, w.wseeds, cnt, d_codes, d_nmask, w.wregs, w.wstatus, &xo, stream)))
            return rc;
        commit_kernel<<<(cnt + tb - 1) / tb, tb, 0, st>>>(d_reads, d_chains, d_seeds, w.wsrc, w.wregs, w.wstatus,
                                                          w.count, state, d_regs);
        if (cudaPeekAtLastError() != cudaSuccess) return G3X_ERR_CUDA;
    }
    finish_kernel<<<nb, tb, 0, st>>>(state, n_reads, d_nregs, d_status);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

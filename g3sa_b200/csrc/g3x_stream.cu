// g3x_stream.cu -- chunked, double-buffered seed-level extension from host memory.
//
// Host seeds are processed in chunks.  For each chunk the library finds the range of plane
// bases its seeds reference, copies the chunk's seeds (re-based to that range) and those
// plane words to one of two device buffer sets on a copy stream, and runs the seed-level
// pipeline of g3x_seeds.cu on a compute stream that waits for the copy.  While chunk k is
// extended, chunk k+1 is copied into the other set.  Results come back through pinned
// staging buffers.  The buffer sets, staging and streams live in the context and are grown
// on demand, so repeated calls allocate nothing.
#include <cuda_runtime.h>
#include <string.h>
#include <algorithm>
#include <vector>
#include "g3x_internal.h"

struct g3x_ctx;  // defined in g3x_api.cu

namespace g3x {

namespace {

struct ChunkRange {
    int64_t first, count;
    uint32_t base;        // first plane base copied (multiple of 32)
    int64_t bases;        // bases copied
};

void release(StreamSet& s) {
    cudaFree(s.d_seeds); cudaFree(s.d_codes); cudaFree(s.d_nmask); cudaFree(s.d_regs);
    cudaFree(s.d_status);
    cudaFreeHost(s.h_seeds); cudaFreeHost(s.h_regs); cudaFreeHost(s.h_status);
    if (s.h2d) cudaEventDestroy(s.h2d);
    if (s.done) cudaEventDestroy(s.done);
    s = StreamSet();
}

// Buffer sets for chunks of `chunk` seeds and the given plane words, kept when large enough.
int grow_stream(StreamScratch& ss, int64_t chunk, int64_t code_words, int64_t mask_words) {
    if (!ss.copy_st && (cudaStreamCreateWithFlags(&ss.copy_st, cudaStreamNonBlocking) != cudaSuccess ||
                        cudaStreamCreateWithFlags(&ss.comp_st, cudaStreamNonBlocking) != cudaSuccess))
        return G3X_ERR_CUDA;
    if (chunk <= ss.seeds && code_words <= ss.code_words && mask_words <= ss.mask_words) return G3X_OK;
    chunk = std::max(chunk, ss.seeds);
    code_words = std::max(code_words, ss.code_words);
    mask_words = std::max(mask_words, ss.mask_words);
    bool ok = true;
    for (int b = 0; b < 2 && ok; ++b) {
        StreamSet& s = ss.set[b];
        release(s);
        ok = cudaMalloc(&s.d_seeds, chunk * sizeof(g3x_seed_t)) == cudaSuccess &&
             cudaMalloc(&s.d_codes, code_words * sizeof(uint32_t)) == cudaSuccess &&
             cudaMalloc(&s.d_nmask, mask_words * sizeof(uint32_t)) == cudaSuccess &&
             cudaMalloc(&s.d_regs, chunk * sizeof(g3x_reg_t)) == cudaSuccess &&
             cudaMalloc(&s.d_status, chunk * sizeof(int32_t)) == cudaSuccess &&
             cudaMallocHost(&s.h_seeds, chunk * sizeof(g3x_seed_t)) == cudaSuccess &&
             cudaMallocHost(&s.h_regs, chunk * sizeof(g3x_reg_t)) == cudaSuccess &&
             cudaMallocHost(&s.h_status, chunk * sizeof(int32_t)) == cudaSuccess &&
             cudaEventCreateWithFlags(&s.h2d, cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) == cudaSuccess;
    }
    if (!ok) {
        for (int b = 0; b < 2; ++b) release(ss.set[b]);
        ss.seeds = ss.code_words = ss.mask_words = 0;
        return G3X_ERR_NOMEM;
    }
    ss.seeds = chunk; ss.code_words = code_words; ss.mask_words = mask_words;
    return G3X_OK;
}

}  // namespace

int extend_seeds_stream(StreamScratch& ss, SeedScratch& ws, int (*grow)(SeedScratch&, int64_t),
                        const g3x_opt_t& opt, const ScoreParams& sp, const g3x_seed_t* h_seeds, int64_t n,
                        const uint32_t* h_codes, const uint32_t* h_nmask, int64_t n_bases,
                        g3x_reg_t* h_regs, int32_t* h_status, int32_t chunk,
                        const LaunchDesc& proto, const WaveRunner* runner) {
    if (chunk <= 0) chunk = 65536;
    const int64_t nchunks = (n + chunk - 1) / chunk;
    std::vector<ChunkRange> ranges((size_t)nchunks);
    int64_t max_bases = 0;
    for (int64_t c = 0; c < nchunks; ++c) {
        ChunkRange& R = ranges[(size_t)c];
        R.first = c * chunk;
        R.count = std::min<int64_t>(chunk, n - R.first);
        int64_t lo = INT64_MAX, hi = 0;
        for (int64_t k = R.first; k < R.first + R.count; ++k) {
            const g3x_seed_t& s = h_seeds[k];
            lo = std::min<int64_t>(lo, std::min<int64_t>(s.read_off, s.win_off));
            hi = std::max<int64_t>(hi, std::max<int64_t>((int64_t)s.read_off + s.l_query,
                                                         (int64_t)s.win_off + (s.rmax1 - s.rmax0)));
        }
        if (hi > n_bases) return G3X_ERR_INVALID;
        R.base = (uint32_t)(lo & ~(int64_t)31);
        R.bases = hi - R.base;
        max_bases = std::max(max_bases, R.bases);
    }
    int rc = grow(ws, chunk);
    if (rc) return rc;
    if ((rc = grow_stream(ss, chunk, (max_bases + 15) / 16 + 2, (max_bases + 31) / 32 + 2))) return rc;
    StreamSet* sets = ss.set;
    cudaStream_t copy_st = ss.copy_st, comp_st = ss.comp_st;
    for (int b = 0; b < 2; ++b) sets[b].pending = -1;
    const int64_t total_code_words = (n_bases + 15) / 16, total_mask_words = (n_bases + 31) / 32;
    auto drain = [&](StreamSet& s) -> int {
        if (s.pending < 0) return G3X_OK;
        if (cudaEventSynchronize(s.done) != cudaSuccess) return G3X_ERR_CUDA;
        const ChunkRange& R = ranges[(size_t)s.pending];
        memcpy(h_regs + R.first, s.h_regs, R.count * sizeof(g3x_reg_t));
        memcpy(h_status + R.first, s.h_status, R.count * sizeof(int32_t));
        s.pending = -1;
        return G3X_OK;
    };
    for (int64_t c = 0; c < nchunks && rc == G3X_OK; ++c) {
        StreamSet& s = sets[c & 1];
        const ChunkRange& R = ranges[(size_t)c];
        if ((rc = drain(s))) break;                      // set free: its last chunk is done
        for (int64_t k = 0; k < R.count; ++k) {
            g3x_seed_t t = h_seeds[R.first + k];
            t.read_off -= R.base;
            t.win_off -= R.base;
            s.h_seeds[k] = t;
        }
        const int64_t cw0 = R.base / 16, mw0 = R.base / 32;
        const int64_t cw = std::min<int64_t>((R.bases + 15) / 16 + 1, total_code_words - cw0);
        const int64_t mw = std::min<int64_t>((R.bases + 31) / 32 + 1, total_mask_words - mw0);
        if (cudaMemcpyAsync(s.d_seeds, s.h_seeds, R.count * sizeof(g3x_seed_t), cudaMemcpyHostToDevice, copy_st) ||
            cudaMemcpyAsync(s.d_codes, h_codes + cw0, cw * sizeof(uint32_t), cudaMemcpyHostToDevice, copy_st) ||
            cudaMemcpyAsync(s.d_nmask, h_nmask + mw0, mw * sizeof(uint32_t), cudaMemcpyHostToDevice, copy_st) ||
            cudaEventRecord(s.h2d, copy_st) || cudaStreamWaitEvent(comp_st, s.h2d, 0)) {
            rc = G3X_ERR_CUDA;
            break;
        }
        LaunchDesc cp = proto;                 // the chunk's planes: its copied words, re-based
        cp.n_bases = std::min<int64_t>(cw * 16, mw * 32);
        if ((rc = extend_seeds(ws, opt, sp, s.d_seeds, (int)R.count, s.d_codes, s.d_nmask, s.d_regs,
                               s.d_status, cp, comp_st, runner)))
            break;
        if (cudaMemcpyAsync(s.h_regs, s.d_regs, R.count * sizeof(g3x_reg_t), cudaMemcpyDeviceToHost, comp_st) ||
            cudaMemcpyAsync(s.h_status, s.d_status, R.count * sizeof(int32_t), cudaMemcpyDeviceToHost, comp_st) ||
            cudaEventRecord(s.done, comp_st)) {
            rc = G3X_ERR_CUDA;
            break;
        }
        s.pending = c;
    }
    for (int b = 0; b < 2; ++b) {
        int r2 = drain(sets[b]);
        if (rc == G3X_OK) rc = r2;
    }
    cudaStreamSynchronize(comp_st);
    cudaStreamSynchronize(copy_st);
    return rc;
}

void free_stream_scratch(StreamScratch& ss) {
    for (int b = 0; b < 2; ++b) release(ss.set[b]);
    if (ss.comp_st) cudaStreamDestroy(ss.comp_st);
    if (ss.copy_st) cudaStreamDestroy(ss.copy_st);
    ss = StreamScratch();
}

}  // namespace g3x

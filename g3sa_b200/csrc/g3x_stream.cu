// g3x_stream.cu -- chunked seed-level extension from host memory, several chunks in flight.
//
// Host seeds are processed in chunks.  For each chunk the library finds the range of plane
// bases its seeds reference, copies the chunk's seeds and those plane words to the device on a
// copy stream, re-bases the seeds' plane offsets to the copied range on the device, and runs the
// seed-level pipeline of g3x_seeds.cu on a compute stream that waits for the copy.
// kStreamLanes chunks run at a time, chunk c on lane c % kStreamLanes: each lane has its own
// compute stream, buffer set, pinned staging, seed scratch and sort scratch, and chains its
// width classes on its stream as programmatic dependent launches (side by side, without side
// streams), so the latency-bound waves of one chunk (a wave's longest job runs alone at the
// end) overlap the next chunks' waves.  The host work of a chunk (its range, its launches)
// overlaps the device work of the chunks before it.  Host buffers that are pinned are copied
// straight to and from; pageable ones go through the lane's pinned staging.  All of it lives in
// the context and is grown on demand, so repeated calls allocate nothing.
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

// The chunk's seeds' plane offsets, made relative to the copied range.
__global__ void rebase_kernel(g3x_seed_t* __restrict__ s, int n, uint32_t base) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) {
        s[k].read_off -= base;
        s[k].win_off -= base;
    }
}

// The lane's buffers and staging (not its stream, events and queue counters).
void release_buffers(StreamSet& s) {
    cudaFree(s.d_seeds); cudaFree(s.d_codes); cudaFree(s.d_nmask); cudaFree(s.d_regs);
    cudaFree(s.d_status);
    cudaFreeHost(s.h_seeds); cudaFreeHost(s.h_regs); cudaFreeHost(s.h_status);
    s.d_seeds = nullptr; s.d_codes = nullptr; s.d_nmask = nullptr; s.d_regs = nullptr;
    s.d_status = nullptr; s.h_seeds = nullptr; s.h_regs = nullptr; s.h_status = nullptr;
}

void release_lane(StreamSet& s) {
    release_buffers(s);
    free_seed_scratch(s.seeds);
    free_sched(s.sched);
    cudaFree(s.queue);
    if (s.h2d) cudaEventDestroy(s.h2d);
    if (s.done) cudaEventDestroy(s.done);
    if (s.comp) cudaStreamDestroy(s.comp);
    s = StreamSet();
}

// Streams, events and queue counters of the lanes, made once per context.
int make_lanes(StreamScratch& ss) {
    if (ss.lanes_ready) return G3X_OK;
    bool ok = cudaStreamCreateWithFlags(&ss.copy_st, cudaStreamNonBlocking) == cudaSuccess;
    for (int l = 0; l < kStreamLanes && ok; ++l) {
        StreamSet& s = ss.set[l];
        ok = cudaStreamCreateWithFlags(&s.comp, cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&s.h2d, cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) == cudaSuccess &&
             cudaMalloc(&s.queue, kMaxBuckets * sizeof(int32_t)) == cudaSuccess;
    }
    if (!ok) {
        free_stream_scratch(ss);
        return G3X_ERR_CUDA;
    }
    ss.lanes_ready = true;
    return G3X_OK;
}

// Buffer sets for chunks of `chunk` seeds and the given plane words, kept when large enough.
// The lanes must be idle.
int grow_stream(StreamScratch& ss, int64_t chunk, int64_t code_words, int64_t mask_words) {
    int rc = make_lanes(ss);
    if (rc) return rc;
    if (chunk <= ss.seeds && code_words <= ss.code_words && mask_words <= ss.mask_words) return G3X_OK;
    chunk = std::max(chunk, ss.seeds);
    code_words = std::max(code_words, ss.code_words);
    mask_words = std::max(mask_words, ss.mask_words);
    bool ok = true;
    for (int l = 0; l < kStreamLanes && ok; ++l) {
        StreamSet& s = ss.set[l];
        release_buffers(s);
        ok = cudaMalloc(&s.d_seeds, chunk * sizeof(g3x_seed_t)) == cudaSuccess &&
             cudaMalloc(&s.d_codes, code_words * sizeof(uint32_t)) == cudaSuccess &&
             cudaMalloc(&s.d_nmask, mask_words * sizeof(uint32_t)) == cudaSuccess &&
             cudaMalloc(&s.d_regs, chunk * sizeof(g3x_reg_t)) == cudaSuccess &&
             cudaMalloc(&s.d_status, chunk * sizeof(int32_t)) == cudaSuccess &&
             cudaMallocHost(&s.h_seeds, chunk * sizeof(g3x_seed_t)) == cudaSuccess &&
             cudaMallocHost(&s.h_regs, chunk * sizeof(g3x_reg_t)) == cudaSuccess &&
             cudaMallocHost(&s.h_status, chunk * sizeof(int32_t)) == cudaSuccess &&
             alloc_seed_scratch(s.seeds, chunk) == G3X_OK && alloc_sched(s.sched, chunk) == G3X_OK;
    }
    if (!ok) {
        for (int l = 0; l < kStreamLanes; ++l) release_buffers(ss.set[l]);
        ss.seeds = ss.code_words = ss.mask_words = 0;
        return G3X_ERR_NOMEM;
    }
    ss.seeds = chunk; ss.code_words = code_words; ss.mask_words = mask_words;
    return G3X_OK;
}

// Whether host memory at p is pinned (page-locked or registered): then the copies go straight
// between it and the device, asynchronously; pageable memory goes through the lane's pinned
// staging, so that the copies still overlap the other lanes' work.
bool pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();                            // older drivers report pageable memory so
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Range of plane bases chunk [first, first + count) reads; G3X_ERR_INVALID when a seed reaches
// past the planes.
int chunk_range(const g3x_seed_t* h_seeds, int64_t first, int64_t count, int64_t n_bases, ChunkRange& R) {
    R.first = first;
    R.count = count;
    int64_t lo = INT64_MAX, hi = 0;
    for (int64_t k = first; k < first + count; ++k) {
        const g3x_seed_t& s = h_seeds[k];
        lo = std::min<int64_t>(lo, std::min<int64_t>(s.read_off, s.win_off));
        hi = std::max<int64_t>(hi, std::max<int64_t>((int64_t)s.read_off + s.l_query,
                                                     (int64_t)s.win_off + (s.rmax1 - s.rmax0)));
    }
    if (hi > n_bases) return G3X_ERR_INVALID;
    R.base = (uint32_t)(lo & ~(int64_t)31);
    R.bases = hi - R.base;
    return G3X_OK;
}

}  // namespace

int extend_seeds_stream(StreamScratch& ss, const g3x_opt_t& opt, const ScoreParams& sp,
                        const g3x_seed_t* h_seeds, int64_t n, const uint32_t* h_codes,
                        const uint32_t* h_nmask, int64_t n_bases, g3x_reg_t* h_regs, int32_t* h_status,
                        int32_t chunk, const LaunchDesc& proto, const WaveRunner* runner) {
    if (chunk <= 0) chunk = 65536;
    const int64_t nchunks = (n + chunk - 1) / chunk;
    int rc = grow_stream(ss, chunk, 1, 1);     // plane words grow with the first chunk's range
    if (rc) return rc;
    // each lane's class waves run on the lane's own sort scratch and queue counters, the classes
    // chained on the lane's stream
    ClassRes res[kStreamLanes];
    ClassWave cw[kStreamLanes];
    WaveRunner wr[kStreamLanes];
    const ClassWave* cw0 = runner ? static_cast<const ClassWave*>(runner->user) : nullptr;
    std::vector<ChunkRange> pend(kStreamLanes);
    for (int l = 0; l < kStreamLanes; ++l) {
        StreamSet& s = ss.set[l];
        s.pending = -1;
        if (!runner) continue;
        res[l] = ClassRes{&s.sched, s.queue, nullptr, nullptr, nullptr, nullptr};
        cw[l] = ClassWave{cw0->ctx, cw0->learned, &res[l]};
        wr[l] = WaveRunner{runner->run, &cw[l]};
    }
    const int64_t total_code_words = (n_bases + 15) / 16, total_mask_words = (n_bases + 31) / 32;
    const bool seeds_pinned = pinned(h_seeds), out_pinned = pinned(h_regs) && pinned(h_status);
    // Each lane's seed pipeline for a full chunk (about 75 launches and copies) is captured as a
    // CUDA graph at the lane's first full chunk of the call and replayed for the next ones: the
    // host work per chunk, not the device, had bounded the stream.  A graph sees the lane's
    // buffers at their capacity (the chunk's seeds lie inside its copied plane range by
    // construction, so no read leaves the copied words), and the seeds are re-based on the copy
    // stream, so nothing in it changes from chunk to chunk.  The last, partial chunk and any
    // failed capture take the direct launches.
    cudaGraphExec_t gx[kStreamLanes] = {};
    bool graphs = true;
    auto drop_graphs = [&]() {
        for (int l = 0; l < kStreamLanes; ++l)
            if (gx[l]) {
                cudaGraphExecDestroy(gx[l]);
                gx[l] = nullptr;
            }
    };
    auto drain = [&](int l) -> int {
        StreamSet& s = ss.set[l];
        if (s.pending < 0) return G3X_OK;
        if (cudaEventSynchronize(s.done) != cudaSuccess) return G3X_ERR_CUDA;
        const ChunkRange& R = pend[(size_t)l];
        if (!out_pinned) {
            memcpy(h_regs + R.first, s.h_regs, R.count * sizeof(g3x_reg_t));
            memcpy(h_status + R.first, s.h_status, R.count * sizeof(int32_t));
        }
        s.pending = -1;
        return G3X_OK;
    };
    for (int64_t c = 0; c < nchunks && rc == G3X_OK; ++c) {
        const int l = (int)(c % kStreamLanes);
        StreamSet& s = ss.set[l];
        ChunkRange R;
        if ((rc = chunk_range(h_seeds, c * chunk, std::min<int64_t>(chunk, n - c * chunk), n_bases, R))) break;
        const int64_t cw0w = R.base / 16, mw0 = R.base / 32;
        const int64_t cwn = std::min<int64_t>((R.bases + 15) / 16 + 1, total_code_words - cw0w);
        const int64_t mwn = std::min<int64_t>((R.bases + 31) / 32 + 1, total_mask_words - mw0);
        if (cwn > ss.code_words || mwn > ss.mask_words) {
            // a wider range than the sets hold: let every lane finish, then grow them
            for (int k = 0; k < kStreamLanes && rc == G3X_OK; ++k) rc = drain(k);
            if (rc) break;
            for (int k = 0; k < kStreamLanes; ++k) cudaStreamSynchronize(ss.set[k].comp);
            drop_graphs();                               // their buffers are about to move
            if ((rc = grow_stream(ss, chunk, cwn + cwn / 4, mwn + mwn / 4))) break;
        }
        if ((rc = drain(l))) break;                      // lane free: its last chunk is done
        const g3x_seed_t* src = h_seeds + R.first;
        if (!seeds_pinned) {
            memcpy(s.h_seeds, src, R.count * sizeof(g3x_seed_t));
            src = s.h_seeds;
        }
        if (cudaMemcpyAsync(s.d_seeds, src, R.count * sizeof(g3x_seed_t), cudaMemcpyHostToDevice, ss.copy_st) ||
            cudaMemcpyAsync(s.d_codes, h_codes + cw0w, cwn * sizeof(uint32_t), cudaMemcpyHostToDevice, ss.copy_st) ||
            cudaMemcpyAsync(s.d_nmask, h_nmask + mw0, mwn * sizeof(uint32_t), cudaMemcpyHostToDevice, ss.copy_st)) {
            rc = G3X_ERR_CUDA;
            break;
        }
        rebase_kernel<<<(unsigned)((R.count + 255) / 256), 256, 0, ss.copy_st>>>(s.d_seeds, (int)R.count, R.base);
        if (cudaEventRecord(s.h2d, ss.copy_st) || cudaStreamWaitEvent(s.comp, s.h2d, 0)) {
            rc = G3X_ERR_CUDA;
            break;
        }
        const WaveRunner* run_l = runner ? &wr[l] : nullptr;
        bool done = false;
        if (graphs && R.count == chunk) {
            if (!gx[l]) {
                LaunchDesc gp = proto;         // the lane's planes at their capacity
                gp.n_bases = std::min<int64_t>(ss.code_words * 16, ss.mask_words * 32);
                cudaGraph_t gph = nullptr;
                if (cudaStreamBeginCapture(s.comp, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                    const int rc2 = extend_seeds(s.seeds, opt, sp, s.d_seeds, (int)R.count, s.d_codes, s.d_nmask,
                                                 s.d_regs, s.d_status, gp, s.comp, run_l);
                    const cudaError_t e = cudaStreamEndCapture(s.comp, &gph);
                    if (rc2 != G3X_OK || e != cudaSuccess || cudaGraphInstantiate(&gx[l], gph, 0) != cudaSuccess)
                        gx[l] = nullptr;
                    if (gph) cudaGraphDestroy(gph);
                }
                if (!gx[l]) {
                    graphs = false;                  // capture refused: direct launches from here on
                    cudaGetLastError();
                }
            }
            if (gx[l]) {
                if (cudaGraphLaunch(gx[l], s.comp) != cudaSuccess) {
                    rc = G3X_ERR_CUDA;
                    break;
                }
                done = true;
            }
        }
        if (!done) {
            LaunchDesc cp = proto;             // the chunk's planes: its copied words, re-based
            cp.n_bases = std::min<int64_t>(cwn * 16, mwn * 32);
            if ((rc = extend_seeds(s.seeds, opt, sp, s.d_seeds, (int)R.count, s.d_codes, s.d_nmask, s.d_regs,
                                   s.d_status, cp, s.comp, run_l)))
                break;
        }
        g3x_reg_t* dst_regs = out_pinned ? h_regs + R.first : s.h_regs;
        int32_t* dst_status = out_pinned ? h_status + R.first : s.h_status;
        if (cudaMemcpyAsync(dst_regs, s.d_regs, R.count * sizeof(g3x_reg_t), cudaMemcpyDeviceToHost, s.comp) ||
            cudaMemcpyAsync(dst_status, s.d_status, R.count * sizeof(int32_t), cudaMemcpyDeviceToHost, s.comp) ||
            cudaEventRecord(s.done, s.comp)) {
            rc = G3X_ERR_CUDA;
            break;
        }
        pend[(size_t)l] = R;
        s.pending = c;
    }
    for (int l = 0; l < kStreamLanes; ++l) {
        int r2 = drain(l);
        if (rc == G3X_OK) rc = r2;
    }
    for (int l = 0; l < kStreamLanes; ++l) cudaStreamSynchronize(ss.set[l].comp);
    cudaStreamSynchronize(ss.copy_st);
    drop_graphs();
    return rc;
}

void free_stream_scratch(StreamScratch& ss) {
    for (int l = 0; l < kStreamLanes; ++l) release_lane(ss.set[l]);
    if (ss.copy_st) cudaStreamDestroy(ss.copy_st);
    ss = StreamScratch();
}

}  // namespace g3x

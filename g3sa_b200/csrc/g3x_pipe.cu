// g3x_pipe.cu -- batches of ksw_extend2 jobs from host memory, pipelined across calls.
//
// A pipe owns two device buffer sets.  Each submit takes the next set and queues three steps
// on three streams of the pipe:
//   h2d   : wait for the caller's stream (work queued there before the submit), and for the
//           set's previous extension (which read the set's inputs); copy jobs, code plane and
//           N plane to the set;
//   comp  : wait for the copies and for the set's previous output copy (which read the set's
//           outputs); run g3x_ksw_extend2_batch on the set (the context's schedule and width
//           classes);
//   d2h   : wait for the extension; copy outputs and statuses back to the caller's host
//           buffers.
// Consecutive submits alternate sets, so batch k+1's input copies and batch k-1's output
// copies run on the copy engines while batch k is extended.  g3x_pipe_wait makes a caller's
// stream wait for every submitted batch.  The extension of all batches is serialised on the
// comp stream, so the context's scratch is used by one batch at a time.
#include <cuda_runtime.h>
#include <algorithm>
#include <string.h>
#include <new>
#include "g3x_internal.h"

namespace {

struct PipeSet {
    g3x_job_t* d_jobs = nullptr;
    uint32_t* d_codes = nullptr;
    uint32_t* d_nmask = nullptr;
    g3x_ext_t* d_out = nullptr;
    int32_t* d_status = nullptr;
    cudaEvent_t in_ready = nullptr, comp_done = nullptr, out_done = nullptr;
};

}  // namespace

struct g3x_pipe {
    g3x_ctx* ctx;
    int device;
    g3x_score_t score;
    int32_t schedule;
    int32_t max_jobs;
    int64_t max_code_words, max_nmask_words;
    cudaStream_t h2d, comp, d2h;
    cudaEvent_t call;
    PipeSet set[2];
    int next;
};

namespace {

void release(g3x_pipe* p) {
    if (!p) return;
    for (PipeSet& s : p->set) {
        cudaFree(s.d_jobs); cudaFree(s.d_codes); cudaFree(s.d_nmask); cudaFree(s.d_out);
        cudaFree(s.d_status);
        if (s.in_ready) cudaEventDestroy(s.in_ready);
        if (s.comp_done) cudaEventDestroy(s.comp_done);
        if (s.out_done) cudaEventDestroy(s.out_done);
    }
    if (p->call) cudaEventDestroy(p->call);
    if (p->h2d) cudaStreamDestroy(p->h2d);
    if (p->comp) cudaStreamDestroy(p->comp);
    if (p->d2h) cudaStreamDestroy(p->d2h);
    delete p;
}

}  // namespace

extern "C" {

int g3x_pipe_create(g3x_ctx* ctx, const g3x_score_t* score, int32_t schedule, int32_t max_jobs,
                    int64_t max_code_words, int64_t max_nmask_words, g3x_pipe** out) {
    if (!ctx || !score || !out || max_jobs <= 0 || max_code_words <= 0 || max_nmask_words <= 0)
        return G3X_ERR_INVALID;
    if (schedule != G3X_SCHED_PLAIN && schedule != G3X_SCHED_SORTED && schedule != G3X_SCHED_LEARNED)
        return G3X_ERR_INVALID;
    *out = nullptr;
    g3x::ScoreParams sp;
    int rc = g3x::score_params(score, &sp);
    if (rc) return rc;
    const int dev = g3x::ctx_device(ctx);
    if (cudaSetDevice(dev) != cudaSuccess) return G3X_ERR_CUDA;
    g3x_pipe* p = new (std::nothrow) g3x_pipe();
    if (!p) return G3X_ERR_NOMEM;
    p->ctx = ctx;
    p->device = dev;
    p->score = *score;
    p->schedule = schedule;
    p->max_jobs = max_jobs;
    p->max_code_words = max_code_words;
    p->max_nmask_words = max_nmask_words;
    p->h2d = p->comp = p->d2h = nullptr;
    p->call = nullptr;
    p->next = 0;
    bool ok = cudaStreamCreateWithFlags(&p->h2d, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&p->comp, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&p->d2h, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&p->call, cudaEventDisableTiming) == cudaSuccess;
    for (PipeSet& s : p->set) {
        ok = ok && cudaEventCreateWithFlags(&s.in_ready, cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&s.comp_done, cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&s.out_done, cudaEventDisableTiming) == cudaSuccess;
        if (!ok) break;
        rc = cudaMalloc(&s.d_jobs, sizeof(g3x_job_t) * (size_t)max_jobs) == cudaSuccess &&
             cudaMalloc(&s.d_codes, sizeof(uint32_t) * (size_t)max_code_words) == cudaSuccess &&
             cudaMalloc(&s.d_nmask, sizeof(uint32_t) * (size_t)max_nmask_words) == cudaSuccess &&
             cudaMalloc(&s.d_out, sizeof(g3x_ext_t) * (size_t)max_jobs) == cudaSuccess &&
             cudaMalloc(&s.d_status, sizeof(int32_t) * (size_t)max_jobs) == cudaSuccess
                 ? G3X_OK : G3X_ERR_NOMEM;
        if (rc) break;
    }
    if (!ok || rc) {
        release(p);
        cudaGetLastError();
        return ok ? rc : G3X_ERR_CUDA;
    }
    *out = p;
    return G3X_OK;
}

int g3x_pipe_submit(g3x_pipe* p, const g3x_job_t* h_jobs, int32_t n, const uint32_t* h_codes,
                    int64_t code_words, const uint32_t* h_nmask, int64_t nmask_words,
                    int32_t max_qlen, int32_t max_tlen, g3x_ext_t* h_out, int32_t* h_status,
                    void* stream) {
    if (!p || n < 0 || code_words < 0 || nmask_words < 0) return G3X_ERR_INVALID;
    if (n > p->max_jobs || code_words > p->max_code_words || nmask_words > p->max_nmask_words)
        return G3X_ERR_INVALID;
    if (n == 0) return G3X_OK;
    if (!h_jobs || !h_codes || !h_nmask || !h_out || !h_status) return G3X_ERR_INVALID;
    if (cudaSetDevice(p->device) != cudaSuccess) return G3X_ERR_CUDA;
    PipeSet& s = p->set[p->next];
    const cudaStream_t caller = (cudaStream_t)stream;
    bool ok = cudaEventRecord(p->call, caller) == cudaSuccess &&
              cudaStreamWaitEvent(p->h2d, p->call, 0) == cudaSuccess &&
              cudaStreamWaitEvent(p->h2d, s.comp_done, 0) == cudaSuccess &&
              cudaMemcpyAsync(s.d_jobs, h_jobs, sizeof(g3x_job_t) * (size_t)n, cudaMemcpyHostToDevice,
                              p->h2d) == cudaSuccess &&
              cudaMemcpyAsync(s.d_codes, h_codes, sizeof(uint32_t) * (size_t)code_words,
                              cudaMemcpyHostToDevice, p->h2d) == cudaSuccess &&
              cudaMemcpyAsync(s.d_nmask, h_nmask, sizeof(uint32_t) * (size_t)nmask_words,
                              cudaMemcpyHostToDevice, p->h2d) == cudaSuccess &&
              cudaEventRecord(s.in_ready, p->h2d) == cudaSuccess &&
              cudaStreamWaitEvent(p->comp, s.in_ready, 0) == cudaSuccess &&
              cudaStreamWaitEvent(p->comp, s.out_done, 0) == cudaSuccess;
    if (!ok) return G3X_ERR_CUDA;
    g3x_batch_opts_t opts;
    memset(&opts, 0, sizeof(opts));
    opts.schedule = p->schedule;
    opts.max_qlen = max_qlen;
    opts.max_tlen = max_tlen;
    opts.kernel = G3X_KERNEL_AUTO;
    // the planes hold the bases their copied words cover
    opts.n_bases = std::min<int64_t>(std::min<int64_t>(code_words * 16, nmask_words * 32), 0x100000000ll);
    int rc = g3x_ksw_extend2_batch(p->ctx, &p->score, s.d_jobs, n, s.d_codes, s.d_nmask, s.d_out,
                                   s.d_status, &opts, p->comp);
    if (rc) return rc;
    ok = cudaEventRecord(s.comp_done, p->comp) == cudaSuccess &&
         cudaStreamWaitEvent(p->d2h, s.comp_done, 0) == cudaSuccess &&
         cudaMemcpyAsync(h_out, s.d_out, sizeof(g3x_ext_t) * (size_t)n, cudaMemcpyDeviceToHost,
                         p->d2h) == cudaSuccess &&
         cudaMemcpyAsync(h_status, s.d_status, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost,
                         p->d2h) == cudaSuccess &&
         cudaEventRecord(s.out_done, p->d2h) == cudaSuccess;
    if (!ok) return G3X_ERR_CUDA;
    p->next ^= 1;
    return G3X_OK;
}

int g3x_pipe_wait(g3x_pipe* p, void* stream) {
    if (!p) return G3X_ERR_INVALID;
    if (cudaSetDevice(p->device) != cudaSuccess) return G3X_ERR_CUDA;
    const cudaStream_t caller = (cudaStream_t)stream;
    // an event never recorded counts as complete
    for (PipeSet& s : p->set)
        if (cudaStreamWaitEvent(caller, s.out_done, 0) != cudaSuccess) return G3X_ERR_CUDA;
    return G3X_OK;
}

int g3x_pipe_destroy(g3x_pipe* p) {
    if (!p) return G3X_ERR_INVALID;
    cudaSetDevice(p->device);
    for (PipeSet& s : p->set) cudaEventSynchronize(s.out_done);
    release(p);
    return G3X_OK;
}

}  // extern "C"

// g3x_api.cu -- host side of the C ABI declared in include/g3x.h.
#include <cuda_runtime.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <new>
#include "g3x_internal.h"

struct g3x_ctx {
    int device;
    int sms;
    int32_t* d_queue;            // persistent-kernel job counters
    g3x::SeedScratch seeds;      // seed-level scratch, grown on demand
};

namespace g3x {

int score_params(const g3x_score_t* s, ScoreParams* sp) {
    if (!s) return G3X_ERR_INVALID;
    if (s->m != 5 || s->e_del <= 0 || s->e_ins <= 0 || s->o_del < 0 || s->o_ins < 0)
        return G3X_ERR_SCORE;
    memset(sp, 0, sizeof(*sp));
    int max_sc = 0;
    for (int k = 0; k < 25; ++k) {
        sp->mat[k] = s->mat[k];
        if (s->mat[k] > max_sc) max_sc = s->mat[k];
    }
    sp->o_del = s->o_del; sp->e_del = s->e_del; sp->o_ins = s->o_ins; sp->e_ins = s->e_ins;
    sp->zdrop = s->zdrop; sp->end_bonus = s->end_bonus; sp->max_sc = max_sc;
    return G3X_OK;
}

// Kernel choice for one batch: schedule, lanes per job and smem bounds.
int batch_proto(const g3x_batch_opts_t* opts, int32_t* queue, LaunchDesc* d) {
    if (!opts) return G3X_ERR_INVALID;
    if (opts->max_qlen < 0 || opts->max_tlen < 0 || opts->max_qlen > 65534 || opts->max_tlen > 65535)
        return G3X_ERR_INVALID;
    memset(d, 0, sizeof(*d));
    d->qmax = opts->max_qlen;
    d->tmax = opts->max_tlen;
    d->cells = opts->d_cells;
    switch (opts->schedule) {
        case G3X_SCHED_PLAIN:
            d->lanes = 32; d->persistent = 0; d->warps_per_block = 1;
            break;
        case G3X_SCHED_SORTED:
        case G3X_SCHED_LEARNED: {
            int lanes = opts->lanes ? opts->lanes : 8;
            if (lanes != 8 && lanes != 16 && lanes != 32) return G3X_ERR_INVALID;
            // Shared memory per job grows with the query; a warp of narrow groups must fit,
            // so the lane count is raised until it does.
            while (lanes < 32 && (32 / lanes) * group_smem_bytes(d->qmax, d->tmax) > 227 * 1024)
                lanes *= 2;
            d->lanes = lanes; d->persistent = 1; d->warps_per_block = 4;
            d->queue = queue;
            break;
        }
        default:
            return G3X_ERR_INVALID;
    }
    return G3X_OK;
}

static void free_seed_scratch(SeedScratch& w) {
    cudaFree(w.ljobs); cudaFree(w.rjobs); cudaFree(w.lext); cudaFree(w.rext);
    cudaFree(w.lstatus); cudaFree(w.rstatus);
    for (int k = 0; k < 4; ++k) cudaFree(w.order[k]);
    cudaFree(w.counters);
    memset(&w, 0, sizeof(w));
}

int alloc_seed_scratch(SeedScratch& w, int64_t n) {
    if (n <= w.cap && w.counters) return G3X_OK;
    free_seed_scratch(w);
    const int64_t cap = std::max<int64_t>(n, 1024);
    bool ok = cudaMalloc(&w.ljobs, cap * sizeof(g3x_job_t)) == cudaSuccess &&
              cudaMalloc(&w.rjobs, cap * sizeof(g3x_job_t)) == cudaSuccess &&
              cudaMalloc(&w.lext, cap * sizeof(g3x_ext_t)) == cudaSuccess &&
              cudaMalloc(&w.rext, cap * sizeof(g3x_ext_t)) == cudaSuccess &&
              cudaMalloc(&w.lstatus, cap * sizeof(int32_t)) == cudaSuccess &&
              cudaMalloc(&w.rstatus, cap * sizeof(int32_t)) == cudaSuccess &&
              cudaMalloc(&w.counters, 16 * sizeof(int32_t)) == cudaSuccess;
    for (int k = 0; k < 4 && ok; ++k) ok = cudaMalloc(&w.order[k], cap * sizeof(int32_t)) == cudaSuccess;
    if (!ok) { free_seed_scratch(w); return G3X_ERR_NOMEM; }
    w.cap = cap;
    return G3X_OK;
}

}  // namespace g3x

extern "C" {

const char* g3x_strerror(int code) {
    switch (code) {
        case G3X_OK: return "ok";
        case G3X_ERR_INVALID: return "invalid argument";
        case G3X_ERR_SCORE: return "unsupported scoring (m must be 5, gap extensions > 0)";
        case G3X_ERR_TOO_LONG: return "job exceeds the length limits";
        case G3X_ERR_CUDA: return "CUDA runtime error";
        case G3X_ERR_TIMEOUT: return "bounded device wait gave up";
        case G3X_ERR_INTERNAL: return "device consistency check failed";
        case G3X_ERR_NOMEM: return "out of device memory for library scratch";
        case G3X_ERR_NOT_TRAINED: return "learned schedule requested before a model was set";
        default: return "unknown error";
    }
}

int g3x_ctx_create(g3x_ctx** out, int device) {
    if (!out) return G3X_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return G3X_ERR_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return G3X_ERR_CUDA;
    g3x_ctx* c = new (std::nothrow) g3x_ctx();
    if (!c) return G3X_ERR_NOMEM;
    memset(&c->seeds, 0, sizeof(c->seeds));
    c->device = device;
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaMalloc(&c->d_queue, 64 * sizeof(int32_t)) != cudaSuccess) {
        delete c;
        return G3X_ERR_NOMEM;
    }
    *out = c;
    return G3X_OK;
}

int g3x_ctx_destroy(g3x_ctx* c) {
    if (!c) return G3X_ERR_INVALID;
    cudaSetDevice(c->device);
    g3x::free_seed_scratch(c->seeds);
    cudaFree(c->d_queue);
    delete c;
    return G3X_OK;
}

int g3x_ksw_extend2_batch(g3x_ctx* ctx, const g3x_score_t* score, const g3x_job_t* d_jobs,
                          int32_t n, const uint32_t* d_codes, const uint32_t* d_nmask,
                          g3x_ext_t* d_out, int32_t* d_status, const g3x_batch_opts_t* opts,
                          void* stream) {
    if (!ctx || !opts || n < 0) return G3X_ERR_INVALID;
    if (n == 0) return G3X_OK;
    if (!d_jobs || !d_codes || !d_nmask || !d_out || !d_status) return G3X_ERR_INVALID;
    g3x::ScoreParams sp;
    int rc = g3x::score_params(score, &sp);
    if (rc) return rc;
    g3x::LaunchDesc d;
    if ((rc = g3x::batch_proto(opts, ctx->d_queue, &d))) return rc;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return G3X_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    d.jobs = d_jobs; d.codes = d_codes; d.nmask = d_nmask; d.out = d_out; d.status = d_status;
    d.n = n;
    if (d.persistent && cudaMemsetAsync(ctx->d_queue, 0, sizeof(int32_t), st) != cudaSuccess)
        return G3X_ERR_CUDA;
    return g3x::launch_extend(d, sp, st);
}

int g3x_extend_seeds(g3x_ctx* ctx, const g3x_opt_t* opt, const g3x_seed_t* d_seeds, int32_t n,
                     const uint32_t* d_codes, const uint32_t* d_nmask, g3x_reg_t* d_regs,
                     int32_t* d_status, const g3x_batch_opts_t* opts, void* stream) {
    if (!ctx || !opt || !opts || n < 0) return G3X_ERR_INVALID;
    if (n == 0) return G3X_OK;
    if (!d_seeds || !d_codes || !d_nmask || !d_regs || !d_status) return G3X_ERR_INVALID;
    g3x::ScoreParams sp;
    int rc = g3x::score_params(&opt->score, &sp);
    if (rc) return rc;
    g3x::LaunchDesc proto;
    if ((rc = g3x::batch_proto(opts, nullptr, &proto))) return rc;
    proto.cells = nullptr;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return G3X_ERR_CUDA;
    if ((rc = g3x::alloc_seed_scratch(ctx->seeds, n))) return rc;
    return g3x::extend_seeds(ctx->seeds, *opt, sp, d_seeds, n, d_codes, d_nmask, d_regs, d_status,
                             proto, (cudaStream_t)stream);
}

int g3x_extend_seeds_stream(g3x_ctx* ctx, const g3x_opt_t* opt, const g3x_seed_t* h_seeds,
                            int64_t n, const uint32_t* h_codes, const uint32_t* h_nmask,
                            int64_t n_bases, g3x_reg_t* h_regs, int32_t* h_status,
                            int32_t chunk, const g3x_batch_opts_t* opts) {
    if (!ctx || !opt || !opts || n < 0 || n_bases < 0) return G3X_ERR_INVALID;
    if (n == 0) return G3X_OK;
    if (!h_seeds || !h_codes || !h_nmask || !h_regs || !h_status) return G3X_ERR_INVALID;
    if (n_bases > 0xFFFFFFFFll) return G3X_ERR_INVALID;
    g3x::ScoreParams sp;
    int rc = g3x::score_params(&opt->score, &sp);
    if (rc) return rc;
    g3x::LaunchDesc proto;
    if ((rc = g3x::batch_proto(opts, nullptr, &proto))) return rc;
    proto.cells = nullptr;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return G3X_ERR_CUDA;
    return g3x::extend_seeds_stream(ctx->seeds, g3x::alloc_seed_scratch, *opt, sp, h_seeds, n,
                                    h_codes, h_nmask, n_bases, h_regs, h_status, chunk, proto);
}

int g3x_int_peak(g3x_ctx* ctx, double* ops_per_s) {
    if (!ctx || !ops_per_s) return G3X_ERR_INVALID;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return G3X_ERR_CUDA;
    return g3x::measure_int_peak(ctx->device, ops_per_s);
}

int g3x_pack_codes(const uint8_t* h_seq, int64_t len, uint32_t* h_codes, uint32_t* h_nmask,
                   int64_t base) {
    if (len < 0 || base < 0 || (len && (!h_seq || !h_codes || !h_nmask))) return G3X_ERR_INVALID;
    for (int64_t k = 0; k < len; ++k) {
        int64_t b = base + k;
        uint32_t c = h_seq[k];
        uint32_t sh = (uint32_t)(b & 15) << 1;
        h_codes[b >> 4] = (h_codes[b >> 4] & ~(3u << sh)) | ((c & 3u) << sh);
        uint32_t nb = 1u << (b & 31);
        if (c > 3) h_nmask[b >> 5] |= nb; else h_nmask[b >> 5] &= ~nb;
    }
    return G3X_OK;
}

}  // extern "C"

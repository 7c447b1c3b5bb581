// g3x_api.cu -- host side of the C ABI declared in include/g3x.h.
#include <cuda_runtime.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <cmath>
#include <new>
#include "g3x_internal.h"

struct g3x_ctx {
    int device;
    int sms;
    int32_t* d_queue;            // persistent-kernel job counters
    g3x::SeedScratch seeds;      // seed-level scratch, grown on demand
    g3x::StreamScratch stream;   // chunked seed stream: buffer sets, staging, streams
    g3x::ModelState model;       // learned cost model
    g3x::SchedScratch sched;     // job order and width classes of a persistent batch
    g3x::ChainScratch chain;     // chain-level call state
    g3x::GlobalScratch global;   // global-alignment backtrack bytes
    g3x::SwScratch sw;           // striped local alignment: job order, XSUBO row maxima
    g3x::TileTable tiles;        // width classes and their kernel configurations
    unsigned long long* d_stats; // occupancy counters of the last persistent batch
    cudaStream_t side[g3x::kMaxBuckets];   // one stream per width class
    cudaEvent_t fork, join[g3x::kMaxBuckets];
    int timing;                             // bracket class launches with timing events
    cudaEvent_t cls0[g3x::kMaxBuckets], cls1[g3x::kMaxBuckets];
    int cls_timed[g3x::kMaxBuckets];        // 1 when the last batch recorded class k
    int64_t step_limit;                     // g3x_set_step_limit (0: the kernels' own bound)
    int no_int16;                           // g3x_set_int16(ctx, 0): width classes in int32 only
};

namespace g3x {

int ctx_device(const g3x_ctx* ctx) { return ctx->device; }
ChainScratch& ctx_chain(g3x_ctx* ctx) { return ctx->chain; }
GlobalScratch& ctx_global(g3x_ctx* ctx) { return ctx->global; }
SwScratch& ctx_sw(g3x_ctx* ctx) { return ctx->sw; }


// The jobs in decreasing order of row count, then of widest row (the counting sort of the
// scheduled batches with one class), so that the jobs a warp takes together are alike.
int cost_order(g3x_ctx* ctx, const g3x_job_t* jobs, int n, const ScoreParams& sp, cudaStream_t st,
               const int32_t** order) {
    int rc = alloc_sched(ctx->sched, n);
    if (rc) return rc;
    TileTable t;
    t.n = 1; t.width[0] = 0x7FFFFFFF; t.lanes[0] = 32; t.tile[0] = 9; t.warp_batch[0] = 0; t.refill[0] = 1;
    if ((rc = schedule_jobs(ctx->sched, jobs, n, sp, nullptr, t, st))) return rc;
    *order = ctx->sched.order;
    return G3X_OK;
}

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
    sp->oe_del = s->o_del + s->e_del; sp->oe_ins = s->o_ins + s->e_ins;
    sp->k16 = 1u << 16; sp->k8 = 1u << 8;
    return G3X_OK;
}

// Kernel choice for one batch: schedule, lanes per job and smem bounds.
int batch_proto(const g3x_batch_opts_t* opts, int32_t* queue, LaunchDesc* d) {
    if (!opts) return G3X_ERR_INVALID;
    if (opts->max_qlen < 0 || opts->max_tlen < 0 || opts->max_qlen > 65534 || opts->max_tlen > 65535)
        return G3X_ERR_INVALID;
    if (opts->n_bases < 1 || opts->n_bases > 0x100000000ll) return G3X_ERR_INVALID;
    memset(d, 0, sizeof(*d));
    d->n_bases = opts->n_bases;
    d->qmax = opts->max_qlen;
    d->tmax = opts->max_tlen;
    d->cells = opts->d_cells;
    d->rows = opts->d_rows;
    if (opts->schedule != G3X_SCHED_PLAIN && opts->schedule != G3X_SCHED_SORTED &&
        opts->schedule != G3X_SCHED_LEARNED)
        return G3X_ERR_INVALID;
    if (opts->kernel < G3X_KERNEL_AUTO || opts->kernel > G3X_KERNEL_BAND) return G3X_ERR_INVALID;
    const bool plain = opts->schedule == G3X_SCHED_PLAIN;
    d->kernel = opts->kernel == G3X_KERNEL_AUTO ? (plain ? kKernelRolling : kKernelRowpar)
                : opts->kernel == G3X_KERNEL_ROLLING ? kKernelRolling
                : opts->kernel == G3X_KERNEL_ROWPAR ? kKernelRowpar
                : opts->kernel == G3X_KERNEL_LANE ? kKernelLane
                : opts->kernel == G3X_KERNEL_LANE16 ? kKernelLane16
                : opts->kernel == G3X_KERNEL_LANE2 ? kKernelLane2 : kKernelBand;
    if (d->kernel == kKernelBand) {
        // one job per warp; tile carries the window (256, 512 or 1024 columns, 0 = 1024)
        const int win = opts->tile ? opts->tile : 1024;
        if (win != 256 && win != 512 && win != 1024) return G3X_ERR_INVALID;
        d->lanes = 32; d->tile = win; d->persistent = plain ? 0 : 1; d->warps_per_block = 4;
        d->queue = plain ? nullptr : queue;
        return G3X_OK;
    }
    if (d->kernel == kKernelLane || d->kernel == kKernelLane16 || d->kernel == kKernelLane2) {
        if (plain) return G3X_ERR_INVALID;            // the lane kernels are persistent only
        d->lanes = 1; d->tile = d->kernel == kKernelLane16 ? 2 : d->kernel == kKernelLane2 ? 4 : 0;
        d->persistent = 1; d->warps_per_block = 4; d->queue = queue;
        d->refill = opts->tile > 0 ? opts->tile : 1;  // tile carries the refill threshold
        return G3X_OK;
    }
    if (plain) {
        // one 32-lane block per job, jobs in the given order
        d->lanes = 32; d->tile = opts->tile ? opts->tile : 9; d->persistent = 0; d->warps_per_block = 1;
    } else {
        int lanes = opts->lanes, tile = opts->tile ? opts->tile : 9;
        if (!lanes) {
            // row-parallel: the narrowest group whose tile covers the widest query;
            // rolling: 8-lane groups
            lanes = 8;
            if (d->kernel == kKernelRowpar) {
                lanes = 4;
                while (lanes < 32 && lanes * tile < d->qmax) lanes *= 2;
            }
        }
        if (lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32) return G3X_ERR_INVALID;
        if (lanes == 4 && d->kernel != kKernelRowpar) return G3X_ERR_INVALID;
        // Shared memory per job grows with the query; a warp of narrow groups must fit,
        // so the lane count is raised until it does.
        while (lanes < 32 && (32 / lanes) * group_smem_bytes(d->qmax, d->tmax) > 227 * 1024)
            lanes *= 2;
        d->lanes = lanes; d->tile = tile; d->persistent = 1; d->warps_per_block = 4;
        d->queue = queue;
    }
    if (d->tile != 5 && d->tile != 9 && d->tile != 13) return G3X_ERR_INVALID;
    return G3X_OK;
}

void free_seed_scratch(SeedScratch& w) {
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

void free_sched(SchedScratch& s) {
    cudaFree(s.bin); cudaFree(s.order); cudaFree(s.hist); cudaFree(s.cursor); cudaFree(s.bucket_oc);
    cudaFree(s.feat); cudaFree(s.pred);
    s = SchedScratch();
}

int alloc_sched(SchedScratch& s, int64_t n) {
    if (n <= s.cap && s.order) return G3X_OK;
    free_sched(s);
    const int64_t cap = std::max<int64_t>(n, 1024);
    const int bins = kMaxBuckets * kSchedLevels;
    if (cudaMalloc(&s.bin, cap * sizeof(int32_t)) || cudaMalloc(&s.order, cap * sizeof(int32_t)) ||
        cudaMalloc(&s.hist, bins * sizeof(int32_t)) || cudaMalloc(&s.cursor, bins * sizeof(int32_t)) ||
        cudaMalloc(&s.bucket_oc, 2 * kMaxBuckets * sizeof(int32_t)) ||
        cudaMalloc(&s.feat, cap * G3X_MLP_FEATURES * sizeof(float)) || cudaMalloc(&s.pred, cap * sizeof(float))) {
        free_sched(s);
        return G3X_ERR_NOMEM;
    }
    s.cap = cap;
    return G3X_OK;
}

// Largest query a class stages: its width, except for the unbounded last class.
int class_qcap(const TileTable& t, int k, int qmax) {
    return k == t.n - 1 ? qmax : std::min(qmax, t.width[k]);
}

// The context's class resources.  The classes chain on the caller's stream as programmatic
// dependent launches; only the per-class timing modes fork them onto the side streams (events
// between chained launches would serialise them).
static ClassRes ctx_res(g3x_ctx* ctx) {
    return ClassRes{&ctx->sched, ctx->d_queue, ctx->timing ? ctx->side : nullptr, ctx->fork, ctx->join,
                    ctx->d_stats};
}

// Runs the persistent kernels over every width class of an ordered batch: one launch per class,
// chained on `st` (or forked onto side streams from `st` and joined back).
static int launch_classes(g3x_ctx* ctx, const LaunchDesc& base, const ScoreParams& sp, cudaStream_t st,
                          int only = -1, const TileTable* tt_override = nullptr, const ClassRes* res_in = nullptr) {
    const TileTable& tt = tt_override ? *tt_override : ctx->tiles;
    const ClassRes res = res_in ? *res_in : ctx_res(ctx);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cap);
    const bool timed = ctx->timing && cap == cudaStreamCaptureStatusNone && !tt_override && !res_in;
    // timing mode 2 runs the classes one after another on `st`, each timed alone.  Resources
    // without side streams chain the classes on `st` as programmatic dependent launches: each
    // class kernel may start as soon as the one before it is running, so they run side by side
    // as on separate streams.
    const bool serial = (timed && ctx->timing == 2) || !res.side;
    const bool chain = serial && !timed;
    bool first = true;
    if (!serial && cudaEventRecord(res.fork, st) != cudaSuccess) return G3X_ERR_CUDA;
    if (timed)
        for (int k = 0; k < kMaxBuckets; ++k) ctx->cls_timed[k] = 0;
    int rc = G3X_OK;
    // Widest class first: its long rows make the longest-running blocks, and the narrow
    // classes' short jobs then fill the SMs its tail leaves idle.
    for (int kk = tt.n - 1; kk >= 0 && rc == G3X_OK; --kk) {
        const int k = kk;
        if (only >= 0 && k != only) continue;
        cudaStream_t cs = serial ? st : res.side[k];
        if (!serial && cudaStreamWaitEvent(cs, res.fork, 0) != cudaSuccess) { rc = G3X_ERR_CUDA; break; }
        LaunchDesc d = base;
        d.kernel = tt.lanes[k] != 1 ? (tt.tile[k] >= 64 ? kKernelBand : kKernelRowpar)
                 : tt.tile[k] == 2 ? kKernelLane16 : tt.tile[k] == 4 ? kKernelLane2 : kKernelLane;
        d.ring = tt.lanes[k] == 1 && tt.tile[k] >= 64 ? tt.tile[k] : 0;
        d.lanes = tt.lanes[k];
        d.tile = tt.tile[k];
        d.warp_batch = tt.warp_batch[k];
        d.refill = tt.refill[k];
        d.persistent = 1;
        d.warps_per_block = 4;
        d.qmax = class_qcap(tt, k, base.qmax);
        d.order = res.sched->order;
        d.order_off = res.sched->bucket_oc + 2 * k;
        d.count = res.sched->bucket_oc + 2 * k + 1;
        d.queue = res.queue + k;
        d.stats = res.stats;
        d.pdl = chain && !first;
        first = false;
        if (timed && cudaEventRecord(ctx->cls0[k], cs) != cudaSuccess) { rc = G3X_ERR_CUDA; break; }
        if (d.kernel == kKernelLane) {
            rc = launch_lane(d, sp, cs);
        } else if (d.kernel == kKernelLane16) {
            rc = launch_lane16(d, sp, cs);
        } else if (d.kernel == kKernelLane2) {
            rc = launch_lane2(d, sp, cs);
        } else if (d.kernel == kKernelBand) {
            rc = launch_band(d, sp, cs);
        } else {
            while (d.lanes < 32 && (32 / d.lanes) * group_smem_bytes(d.qmax, d.tmax) > 227 * 1024) d.lanes *= 2;
            rc = launch_rowpar(d, sp, cs);
        }
        if (rc == G3X_OK && timed) {
            if (cudaEventRecord(ctx->cls1[k], cs) != cudaSuccess) rc = G3X_ERR_CUDA;
            else ctx->cls_timed[k] = 1;
        }
        if (serial) continue;
        if (rc == G3X_OK && cudaEventRecord(res.join[k], cs) != cudaSuccess) rc = G3X_ERR_CUDA;
        if (rc == G3X_OK && cudaStreamWaitEvent(st, res.join[k], 0) != cudaSuccess) rc = G3X_ERR_CUDA;
    }
    return rc;
}

// Schedules and runs a persistent batch: cost per job (length, or the model's prediction),
// counting sort into width classes, one launch per class.
static int run_scheduled(g3x_ctx* ctx, const LaunchDesc& base, const ScoreParams& sp, bool learned,
                         cudaStream_t st) {
    int rc = alloc_sched(ctx->sched, base.n);
    if (rc) return rc;
    if (learned && (!ctx->model.params || !ctx->model.trained)) return G3X_ERR_NOT_TRAINED;
    rc = learned && ctx->model.active
             ? schedule_jobs_learned(ctx->sched, base.jobs, base.n, base.codes, base.nmask, base.n_bases,
                                     ctx->model.params, sp, ctx->tiles, st)
             : schedule_jobs(ctx->sched, base.jobs, base.n, sp, nullptr, ctx->tiles, st);
    if (rc) return rc;
    if (cudaMemsetAsync(ctx->d_queue, 0, kMaxBuckets * sizeof(int32_t), st) != cudaSuccess ||
        cudaMemsetAsync(ctx->d_stats, 0, 4 * sizeof(unsigned long long), st) != cudaSuccess)
        return G3X_ERR_CUDA;
    return launch_classes(ctx, base, sp, st);
}

int run_class_wave(void* user, const LaunchDesc& d, const ScoreParams& sp, cudaStream_t st) {
    const ClassWave* w = static_cast<const ClassWave*>(user);
    g3x_ctx* ctx = w->ctx;
    const ClassRes res = w->res ? *w->res : ctx_res(ctx);
    SchedScratch& sched = *res.sched;
    int rc = w->learned && ctx->model.active
                 ? schedule_jobs_learned(sched, d.jobs, d.n, d.codes, d.nmask, d.n_bases, ctx->model.params, sp,
                                         ctx->tiles, st, d.order, d.count)
                 : schedule_jobs(sched, d.jobs, d.n, sp, nullptr, ctx->tiles, st, d.order, d.count);
    if (rc) return rc;
    if (cudaMemsetAsync(res.queue, 0, kMaxBuckets * sizeof(int32_t), st) != cudaSuccess) return G3X_ERR_CUDA;
    LaunchDesc base = d;
    base.order = nullptr; base.count = nullptr; base.order_off = nullptr; base.queue = nullptr;
    return launch_classes(ctx, base, sp, st, -1, nullptr, w->res);
}

// Whether a seed-level call goes through the width classes, and how to run its waves.
static int seed_waves(g3x_ctx* ctx, const g3x_batch_opts_t* opts, const LaunchDesc& proto, int64_t n,
                      ClassWave* cw, WaveRunner* wr, const WaveRunner** out) {
    *out = nullptr;
    if (!(proto.persistent && proto.kernel == kKernelRowpar && opts->kernel == G3X_KERNEL_AUTO &&
          opts->lanes == 0 && opts->tile == 0))
        return opts->schedule == G3X_SCHED_LEARNED ? G3X_ERR_INVALID : G3X_OK;
    const bool learned = opts->schedule == G3X_SCHED_LEARNED;
    if (learned && (!ctx->model.params || !ctx->model.trained)) return G3X_ERR_NOT_TRAINED;
    int rc = alloc_sched(ctx->sched, n);
    if (rc) return rc;
    cw->ctx = ctx;
    cw->learned = learned;
    cw->res = nullptr;
    wr->run = run_class_wave;
    wr->user = cw;
    *out = wr;
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
        case G3X_ERR_SCRATCH: return "batch exceeds the static scratch of g3x_ksw_extend2_batch_noalloc (at most G3X_NOALLOC_MAX_JOBS = 1048576 jobs)";
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
    g3x::context_tiles(c->tiles);
    bool ok = cudaMalloc(&c->d_queue, 64 * sizeof(int32_t)) == cudaSuccess &&
              cudaMalloc(&c->d_stats, 4 * sizeof(unsigned long long)) == cudaSuccess &&
              cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming) == cudaSuccess;
    for (int k = 0; k < g3x::kMaxBuckets && ok; ++k)
        ok = cudaStreamCreateWithFlags(&c->side[k], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&c->join[k], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreate(&c->cls0[k]) == cudaSuccess && cudaEventCreate(&c->cls1[k]) == cudaSuccess;
    if (!ok) {
        delete c;
        return G3X_ERR_NOMEM;
    }
    cudaMemset(c->d_stats, 0, 4 * sizeof(unsigned long long));
    *out = c;
    return G3X_OK;
}

int g3x_ctx_destroy(g3x_ctx* c) {
    if (!c) return G3X_ERR_INVALID;
    cudaSetDevice(c->device);
    cudaDeviceSynchronize();
    g3x::free_seed_scratch(c->seeds);
    g3x::free_stream_scratch(c->stream);
    g3x::model_free(c->model);
    g3x::free_sched(c->sched);
    g3x::free_chain_scratch(c->chain);
    cudaFree(c->global.z);
    cudaFree(c->global.queue);
    cudaFree(c->sw.buf);
    cudaFree(c->sw.sub);
    cudaFree(c->sw.flt);
    for (int k = 0; k < g3x::kMaxBuckets; ++k) {
        cudaStreamDestroy(c->side[k]);
        cudaEventDestroy(c->join[k]);
        cudaEventDestroy(c->cls0[k]);
        cudaEventDestroy(c->cls1[k]);
    }
    cudaEventDestroy(c->fork);
    cudaFree(c->d_stats);
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
    d.step_limit = ctx->step_limit;
    // Persistent batches without a fixed kernel shape go through the scheduler.
    if (d.persistent && d.kernel == g3x::kKernelRowpar && opts->kernel == G3X_KERNEL_AUTO &&
        opts->lanes == 0 && opts->tile == 0)
        return g3x::run_scheduled(ctx, d, sp, opts->schedule == G3X_SCHED_LEARNED, st);
    if (opts->schedule == G3X_SCHED_LEARNED) return G3X_ERR_INVALID;   // needs the scheduler
    if (d.persistent) {
        d.stats = ctx->d_stats;
        if (cudaMemsetAsync(ctx->d_queue, 0, sizeof(int32_t), st) != cudaSuccess ||
            cudaMemsetAsync(ctx->d_stats, 0, 4 * sizeof(unsigned long long), st) != cudaSuccess)
            return G3X_ERR_CUDA;
    }
    return g3x::launch_extend(d, sp, st);
}

struct g3x_graph {
    cudaGraph_t graph;
    cudaGraphExec_t exec;
};

int g3x_graph_capture(g3x_ctx* ctx, const g3x_score_t* score, const g3x_job_t* d_jobs, int32_t n,
                      const uint32_t* d_codes, const uint32_t* d_nmask, g3x_ext_t* d_out,
                      int32_t* d_status, const g3x_batch_opts_t* opts, g3x_graph** out) {
    if (!ctx || !out) return G3X_ERR_INVALID;
    *out = nullptr;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return G3X_ERR_CUDA;
    // Scratch must exist before capture (allocation is not a graph operation).
    if (opts && opts->schedule != G3X_SCHED_PLAIN) {
        int rc = g3x::alloc_sched(ctx->sched, n);
        if (rc) return rc;
    }
    cudaStream_t cs;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return G3X_ERR_CUDA;
    g3x_graph* g = new (std::nothrow) g3x_graph();
    if (!g) { cudaStreamDestroy(cs); return G3X_ERR_NOMEM; }
    int rc = G3X_OK;
    if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) rc = G3X_ERR_CUDA;
    if (rc == G3X_OK) {
        rc = g3x_ksw_extend2_batch(ctx, score, d_jobs, n, d_codes, d_nmask, d_out, d_status, opts, cs);
        cudaGraph_t graph = nullptr;
        const cudaError_t e = cudaStreamEndCapture(cs, &graph);
        if (rc == G3X_OK && e != cudaSuccess) rc = G3X_ERR_CUDA;
        g->graph = graph;
        if (rc == G3X_OK && cudaGraphInstantiate(&g->exec, graph, 0) != cudaSuccess) rc = G3X_ERR_CUDA;
    }
    cudaStreamDestroy(cs);
    if (rc != G3X_OK) {
        if (g->graph) cudaGraphDestroy(g->graph);
        delete g;
        cudaGetLastError();
        return rc;
    }
    *out = g;
    return G3X_OK;
}

int g3x_graph_launch(g3x_graph* g, void* stream) {
    if (!g) return G3X_ERR_INVALID;
    return cudaGraphLaunch(g->exec, (cudaStream_t)stream) == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

int g3x_graph_destroy(g3x_graph* g) {
    if (!g) return G3X_ERR_INVALID;
    cudaGraphExecDestroy(g->exec);
    cudaGraphDestroy(g->graph);
    delete g;
    return G3X_OK;
}

int g3x_get_tiles(g3x_ctx* ctx, g3x_tile_t* h, int32_t* n) {
    if (!ctx || !h || !n) return G3X_ERR_INVALID;
    for (int k = 0; k < ctx->tiles.n; ++k)
        h[k] = g3x_tile_t{ctx->tiles.width[k], ctx->tiles.lanes[k], ctx->tiles.tile[k],
                          ctx->tiles.warp_batch[k], ctx->tiles.refill[k]};
    *n = ctx->tiles.n;
    return G3X_OK;
}

int g3x_set_tiles(g3x_ctx* ctx, const g3x_tile_t* h, int32_t n) {
    if (!ctx || !h || n < 1 || n > G3X_MAX_CLASSES) return G3X_ERR_INVALID;
    for (int k = 0; k < n; ++k) {
        const g3x_tile_t& t = h[k];
        const bool lane = t.lanes == 1;
        // the band kernel (32 lanes, a window of 256, 512 or 1024 columns) holds only bands that
        // fit its window, so it cannot be the last class, which takes every job
        const bool band = t.lanes == 32 && (t.tile == 256 || t.tile == 512 || t.tile == 1024) && k < n - 1;
        if ((!lane && t.lanes != 4 && t.lanes != 8 && t.lanes != 16 && t.lanes != 32) ||
            (!lane && !band && t.tile != 5 && t.tile != 9 && t.tile != 13) ||
            (lane && t.tile != 0 && t.tile != 2 && t.tile != 4 && (t.tile < 64 || t.tile % 16)) ||
            (lane && t.tile == 2 && ctx->no_int16) ||
            t.width < 1 ||
            (k && t.width <= h[k - 1].width) || (t.warp_batch != 0 && t.warp_batch != 1) ||
            (lane && (t.refill < 1 || t.refill > 32)))
            return G3X_ERR_INVALID;
    }
    ctx->tiles.n = n;
    for (int k = 0; k < n; ++k) {
        ctx->tiles.width[k] = k == n - 1 ? 0x7FFFFFFF : h[k].width;
        ctx->tiles.lanes[k] = h[k].lanes;
        ctx->tiles.tile[k] = h[k].tile;
        ctx->tiles.warp_batch[k] = h[k].warp_batch;
        ctx->tiles.refill[k] = h[k].refill < 1 ? 1 : h[k].refill;
    }
    return G3X_OK;
}

int g3x_set_int16(g3x_ctx* ctx, int32_t enable) {
    if (!ctx || (enable != 0 && enable != 1)) return G3X_ERR_INVALID;
    ctx->no_int16 = !enable;
    if (!enable)
        for (int k = 0; k < ctx->tiles.n; ++k)
            if (ctx->tiles.lanes[k] == 1 && ctx->tiles.tile[k] == 2) ctx->tiles.tile[k] = 0;
    return G3X_OK;
}

int g3x_set_step_limit(g3x_ctx* ctx, int64_t limit) {
    if (!ctx || limit < 0) return G3X_ERR_INVALID;
    ctx->step_limit = limit;
    return G3X_OK;
}

int g3x_set_timing(g3x_ctx* ctx, int32_t on) {
    if (!ctx || on < 0 || on > 2) return G3X_ERR_INVALID;
    ctx->timing = on;
    return G3X_OK;
}

int g3x_class_times(g3x_ctx* ctx, float* h_ms, int32_t* h_jobs, int32_t* n) {
    if (!ctx || !h_ms || !h_jobs || !n) return G3X_ERR_INVALID;
    if (cudaSetDevice(ctx->device) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return G3X_ERR_CUDA;
    int32_t oc[2 * g3x::kMaxBuckets] = {0};
    if (ctx->sched.bucket_oc &&
        cudaMemcpy(oc, ctx->sched.bucket_oc, sizeof(oc), cudaMemcpyDeviceToHost) != cudaSuccess)
        return G3X_ERR_CUDA;
    for (int k = 0; k < ctx->tiles.n; ++k) {
        h_ms[k] = -1.0f;
        if (ctx->cls_timed[k] && cudaEventElapsedTime(&h_ms[k], ctx->cls0[k], ctx->cls1[k]) != cudaSuccess)
            return G3X_ERR_CUDA;
        h_jobs[k] = oc[2 * k + 1];
    }
    *n = ctx->tiles.n;
    return G3X_OK;
}

int g3x_last_stats(g3x_ctx* ctx, uint64_t* h) {
    if (!ctx || !h) return G3X_ERR_INVALID;
    if (cudaSetDevice(ctx->device) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return G3X_ERR_CUDA;
    unsigned long long v[4];
    if (cudaMemcpy(v, ctx->d_stats, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) return G3X_ERR_CUDA;
    for (int k = 0; k < 3; ++k) h[k] = v[k];
    return G3X_OK;
}

int g3x_autotune_schedule(g3x_ctx* ctx, int32_t schedule, const g3x_score_t* score, const g3x_job_t* d_jobs,
                          int32_t n, const uint32_t* d_codes, const uint32_t* d_nmask, int64_t n_bases,
                          int32_t max_qlen, int32_t max_tlen, g3x_tile_t* h_tiles, int32_t* n_tiles) {
    if (!ctx || !d_jobs || !d_codes || !d_nmask || n <= 0) return G3X_ERR_INVALID;
    if (n_bases < 1 || n_bases > 0x100000000ll) return G3X_ERR_INVALID;
    if (schedule != G3X_SCHED_SORTED && schedule != G3X_SCHED_LEARNED) return G3X_ERR_INVALID;
    if (schedule == G3X_SCHED_LEARNED && (!ctx->model.params || !ctx->model.trained)) return G3X_ERR_NOT_TRAINED;
    g3x::ScoreParams sp;
    int rc = g3x::score_params(score, &sp);
    if (rc) return rc;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return G3X_ERR_CUDA;
    if ((rc = g3x::alloc_sched(ctx->sched, n))) return rc;
    g3x_ext_t* out = nullptr;
    int32_t* status = nullptr;
    if (cudaMalloc(&out, (size_t)n * sizeof(g3x_ext_t)) || cudaMalloc(&status, (size_t)n * sizeof(int32_t))) {
        cudaFree(out);
        return G3X_ERR_NOMEM;
    }
    g3x::LaunchDesc base;
    memset(&base, 0, sizeof(base));
    base.jobs = d_jobs; base.codes = d_codes; base.nmask = d_nmask; base.out = out; base.status = status;
    base.n = n; base.qmax = max_qlen; base.tmax = max_tlen; base.n_bases = n_bases;
    cudaStream_t st = nullptr;
    // Class widths follow the batch: up to seven classes at max_qlen times the fractions below,
    // rounded up to eight columns, then the unbounded class.  A class's shared memory per job is
    // sized by its width: the steps grow at the low end, where rows are short and few cells lie,
    // and stay dense at the top, where shared memory bounds the resident warps (for max_qlen 231:
    // 32, 56, 88, 128, 168, 200, 232, the fastest of the layouts measured on the benchmark batch).
    {
        static const double kFrac[7] = {0.138, 0.241, 0.379, 0.552, 0.724, 0.862, 1.0};
        g3x::TileTable t;
        t.n = 0;
        for (int k = 1; k <= 7; ++k) {
            int wk = (int)(max_qlen * kFrac[k - 1] + 0.999);
            wk = std::max(8, (wk + 7) & ~7);
            if (t.n && wk <= t.width[t.n - 1]) continue;
            t.width[t.n] = wk;
            t.lanes[t.n] = 4;
            while (t.lanes[t.n] < 32 && t.lanes[t.n] * 9 < wk) t.lanes[t.n] *= 2;
            t.tile[t.n] = 9; t.warp_batch[t.n] = 0; t.refill[t.n] = 1;
            ++t.n;
        }
        t.width[t.n] = 0x7FFFFFFF; t.lanes[t.n] = 32; t.tile[t.n] = 9; t.warp_batch[t.n] = 0; t.refill[t.n] = 1;
        ++t.n;
        ctx->tiles = t;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    if (rc == G3X_OK)
        rc = schedule == G3X_SCHED_LEARNED && ctx->model.active
                 ? g3x::schedule_jobs_learned(ctx->sched, d_jobs, n, d_codes, d_nmask, n_bases, ctx->model.params, sp,
                                              ctx->tiles, st)
                 : g3x::schedule_jobs(ctx->sched, d_jobs, n, sp, nullptr, ctx->tiles, st);
    // ring of the lane kernel's ring form: every band of the batch, 2w + 16 columns, rounded up
    int32_t wmax = 0, ring = 0;
    if (rc == G3X_OK) rc = g3x::batch_max_w(d_jobs, n, sp, ctx->d_queue + 32, &wmax, st);
    if (rc == G3X_OK && wmax > 0) ring = (2 * wmax + 16 + 15) & ~15;
    int32_t oc[2 * g3x::kMaxBuckets];
    if (rc == G3X_OK && cudaMemcpy(oc, ctx->sched.bucket_oc, sizeof(oc), cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = G3X_ERR_CUDA;
    // Candidates per class: the lane-per-job kernel with refill waves of 1, 8 or 32 lanes
    // (where a warp's working set fits), and row-parallel groups whose tile covers the class
    // width (the unbounded class: 32-lane groups), each refilling per group or per warp.
    struct Cand { int lanes, tile, wb, refill; };
    Cand cands[64];
    g3x::TileTable best = ctx->tiles, best_nb = ctx->tiles;   // best_nb: the best without band classes
    for (int k = 0; k < ctx->tiles.n && rc == G3X_OK; ++k) {
        if (oc[2 * k + 1] == 0) continue;
        const int width = std::min(ctx->tiles.width[k], max_qlen);
        const bool last = k == ctx->tiles.n - 1;
        int nc = 0;
        if (!last && g3x::lane_smem_per_warp(g3x::class_qcap(ctx->tiles, k, max_qlen), max_tlen) <= 200 * 1024)
            for (int rf : {1, 8, 32}) cands[nc++] = Cand{1, 0, 0, rf};
        if (!last && !ctx->no_int16 &&
            g3x::lane16_smem_per_warp(g3x::class_qcap(ctx->tiles, k, max_qlen)) <= 200 * 1024)
            for (int rf : {1, 8, 32}) cands[nc++] = Cand{1, 2, 0, rf};
        if (!last && g3x::lane2_smem_per_warp(g3x::class_qcap(ctx->tiles, k, max_qlen)) <= 200 * 1024)
            for (int rf : {1, 8, 32}) cands[nc++] = Cand{1, 4, 0, rf};
        // the ring form of the lane kernel, where the band is narrower than the class's queries
        if (!last && ring > 0 && ring < g3x::class_qcap(ctx->tiles, k, max_qlen) + 19 &&
            g3x::lane_ring_smem_per_warp(ring) <= 200 * 1024)
            for (int rf : {1, 8, 32}) cands[nc++] = Cand{1, ring, 0, rf};
        // the band kernel (one warp per job), with the narrowest window that holds every band
        if (!last && wmax > 0 && 2 * wmax + 2 <= 1024) {
            const int win = 2 * wmax + 2 <= 256 ? 256 : 2 * wmax + 2 <= 512 ? 512 : 1024;
            cands[nc++] = Cand{32, win, 0, 1};
        }
        for (int l : {4, 8, 16, 32})
            for (int c : {5, 9, 13}) {
                const int S = l * c;
                if (last ? l != 32 : (S < width || S > 2 * width + 40)) continue;
                for (int wb = 0; wb < 2; ++wb) cands[nc++] = Cand{l, c, wb, 1};
            }
        float best_ms = 1e30f, best_nb_ms = 1e30f;
        for (int ci = 0; ci < nc && rc == G3X_OK; ++ci) {
            g3x::TileTable tt = ctx->tiles;
            tt.lanes[k] = cands[ci].lanes; tt.tile[k] = cands[ci].tile;
            tt.warp_batch[k] = cands[ci].wb; tt.refill[k] = cands[ci].refill;
            float ms = 0;
            for (int rep = 0; rep < 2 && rc == G3X_OK; ++rep) {
                cudaMemsetAsync(ctx->d_queue, 0, g3x::kMaxBuckets * sizeof(int32_t), st);
                cudaEventRecord(e0, st);
                rc = g3x::launch_classes(ctx, base, sp, st, k, &tt);
                cudaEventRecord(e1, st);
                if (cudaEventSynchronize(e1) != cudaSuccess) rc = G3X_ERR_CUDA;
                cudaEventElapsedTime(&ms, e0, e1);
            }
            if (rc == G3X_OK && ms < best_ms) {
                best_ms = ms;
                best.lanes[k] = tt.lanes[k]; best.tile[k] = tt.tile[k];
                best.warp_batch[k] = tt.warp_batch[k]; best.refill[k] = tt.refill[k];
            }
            const bool band = tt.lanes[k] == 32 && tt.tile[k] >= 64;
            if (rc == G3X_OK && !band && ms < best_nb_ms) {
                best_nb_ms = ms;
                best_nb.lanes[k] = tt.lanes[k]; best_nb.tile[k] = tt.tile[k];
                best_nb.warp_batch[k] = tt.warp_batch[k]; best_nb.refill[k] = tt.refill[k];
            }
        }
    }
    // Each class was timed alone; side by side, the band kernel's register-heavy warps and the
    // lane kernels' shared-memory-heavy warps compete for the same SMs.  So a table with band
    // classes is kept only if the whole batch runs faster with it than with those classes on
    // their best other kernel.
    bool has_band = false;
    for (int k = 0; k < best.n; ++k) has_band |= best.lanes[k] == 32 && best.tile[k] >= 64;
    if (rc == G3X_OK && has_band) {
        auto whole = [&](const g3x::TileTable& tt, float* out_ms) -> int {
            int r = G3X_OK;
            for (int rep = 0; rep < 2 && r == G3X_OK; ++rep) {
                cudaMemsetAsync(ctx->d_queue, 0, g3x::kMaxBuckets * sizeof(int32_t), st);
                cudaEventRecord(e0, st);
                r = g3x::launch_classes(ctx, base, sp, st, -1, &tt);
                cudaEventRecord(e1, st);
                if (cudaEventSynchronize(e1) != cudaSuccess) r = G3X_ERR_CUDA;
                cudaEventElapsedTime(out_ms, e0, e1);
            }
            return r;
        };
        float ms_band = 0, ms_alt = 0;
        rc = whole(best, &ms_band);
        if (rc == G3X_OK) rc = whole(best_nb, &ms_alt);
        if (rc == G3X_OK && ms_alt < ms_band) best = best_nb;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    cudaFree(status);
    if (rc == G3X_OK) {
        ctx->tiles = best;
        if (h_tiles && n_tiles) rc = g3x_get_tiles(ctx, h_tiles, n_tiles);
    }
    return rc;
}

int g3x_autotune(g3x_ctx* ctx, const g3x_score_t* score, const g3x_job_t* d_jobs, int32_t n,
                 const uint32_t* d_codes, const uint32_t* d_nmask, int64_t n_bases, int32_t max_qlen,
                 int32_t max_tlen, g3x_tile_t* h_tiles, int32_t* n_tiles) {
    return g3x_autotune_schedule(ctx, G3X_SCHED_SORTED, score, d_jobs, n, d_codes, d_nmask, n_bases, max_qlen,
                                 max_tlen, h_tiles, n_tiles);
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
    g3x::ClassWave cw;
    g3x::WaveRunner wr;
    const g3x::WaveRunner* runner = nullptr;
    if ((rc = g3x::seed_waves(ctx, opts, proto, n, &cw, &wr, &runner))) return rc;
    return g3x::extend_seeds(ctx->seeds, *opt, sp, d_seeds, n, d_codes, d_nmask, d_regs, d_status,
                             proto, (cudaStream_t)stream, runner);
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
    g3x_batch_opts_t so = *opts;          // the planes' length is this call's n_bases
    so.n_bases = n_bases > 0 ? n_bases : 1;
    if ((rc = g3x::batch_proto(&so, nullptr, &proto))) return rc;
    proto.cells = nullptr;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return G3X_ERR_CUDA;
    g3x::ClassWave cw;
    g3x::WaveRunner wr;
    const g3x::WaveRunner* runner = nullptr;
    if ((rc = g3x::seed_waves(ctx, opts, proto, chunk > 0 ? chunk : 65536, &cw, &wr, &runner))) return rc;
    return g3x::extend_seeds_stream(ctx->stream, *opt, sp, h_seeds, n,
                                    h_codes, h_nmask, n_bases, h_regs, h_status, chunk, proto, runner);
}

int g3x_features(g3x_ctx* ctx, const g3x_job_t* d_jobs, int32_t n, const uint32_t* d_codes,
                 const uint32_t* d_nmask, int64_t n_bases, float* d_feat, void* stream) {
    if (!ctx || n < 0 || (n && (!d_jobs || !d_codes || !d_nmask || !d_feat))) return G3X_ERR_INVALID;
    if (n_bases < 0 || n_bases > 0x100000000ll) return G3X_ERR_INVALID;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return G3X_ERR_CUDA;
    return g3x::model_features(d_jobs, n, d_codes, d_nmask, n_bases, d_feat, (cudaStream_t)stream);
}

int g3x_mlp_init(g3x_ctx* ctx, uint64_t seed) {
    if (!ctx) return G3X_ERR_INVALID;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return G3X_ERR_CUDA;
    return g3x::model_init(ctx->model, seed);
}

int g3x_mlp_train(g3x_ctx* ctx, const float* d_feat, const float* d_target, int32_t n,
                  int32_t epochs, int32_t batch, float lr, uint64_t seed, float* h_epoch_loss) {
    if (!ctx || !d_feat || !d_target || n <= 0 || epochs < 0 || batch <= 0 || batch > n) return G3X_ERR_INVALID;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return G3X_ERR_CUDA;
    if (!ctx->model.params) {
        int rc = g3x::model_init(ctx->model, seed);
        if (rc) return rc;
    }
    int rc = g3x::model_train(ctx->model, d_feat, d_target, n, epochs, batch, lr, seed, h_epoch_loss, 0);
    if (rc == G3X_OK && cudaDeviceSynchronize() != cudaSuccess) rc = G3X_ERR_CUDA;
    if (rc == G3X_OK) ctx->model.trained = 1;
    return rc;
}

int g3x_mlp_gradient(g3x_ctx* ctx, const float* d_feat, const float* d_target, int32_t n,
                     float* h_grad, float* h_loss) {
    if (!ctx || !d_feat || !d_target || n <= 0 || !h_grad) return G3X_ERR_INVALID;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return G3X_ERR_CUDA;
    if (!ctx->model.params) return G3X_ERR_NOT_TRAINED;
    return g3x::model_gradient(ctx->model, d_feat, d_target, n, h_grad, h_loss, 0);
}

int g3x_mlp_predict(g3x_ctx* ctx, const float* d_feat, int32_t n, float* d_pred, void* stream) {
    if (!ctx || n < 0 || (n && (!d_feat || !d_pred))) return G3X_ERR_INVALID;
    if (!ctx->model.params) return G3X_ERR_NOT_TRAINED;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return G3X_ERR_CUDA;
    return g3x::model_predict(ctx->model.params, d_feat, n, d_pred, (cudaStream_t)stream);
}

int g3x_mlp_predict_jobs(g3x_ctx* ctx, const g3x_job_t* d_jobs, int32_t n, const uint32_t* d_codes,
                         const uint32_t* d_nmask, int64_t n_bases, float* d_pred, void* stream) {
    if (!ctx || n < 0 || (n && (!d_jobs || !d_codes || !d_nmask || !d_pred))) return G3X_ERR_INVALID;
    if (n_bases < 1 || n_bases > 0x100000000ll) return G3X_ERR_INVALID;
    if (!ctx->model.params) return G3X_ERR_NOT_TRAINED;
    if (n == 0) return G3X_OK;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return G3X_ERR_CUDA;
    int rc = g3x::alloc_sched(ctx->sched, n);
    if (rc) return rc;
    // the sort keys the kernel also forms land in the context's sort scratch and are not used
    // here; they take BWA's default scoring
    g3x::ScoreParams sp;
    g3x_score_t sc;
    memset(&sc, 0, sizeof(sc));
    for (int a = 0; a < 5; ++a)
        for (int b = 0; b < 5; ++b) sc.mat[a * 5 + b] = a == b ? 1 : -4;
    sc.o_del = sc.o_ins = 6; sc.e_del = sc.e_ins = 1; sc.zdrop = 100; sc.end_bonus = 5; sc.m = 5;
    if ((rc = g3x::score_params(&sc, &sp))) return rc;
    return g3x::schedule_jobs_learned(ctx->sched, d_jobs, n, d_codes, d_nmask, n_bases, ctx->model.params, sp,
                                      ctx->tiles, (cudaStream_t)stream, nullptr, nullptr, d_pred);
}

int g3x_mlp_set_active(g3x_ctx* ctx, int32_t active) {
    if (!ctx || (active != 0 && active != 1)) return G3X_ERR_INVALID;
    ctx->model.active = active;
    return G3X_OK;
}

int g3x_mlp_get_params(g3x_ctx* ctx, float* h_params) {
    if (!ctx || !h_params) return G3X_ERR_INVALID;
    if (!ctx->model.params) return G3X_ERR_NOT_TRAINED;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return G3X_ERR_CUDA;
    return cudaMemcpy(h_params, ctx->model.params, G3X_MLP_PARAMS * sizeof(float),
                      cudaMemcpyDeviceToHost) == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

int g3x_mlp_set_params(g3x_ctx* ctx, const float* h_params) {
    if (!ctx || !h_params) return G3X_ERR_INVALID;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return G3X_ERR_CUDA;
    int rc = g3x::model_alloc(ctx->model, 256);
    if (rc) return rc;
    if (cudaMemcpy(ctx->model.params, h_params, G3X_MLP_PARAMS * sizeof(float),
                   cudaMemcpyHostToDevice) != cudaSuccess)
        return G3X_ERR_CUDA;
    cudaMemset(ctx->model.m, 0, G3X_MLP_PARAMS * sizeof(float));
    cudaMemset(ctx->model.v, 0, G3X_MLP_PARAMS * sizeof(float));
    ctx->model.t = 0;
    ctx->model.trained = 1;
    return G3X_OK;
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

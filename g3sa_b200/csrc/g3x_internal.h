// g3x_internal.h -- declarations shared by the library's translation units.
#pragma once
#include <mutex>
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/g3x.h"

namespace g3x {

// Scoring as the kernels consume it (passed by value as a kernel parameter).
struct ScoreParams {
    int8_t mat[25];
    int8_t pad_[3];
    int32_t o_del, e_del, o_ins, e_ins, zdrop, end_bonus, max_sc;
    int32_t oe_del, oe_ins;   // o + e
    // 2^16 and 2^8 as run-time values: multiplying by them keeps 16-bit field packing and
    // unpacking on the FMA pipe (IMAD), which the compiler would turn into ALU shifts and
    // logic operations for literal constants, and the ALU pipe is the one the DP saturates
    uint32_t k16, k8;
};

// One launch of the extension kernel family.
struct LaunchDesc {
    const g3x_job_t* jobs;
    const uint32_t* codes;
    const uint32_t* nmask;
    g3x_ext_t* out;
    int32_t* status;
    int32_t* cells;        // optional
    int32_t* rows;         // optional: rows of the row loop each job ran
    const int32_t* order;  // optional permutation: queue slot -> job index
    const int32_t* count;  // optional device-side job count (overrides n when set)
    int32_t* queue;        // persistent kernels: device counter (zeroed by the caller)
    const int32_t* order_off;  // optional device offset added to `order` (bucket start)
    unsigned long long* stats; // optional: [0] group-rows computed, [1] group-rows idle
                               // (warp-batched pulling), [2] warp batches
    int32_t n;
    int32_t qmax, tmax;    // smem sizing bounds
    int32_t kernel;        // kKernelRolling or kKernelRowpar
    int32_t lanes;         // lanes per job
    int32_t tile;          // row-parallel kernel: cells per lane per tile
    int32_t persistent;    // 0: one group per job slot; 1: groups pull from `queue`
    int32_t warps_per_block;
    int32_t blocks;        // persistent grid size (0 = derive from occupancy)
    int32_t warp_batch;    // persistent row-parallel: 1 = a warp pulls one job per group at
                           // once and waits for all of them; 0 = each group refills alone
    int32_t refill;        // lane-per-job kernel: idle lanes that trigger a refill wave
    int32_t ring;          // lane-per-job kernel: 0, or the columns of its row-buffer ring
    int32_t pdl;           // class kernels: 1 = launched as a programmatic dependent of the
                           // class kernel before it on the stream (launch_class_kernel)
    int64_t n_bases;       // bases the planes hold: jobs reaching past them are refused
    int64_t step_limit;    // plain (rolling) kernel: per-job step bound, 0 = the default bound
};

// A job whose query or target reaches past the planes' n_bases bases is refused before any of
// its bases is read (per-job G3X_ERR_INVALID).
__host__ __device__ __forceinline__ bool job_in_planes(const g3x_job_t& jb, int64_t n_bases) {
    return (int64_t)jb.q_off + jb.qlen <= n_bases && (int64_t)jb.t_off + jb.tlen <= n_bases;
}

// Tile configurations by job width class (ascending width; the last class is unbounded).
constexpr int kMaxBuckets = 8;
struct TileTable {
    int32_t n;
    int32_t width[kMaxBuckets];   // widest row this class holds
    int32_t lanes[kMaxBuckets];
    int32_t tile[kMaxBuckets];
    int32_t warp_batch[kMaxBuckets];
    int32_t refill[kMaxBuckets];
};

// The width classes a new context starts with (and the no-alloc entry point always uses): each
// runs the row-parallel kernel with the narrowest group whose tile (lanes x odd cells per lane)
// covers the class width; the last class tiles wider rows.
inline void default_tiles(TileTable& t) {
    const int w[] = {20, 36, 72, 144, 288, 0x7FFFFFFF};
    const int l[] = {4, 4, 8, 16, 32, 32};
    const int c[] = {5, 9, 9, 9, 9, 9};
    t.n = 6;
    for (int k = 0; k < t.n; ++k) {
        t.width[k] = w[k]; t.lanes[k] = l[k]; t.tile[k] = c[k]; t.warp_batch[k] = 0; t.refill[k] = 1;
    }
}

// The width classes a new context starts with: the int16x2 lane kernel (g3x_lane16.cu) over
// seven classes of query length up to 256, refilling in waves of 8 lanes -- the layout the
// autotuner settles on for reads of 100-250 bp -- then the row-parallel kernel for longer
// queries and for jobs outside the int16 fit.
inline void context_tiles(TileTable& t) {
    const int w[] = {32, 56, 88, 128, 168, 200, 256};
    t.n = 8;
    for (int k = 0; k < 7; ++k) {
        t.width[k] = w[k]; t.lanes[k] = 1; t.tile[k] = 2; t.warp_batch[k] = 0; t.refill[k] = 8;
    }
    t.width[7] = 0x7FFFFFFF; t.lanes[7] = 32; t.tile[7] = 9; t.warp_batch[7] = 0; t.refill[7] = 1;
}

// Sort bins per width class of schedule_jobs (its histogram holds kMaxBuckets * kSchedLevels).
constexpr int kSchedLevels = 2048;

// Device scratch of the scheduler and of the learned schedule (capacity >= n jobs).
struct SchedScratch {
    int32_t *bin = nullptr, *order = nullptr, *hist = nullptr, *cursor = nullptr;
    int32_t* bucket_oc = nullptr;  // [offset, count] per bucket
    float *feat = nullptr, *pred = nullptr;
    int64_t cap = 0;
};
// Sorts jobs 0..n-1, or with `subset` the *subset_n jobs subset[0..] (device arrays, at most
// n), into width classes; s.order receives job indices.
int schedule_jobs(SchedScratch& s, const g3x_job_t* jobs, int n, const ScoreParams& sp,
                  const float* pred, const TileTable& tt, cudaStream_t st,
                  const int32_t* subset = nullptr, const int32_t* subset_n = nullptr);
// The same sort with the learned schedule's keys: the jobs' features, the network (params) and
// the keys in one kernel (g3x_model.cu); pred_out (optional) receives each job's prediction.
int schedule_jobs_learned(SchedScratch& s, const g3x_job_t* jobs, int n, const uint32_t* codes,
                          const uint32_t* nmask, int64_t n_bases, const float* params, const ScoreParams& sp,
                          const TileTable& tt, cudaStream_t st, const int32_t* subset = nullptr,
                          const int32_t* subset_n = nullptr, float* pred_out = nullptr);
int launch_learned_keys(const float* params, const g3x_job_t* jobs, int n, const uint32_t* codes,
                        const uint32_t* nmask, int64_t n_bases, const ScoreParams& sp, const TileTable& tt,
                        int32_t* bin, int32_t* hist, cudaStream_t st, const int32_t* subset,
                        const int32_t* subset_n, float* pred_out);
// Largest band width w (after the clamp of ksw.cu:321-329) over n jobs; blocks.
int batch_max_w(const g3x_job_t* jobs, int n, const ScoreParams& sp, int32_t* d_tmp, int32_t* h_out,
                cudaStream_t st);

constexpr int32_t kKernelRolling = 1;   // anti-diagonal wavefront, rows on lanes
constexpr int32_t kKernelRowpar = 2;    // one row per step, columns on lanes
constexpr int32_t kKernelLane = 3;      // one job per lane
constexpr int32_t kKernelLane16 = 4;    // one job per lane, int16x2 pair-column blocks
constexpr int32_t kKernelLane2 = 5;     // one job per lane, two rows in flight
constexpr int32_t kKernelBand = 6;      // one job per warp, the band's row buffer in registers

int launch_extend(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream);

// Launch facts that never change for a kernel on a device, cached for the process: the SM
// count, the dynamic shared memory a block of a kernel may use (after its limit was raised once),
// and the resident blocks per SM at a block size and dynamic shared memory.  Each CUDA query
// costs microseconds of host time, and a chunked seed stream makes thousands of class launches
// with a handful of configurations.
struct LaunchCache {
    struct Ent {
        int kind;            // 0: dynamic shared memory limit, 1: resident blocks, 2: SMs
        const void* fn;
        int dev, threads;
        size_t smem;
        long long val;
    };
    std::mutex mu;
    Ent e[1024];
    int n = 0;
    bool get(int kind, const void* fn, int dev, int threads, size_t smem, long long* val) {
        std::lock_guard<std::mutex> g(mu);
        for (int k = 0; k < n; ++k)
            if (e[k].kind == kind && e[k].fn == fn && e[k].dev == dev && e[k].threads == threads &&
                e[k].smem == smem) {
                *val = e[k].val;
                return true;
            }
        return false;
    }
    void put(int kind, const void* fn, int dev, int threads, size_t smem, long long val) {
        std::lock_guard<std::mutex> g(mu);
        if (n < 1024) e[n++] = Ent{kind, fn, dev, threads, smem, val};
    }
};
inline LaunchCache& launch_cache() {
    static LaunchCache c;
    return c;
}

inline int sm_count() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    long long v;
    if (launch_cache().get(2, nullptr, dev, 0, 0, &v)) return (int)v;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) return 1;
    launch_cache().put(2, nullptr, dev, 0, 0, sms);
    return sms;
}

// Lets kernel `fn` launch with all the dynamic shared memory a block can have on this device
// (the opt-in maximum less the kernel's static shared memory), which *limit receives.  Always
// the same value, set once per device: a kernel launched by several width classes (possibly
// captured in one CUDA graph) must never see another launch lower its limit below its own size.
template <class F>
inline cudaError_t allow_max_smem(F* fn, size_t* limit = nullptr) {
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    long long v;
    if (launch_cache().get(0, (const void*)fn, dev, 0, 0, &v)) {
        if (limit) *limit = (size_t)v;
        return cudaSuccess;
    }
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes a;
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, fn);
    if (e != cudaSuccess) return e;
    const int dyn = optin - (int)a.sharedSizeBytes;
    if (limit) *limit = (size_t)dyn;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
    if (e == cudaSuccess) launch_cache().put(0, (const void*)fn, dev, 0, 0, dyn);
    return e;
}

// Resident blocks per SM of `fn` with `threads` threads and `smem` bytes of dynamic shared
// memory per block (0 when it does not fit).
template <class F>
inline int resident_blocks(F* fn, int threads, size_t smem) {
    int dev = 0, per_sm = 0;
    cudaGetDevice(&dev);
    long long v;
    if (launch_cache().get(1, (const void*)fn, dev, threads, smem, &v)) return (int)v;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess) per_sm = 0;
    launch_cache().put(1, (const void*)fn, dev, threads, smem, per_sm);
    return per_sm;
}

// Launches a width-class kernel fn<<<grid, block, smem, st>>>(d, sp).  With d.pdl it goes out
// as a programmatic dependent of the kernel before it on `st`: it may start as soon as every
// block of that kernel has called pdl_trigger(), so the classes of one stream run side by side
// like launches on separate streams, without the streams.
template <class K>
inline cudaError_t launch_class_kernel(K* fn, int grid, int block, size_t smem, cudaStream_t st,
                                       const LaunchDesc& d, const ScoreParams& sp) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = d.pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, fn, d, sp);
}
int launch_rolling(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream);
int launch_rowpar(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream);
int launch_lane(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream);
int launch_lane16(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream);
int launch_lane2(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream);
int launch_band(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream);
size_t band_smem_per_warp(int qcap);
size_t lane2_smem_per_warp(int qcap);
size_t lane16_smem_per_warp(int qcap);
size_t lane_ring_smem_per_warp(int ring);
size_t lane_smem_per_warp(int qcap, int tcap);

// Device scratch of one seed-level call (capacity >= n seeds).
struct SeedScratch {
    g3x_job_t *ljobs, *rjobs;
    g3x_ext_t *lext, *rext;
    int32_t *lstatus, *rstatus;
    int32_t* order[4];     // left wave 1/2, right wave 1/2
    int32_t* counters;     // 16 ints
    int64_t cap;
};

int alloc_seed_scratch(SeedScratch& w, int64_t n);   // grown to >= n seeds, kept when large enough
void free_seed_scratch(SeedScratch& w);

// Runs one wave of a seed-level call: d names the wave's job array (d.n entries) and its jobs
// (d.order[0 .. *d.count)); by default one launch of d.kernel over them.
struct WaveRunner {
    int (*run)(void* user, const LaunchDesc& d, const ScoreParams& sp, cudaStream_t st);
    void* user;
};

int extend_seeds(const SeedScratch& ws, const g3x_opt_t& opt, const ScoreParams& sp,
                 const g3x_seed_t* seeds, int n, const uint32_t* codes, const uint32_t* nmask,
                 g3x_reg_t* regs, int32_t* status, const LaunchDesc& proto, cudaStream_t st,
                 const WaveRunner* runner = nullptr);
// What one width-class pipeline uses: the sort scratch, the classes' job-queue counters
// (kMaxBuckets), one stream per class and the events that fork the classes from the caller's
// stream and join them back (side null: the classes chain on the caller's stream as
// programmatic dependent launches), the occupancy counters (or none).  A context has one; the seed stream keeps one per
// chunk it runs at a time.
struct ClassRes {
    SchedScratch* sched;
    int32_t* queue;
    cudaStream_t* side;
    cudaEvent_t fork;
    cudaEvent_t* join;
    unsigned long long* stats;
};
int alloc_sched(SchedScratch& s, int64_t n);
void free_sched(SchedScratch& s);

// A seed-level wave through the width classes (g3x_api.cu): the wave's jobs sorted like a batch
// (length-sorted, or by the cost model's predictions) with res's scratch, then one persistent
// launch per class on res's streams (res null: the context's own).
struct ClassWave {
    g3x_ctx* ctx;
    bool learned;
    const ClassRes* res;
};
int run_class_wave(void* user, const LaunchDesc& d, const ScoreParams& sp, cudaStream_t st);

// The chunked seed stream (g3x_stream.cu) runs kStreamLanes chunks at a time, each on its own
// compute stream with its own device buffer set, pinned staging, seed scratch and width-class
// scratch, so one chunk's latency-bound waves overlap the next chunks' work.  A lane chains its
// classes on its own stream as programmatic dependent launches (they still run side by side),
// so the whole stream stays within eight CUDA streams (seven lanes and the copy stream), the
// hardware work queues a context has by default: more streams than queues alias onto the same
// queues and serialise.  Config 5 (2M seeds, 32k-seed chunks): 40.6 ms with four lanes, 33.8 with
// six, 33.0 with seven.  Kept in the context between calls and grown on demand.
constexpr int kStreamLanes = 7;
struct StreamSet {
    g3x_seed_t* d_seeds = nullptr;
    uint32_t* d_codes = nullptr;
    uint32_t* d_nmask = nullptr;
    g3x_reg_t* d_regs = nullptr;
    int32_t* d_status = nullptr;
    g3x_seed_t* h_seeds = nullptr;   // pinned staging
    g3x_reg_t* h_regs = nullptr;
    int32_t* h_status = nullptr;
    cudaEvent_t h2d = nullptr, done = nullptr;
    int64_t pending = -1;            // chunk whose results sit in this set
    cudaStream_t comp = nullptr;     // the lane's compute stream
    SeedScratch seeds = {};          // the lane's seed-level scratch
    SchedScratch sched;              // the lane's width-class sort scratch
    int32_t* queue = nullptr;        // and job-queue counters
};
struct StreamScratch {
    StreamSet set[kStreamLanes];
    cudaStream_t copy_st = nullptr;
    int64_t seeds = 0, code_words = 0, mask_words = 0;   // capacities of each set
    bool lanes_ready = false;        // streams, events and queues of the lanes created
};
void free_stream_scratch(StreamScratch& s);

// runner: the class-wave runner of the call (its ClassWave user is copied per lane with the
// lane's resources), or null for the call's single kernel.
int extend_seeds_stream(StreamScratch& ss, const g3x_opt_t& opt,
                        const ScoreParams& sp, const g3x_seed_t* h_seeds, int64_t n,
                        const uint32_t* h_codes, const uint32_t* h_nmask, int64_t n_bases,
                        g3x_reg_t* h_regs, int32_t* h_status, int32_t chunk,
                        const LaunchDesc& proto, const WaveRunner* runner = nullptr);
int score_params(const g3x_score_t* s, ScoreParams* sp);
int ctx_device(const g3x_ctx* ctx);   // the CUDA device a context is bound to

// Scratch of the chain-level call (g3x_chain.cu), grown on demand.
struct ChainScratch {
    int64_t* win = nullptr;          // per chain: reference window [r0, r1)
    uint64_t* srt = nullptr;         // per seed: its chain's processing keys
    void* state = nullptr;           // per read: 16-byte walk state
    g3x_seed_t* xseeds = nullptr;    // per seed: its seed-level extension record ...
    g3x_reg_t* xregs = nullptr;      // ... and result
    int32_t* xstatus = nullptr;
    int32_t* maxlen = nullptr;       // longest read and window of the call
    int32_t* h_maxlen = nullptr;     // pinned copy of the two bounds
    int64_t reads = 0, chains = 0, seeds = 0;
};
ChainScratch& ctx_chain(g3x_ctx* ctx);

// Direction bytes of the global-alignment backtrack (g3x_global.cu), grown on demand.
struct GlobalScratch {
    uint8_t* z = nullptr;
    int32_t* queue = nullptr;
    int64_t bytes = 0;
};
GlobalScratch& ctx_global(g3x_ctx* ctx);
// Scratch of the striped local alignment: sort arrays and counters (int32), XSUBO row maxima.
struct SwScratch {
    int32_t* buf = nullptr;
    uint32_t* sub = nullptr;
    int64_t cap = 0, sub_cap = 0;
    uint8_t* flt = nullptr;        // the seed filter: its jobs, results and per-read values
    int64_t flt_cap = 0;
};
SwScratch& ctx_sw(g3x_ctx* ctx);
// The context's job order by decreasing row count and row width (its scheduling scratch).
int cost_order(g3x_ctx* ctx, const g3x_job_t* jobs, int n, const ScoreParams& sp, cudaStream_t st,
               const int32_t** order);
void free_chain_scratch(ChainScratch& w);

// Learned cost model state (device buffers; g3x_model.cu).
struct ModelState {
    float *params = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
    float *h1 = nullptr, *h2 = nullptr, *dh1 = nullptr, *dh2 = nullptr, *dy = nullptr;
    float* loss_part = nullptr;
    int* perm = nullptr;
    int batch_cap = 0, perm_cap = 0;
    long long t = 0;       // Adam step
    int trained = 0;       // parameters set by training or by the caller
    int active = 1;        // 0: the learned schedule uses the length order (no inference)
};
int model_alloc(ModelState& M, int batch);
void model_free(ModelState& M);
int model_init(ModelState& M, uint64_t seed);
int model_features(const g3x_job_t* jobs, int n, const uint32_t* codes, const uint32_t* nmask,
                   int64_t n_bases, float* feat, cudaStream_t st,
                   const int32_t* subset = nullptr, const int32_t* subset_n = nullptr);
int model_predict(const float* params, const float* feat, int n, float* out, cudaStream_t st);
int model_gradient(ModelState& M, const float* X, const float* T, int B, float* h_grad,
                   float* h_loss, cudaStream_t st);
int model_train(ModelState& M, const float* X, const float* T, int n, int epochs, int batch,
                float lr, uint64_t seed, float* h_epoch_loss, cudaStream_t st);
int batch_proto(const g3x_batch_opts_t* opts, int32_t* queue, LaunchDesc* d);
size_t group_smem_bytes(int qmax, int tmax);
int measure_int_peak(int device, double* ops_per_s);

}  // namespace g3x

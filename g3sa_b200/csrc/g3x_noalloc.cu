// g3x_noalloc.cu -- length-sorted ksw_extend2 batch that allocates no memory.
//
// g3x_ksw_extend2_batch_noalloc runs the same scheduled path as g3x_ksw_extend2_batch with
// G3X_SCHED_SORTED (counting sort into width classes, one persistent row-parallel launch per
// class), but takes its scratch -- the per-job sort keys and job order, the sort histogram and
// cursors, each class's (offset, count) and job-queue counter -- from one file-scope device
// array of fixed size instead of a context's cudaMalloc'd buffers.  It needs no context.
//
// Who needs it: a caller that must not allocate device memory while it runs -- a pipeline
// stage that runs between other stages' kernels on its own streams, where cudaMalloc and
// cudaFree would synchronise with the whole device; a caller that has reserved nearly all of
// the GPU's memory for its index and batches up front (as the reference's pipeline does in
// device_alloc) and has nothing left for a library to grow into; and a caller inside a
// framework whose allocator owns all device memory.
//
// Set-up: CUDA loads a library's device code, and with it this array, on first use (lazy
// module loading, the default unless CUDA_MODULE_LOADING=EAGER), and loading may allocate
// device memory and synchronise.  So the first call on a device -- which also looks the array's
// address up with cudaGetSymbolAddress, once per device -- belongs before the phase in which
// nothing may allocate: one call with a small batch loads every kernel the entry point
// launches, and a call with n = 0 does the address look-up alone.  The address is kept per
// device index and belongs to the device's primary context (the one the runtime API uses):
// the entry point assumes that context throughout, with no cudaDeviceReset between calls.
//
// Limits: at most G3X_NOALLOC_MAX_JOBS jobs per call (larger batches return
// G3X_ERR_SCRATCH).  Every call on a device shares the one array, so calls that overlap on
// the GPU -- on two streams, or from two host threads -- race on it and corrupt each other;
// serialise them (one stream, or events between them).
#include <cuda_runtime.h>
#include <mutex>
#include <string.h>
#include "g3x_internal.h"

namespace g3x {

namespace {

constexpr int kBins = kMaxBuckets * kSchedLevels;         // schedule_jobs' histogram bins
// Word layout of the scratch array (int32 words).
constexpr int64_t kQueueAt = 0;                           // kMaxBuckets job-queue counters
constexpr int64_t kBucketAt = 64;                         // 2 * kMaxBuckets (offset, count)
constexpr int64_t kHistAt = 128;                          // kBins
constexpr int64_t kCursorAt = kHistAt + kBins;            // kBins
constexpr int64_t kBinAt = kCursorAt + kBins;             // G3X_NOALLOC_MAX_JOBS
constexpr int64_t kOrderAt = kBinAt + G3X_NOALLOC_MAX_JOBS;  // G3X_NOALLOC_MAX_JOBS
constexpr int64_t kWords = kOrderAt + G3X_NOALLOC_MAX_JOBS;  // 8.13 MiB in all

static_assert(kBinAt % 64 == 0 && kOrderAt % 64 == 0, "256-byte aligned sub-arrays");

__device__ __align__(256) int32_t g_scratch[kWords];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
int32_t* g_scratch_ptr[kMaxDevices];                      // per device, set up once

// Address of the scratch array on the current device, looked up once per device.
int scratch_of(int device, int32_t** out) {
    if (device < 0 || device >= kMaxDevices) return G3X_ERR_INVALID;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[device]) {
        int32_t* p = nullptr;
        if (cudaGetSymbolAddress((void**)&p, g_scratch) != cudaSuccess || !p) return G3X_ERR_CUDA;
        g_scratch_ptr[device] = p;
    }
    *out = g_scratch_ptr[device];
    return G3X_OK;
}

}  // namespace

}  // namespace g3x

extern "C" int g3x_ksw_extend2_batch_noalloc(int device, const g3x_score_t* score,
                                             const g3x_job_t* d_jobs, int32_t n,
                                             const uint32_t* d_codes, const uint32_t* d_nmask,
                                             int64_t n_bases, g3x_ext_t* d_out, int32_t* d_status,
                                             int32_t max_qlen, int32_t max_tlen, void* stream) {
    using namespace g3x;
    if (n < 0) return G3X_ERR_INVALID;
    if (n > G3X_NOALLOC_MAX_JOBS) return G3X_ERR_SCRATCH;
    if (n > 0 && (n_bases < 1 || n_bases > 0x100000000ll)) return G3X_ERR_INVALID;
    int rc;
    if (cudaSetDevice(device) != cudaSuccess) return G3X_ERR_CUDA;
    int32_t* s = nullptr;
    if ((rc = scratch_of(device, &s))) return rc;
    if (n == 0) return G3X_OK;
    if (!d_jobs || !d_codes || !d_nmask || !d_out || !d_status) return G3X_ERR_INVALID;
    if (max_qlen < 0 || max_tlen < 0 || max_qlen > 65534 || max_tlen > 65535) return G3X_ERR_INVALID;
    ScoreParams sp;
    if ((rc = score_params(score, &sp))) return rc;
    cudaStream_t st = (cudaStream_t)stream;

    // Sort scratch: schedule_jobs clears the histogram itself and writes the keys, cursors,
    // order and class (offset, count) before reading them.
    SchedScratch sc;
    sc.hist = s + kHistAt;
    sc.cursor = s + kCursorAt;
    sc.bin = s + kBinAt;
    sc.order = s + kOrderAt;
    sc.bucket_oc = s + kBucketAt;
    sc.cap = G3X_NOALLOC_MAX_JOBS;
    TileTable tt;
    default_tiles(tt);
    if ((rc = schedule_jobs(sc, d_jobs, n, sp, nullptr, tt, st))) return rc;
    // The persistent kernels take jobs from a counter that must start at zero.
    if (cudaMemsetAsync(s + kQueueAt, 0, kMaxBuckets * sizeof(int32_t), st) != cudaSuccess)
        return G3X_ERR_CUDA;
    // One launch per width class, in order on the caller's stream.
    for (int k = 0; k < tt.n; ++k) {
        LaunchDesc d;
        memset(&d, 0, sizeof(d));
        d.jobs = d_jobs; d.codes = d_codes; d.nmask = d_nmask; d.out = d_out; d.status = d_status;
        d.n = n;
        d.tmax = max_tlen;
        d.n_bases = n_bases;
        d.qmax = k == tt.n - 1 ? max_qlen : (max_qlen < tt.width[k] ? max_qlen : tt.width[k]);
        d.kernel = kKernelRowpar;
        d.lanes = tt.lanes[k];
        d.tile = tt.tile[k];
        d.persistent = 1;
        d.warps_per_block = 4;
        d.order = sc.order;
        d.order_off = sc.bucket_oc + 2 * k;
        d.count = sc.bucket_oc + 2 * k + 1;
        d.queue = s + kQueueAt + k;
        while (d.lanes < 32 && (32 / d.lanes) * group_smem_bytes(d.qmax, d.tmax) > 227 * 1024) d.lanes *= 2;
        if ((rc = launch_rowpar(d, sp, st))) return rc;
    }
    return G3X_OK;
}

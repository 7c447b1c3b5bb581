// g3x_sched.cu -- job scheduling for the persistent row-parallel kernels.
//
// Every job gets
//   a bucket : the first width class that holds its query (the class's tile, G lanes x C
//              cells, covers the class width, so it covers the job's widest possible row
//              min(qlen, 2w' + 1), w' the clamped band of ksw.cu:321-329); one persistent
//              launch per class;
//   a key    : the job's row count, then its widest row.  The row count is the length-sorted
//              fallback's bound tlen, or, learned, that bound corrected by the cost model: the
//              model predicts log2(1 + rows) less log2(1 + tlen), at most 0 (a job runs at most
//              tlen rows), and the key's log2 row count is log2(1 + tlen) plus
//              min(0, correction + 1); the widest row is min(qlen, 2w' + 1).
//              A warp of a row-synchronous kernel takes consecutive jobs, so jobs of similar
//              row count and similar row width run together, longest first.
// A device counting sort over (bucket, key) bins -- histogram, exclusive scan, scatter --
// writes the job order with each bucket's jobs contiguous and in decreasing row count, plus
// each bucket's (offset, count).  Nothing returns to the host, so the whole
// batch (features, prediction, sort, launches) can be captured in one CUDA graph.
#include <cuda_runtime.h>
#include <math.h>
#include "g3x_core.h"
#include "g3x_internal.h"
#include "g3x_schedkey.cuh"

namespace g3x {

namespace {

constexpr int kLevels = kSchedLevels;  // key levels per bucket: 64 row-count x 32 width bins
static_assert(kLevels % 1024 == 0 && kMaxBuckets * kLevels <= 16 * 1024, "scan: 1..16 bins per thread");

// Job of sort position k: k itself, or subset[k] when sorting a subset of *subset_n jobs.
__device__ __forceinline__ int job_at(int k, const int32_t* subset) { return subset ? subset[k] : k; }

__global__ void cost_kernel(const g3x_job_t* __restrict__ jobs, int n, ScoreParams sp,
                            const float* __restrict__ pred, TileTable tt,
                            int32_t* __restrict__ bin, int32_t* __restrict__ hist,
                            const int32_t* __restrict__ subset, const int32_t* __restrict__ subset_n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n || (subset_n && k >= *subset_n)) return;
    const int job = job_at(k, subset);
    const int bn = sched_key(jobs[job], sp, tt, pred != nullptr, pred ? pred[job] : 0.0f);
    bin[k] = bn;
    sched_count(hist, bn);
}

// Exclusive scan of the nb bins in one block; also each bucket's (offset, count).  nb is a
// multiple of 1024 with at most 16 bins per thread (nb = classes x kLevels): each thread sums
// its consecutive bins with independent loads, the warps scan their sums with shuffles and warp
// 0 scans the 32 warp totals.
__global__ void __launch_bounds__(1024) scan_kernel(const int32_t* __restrict__ hist, int nb,
                                                    int32_t* __restrict__ cursor, int32_t* __restrict__ bucket_oc,
                                                    int nbuckets) {
    __shared__ int32_t wsum[32];
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    const int per = nb >> 10;
    int v[16];
    int s = 0;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        v[k] = k < per ? hist[t * per + k] : 0;
        s += v[k];
    }
    int inc = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) wsum[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        int w = wsum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xFFFFFFFFu, w, o);
            if (lane >= o) w += u;
        }
        wsum[lane] = w;                       // inclusive over warps
    }
    __syncthreads();
    int run = (wid ? wsum[wid - 1] : 0) + inc - s;
#pragma unroll
    for (int k = 0; k < 16; ++k)
        if (k < per) {
            cursor[t * per + k] = run;
            run += v[k];
        }
    __syncthreads();
    if (t < nbuckets) {
        const int lo = cursor[t * kLevels];
        const int hi = t + 1 < nbuckets ? cursor[(t + 1) * kLevels] : wsum[31];
        bucket_oc[2 * t] = lo;
        bucket_oc[2 * t + 1] = hi - lo;
    }
}

__global__ void scatter_kernel(const int32_t* __restrict__ bin, int n, int32_t* __restrict__ cursor,
                               int32_t* __restrict__ order, const int32_t* __restrict__ subset,
                               const int32_t* __restrict__ subset_n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n || (subset_n && k >= *subset_n)) return;
    const int bn = bin[k];
    // the warp's jobs of one bin take consecutive slots with one atomic
    const unsigned peers = __match_any_sync(__activemask(), bn);
    const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
    int at = 0;
    if (lane == leader) at = atomicAdd(cursor + bn, __popc(peers));
    at = __shfl_sync(peers, at, leader) + __popc(peers & ((1u << lane) - 1u));
    order[at] = job_at(k, subset);
}

__global__ void max_w_kernel(const g3x_job_t* __restrict__ jobs, int n, ScoreParams sp, int32_t* out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    int32_t w = 0;
    if (k < n) {
        const g3x_job_t jb = jobs[k];
        w = clamp_w(jb.w, jb.qlen, sp.max_sc, sp.end_bonus, sp.o_del, sp.e_del, sp.o_ins, sp.e_ins);
    }
    w = (int32_t)__reduce_max_sync(0xFFFFFFFFu, (unsigned)(w > 0 ? w : 0));
    if ((threadIdx.x & 31) == 0) atomicMax(out, w);
}

}  // namespace

int batch_max_w(const g3x_job_t* jobs, int n, const ScoreParams& sp, int32_t* d_tmp, int32_t* h_out,
                cudaStream_t st) {
    if (cudaMemsetAsync(d_tmp, 0, sizeof(int32_t), st) != cudaSuccess) return G3X_ERR_CUDA;
    max_w_kernel<<<(n + 255) / 256, 256, 0, st>>>(jobs, n, sp, d_tmp);
    if (cudaMemcpyAsync(h_out, d_tmp, sizeof(int32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return G3X_ERR_CUDA;
    return G3X_OK;
}

int schedule_jobs(SchedScratch& s, const g3x_job_t* jobs, int n, const ScoreParams& sp,
                  const float* pred, const TileTable& tt, cudaStream_t st, const int32_t* subset,
                  const int32_t* subset_n) {
    const int nbins = tt.n * kLevels;
    if (cudaMemsetAsync(s.hist, 0, nbins * sizeof(int32_t), st) != cudaSuccess) return G3X_ERR_CUDA;
    const int tb = 256, nb = (n + tb - 1) / tb;
    cost_kernel<<<nb, tb, 0, st>>>(jobs, n, sp, pred, tt, s.bin, s.hist, subset, subset_n);
    scan_kernel<<<1, 1024, 0, st>>>(s.hist, nbins, s.cursor, s.bucket_oc, tt.n);
    scatter_kernel<<<nb, tb, 0, st>>>(s.bin, n, s.cursor, s.order, subset, subset_n);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

int schedule_jobs_learned(SchedScratch& s, const g3x_job_t* jobs, int n, const uint32_t* codes,
                          const uint32_t* nmask, int64_t n_bases, const float* params, const ScoreParams& sp,
                          const TileTable& tt, cudaStream_t st, const int32_t* subset, const int32_t* subset_n,
                          float* pred_out) {
    const int nbins = tt.n * kLevels;
    if (cudaMemsetAsync(s.hist, 0, nbins * sizeof(int32_t), st) != cudaSuccess) return G3X_ERR_CUDA;
    int rc = launch_learned_keys(params, jobs, n, codes, nmask, n_bases, sp, tt, s.bin, s.hist, st, subset, subset_n,
                                 pred_out);
    if (rc) return rc;
    const int tb = 256, nb = (n + tb - 1) / tb;
    scan_kernel<<<1, 1024, 0, st>>>(s.hist, nbins, s.cursor, s.bucket_oc, tt.n);
    if (nb > 0) scatter_kernel<<<nb, tb, 0, st>>>(s.bin, n, s.cursor, s.order, subset, subset_n);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

}  // namespace g3x

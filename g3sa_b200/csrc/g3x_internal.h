// g3x_internal.h -- declarations shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/g3x.h"

namespace g3x {

// Scoring as the kernels consume it (passed by value as a kernel parameter).
struct ScoreParams {
    int8_t mat[25];
    int8_t pad_[3];
    int32_t o_del, e_del, o_ins, e_ins, zdrop, end_bonus, max_sc;
};

// One launch of the extension kernel family.
struct LaunchDesc {
    const g3x_job_t* jobs;
    const uint32_t* codes;
    const uint32_t* nmask;
    g3x_ext_t* out;
    int32_t* status;
    int32_t* cells;        // optional
    const int32_t* order;  // optional permutation: queue slot -> job index
    const int32_t* count;  // optional device-side job count (overrides n when set)
    int32_t* queue;        // persistent kernels: device counter (zeroed by the caller)
    int32_t n;
    int32_t qmax, tmax;    // smem sizing bounds
    int32_t lanes;         // 8, 16 or 32
    int32_t persistent;    // 0: one group per job slot; 1: groups pull from `queue`
    int32_t warps_per_block;
    int32_t blocks;        // persistent grid size (0 = derive from occupancy)
};

int launch_extend(const LaunchDesc& d, const ScoreParams& sp, cudaStream_t stream);

// Device scratch of one seed-level call (capacity >= n seeds).
struct SeedScratch {
    g3x_job_t *ljobs, *rjobs;
    g3x_ext_t *lext, *rext;
    int32_t *lstatus, *rstatus;
    int32_t* order[4];     // left wave 1/2, right wave 1/2
    int32_t* counters;     // 16 ints
    int64_t cap;
};

int extend_seeds(const SeedScratch& ws, const g3x_opt_t& opt, const ScoreParams& sp,
                 const g3x_seed_t* seeds, int n, const uint32_t* codes, const uint32_t* nmask,
                 g3x_reg_t* regs, int32_t* status, const LaunchDesc& proto, cudaStream_t st);
int extend_seeds_stream(SeedScratch& ws, int (*grow)(SeedScratch&, int64_t), const g3x_opt_t& opt,
                        const ScoreParams& sp, const g3x_seed_t* h_seeds, int64_t n,
                        const uint32_t* h_codes, const uint32_t* h_nmask, int64_t n_bases,
                        g3x_reg_t* h_regs, int32_t* h_status, int32_t chunk,
                        const LaunchDesc& proto);
int score_params(const g3x_score_t* s, ScoreParams* sp);
int batch_proto(const g3x_batch_opts_t* opts, int32_t* queue, LaunchDesc* d);
size_t group_smem_bytes(int qmax, int tmax);
int measure_int_peak(int device, double* ops_per_s);

}  // namespace g3x

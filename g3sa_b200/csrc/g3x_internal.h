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
size_t group_smem_bytes(int qmax, int tmax);
int measure_int_peak(int device, double* ops_per_s);

}  // namespace g3x

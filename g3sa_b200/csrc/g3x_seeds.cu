// g3x_seeds.cu -- seed-level extension with BWA's band-retry loop on the GPU.
//
// Restates, per seed, the left/right extension block of mem_chain2aln
// (bwa/src/aux.cu:250-310) as a sequence of device passes, all asynchronous on one stream
// and with every count kept on the device:
//   1. left jobs    : seeds with qbeg > 0 get a job on the reversed read prefix and the
//                     reversed window prefix (aux.cu:258-265), h0 = len * a, band w
//   2. wave, retry  : the extension kernel runs the jobs; a job is re-run with band 2w when
//                     its score differs from `prev` and max_off >= (w>>1)+(w>>2)
//                     (aux.cu:266-271, MAX_BAND_TRY = 2 at aux.cuh:401)
//   3. left finish  : local vs to-end choice (aux.cu:273-280) and the right jobs: the read
//                     suffix and the window after the seed, h0 = sc0 = the left score
//                     (aux.cu:283-286)
//   4. wave, retry  : as 2, with prev = sc0 (aux.cu:287-292)
//   5. right finish : aux.cu:294-301 and the band width of the region (aux.cu:309)
#include <cuda_runtime.h>
#include "g3x_internal.h"

namespace g3x {

namespace {

constexpr uint32_t kRetried = 0x100u;   // job flag: re-run with the doubled band

__device__ __forceinline__ void push(int32_t* order, int32_t* count, int32_t k) {
    const int32_t at = atomicAdd(count, 1);
    order[at] = k;
}

__global__ void left_jobs_kernel(const g3x_seed_t* __restrict__ seeds, int n, g3x_opt_t opt,
                                 int64_t n_bases, g3x_job_t* jobs, int32_t* order, int32_t* count,
                                 g3x_reg_t* regs, int32_t* status) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const g3x_seed_t s = seeds[k];
    g3x_reg_t a;
    a.rb = a.re = 0; a.qb = a.qe = 0;
    a.score = a.truesc = -1;                       // aux.cu:254-255
    a.w = opt.w;
    a.tries_left = a.tries_right = 0;
    a.pad_[0] = a.pad_[1] = 0;
    status[k] = G3X_OK;
    const int64_t tl = s.rbeg - s.rmax0;
    const int64_t tr = s.rmax1 - (s.rbeg + s.len);
    if (s.qbeg < 0 || s.len < 0 || s.qbeg + s.len > s.l_query || tl < 0 || tr < 0 ||
        s.qbeg > 65534 || s.l_query - s.qbeg - s.len > 65534 || tl > 65535 || tr > 65535) {
        status[k] = G3X_ERR_TOO_LONG;
        regs[k] = a;
        return;
    }
    // the read and the window must lie in the planes: no job of this seed reads past them
    if ((int64_t)s.read_off + s.l_query > n_bases || (int64_t)s.win_off + (s.rmax1 - s.rmax0) > n_bases) {
        status[k] = G3X_ERR_INVALID;
        regs[k] = a;
        return;
    }
    if (s.qbeg) {
        g3x_job_t j;
        j.q_off = s.read_off; j.qlen = (uint16_t)s.qbeg;
        j.t_off = s.win_off; j.tlen = (uint16_t)tl;
        j.h0 = s.len * opt.a; j.w = opt.w; j.flags = G3X_JOB_QREV | G3X_JOB_TREV;
        jobs[k] = j;
        push(order, count, k);
    } else {                                        // aux.cu:282
        a.score = a.truesc = s.len * opt.a;
        a.qb = 0; a.rb = s.rbeg;
    }
    regs[k] = a;
}

// Selects the jobs of one wave that BWA retries with a doubled band.  prev is -1 for the
// left side and sc0 (= the job's h0) for the right side.
__global__ void retry_kernel(const int32_t* __restrict__ order, const int32_t* __restrict__ count,
                             g3x_job_t* jobs, const g3x_ext_t* __restrict__ ext,
                             const int32_t* __restrict__ status, int right, int32_t* order2,
                             int32_t* count2) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= *count) return;
    const int k = order[t];
    if (status[k] != G3X_OK) return;
    const g3x_job_t j = jobs[k];
    const int prev = right ? j.h0 : -1;
    const g3x_ext_t e = ext[k];
    if (e.score == prev || e.max_off < (j.w >> 1) + (j.w >> 2)) return;
    jobs[k].w = j.w << 1;
    jobs[k].flags = j.flags | kRetried;
    push(order2, count2, k);
}

__global__ void left_finish_kernel(const g3x_seed_t* __restrict__ seeds, int n, g3x_opt_t opt,
                                   const g3x_job_t* __restrict__ ljobs,
                                   const g3x_ext_t* __restrict__ lext, g3x_job_t* rjobs,
                                   int32_t* rorder, int32_t* rcount, g3x_reg_t* regs,
                                   const int32_t* __restrict__ lstatus, int32_t* status) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (status[k] != G3X_OK) return;
    const g3x_seed_t s = seeds[k];
    g3x_reg_t a = regs[k];
    if (s.qbeg) {
        if (lstatus[k] != G3X_OK) { status[k] = lstatus[k]; return; }
        const g3x_ext_t e = lext[k];
        const int aw0 = ljobs[k].w;
        a.score = e.score;
        a.tries_left = (uint8_t)((ljobs[k].flags & kRetried) ? 2 : 1);
        if (e.gscore <= 0 || e.gscore <= e.score - opt.pen_clip5) {     // aux.cu:273-276
            a.qb = s.qbeg - e.qle; a.rb = s.rbeg - e.tle; a.truesc = e.score;
        } else {                                                       // aux.cu:277-279
            a.qb = 0; a.rb = s.rbeg - e.gtle; a.truesc = e.gscore;
        }
        a.w = aw0;
    }
    const int qe = s.qbeg + s.len;
    if (qe != s.l_query) {                                             // aux.cu:283-286
        const int64_t re = s.rbeg + s.len - s.rmax0;
        g3x_job_t j;
        j.q_off = s.read_off + (uint32_t)qe; j.qlen = (uint16_t)(s.l_query - qe);
        j.t_off = s.win_off + (uint32_t)re; j.tlen = (uint16_t)(s.rmax1 - s.rmax0 - re);
        j.h0 = a.score; j.w = opt.w; j.flags = 0;
        rjobs[k] = j;
        push(rorder, rcount, k);
    } else {                                                           // aux.cu:301
        a.qe = s.l_query; a.re = s.rbeg + s.len;
    }
    regs[k] = a;
}

__global__ void right_finish_kernel(const g3x_seed_t* __restrict__ seeds, int n, g3x_opt_t opt,
                                    const g3x_job_t* __restrict__ rjobs,
                                    const g3x_ext_t* __restrict__ rext, g3x_reg_t* regs,
                                    const int32_t* __restrict__ rstatus, int32_t* status) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (status[k] != G3X_OK) return;
    const g3x_seed_t s = seeds[k];
    g3x_reg_t a = regs[k];
    const int qe = s.qbeg + s.len;
    int aw1 = opt.w;
    if (qe != s.l_query) {
        if (rstatus[k] != G3X_OK) { status[k] = rstatus[k]; return; }
        const g3x_ext_t e = rext[k];
        const g3x_job_t j = rjobs[k];
        const int sc0 = j.h0;
        const int64_t re = s.rbeg + s.len - s.rmax0;
        aw1 = j.w;
        a.score = e.score;
        a.tries_right = (uint8_t)((j.flags & kRetried) ? 2 : 1);
        if (e.gscore <= 0 || e.gscore <= e.score - opt.pen_clip3) {     // aux.cu:294-296
            a.qe = qe + e.qle; a.re = s.rmax0 + re + e.tle; a.truesc += e.score - sc0;
        } else {                                                       // aux.cu:297-299
            a.qe = s.l_query; a.re = s.rmax0 + re + e.gtle; a.truesc += e.gscore - sc0;
        }
    }
    const int aw0 = a.w;
    a.w = aw0 > aw1 ? aw0 : aw1;                                       // aux.cu:309
    regs[k] = a;
}

}  // namespace

int extend_seeds(const SeedScratch& ws, const g3x_opt_t& opt, const ScoreParams& sp,
                 const g3x_seed_t* seeds, int n, const uint32_t* codes, const uint32_t* nmask,
                 g3x_reg_t* regs, int32_t* status, const LaunchDesc& proto, cudaStream_t st,
                 const WaveRunner* runner) {
    if (n == 0) return G3X_OK;
    // counters: [0] left wave 1, [1] left wave 2, [2] right wave 1, [3] right wave 2;
    // queue counters of the four persistent launches at [8 .. 11]
    if (cudaMemsetAsync(ws.counters, 0, 16 * sizeof(int32_t), st) != cudaSuccess) return G3X_ERR_CUDA;
    const int tb = 256, nb = (n + tb - 1) / tb;
    left_jobs_kernel<<<nb, tb, 0, st>>>(seeds, n, opt, proto.n_bases, ws.ljobs, ws.order[0], ws.counters + 0,
                                        regs, status);
    auto wave = [&](g3x_job_t* jobs, g3x_ext_t* ext, int32_t* jst, int32_t* order, int32_t* count,
                    int32_t* queue) -> int {
        LaunchDesc d = proto;
        d.jobs = jobs; d.codes = codes; d.nmask = nmask; d.out = ext; d.status = jst;
        d.cells = nullptr; d.rows = nullptr; d.order = order; d.count = count; d.queue = queue; d.n = n;
        return runner ? runner->run(runner->user, d, sp, st) : launch_extend(d, sp, st);
    };
    int rc;
    if ((rc = wave(ws.ljobs, ws.lext, ws.lstatus, ws.order[0], ws.counters + 0, ws.counters + 8))) return rc;
    retry_kernel<<<nb, tb, 0, st>>>(ws.order[0], ws.counters + 0, ws.ljobs, ws.lext, ws.lstatus, 0,
                                    ws.order[1], ws.counters + 1);
    if ((rc = wave(ws.ljobs, ws.lext, ws.lstatus, ws.order[1], ws.counters + 1, ws.counters + 9))) return rc;
    left_finish_kernel<<<nb, tb, 0, st>>>(seeds, n, opt, ws.ljobs, ws.lext, ws.rjobs, ws.order[2],
                                          ws.counters + 2, regs, ws.lstatus, status);
    if ((rc = wave(ws.rjobs, ws.rext, ws.rstatus, ws.order[2], ws.counters + 2, ws.counters + 10))) return rc;
    retry_kernel<<<nb, tb, 0, st>>>(ws.order[2], ws.counters + 2, ws.rjobs, ws.rext, ws.rstatus, 1,
                                    ws.order[3], ws.counters + 3);
    if ((rc = wave(ws.rjobs, ws.rext, ws.rstatus, ws.order[3], ws.counters + 3, ws.counters + 11))) return rc;
    right_finish_kernel<<<nb, tb, 0, st>>>(seeds, n, opt, ws.rjobs, ws.rext, regs, ws.rstatus, status);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

}  // namespace g3x

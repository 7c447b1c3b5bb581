// g3x_schedkey.cuh -- the counting sort's key of one job (g3x_sched.cu), shared by the cost
// kernel of the length-sorted schedule and the learned schedule's fused key kernel
// (g3x_model.cu), so both order jobs by exactly the same rules.
//
// A job's key is its width class, then a row-count bin, then a row-width bin:
//   class : the first class that holds its query (the class's kernel stages queries up to its
//           width; the last class takes any), or the last class when the class's kernel cannot
//           take the job (scores outside its 16-bit fields or int16 fit, a band wider than its
//           ring or window);
//   rows  : log2(1 + tlen), four bins per doubling, more rows first; learned, plus the model's
//           correction soft-thresholded by one halving, min(0, pred + 1): a job moves ahead of
//           the length order only where the network predicts that it ends before half its rows
//           (a z-drop on an unrelated target), and by how much further; its error on jobs that
//           run to their end leaves them in length order, which is already near the true order
//           for them.  Continuous, so jobs of equal predicted rows stay together;
//   width : eight-column blocks of the widest row min(qlen, 2w' + 1), wider first.
#pragma once
#include <math.h>
#include "g3x_core.h"
#include "g3x_internal.h"

namespace g3x {

constexpr int kSchedRowBins = 64, kSchedWidthBins = 32;
constexpr float kLearnedSlack = 1.0f;   // log2 rows the learned correction must exceed
static_assert(kSchedRowBins * kSchedWidthBins == kSchedLevels, "key layout");

// has_pred: the learned schedule, with the model's correction `pred` for this job.
__device__ __forceinline__ int sched_key(const g3x_job_t& jb, const ScoreParams& sp, const TileTable& tt,
                                         bool has_pred, float pred) {
    const int w = clamp_w(jb.w, jb.qlen, sp.max_sc, sp.end_bonus, sp.o_del, sp.e_del, sp.o_ins, sp.e_ins);
    const int wide = jb.qlen < 2 * w + 1 ? jb.qlen : 2 * w + 1;
    int b = tt.n - 1;
    for (int t = 0; t < tt.n; ++t)
        if (tt.width[t] >= jb.qlen) { b = t; break; }
    if (tt.lanes[b] == 1 && b != tt.n - 1) {
        JobConst c;
        c.qlen = jb.qlen; c.tlen = jb.tlen; c.h0 = jb.h0; c.w = w;
        c.o_del = sp.o_del; c.e_del = sp.e_del; c.o_ins = sp.o_ins; c.e_ins = sp.e_ins;
        c.oe_del = sp.oe_del; c.oe_ins = sp.oe_ins; c.zdrop = sp.zdrop;
        bool fits = tt.tile[b] == 2 ? job_fits_int16(c, sp.max_sc) : job_fits_lane(c, sp.max_sc);
        if (tt.tile[b] >= 64 && 2 * w + 16 > tt.tile[b]) fits = false;   // band wider than the ring
        if (!fits) b = tt.n - 1;
    } else if (tt.lanes[b] == 32 && tt.tile[b] >= 64 && b != tt.n - 1) {
        // the band kernel: the band's 2w' + 2 entries fit its window, and every H stays below 2^21
        const int64_t hmax = (int64_t)jb.qlen * sp.max_sc + (jb.h0 > 0 ? jb.h0 : 0);
        if (2 * w + 2 > tt.tile[b] || hmax >= (1 << 21)) b = tt.n - 1;
    }
    float lr = log2f(1.0f + (float)jb.tlen);
    if (has_pred) lr += fminf(pred + kLearnedSlack, 0.0f);
    int rb = (int)((16.0f - lr) * (kSchedRowBins / 16.0f));
    rb = rb < 0 ? 0 : (rb >= kSchedRowBins ? kSchedRowBins - 1 : rb);
    int wb = (wide + 7) >> 3;
    wb = kSchedWidthBins - 1 - (wb < kSchedWidthBins - 1 ? wb : kSchedWidthBins - 1);
    return b * kSchedLevels + rb * kSchedWidthBins + wb;
}

// One histogram atomic per distinct key of the warp (a batch has few populated bins).
__device__ __forceinline__ void sched_count(int32_t* hist, int bn) {
    const unsigned peers = __match_any_sync(__activemask(), bn);
    if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(hist + bn, __popc(peers));
}

}  // namespace g3x

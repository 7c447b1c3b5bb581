// g3x_core.h -- per-lane step logic of the banded-extension wavefront.
//
// One job (one ksw_extend2 call, bwa/src/ksw.cu:303-401) is processed by a group of G
// lanes.  Lane r of the group owns target rows r, r+G, r+2G, ... ("rolling rows"); a lane
// walks its row left to right, up to one aligned block of four cells per step, and trails
// the lane that owns the previous row, so the group sweeps anti-diagonals.  The
// reference's single row buffer eh[] (ksw.cu:310) is kept verbatim in shared memory: every
// row reads and overwrites it at the same positions, in the same row order, as the scalar
// loop does, so the stale entries the reference reads when its band grows by two columns
// (ksw.cu:388-391) hold the same values here.
//
// The scalar loop decides the band of row i+1 only after row i has finished
// (ksw.cu:388-391).  Here the lane that owns row i+1 instead watches, every step, how far
// row i has got (`col`: columns < col are final) and the last non-zero entry row i has
// written (`lnz1` = that column + 1).  Column j of row i+1 is inside the reference's band
// exactly when j <= L_i + 1 (L_i = row i's last non-zero), so the lane computes cell j as
// soon as row i has written a non-zero entry at column >= j-1, and ends the row once row i
// is finished and has none.  The left edge uses the first non-zero entry of row i
// (`fnz`), and the fixed band limits i-w and i+w+1 are applied as in ksw.cu:338-340.
// Rows therefore end in row order, one per step at most, and the per-row bookkeeping of
// ksw.cu:371-386 (to-end score, max tracking, z-drop) is applied in row order by a
// uniform "commit" over the group.  Rows started after the row that ends the extension
// are speculative and are discarded.
//
// A finished row publishes its final words for exactly one step; its successor latches
// them, so the lane can take its next row immediately.
//
// Everything in this header is plain C++ usable on the host as well, so a CPU model of
// the warp protocol (g3x_emu.cpp, test-only) runs this same code.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define G3X_HD __host__ __device__ __forceinline__
#else
#define G3X_HD inline
#endif

namespace g3x {

constexpr uint32_t kNone = 0xFFFFu;   // "no column yet" / "row finished" marker
constexpr int kBlock = 4;             // cells per lane-step (one aligned block)

enum LaneState : int32_t { kIdle = 0, kWait = 1, kRun = 2, kDone = 3 };

// Per-job constants, derived once at job start (ksw.cu:305-333).
struct JobConst {
    int32_t qlen, tlen, w, h0;
    int32_t o_del, e_del, o_ins, e_ins, oe_del, oe_ins, zdrop;
};

struct EhCell {
    int32_t h, e;
};

// What one lane carries for the row it owns.
struct Lane {
    int32_t st;     // LaneState
    int32_t i;      // row (target position)
    int32_t j;      // next column to compute
    int32_t beg;    // first column of the row
    int32_t cap;    // min(i + w + 1, qlen): fixed right limit of the band
    int32_t h1;     // H(i, j-1)
    int32_t f;      // F(i, j)
    int32_t key;    // narrow rows: (row max << 16) | last column reaching it; -1 = none
    int32_t m, mj;  // wide rows: row maximum and the last column reaching it
    int32_t fnz;    // first column whose new eh entry is non-zero (kNone: none yet)
    int32_t lnz1;   // 1 + last column whose new eh entry is non-zero (0: none)
    int32_t qrow;   // offset of this row's query-profile row
    uint32_t lat_prog, lat_fnz;  // predecessor's final words, latched when it finished
    int32_t lat;    // 1 when the latch holds the predecessor row of this lane's row
};

// What a lane hands to the group when its row ends.
struct RowDone {
    int32_t m, mj;
    int32_t gval;   // H at the last column when the row reached qlen, else -1
    int32_t ncells; // cells computed in the row (trip count of ksw.cu:346)
};

// Group-uniform result state (ksw.cu:331-333 and the outputs of ksw.cu:395-400).
struct Commit {
    int32_t next;       // next row to commit
    int32_t stop;       // extension finished (break or last row)
    int32_t best, best_i, best_j;
    int32_t gscore, max_ie, max_off;
    int64_t cells;
};

// Band clamp, ksw.cu:321-329, in integer form: (int)((double)num/e + 1.) clamped to >= 1
// equals num/e + 1 for num >= 0 and 1 for num < 0 (e > 0).
G3X_HD int32_t gap_limit(int32_t qlen, int32_t max_sc, int32_t end_bonus, int32_t o, int32_t e) {
    int32_t num = qlen * max_sc + end_bonus - o;
    int32_t v = num >= 0 ? num / e + 1 : 1;
    return v > 1 ? v : 1;
}

G3X_HD int32_t clamp_w(int32_t w, int32_t qlen, int32_t max_sc, int32_t end_bonus,
                       int32_t o_del, int32_t e_del, int32_t o_ins, int32_t e_ins) {
    int32_t a = gap_limit(qlen, max_sc, end_bonus, o_ins, e_ins);
    int32_t b = gap_limit(qlen, max_sc, end_bonus, o_del, e_del);
    w = w < a ? w : a;
    return w < b ? w : b;
}

// Row "-1" of the buffer (ksw.cu:317-319) in closed form: h0 at 0, then the insertion
// scores h0 - oe_ins - (j-1)*e_ins while positive, zero beyond; e is zero everywhere.
G3X_HD int32_t init_h(int32_t j, const JobConst& c) {
    if (j == 0) return c.h0;
    int32_t v1 = c.h0 > c.oe_ins ? c.h0 - c.oe_ins : 0;
    if (j > c.qlen) return j == 1 ? v1 : 0;   // only eh[1] of an empty query is written
    int32_t v = v1 - (j - 1) * c.e_ins;
    return v > 0 ? v : 0;
}

// A job is "narrow" when every H it can produce is below 2^15: then a row's maximum and
// its column pack into one int32 key.  H <= h0 + max_sc * min(qlen, tlen).
G3X_HD bool job_is_narrow(const JobConst& c, int32_t max_sc) {
    int64_t mn = c.qlen < c.tlen ? c.qlen : c.tlen;
    int64_t hmax = (int64_t)(c.h0 > 0 ? c.h0 : 0) + (int64_t)max_sc * mn;
    return hmax < 32768 && c.qlen < 65535;
}

// The lane-per-job kernel keeps H and E of a job in 16-bit fields: it takes narrow jobs with
// h0 >= 0 (its M = min(H + S, 256 H) form needs H >= 0).
G3X_HD bool job_fits_lane(const JobConst& c, int32_t max_sc) {
    return c.h0 >= 0 && job_is_narrow(c, max_sc);
}

// Shift k of the int16x2 kernel's M = min(H + S, H << k): the smallest k with 2^k >= 1 + max_sc,
// so that H << k >= H + S for every H > 0.
G3X_HD int32_t int16_shift(int32_t max_sc) {
    int32_t k = 0;
    while ((1 << k) < 1 + max_sc && k < 15) ++k;
    return k;
}

// A job fits the int16x2 kernel when every value of its DP, H << k included, stays below 2^15:
// 0 <= H <= h0 + max_sc * min(qlen, tlen) (E and F are bounded by H), and the penalties keep
// M - o - e and F - 8 e_ins above -2^15.
G3X_HD bool job_fits_int16(const JobConst& c, int32_t max_sc) {
    if (c.h0 < 0 || c.qlen >= 65535 || c.oe_del >= 16384 || c.oe_ins >= 16384) return false;
    if (c.e_ins > 4095 || c.e_del > 4095) return false;
    const int64_t mn = c.qlen < c.tlen ? c.qlen : c.tlen;
    const int64_t hmax = (int64_t)c.h0 + (int64_t)(max_sc > 0 ? max_sc : 0) * mn;
    return (hmax << int16_shift(max_sc)) < 32768;
}

G3X_HD void commit_init(Commit& k, const JobConst& c) {
    k.next = 0;
    k.stop = c.tlen <= 0;
    k.best = c.h0; k.best_i = -1; k.best_j = -1;
    k.gscore = -1; k.max_ie = -1; k.max_off = 0;
    k.cells = 0;
}

// Row bookkeeping of ksw.cu:372-386 for the next row in order.
G3X_HD void commit_row(Commit& k, const JobConst& c, const RowDone& d) {
    const int32_t i = k.next;
    if (d.gval >= 0) {                                   // row reached qlen (ksw.cu:372-375)
        if (!(k.gscore > d.gval)) k.max_ie = i;
        if (d.gval > k.gscore) k.gscore = d.gval;
    }
    k.cells += d.ncells;
    k.next = i + 1;
    if (d.m == 0) { k.stop = 1; return; }                // ksw.cu:376
    if (d.m > k.best) {                                  // ksw.cu:377-379
        k.best = d.m; k.best_i = i; k.best_j = d.mj;
        int32_t off = d.mj > i ? d.mj - i : i - d.mj;
        if (off > k.max_off) k.max_off = off;
    } else if (c.zdrop > 0) {                            // ksw.cu:380-386
        int32_t di = i - k.best_i, dj = d.mj - k.best_j;
        if (di > dj) {
            if (k.best - d.m - (di - dj) * c.e_del > c.zdrop) { k.stop = 1; return; }
        } else {
            if (k.best - d.m - (dj - di) * c.e_ins > c.zdrop) { k.stop = 1; return; }
        }
    }
    if (k.next >= c.tlen) k.stop = 1;
}

G3X_HD void lane_init(Lane& L, int32_t r, int32_t tlen) {
    L.st = r < tlen ? kWait : kIdle;
    L.i = r;
    L.j = L.beg = L.cap = L.h1 = L.f = L.m = L.qrow = 0;
    L.mj = -1; L.key = -1;
    L.fnz = (int32_t)kNone; L.lnz1 = 0;
    L.lat_prog = 0; L.lat_fnz = kNone; L.lat = 0;
}

// The words a lane publishes to its successor each step.
G3X_HD uint32_t lane_prog(const Lane& L) {
    uint32_t col = L.st == kDone ? kNone : (L.st == kRun ? (uint32_t)L.j : 0u);
    uint32_t lnz = (L.st == kDone || L.st == kRun) ? (uint32_t)L.lnz1 : 0u;
    return (col << 16) | lnz;
}
G3X_HD uint32_t lane_fnz(const Lane& L) {
    return (L.st == kDone || L.st == kRun) ? (uint32_t)L.fnz : kNone;
}

G3X_HD void lane_begin_row(Lane& L, int32_t beg, const JobConst& c, int32_t tcode,
                           int32_t qstride) {
    L.st = kRun;
    L.beg = beg;
    L.j = beg;
    int32_t cap = L.i + c.w + 1;
    L.cap = cap < c.qlen ? cap : c.qlen;
    if (beg == 0) {                                      // ksw.cu:342-345
        int32_t h = c.h0 - (c.o_del + c.e_del * (L.i + 1));
        L.h1 = h > 0 ? h : 0;
    } else {
        L.h1 = 0;
    }
    L.f = 0; L.m = 0; L.mj = -1; L.key = -1;
    L.fnz = (int32_t)kNone; L.lnz1 = 0;
    L.qrow = tcode * qstride;
}

#if defined(__CUDACC__)
G3X_HD int32_t max3_i32(int32_t a, int32_t b, int32_t c) {
#if defined(__CUDA_ARCH__)
    return __vimax3_s32(a, b, c);
#else
    int32_t m = a > b ? a : b; return m > c ? m : c;
#endif
}
// max(a + b, c)
G3X_HD int32_t addmax_i32(int32_t a, int32_t b, int32_t c) {
#if defined(__CUDA_ARCH__)
    return __viaddmax_s32(a, b, c);
#else
    int32_t s = a + b; return s > c ? s : c;
#endif
}
// min(a + b, c)
G3X_HD int32_t addmin_i32(int32_t a, int32_t b, int32_t c) {
#if defined(__CUDA_ARCH__)
    return __viaddmin_s32(a, b, c);
#else
    int32_t s = a + b; return s < c ? s : c;
#endif
}
#else
inline int32_t max3_i32(int32_t a, int32_t b, int32_t c) { int32_t m = a > b ? a : b; return m > c ? m : c; }
inline int32_t addmax_i32(int32_t a, int32_t b, int32_t c) { int32_t s = a + b; return s > c ? s : c; }
inline int32_t addmin_i32(int32_t a, int32_t b, int32_t c) { int32_t s = a + b; return s < c ? s : c; }
#endif

// Row end, ksw.cu:371-375.  For an empty row (j == beg) the reference's loop variable is
// beg, its eh[end] write is never read again (the row breaks), and the to-end test uses
// the row's initial h1.
template <bool kNarrow, class Buf>
G3X_HD void lane_end_row(Lane& L, const JobConst& c, Buf& buf, RowDone* done) {
    const int32_t jn = L.j;
    if (jn > L.beg) {
        buf.store(jn, L.h1, 0);
        if (L.h1 != 0) L.lnz1 = jn + 1;
    }
    if (L.fnz == (int32_t)kNone) L.fnz = jn;
    if (kNarrow) {
        done->m = L.key < 0 ? 0 : (L.key >> 16);
        done->mj = L.key < 0 ? -1 : (L.key & 0xFFFF);
    } else {
        done->m = L.m;
        done->mj = L.mj;
    }
    done->gval = jn == c.qlen ? L.h1 : -1;
    done->ncells = jn - L.beg;
    L.st = kDone;
    L.lat = 0;
}

// One cell of ksw.cu:346-370 on the lane's running state.  M = H(i-1,j-1) ? H(i-1,j-1) + S : 0
// is written as min(H + S, 256 H): equal when H > 0, and <= 0 when H == 0, which every use
// below clips to 0 exactly like the reference's 0.  Writes eh[col] = {H(i,col-1), E(i+1,col)}
// and returns that entry's "non-zero" word.
template <bool kNarrow, class Buf>
G3X_HD int32_t dp_cell(const JobConst& c, Buf& buf, int32_t col, EhCell v, int32_t s,
                       int32_t& h1, int32_t& f, int32_t& key, int32_t& m, int32_t& mj) {
    const int32_t M = addmin_i32(v.h, s, v.h << 8);
    const int32_t h = max3_i32(M, v.e, f);
    const int32_t te = addmax_i32(M, -c.oe_del, 0);
    const int32_t e2 = addmax_i32(v.e, -c.e_del, te);
    buf.store(col, h1, e2);
    const int32_t nz = h1 | e2;
    if (kNarrow) {
        const int32_t k2 = (h << 16) | col;
        key = key > k2 ? key : k2;
    } else {
        if (h >= m) { m = h; mj = col; }
    }
    const int32_t tf = addmax_i32(M, -c.oe_ins, 0);
    f = addmax_i32(f, -c.e_ins, tf);
    h1 = h;
    return nz;
}

// Lane transitions outside a running row: a finished row is published for one step, then
// the lane takes row i+G; a waiting lane starts once its predecessor row has a first
// non-zero column (or is finished).
template <int G, class Tgt>
G3X_HD void lane_advance(Lane& L, const JobConst& c, uint32_t pfnz, const Tgt& tgt,
                         int32_t qstride) {
    if (L.st == kDone) {
        L.i += G;
        L.st = L.i < c.tlen ? kWait : kIdle;
    }
    if (L.st == kWait) {
        if (L.i == 0) {
            int32_t b = -c.w;
            lane_begin_row(L, b > 0 ? b : 0, c, tgt.code(0), qstride);
        } else if (pfnz != kNone) {
            int32_t b = L.i - c.w;
            lane_begin_row(L, (int32_t)pfnz > b ? (int32_t)pfnz : b, c, tgt.code(L.i), qstride);
        }
    }
}

// One step of one lane.  `pprog`/`pfnz` are the predecessor's published words at the start
// of the step.  Returns true when the lane's row ended in this step (then *done is
// filled).  `buf` gives the job's row buffer, `qp` the query profile, `tgt` the target.
//
// Buf interface:  load4(jb, EhCell v[4])  -- the four slots of the aligned block at jb
//                 store(c, h, e)          -- write slot c
//                 note_read(c)            -- the lane consumed slot c (test hook)
// Tgt interface:  code(i)                 -- target code (0-4) of row i
template <int G, bool kNarrow, class Buf, class Tgt>
G3X_HD bool lane_step(Lane& L, const JobConst& c, uint32_t pprog, uint32_t pfnz, Buf& buf,
                      const int8_t* qp, const Tgt& tgt, int32_t qstride, RowDone* done) {
    // Latch the predecessor's final words the step they appear (it moves on next step).
    if ((pprog >> 16) == kNone) { L.lat_prog = pprog; L.lat_fnz = pfnz; L.lat = 1; }
    if (L.lat) { pprog = L.lat_prog; pfnz = L.lat_fnz; }
    if (L.st != kRun) {
        lane_advance<G>(L, c, pfnz, tgt, qstride);
        if (L.st != kRun) return false;
    }

    uint32_t colp = pprog >> 16, lnzp = pprog & 0xFFFFu;
    if (L.i == 0) { colp = kNone; lnzp = kNone; }        // row 0 reads the initial buffer
    const bool pdone = colp == kNone;
    int32_t lim = L.cap;                                  // cells j < lim may be computed
    if ((int32_t)colp < lim) lim = (int32_t)colp;
    if ((int32_t)lnzp + 1 < lim) lim = (int32_t)lnzp + 1;
    const int32_t j0 = L.j;
    if (j0 < lim) {
        const int32_t jb = j0 & ~(kBlock - 1);
        EhCell v[kBlock];
        buf.load4(jb, v);
        const uint32_t sc4 = *reinterpret_cast<const uint32_t*>(qp + L.qrow + jb);
        int32_t h1 = L.h1, f = L.f, key = L.key, m = L.m, mj = L.mj, lnz1 = L.lnz1;
        int32_t nzw[kBlock];
        if (j0 == jb && jb + kBlock <= lim) {
            // whole block inside the band: no per-cell predicates
#pragma unroll
            for (int t = 0; t < kBlock; ++t) {
                buf.note_read(jb + t);
                nzw[t] = dp_cell<kNarrow>(c, buf, jb + t, v[t], (int32_t)(int8_t)(sc4 >> (8 * t)),
                                          h1, f, key, m, mj);
                if (nzw[t]) lnz1 = jb + t + 1;
            }
            L.j = jb + kBlock;
        } else {
#pragma unroll
            for (int t = 0; t < kBlock; ++t) {
                const int32_t col = jb + t;
                nzw[t] = 0;
                if (col >= j0 && col < lim) {
                    buf.note_read(col);
                    nzw[t] = dp_cell<kNarrow>(c, buf, col, v[t], (int32_t)(int8_t)(sc4 >> (8 * t)),
                                              h1, f, key, m, mj);
                    if (nzw[t]) lnz1 = col + 1;
                }
            }
            L.j = jb + kBlock < lim ? jb + kBlock : lim;
        }
        if (L.fnz == (int32_t)kNone) {            // first non-zero entry of the row (rare path)
#pragma unroll
            for (int t = kBlock - 1; t >= 0; --t)
                if (nzw[t]) L.fnz = jb + t;
        }
        L.h1 = h1; L.f = f; L.key = key; L.m = m; L.mj = mj; L.lnz1 = lnz1;
    }
    const int32_t jn = L.j;
    if (jn >= L.cap || (pdone && (uint32_t)jn > lnzp)) {
        lane_end_row<kNarrow>(L, c, buf, done);
        return true;
    }
    return false;
}

}  // namespace g3x

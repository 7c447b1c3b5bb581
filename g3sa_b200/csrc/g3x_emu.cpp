// g3x_emu.cpp -- CPU model of the group wavefront protocol, for tests only.
//
// Runs the same per-lane step logic as the sm_100a kernels (g3x_core.h) with G emulated
// lanes: every step snapshots the words each lane publishes (the warp shuffle), lets every
// lane act, then applies the uniform row commit.  It additionally checks the property the
// kernels rely on -- within one step no two lanes touch the same row-buffer slot -- and
// that at most one row ends per step.  It is built as its own library (libg3x_emu.so),
// loaded only by tests, and is never part of the product path.
#include <stdint.h>
#include <string.h>
#include <vector>
#include "g3x_core.h"
#include "../../include/g3x.h"

namespace {

struct Tracker {
    std::vector<int32_t> owner;   // lane that touched the slot in the current step
    std::vector<int32_t> stamp;   // step of that touch
    int32_t step = 0, lane = 0;
    bool conflict = false;
};

struct EmuBuf {
    std::vector<g3x::EhCell> slot;
    Tracker* tr;
    void touch(int idx) const {
        if (tr->stamp[idx] == tr->step && tr->owner[idx] != tr->lane) tr->conflict = true;
        tr->stamp[idx] = tr->step;
        tr->owner[idx] = tr->lane;
    }
    void load4(int jb, g3x::EhCell v[4]) const {
        for (int t = 0; t < 4; ++t) v[t] = slot.at((size_t)(jb + t));
    }
    void store(int c, int32_t h, int32_t e) { touch(c); slot.at((size_t)c) = g3x::EhCell{h, e}; }
    void note_read(int c) const { touch(c); }
};

struct EmuTgt {
    const uint8_t* p;
    int32_t code(int32_t i) const { return p[i]; }
};

template <int G>
bool step_g(bool narrow, g3x::Lane& L, const g3x::JobConst& c, uint32_t pp, uint32_t pf, EmuBuf& eh,
            const int8_t* qp, const uint8_t* tgt, int qs, g3x::RowDone* rd) {
    const EmuTgt tg{tgt};
    return narrow ? g3x::lane_step<G, true>(L, c, pp, pf, eh, qp, tg, qs, rd)
                  : g3x::lane_step<G, false>(L, c, pp, pf, eh, qp, tg, qs, rd);
}

// The lane count is a template parameter of lane_step (it sets the row stride).
bool step(bool narrow, int G, g3x::Lane& L, const g3x::JobConst& c, uint32_t pp, uint32_t pf,
          EmuBuf& eh, const int8_t* qp, const uint8_t* tgt, int qs, g3x::RowDone* rd) {
    switch (G) {
        case 2: return step_g<2>(narrow, L, c, pp, pf, eh, qp, tgt, qs, rd);
        case 3: return step_g<3>(narrow, L, c, pp, pf, eh, qp, tgt, qs, rd);
        case 4: return step_g<4>(narrow, L, c, pp, pf, eh, qp, tgt, qs, rd);
        case 8: return step_g<8>(narrow, L, c, pp, pf, eh, qp, tgt, qs, rd);
        case 16: return step_g<16>(narrow, L, c, pp, pf, eh, qp, tgt, qs, rd);
        default: return step_g<32>(narrow, L, c, pp, pf, eh, qp, tgt, qs, rd);
    }
}

int decode(const uint32_t* codes, const uint32_t* nmask, uint32_t off, int k, int len, bool rev) {
    uint32_t p = rev ? off + (uint32_t)(len - 1 - k) : off + (uint32_t)k;
    uint32_t c = (codes[p >> 4] >> ((p & 15u) << 1)) & 3u;
    return ((nmask[p >> 5] >> (p & 31u)) & 1u) ? 4 : (int)c;
}

}  // namespace

extern "C" {

// Emulates one group of G lanes per job.  stats[k] = {steps, lane_cells, max_ends_per_step,
// conflict}.  Returns 0, or -1 on bad arguments.
int g3x_emu_extend_batch(const g3x_score_t* s, const g3x_job_t* jobs, int32_t n,
                         const uint32_t* codes, const uint32_t* nmask, int32_t G,
                         g3x_ext_t* out, int32_t* status, int32_t* cells, int64_t* stats) {
    if (!s || !jobs || !out || !status || (G != 2 && G != 3 && G != 4 && G != 8 && G != 16 && G != 32)) return -1;
    int max_sc = 0;
    for (int k = 0; k < 25; ++k) max_sc = s->mat[k] > max_sc ? s->mat[k] : max_sc;
    for (int32_t jid = 0; jid < n; ++jid) {
        const g3x_job_t& jb = jobs[jid];
        const int qlen = jb.qlen, tlen = jb.tlen;
        g3x::JobConst c;
        c.qlen = qlen; c.tlen = tlen; c.h0 = jb.h0;
        c.o_del = s->o_del; c.e_del = s->e_del; c.o_ins = s->o_ins; c.e_ins = s->e_ins;
        c.oe_del = s->o_del + s->e_del; c.oe_ins = s->o_ins + s->e_ins; c.zdrop = s->zdrop;
        c.w = g3x::clamp_w(jb.w, qlen, max_sc, s->end_bonus, s->o_del, s->e_del, s->o_ins, s->e_ins);
        const int qs = (qlen + 4) & ~3;           // as qstride_of() in the kernels
        const int nslots = (qlen + 8) & ~3;       // as eh_slots() in the kernels
        std::vector<int8_t> qp((size_t)5 * qs + 4, 0);
        std::vector<uint8_t> tgt((size_t)tlen + 1, 0);
        Tracker tr;
        tr.owner.assign((size_t)nslots, -1);
        tr.stamp.assign((size_t)nslots, -1);
        EmuBuf eh;
        eh.tr = &tr;
        eh.slot.assign((size_t)nslots, g3x::EhCell{0, 0});
        for (int k = 0; k < qlen; ++k) {
            int code = decode(codes, nmask, jb.q_off, k, qlen, jb.flags & G3X_JOB_QREV);
            for (int a = 0; a < 5; ++a) qp[(size_t)a * qs + k] = s->mat[a * 5 + code];
        }
        for (int k = 0; k < tlen; ++k) tgt[k] = (uint8_t)decode(codes, nmask, jb.t_off, k, tlen, jb.flags & G3X_JOB_TREV);
        for (int k = 0; k <= qlen + 1; ++k) eh.slot[k] = g3x::EhCell{g3x::init_h(k, c), 0};
        const bool narrow = g3x::job_is_narrow(c, max_sc);
        std::vector<g3x::Lane> L((size_t)G);
        for (int r = 0; r < G; ++r) g3x::lane_init(L[r], r, tlen);
        g3x::Commit K;
        g3x::commit_init(K, c);
        std::vector<uint32_t> prog((size_t)G), fnz((size_t)G);
        const long long limit = 8LL * ((long long)tlen + 2) * ((long long)qlen + 8) + 4096;
        long long steps = 0, lane_cells = 0;
        int max_ends = 0;
        int32_t err = G3X_OK;
        while (!K.stop) {
            for (int r = 0; r < G; ++r) { prog[r] = g3x::lane_prog(L[r]); fnz[r] = g3x::lane_fnz(L[r]); }
            int ends = 0;
            g3x::RowDone fin{};
            tr.step = (int32_t)steps;
            for (int r = 0; r < G; ++r) {
                int pr = (r + G - 1) % G;
                g3x::RowDone rd;
                const int32_t j0 = L[r].j, st0 = L[r].st, i0 = L[r].i;
                tr.lane = r;
                bool f = step(narrow, G, L[r], c, prog[pr], fnz[pr], eh, qp.data(), tgt.data(), qs, &rd);
                if (st0 == g3x::kRun)
                    lane_cells += L[r].j - j0;                       // continued its row
                else if ((L[r].st == g3x::kRun || L[r].st == g3x::kDone) && (L[r].i != i0 || st0 == g3x::kWait))
                    lane_cells += L[r].j - L[r].beg;                 // started a row this step
                if (f) { ++ends; fin = rd; }
            }
            if (ends > max_ends) max_ends = ends;
            if (ends > 1) { err = G3X_ERR_INTERNAL; break; }
            if (ends == 1) g3x::commit_row(K, c, fin);
            if (++steps > limit) { err = G3X_ERR_TIMEOUT; break; }
        }
        out[jid] = g3x_ext_t{K.best, K.best_j + 1, K.best_i + 1, K.max_ie + 1, K.gscore, K.max_off};
        status[jid] = err;
        if (cells) cells[jid] = (int32_t)K.cells;
        if (stats) {
            stats[4 * (int64_t)jid + 0] = steps;
            stats[4 * (int64_t)jid + 1] = lane_cells;
            stats[4 * (int64_t)jid + 2] = max_ends;
            stats[4 * (int64_t)jid + 3] = tr.conflict ? 1 : 0;
        }
    }
    return 0;
}

}  // extern "C"

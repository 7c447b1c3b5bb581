// g3x_emu16.cu -- CPU model of the int16x2 lane kernel's per-lane logic (test-only; built as
// host code into libg3x_emu16.so, loaded only by tests).
//
// It runs each job through the same functions the kernel runs per lane (g3x_lane16.cuh): row
// begin, the row's blocks, the row end with its band trims, on a row buffer with the kernel's
// layout, so the arithmetic and the band handling of the kernel can be checked against the
// oracle on the CPU.  What only the kernel has -- the warp's refill waves, its warp-uniform
// block loop and the staging from the bit planes -- does not change a lane's results: every lane
// computes its own job, and lanes with shorter rows skip the extra iterations.
#include <stdint.h>
#include <string.h>
#include <vector>
#include "g3x_internal.h"
#include "g3x_lane16.cuh"

using namespace g3x;

namespace {

ScoreParams score_of(const g3x_score_t& s) {
    ScoreParams sp;
    memset(&sp, 0, sizeof(sp));
    int max_sc = 0;
    for (int k = 0; k < 25; ++k) {
        sp.mat[k] = s.mat[k];
        if (s.mat[k] > max_sc) max_sc = s.mat[k];
    }
    sp.o_del = s.o_del; sp.e_del = s.e_del; sp.o_ins = s.o_ins; sp.e_ins = s.e_ins;
    sp.zdrop = s.zdrop; sp.end_bonus = s.end_bonus; sp.max_sc = max_sc;
    sp.oe_del = s.o_del + s.e_del; sp.oe_ins = s.o_ins + s.e_ins;
    return sp;
}

uint8_t base_at(const uint8_t* u8, uint32_t off, int len, int k, bool rev) {
    const uint8_t c = u8[rev ? off + (uint32_t)(len - 1 - k) : off + (uint32_t)k];
    return c < 4 ? c : 4;
}

template <bool kSym>
int run_job(const g3x_job_t& jb, const uint8_t* u8, const ScoreParams& sp, const uint2* pools,
            const uint4* ge, g3x_ext_t* out, int32_t* cells) {
    JobConst c;
    c.qlen = jb.qlen; c.tlen = jb.tlen; c.h0 = jb.h0;
    c.o_del = sp.o_del; c.e_del = sp.e_del; c.o_ins = sp.o_ins; c.e_ins = sp.e_ins;
    c.oe_del = sp.oe_del; c.oe_ins = sp.oe_ins; c.zdrop = sp.zdrop;
    c.w = clamp_w(jb.w, c.qlen, sp.max_sc, sp.end_bonus, sp.o_del, sp.e_del, sp.o_ins, sp.e_ins);
    if (!job_fits_int16(c, sp.max_sc)) return G3X_ERR_TOO_LONG;
    const int qcap = c.qlen;
    const int nb = l16::blocks_of(qcap);
    // one lane (lane 0) of a warp-sized buffer, the kernel's layout
    std::vector<uint4> H((size_t)nb * 32), E((size_t)nb * 32);
    std::vector<uint32_t> qn((size_t)l16::nib_words(qcap) * 32);
    const bool qrev = (jb.flags & G3X_JOB_QREV) != 0, trev = (jb.flags & G3X_JOB_TREV) != 0;
    for (int k = 0; k < c.qlen; ++k)
        qn[(size_t)(k >> 3) * 32] |= (uint32_t)base_at(u8, jb.q_off, c.qlen, k, qrev) << ((k & 7) * 4);
    // stale words from an earlier job, as a lane of the kernel finds its row buffer
    for (auto& v : H) v = make_uint4(0x1357u, 0x2468u, 0x1111u, 0x2222u);
    for (auto& v : E) v = make_uint4(0x0123u, 0x0456u, 0x0789u, 0x0abcu);
    l16::Planes P;
    P.H = H.data(); P.E = E.data();
    P.H32 = reinterpret_cast<uint32_t*>(P.H);
    P.E32 = reinterpret_cast<uint32_t*>(P.E);
    P.qn = qn.data();
    const l16::PairConst pc = l16::pair_const(sp);
    l16::init_row(P, 0, c.qlen, c.h0, sp, pc, ge);
    for (int b = 0; b <= ((c.qlen + 1) >> 3); ++b) {      // the closed form against init_h
        const uint32_t* h = reinterpret_cast<const uint32_t*>(&H[(size_t)b * 32]);
        for (int p = 0; p < 4; ++p)
            if (h[p] != (((uint32_t)init_h(8 * b + p, c) & 0xFFFFu) | ((uint32_t)init_h(8 * b + p + 4, c) << 16)))
                return G3X_ERR_INTERNAL;
    }
    l16::LaneJob J;
    J.job = 0;
    J.qlen = c.qlen; J.tlen = c.tlen; J.w = c.w; J.h0 = c.h0;
    J.t_off = jb.t_off; J.trev = trev;
    commit_init(J.K, c);
    J.beg = 0; J.end = c.qlen;
    while (!J.K.stop) {
        const int32_t i = J.K.next;
        J.tx = J.tn = 0;
        for (int k = 0; k < 16 && (i & ~15) + k < c.tlen; ++k) {
            const uint8_t t = base_at(u8, jb.t_off, c.tlen, (i & ~15) + k, trev);
            J.tx |= (uint32_t)(t & 3) << (2 * k);
            J.tn |= (uint32_t)(t == 4) << k;
        }
        l16::RowState r;
        l16::row_begin(J, sp, pools, r);
        const bool nonempty = r.beg < r.end;
        const int nblk = l16::blocks_in_row(r);
        // the warp's widest row in the kernel can have more blocks than this lane's: vary it
        const int kmax = nblk + (int)((i * 2654435761u + (uint32_t)jb.q_off) >> 30);
        uint32_t mF, mL;
        // a one-block row elsewhere in the warp masks this lane's last block too: vary it
        const bool any_single = nblk == 1 || ((i * 2246822519u + (uint32_t)jb.t_off) >> 31);
        l16::row_blocks<kSym>(P, 0, r, pc, ge, nblk, kmax, any_single, mF, mL);
        l16::row_end(J, P, 0, r, sp, nonempty, mF, mL);
    }
    const Commit& K = J.K;
    *out = g3x_ext_t{K.best, K.best_j + 1, K.best_i + 1, K.max_ie + 1, K.gscore, K.max_off};
    *cells = (int32_t)K.cells;
    return G3X_OK;
}

}  // namespace

// n jobs through the model; status G3X_ERR_TOO_LONG for jobs outside the int16 fit.
extern "C" int g3x_emu16_extend(const g3x_job_t* jobs, int32_t n, const uint8_t* u8,
                                const g3x_score_t* score, g3x_ext_t* out, int32_t* cells,
                                int32_t* status) {
    if (!jobs || !u8 || !score || !out || !cells || !status || n < 0) return G3X_ERR_INVALID;
    const ScoreParams sp = score_of(*score);
    uint2 pools[5];
    for (int a = 0; a < 5; ++a) {
        pools[a].x = (uint32_t)(uint8_t)sp.mat[a * 5 + 0] | ((uint32_t)(uint8_t)sp.mat[a * 5 + 1] << 8) |
                     ((uint32_t)(uint8_t)sp.mat[a * 5 + 2] << 16) | ((uint32_t)(uint8_t)sp.mat[a * 5 + 3] << 24);
        pools[a].y = (uint32_t)(uint8_t)sp.mat[a * 5 + 4] * 0x01010101u;
    }
    uint4 ge[10];
    for (int o = 0; o < 10; ++o)
        ge[o] = make_uint4(l16::ge_word(o, 0), l16::ge_word(o, 1), l16::ge_word(o, 2), l16::ge_word(o, 3));
    const bool sym = sp.oe_del == sp.oe_ins;
    for (int32_t k = 0; k < n; ++k) {
        out[k] = g3x_ext_t{0, 0, 0, 0, 0, 0};
        cells[k] = 0;
        status[k] = sym ? run_job<true>(jobs[k], u8, sp, pools, ge, &out[k], &cells[k])
                        : run_job<false>(jobs[k], u8, sp, pools, ge, &out[k], &cells[k]);
    }
    return G3X_OK;
}

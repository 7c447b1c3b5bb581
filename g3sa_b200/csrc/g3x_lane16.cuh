// g3x_lane16.cuh -- per-lane logic of the int16x2 lane-per-job kernel for batched ksw_extend2
// (bwa/src/ksw.cu:303-401), shared by the sm_100a kernel (g3x_lane16.cu) and its CPU model
// (g3x_emu16.cu, test-only).
//
// One lane runs one job through the reference's row loop.  The lane's row buffer (ksw.cu:310,
// eh[j] = {H(i-1, j-1), E(i, j)} before row i) lives in shared memory as int16 fields grouped in
// 8-column blocks: per block four int16x2 words of H and four of E, word p holding columns
// jb+p (low half) and jb+p+4 (high half).  A row is walked in aligned blocks; every step of the
// recurrence is one Blackwell DPX int16x2 instruction for two cells.
//
// The recurrence of ksw.cu:346-370, per column j of row i:
//   M = H(i-1,j-1) ? H(i-1,j-1) + S : 0;  H = max(M, E, F);
//   E' = max(E - e_del, max(M - oe_del, 0));  F' = max(F - e_ins, max(M - oe_ins, 0)).
// E and F are computed from M, never from H, so inside a row F is a max-plus prefix over the
// row's M values: with T(t) = max(M(t) - oe_ins, 0) and V(t) = max_{s<t} T(s) - (t-1-s) e_ins,
//   F(t) = max(F_in - t e_ins, V(t))           (F_in = F entering the block).
// A block computes each half's own prefix of T over its four columns (the L words: low half
// over columns 0-3, high half over 4-7), then F(4) = max(F_in - 4e, V(4)) with V(4) the low
// half's full prefix, and every F of the block from the pair (F_in, F(4)):
//   (F(p), F(p+4)) = max((F_in, F(4)) - p e, L[p-1]),     F(8) = max(F(4) - 4e, L[3].hi).
//
// Exactness in 16 bits: a job runs here only when every value of its DP fits (job_fits_int16):
// 0 <= h0, K (h0 + max_score min(qlen, tlen)) < 2^15 with K the smallest power of two
// >= 1 + max_score, small gap penalties.  Then M = H ? H + S : 0 equals min(H + S, K H) where
// H > 0 and is <= 0 where H == 0, which every use clips to 0 as the reference's 0.
//
// Band edges.  Columns left of beg are never read again (beg only grows), and the reference's
// trim (ksw.cu:388-389) only moves beg past columns whose H and E words are zero, so every such
// "dead" column holds zeros -- except those the band clamp beg >= i - w (ksw.cu:338) cuts off.
// The first block of a row therefore zeroes the H and E words left of beg as it loads them; a
// dead column then computes M <= 0, T = 0, E' = 0, F = 0 and H = 0, so it adds nothing to F or
// to the row maximum and writes zeros back, and the H word of column beg (H(i, beg-1), 0 for
// beg > 0 as ksw.cu:344-345 sets it) comes out right.  The last block keeps the words right of
// column end as they were (the band can grow back into them, ksw.cu:390-391), and leaves
// columns >= end out of the row maximum.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "g3x_core.h"

namespace g3x {
namespace l16 {

constexpr int kLB = 8;   // columns per block

// Blocks per lane: columns up to qcap + 8 (block loads reach (end - 1) | 7 <= qcap - 1 | 7, the
// row end writes column end <= qcap, the column-of-maximum search reads one block past the
// winning block, which starts at most at (qcap - 1) & ~7).
G3X_HD int blocks_of(int qcap) { return (qcap + 7) / 8 + 1; }
G3X_HD int nib_words(int qcap) { return 2 * ((qcap + 15) / 16); }
G3X_HD size_t warp_bytes(int qcap) {
    return (size_t)32 * blocks_of(qcap) * 32 + (size_t)128 * nib_words(qcap);
}

// PTX prmt (default mode): result byte k = byte (s_k & 7) of {b, a}, sign-replicated when s_k & 8.
G3X_HD uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
#if defined(__CUDA_ARCH__)
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(sel));
    return r;
#else
    const uint64_t v = (uint64_t)a | ((uint64_t)b << 32);
    uint32_t r = 0;
    for (int k = 0; k < 4; ++k) {
        const uint32_t s = (sel >> (4 * k)) & 15u;
        uint32_t byte = (uint32_t)(v >> (8 * (s & 7u))) & 0xFFu;
        if (s & 8u) byte = (byte & 0x80u) ? 0xFFu : 0u;
        r |= byte << (8 * k);
    }
    return r;
#endif
}

G3X_HD int ffs32(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __ffs(x);
#else
    return x ? __builtin_ctz(x) + 1 : 0;
#endif
}
G3X_HD int clz32(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __clz(x);
#else
    return x ? __builtin_clz(x) : 32;
#endif
}
// Index of the highest set bit, -1 for 0 (PTX bfind.u32).
G3X_HD int msb32(uint32_t x) {
#if defined(__CUDA_ARCH__)
    int r;
    asm("bfind.u32 %0, %1;" : "=r"(r) : "r"(x));
    return r;
#else
    return x ? 31 - __builtin_clz(x) : -1;
#endif
}
// Bits pos .. pos + width - 1 set, for 0 <= pos < 32 and 0 < width <= 8 (PTX bmsk.clamp.b32;
// other arguments give some mask that callers discard).
G3X_HD uint32_t bits_at(int pos, int width) {
#if defined(__CUDA_ARCH__)
    uint32_t r;
    asm("bmsk.clamp.b32 %0, %1, %2;" : "=r"(r) : "r"(pos), "r"(width));
    return r;
#else
    if (width <= 0 || pos < 0 || pos >= 32) return 0u;
    return (uint32_t)((((uint64_t)1 << (width < 32 ? width : 32)) - 1u) << pos);
#endif
}

// Scores of columns p and p+4 of a block as int16x2: byte p of lo and byte p of hi, each
// sign-extended to 16 bits.
template <int p>
G3X_HD uint32_t pair_score(uint32_t lo, uint32_t hi) {
    constexpr uint32_t sel = (uint32_t)p | ((8u | p) << 4) | ((4u + p) << 8) | ((8u | (4u + p)) << 12);
    return prmt(lo, hi, sel);
}

// Lane-interleaved layout: block b of lane L at uint4 index b * 32 + L; the 32-bit word of
// column c is word (c & 3) of its block's uint4, in the half (c & 4).
G3X_HD int word_of(int c, int L) { return ((((c >> 3) << 5) + L) << 2) + (c & 3); }

struct Planes {
    uint4* H;
    uint4* E;
    uint32_t* H32;
    uint32_t* E32;
    const uint32_t* qn;   // query codes, 8 nibbles per word, word k of lane L at qn[k * 32 + L]
};

G3X_HD void set_col(uint32_t* P, int c, int L, int32_t v) {
    uint32_t& w = P[word_of(c, L)];
    w = (c & 4) ? ((w & 0x0000FFFFu) | ((uint32_t)v << 16)) : ((w & 0xFFFF0000u) | ((uint32_t)v & 0xFFFFu));
}

// Constants of the recurrence, replicated in both halves.
struct PairConst {
    uint32_t noe_del, ne_del, noe_ins, ne_ins;
    uint32_t nt[4];     // -p e_ins
    uint32_t n4;        // -4 e_ins
    uint32_t ni[4];     // (-p e_ins, -(p + 4) e_ins)
    uint32_t kmul;      // 2^k: M = min(H + S, H * 2^k)
};

G3X_HD uint32_t rep16(int32_t v) { return ((uint32_t)v & 0xFFFFu) * 0x00010001u; }

G3X_HD PairConst pair_const(const ScoreParams& sp) {
    PairConst pc;
    pc.noe_del = rep16(-sp.oe_del);
    pc.ne_del = rep16(-sp.e_del);
    pc.noe_ins = rep16(-sp.oe_ins);
    pc.ne_ins = rep16(-sp.e_ins);
    for (int p = 0; p < 4; ++p) pc.nt[p] = rep16(-p * sp.e_ins);
    pc.n4 = rep16(-4 * sp.e_ins);
    for (int p = 0; p < 4; ++p)
        pc.ni[p] = ((uint32_t)(-p * sp.e_ins) & 0xFFFFu) | ((uint32_t)(-(p + 4) * sp.e_ins) << 16);
    pc.kmul = 1u << int16_shift(sp.max_sc);
    return pc;
}

// Masks per column offset o (0..9) within a block: in each pair word, 0xFFFF in each half whose
// column offset (p, p + 4) is >= o.
G3X_HD uint32_t ge_word(int o, int p) {
    return (p >= o ? 0x0000FFFFu : 0u) | (p + 4 >= o ? 0xFFFF0000u : 0u);
}

// State of one row of one lane.
struct RowState {
    int32_t beg, end, h1;
    uint32_t plo, phi;   // the row's score pools (target code vs query codes 0-3 and N)
    uint32_t fr;         // high half: F entering the next block
    uint32_t hlast;      // high half: H of the column before the next block
    int32_t key;         // row maximum << 16 | block index of its last block reaching it
};

// The part of a block that does not depend on F entering it: scores, M, each half's prefix of
// T (L), and the E step, which uses M only.
struct BlockA {
    uint32_t M2[4], E2[4], L2[4];
};

// kSym: oe_del == oe_ins, so the E step reuses max(M - oe_ins, 0).
template <bool kSym>
G3X_HD void phase_a(const uint32_t (&H2)[4], const uint32_t (&E2)[4], uint32_t qw, const RowState& r,
                    const PairConst& pc, BlockA& a, uint32_t (&ne)[4]) {
    const uint32_t sc_lo = prmt(r.plo, r.phi, qw);   // prmt reads selector bits 0-15 only
    const uint32_t sc_hi = prmt(r.plo, r.phi, qw >> 16);
    const uint32_t S2[4] = {pair_score<0>(sc_lo, sc_hi), pair_score<1>(sc_lo, sc_hi),
                            pair_score<2>(sc_lo, sc_hi), pair_score<3>(sc_lo, sc_hi)};
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        a.E2[p] = E2[p];
        a.M2[p] = __viaddmin_s16x2(H2[p], S2[p], H2[p] * pc.kmul);
        const uint32_t T2 = __viaddmax_s16x2(a.M2[p], pc.noe_ins, 0u);
        a.L2[p] = p == 0 ? T2 : __viaddmax_s16x2(a.L2[p - 1], pc.ne_ins, T2);
        const uint32_t te = kSym ? T2 : __viaddmax_s16x2(a.M2[p], pc.noe_del, 0u);
        ne[p] = __viaddmax_s16x2(E2[p], pc.ne_del, te);
    }
}

// The part that takes F in: (F_in, F(4)), every F and H of the block, the new H words; advances
// fr and hlast.
G3X_HD void phase_b(const BlockA& a, RowState& r, const PairConst& pc, uint32_t (&nh)[4], uint32_t (&h2)[4]) {
    const uint32_t fin = prmt(r.fr, r.fr, 0x3232u);
    const uint32_t x = __viaddmax_s16x2(fin, pc.n4, a.L2[3]);                // low half: F(4)
    const uint32_t fp = prmt(r.fr, x, 0x5432u);
    r.fr = __viaddmax_s16x2(fp, pc.n4, a.L2[3]);                             // high half: F(8)
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const uint32_t F2 = p == 0 ? fp : __viaddmax_s16x2(fp, pc.nt[p], a.L2[p - 1]);
        h2[p] = __vimax3_s16x2(a.M2[p], a.E2[p], F2);
    }
    nh[0] = prmt(r.hlast, h2[3], 0x5432u);
    nh[1] = h2[0]; nh[2] = h2[1]; nh[3] = h2[2];
    r.hlast = h2[3];
}

// The whole block on loaded (and masked) words: the new H and E words and the H of the block's
// columns (h2); advances fr and hlast.
template <bool kSym>
G3X_HD void block_core(const uint32_t (&H2)[4], const uint32_t (&E2)[4], uint32_t qw, RowState& r,
                       const PairConst& pc, uint32_t (&nh)[4], uint32_t (&ne)[4], uint32_t (&h2)[4]) {
    BlockA a;
    phase_a<kSym>(H2, E2, qw, r, pc, a, ne);
    phase_b(a, r, pc, nh, h2);
}

// Row maximum of a block (of the given H words) into the running key (max << 16) | kb: one key
// per half of the block's pair maximum, the larger of the two and the running key kept (on
// ties the later block, whose index is larger).
G3X_HD void block_max(const uint32_t (&hm)[4], int32_t kb, RowState& r) {
    const uint32_t b2 = __vimax3_s16x2(__vimax3_s16x2(hm[0], hm[1], hm[2]), hm[3], hm[3]);
    const int32_t klo = (int32_t)prmt((uint32_t)kb, b2, 0x5410u);   // (low half << 16) | kb
    const int32_t khi = (int32_t)prmt((uint32_t)kb, b2, 0x7610u);   // (high half << 16) | kb
    r.key = __vimax3_s32(r.key, klo, khi);
}

// Bit t set when column jb+t of a block's words (H and E pairs in registers) is non-zero, for the
// columns in keep (a mask within bits 0-7): every half-word pair becomes min(H + E, 1) (H, E >= 0
// below 2^15 in the band, so the sum does not wrap; columns outside keep may hold anything),
// then the four pairs are summed with weights 1-8 (each half stays below 16), which leaves
// columns 0-3 in bits 0-3 and 4-7 in bits 16-19, folded down to bits 4-7.
G3X_HD uint32_t nonzero_mask(const uint32_t (&h)[4], const uint32_t (&e)[4], uint32_t keep) {
    const uint32_t one = 0x00010001u;
    const uint32_t z0 = __viaddmin_u16x2(h[0], e[0], one), z1 = __viaddmin_u16x2(h[1], e[1], one);
    const uint32_t z2 = __viaddmin_u16x2(h[2], e[2], one), z3 = __viaddmin_u16x2(h[3], e[3], one);
    const uint32_t s = z0 + 2u * z1 + 4u * z2 + 8u * z3;
    return (s | (s >> 12)) & keep;
}

// A block strictly inside the row.
template <bool kSym>
G3X_HD void block_mid(const Planes& P, int at, int32_t kb, RowState& r, const PairConst& pc) {
    const uint4 hq = P.H[at], eq = P.E[at];
    const uint32_t H2[4] = {hq.x, hq.y, hq.z, hq.w}, E2[4] = {eq.x, eq.y, eq.z, eq.w};
    uint32_t nh[4], ne[4], h2[4];
    block_core<kSym>(H2, E2, P.qn[at], r, pc, nh, ne, h2);
    P.H[at] = make_uint4(nh[0], nh[1], nh[2], nh[3]);
    P.E[at] = make_uint4(ne[0], ne[1], ne[2], ne[3]);
    block_max(h2, kb, r);
}

// Two consecutive blocks strictly inside the row, the second only when `second` (else nothing of
// it is stored and the row state stays as the first block leaves it).  The F-independent
// phases of both blocks come first, so the two blocks' instructions interleave.
template <bool kSym>
G3X_HD void block_mid2(const Planes& P, int at, int32_t kb, bool second, RowState& r, const PairConst& pc) {
    const uint4 hq0 = P.H[at], eq0 = P.E[at], hq1 = P.H[at + 32], eq1 = P.E[at + 32];
    const uint32_t qw0 = P.qn[at], qw1 = P.qn[at + 32];
    BlockA a0, a1;
    uint32_t ne0[4], ne1[4];
    {
        const uint32_t H2[4] = {hq0.x, hq0.y, hq0.z, hq0.w}, E2[4] = {eq0.x, eq0.y, eq0.z, eq0.w};
        phase_a<kSym>(H2, E2, qw0, r, pc, a0, ne0);
    }
    {
        const uint32_t H2[4] = {hq1.x, hq1.y, hq1.z, hq1.w}, E2[4] = {eq1.x, eq1.y, eq1.z, eq1.w};
        phase_a<kSym>(H2, E2, qw1, r, pc, a1, ne1);
    }
    uint32_t nh0[4], h20[4], nh1[4], h21[4];
    phase_b(a0, r, pc, nh0, h20);
    RowState r1 = r;
    phase_b(a1, r1, pc, nh1, h21);
    P.E[at] = make_uint4(ne0[0], ne0[1], ne0[2], ne0[3]);
    P.H[at] = make_uint4(nh0[0], nh0[1], nh0[2], nh0[3]);
    block_max(h20, kb, r);
    if (second) {
        P.E[at + 32] = make_uint4(ne1[0], ne1[1], ne1[2], ne1[3]);
        P.H[at + 32] = make_uint4(nh1[0], nh1[1], nh1[2], nh1[3]);
        r.fr = r1.fr;
        r.hlast = r1.hlast;
        block_max(h21, kb + 1, r);
    }
}

// The first block of a row with two or more blocks: the words left of beg are zeroed on load.
// Returns the columns of the block at or right of beg whose new H or E word is non-zero.
template <bool kSym>
G3X_HD uint32_t block_first(const Planes& P, int at, int32_t kb, RowState& r, const PairConst& pc,
                            const uint4* ge) {
    const int32_t jb = kb << 3;
    const uint4 hq = P.H[at], eq = P.E[at];
    const uint4 A = ge[r.beg - jb];
    const uint32_t H2[4] = {hq.x & A.x, hq.y & A.y, hq.z & A.z, hq.w & A.w};
    const uint32_t E2[4] = {eq.x & A.x, eq.y & A.y, eq.z & A.z, eq.w & A.w};
    uint32_t nh[4], ne[4], h2[4];
    block_core<kSym>(H2, E2, P.qn[at], r, pc, nh, ne, h2);
    P.H[at] = make_uint4(nh[0], nh[1], nh[2], nh[3]);
    P.E[at] = make_uint4(ne[0], ne[1], ne[2], ne[3]);
    block_max(h2, kb, r);
    return nonzero_mask(nh, ne, 0xFFu << (r.beg - jb));
}

// The last block of a row (first == true: also its first, the row's only block): columns right of
// end keep their words, columns >= end stay out of the row maximum, r.h1 = H(i, end - 1).  When
// column end is in the block its words become {h1, 0} here (ksw.cu:371): its H word is H(i, end-1)
// as computed, its E word is cleared.  Returns the columns of the block up to column end whose
// new H or E word is non-zero.  mask_beg: some lane of the warp runs a one-block row (the same
// for every lane, so the branch is uniform); only then are words left of beg zeroed here.
template <bool kSym>
G3X_HD uint32_t block_last(const Planes& P, int at, int32_t kb, bool first, bool mask_beg, RowState& r,
                           const PairConst& pc, const uint4* ge) {
    const int32_t jb = kb << 3;
    const uint4 hq = P.H[at], eq = P.E[at];
    const int hi = r.end - jb;                       // 1 .. 8
    const uint4 gv = ge[hi], gw = ge[hi + 1];
    const uint32_t Hq[4] = {hq.x, hq.y, hq.z, hq.w}, Eq[4] = {eq.x, eq.y, eq.z, eq.w};
    const uint32_t V[4] = {~gv.x, ~gv.y, ~gv.z, ~gv.w};
    const uint32_t G[4] = {gw.x, gw.y, gw.z, gw.w};   // columns right of end
    uint32_t H2[4] = {Hq[0], Hq[1], Hq[2], Hq[3]}, E2[4] = {Eq[0], Eq[1], Eq[2], Eq[3]};
    if (mask_beg) {
        const uint4 A = ge[first ? r.beg - jb : 0];
        const uint32_t Am[4] = {A.x, A.y, A.z, A.w};
#pragma unroll
        for (int p = 0; p < 4; ++p) { H2[p] &= Am[p]; E2[p] &= Am[p]; }
    }
    uint32_t nh[4], ne[4], h2[4], hm[4];
    block_core<kSym>(H2, E2, P.qn[at], r, pc, nh, ne, h2);
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        nh[p] = (nh[p] & ~G[p]) | (Hq[p] & G[p]);   // columns <= end: new; beyond: as they were
        ne[p] = (ne[p] & V[p]) | (Eq[p] & G[p]);    // columns < end: new; end: 0; beyond: as they were
        hm[p] = h2[p] & V[p];
    }
    P.H[at] = make_uint4(nh[0], nh[1], nh[2], nh[3]);
    P.E[at] = make_uint4(ne[0], ne[1], ne[2], ne[3]);
    block_max(hm, kb, r);
    // H(i, end - 1): column t = hi - 1, half t >> 2 of word t & 3, taken from the words (t & 2,
    // (t & 2) + 1) by one permute of bytes off, off + 1 with off = 4 (t & 1) + 2 (t >> 2) (the
    // nibbles of 0x62624040), zero-extended (the sign of H's high byte: H >= 0)
    const int t = hi - 1;
    const bool w2 = (t & 2) != 0;
    const uint32_t off = (0x62624040u >> (t << 2)) & 0xFu;
    r.h1 = (int32_t)prmt(w2 ? h2[2] : h2[0], w2 ? h2[3] : h2[1], off * 0x1111u + 0x9910u);
    return nonzero_mask(nh, ne, 0xFFu >> (7 - (hi < 8 ? hi : 7)));
}

// Bit t set when column b+t (b a multiple of 8) has a non-zero H or E word: every half-word is
// reduced to 0 or 1 by an unsigned min, then the four pairs are summed with weights 1-8 (each
// half stays below 16), which leaves columns 0-3 in bits 0-3 and 4-7 in bits 16-19.
G3X_HD uint32_t nonzero_cols(const Planes& P, int32_t b, int lane) {
    const int at = ((b >> 3) << 5) + lane;
    const uint4 hq = P.H[at], eq = P.E[at];
    const uint32_t one = 0x00010001u;
    const uint32_t z0 = __vimin3_u16x2(hq.x | eq.x, one, one), z1 = __vimin3_u16x2(hq.y | eq.y, one, one);
    const uint32_t z2 = __vimin3_u16x2(hq.z | eq.z, one, one), z3 = __vimin3_u16x2(hq.w | eq.w, one, one);
    const uint32_t s = z0 + 2u * z1 + 4u * z2 + 8u * z3;
    return (s | (s >> 12)) & 0xFFu;
}

// The column of the row maximum (ksw.cu:362-364, the last column reaching it): the last column c
// in [beg, end) of the block in the key's low half with H(i, c) == m, the key's high half.
// Every H of those columns is <= m and one of them equals it (the key's block reached m inside
// the band), when m > 0; for m == 0 the result is meaningless and the caller discards it.
// H(i, c) sits in the H word of column c + 1: columns mjb .. mjb + 2 in the low halves of words
// 1-3, mjb + 3 .. mjb + 6 in the high halves of words 0-3, mjb + 7 in the low half of the next
// block's word 0.  max(H - m, -1) makes each half-word 0 where H == m and all ones where
// H < m (other values only outside [beg, end), masked off).
G3X_HD int32_t max_col(const Planes& P, int lane, int32_t key, int32_t beg, int32_t end) {
    const int32_t kb = key & 0xFFFF, mjb = kb << 3;
    const int at = (kb << 5) + lane;
    const uint4 hq = P.H[at];
    const uint32_t nx = P.H32[(at + 32) << 2];
    const int32_t nm = -(key >> 16);
    const uint32_t nm2 = prmt((uint32_t)nm, (uint32_t)nm, 0x1010u), lt = 0xFFFFFFFFu;
    const uint32_t d0 = __viaddmax_s16x2(hq.x, nm2, lt), d1 = __viaddmax_s16x2(hq.y, nm2, lt);
    const uint32_t d2 = __viaddmax_s16x2(hq.z, nm2, lt), d3 = __viaddmax_s16x2(hq.w, nm2, lt);
    const uint32_t dn = __viaddmax_s16x2(nx, nm2, lt);
    // bit t (low half: t = 0..3, high half: bits 16-19 for t = 4..7) set where H < m
    const uint32_t s = (d1 & 0x00010001u) | (d2 & 0x00020002u) | (d3 & 0x00040004u) |
                       (prmt(d0, dn, 0x5432u) & 0x00080008u);
    const int32_t lo = beg - mjb > 0 ? beg - mjb : 0, hi = end - mjb < kLB ? end - mjb : kLB;
    const uint32_t eq = ~(s | (s >> 12)) & bits_at(lo, hi - lo);
    return mjb + msb32(eq);
}

// Per-lane job state.
struct LaneJob {
    int job;                 // -1 = none
    int32_t qlen, tlen, w, h0;
    uint32_t t_off;
    int32_t trev;
    Commit K;
    int32_t beg, end;        // band of the next row before the clamps of ksw.cu:338-340
    uint32_t tx, tn;         // target chunk K.next >> 4: 2-bit codes and N bits
    uint64_t pv, pm;         // the plane words of the next chunk (kernel prefetch)
};

G3X_HD JobConst job_const(const LaneJob& J, const ScoreParams& sp) {
    JobConst c;
    c.qlen = J.qlen; c.tlen = J.tlen; c.w = J.w; c.h0 = J.h0;
    c.o_del = sp.o_del; c.e_del = sp.e_del; c.o_ins = sp.o_ins; c.e_ins = sp.e_ins;
    c.oe_del = sp.oe_del; c.oe_ins = sp.oe_ins; c.zdrop = sp.zdrop;
    return c;
}

// Row begin (ksw.cu:335-345): the band after the clamps, the first column's h1, the pools of the
// row's target code (target chunks as 2-bit fields x and N bits n, 16 rows per chunk).
G3X_HD void row_begin(const LaneJob& J, const ScoreParams& sp, const uint2* pools, RowState& r) {
    const int32_t i = J.K.next;
    r.beg = J.beg > i - J.w ? J.beg : i - J.w;
    r.end = J.end < i + J.w + 1 ? J.end : i + J.w + 1;
    if (r.end > J.qlen) r.end = J.qlen;
    r.h1 = 0;
    if (r.beg == 0) {
        const int32_t h = J.h0 - (sp.o_del + sp.e_del * (i + 1));
        r.h1 = h > 0 ? h : 0;
    }
    uint32_t code = (J.tx >> ((i & 15) << 1)) & 3u;
    if ((J.tn >> (i & 15)) & 1u) code = 4;
    const uint2 p = pools[code];
    r.plo = p.x;
    r.phi = p.y;
    r.fr = 0;
    r.hlast = (uint32_t)r.h1 << 16;
    r.key = 0;
}

// The row bookkeeping of ksw.cu:372-386 (the same as commit_row) with selects in place of
// branches: to-end score, cell count, new maximum or z-drop, last row.
G3X_HD void commit_row_sel(Commit& k, const JobConst& c, const RowDone& d) {
    const int32_t i = k.next;
    // ksw.cu:372-375 for gval >= 0 (gval -1: no to-end score this row); gscore starts at -1 and
    // only grows, so it is the running maximum of gval, and max_ie moves to i where gval >= 0
    // reaches it
    k.max_ie = d.gval >= (k.gscore > 0 ? k.gscore : 0) ? i : k.max_ie;
    k.gscore = d.gval > k.gscore ? d.gval : k.gscore;
    k.cells += d.ncells;
    k.next = i + 1;
    const bool up = d.m > k.best;                                            // ksw.cu:377-379
    const int32_t di = i - k.best_i, dj = d.mj - k.best_j;                   // ksw.cu:380-386
    const int32_t drop = di > dj ? k.best - d.m - (di - dj) * c.e_del : k.best - d.m - (dj - di) * c.e_ins;
    const bool zstop = !up && c.zdrop > 0 && drop > c.zdrop;
    const int32_t off = abs(d.mj - i);
    k.max_off = up ? (off > k.max_off ? off : k.max_off) : k.max_off;
    k.best = d.m > k.best ? d.m : k.best;
    k.best_i = up ? i : k.best_i;
    k.best_j = up ? d.mj : k.best_j;
    k.stop = d.m == 0 || zstop || k.next >= c.tlen;                         // ksw.cu:376, the row loop
}

// Row end (ksw.cu:371-391) for a running lane: column end's words, the row's bookkeeping, and
// the band of the next row.  mF: the columns >= beg of the row's first block with a non-zero new
// word (rows of two or more blocks); mL: those up to column end of its last block.  The first
// non-zero column from beg and the last one back from end are almost always found in them; the
// row buffer is read only when not.
G3X_HD void row_end(LaneJob& J, const Planes& P, int lane, const RowState& r, const ScoreParams& sp,
                    bool nonempty, uint32_t mF, uint32_t mL) {
    const int32_t beg = r.beg, end = r.end;
    const int32_t jb0 = beg & ~(kLB - 1), jbl = (end - 1) & ~(kLB - 1);
    // column end starts the block after the last one: its words {h1, 0} (ksw.cu:371)
    const bool end_next = nonempty && end - jbl == kLB;
    if (end_next) {
        set_col(P.H32, end, lane, r.h1);
        set_col(P.E32, end, lane, 0);
    }
    RowDone rd;
    rd.m = r.key >> 16;
    const int32_t mj = max_col(P, lane, r.key, beg, end);
    rd.mj = rd.m > 0 ? mj : -1;
    rd.gval = (nonempty ? end : beg) == J.qlen ? r.h1 : -1;
    rd.ncells = nonempty ? end - beg : 0;
    commit_row_sel(J.K, job_const(J, sp), rd);
    if (J.K.stop) return;
    // (a row that does not stop has a non-empty band)
    // ksw.cu:388-389: the first column of [beg, end) whose H or E word is non-zero, else end
    const uint32_t mk = jb0 < jbl ? mF : (mL & (0xFFu << (beg - jb0)) & (0xFFu >> (kLB - (end - jb0))));
    int32_t nb = end;
    if (mk) {
        nb = jb0 + ffs32(mk) - 1;
    } else {
        for (int32_t b = jb0 + kLB; b < end; b += kLB) {
            uint32_t m2 = nonzero_cols(P, b, lane);
            if (end - b < kLB) m2 &= 0xFFu >> (kLB - (end - b));
            if (m2) {
                nb = b + ffs32(m2) - 1;
                break;
            }
        }
    }
    // ksw.cu:390-391: the last column of [nb, end] whose word is non-zero, else nb - 1
    int32_t last = nb - 1;
    if (end_next && r.h1 != 0) {
        last = end;
    } else if (nb <= jbl + kLB - 1) {
        const uint32_t ml = nb > jbl ? mL & (0xFFu << (nb - jbl)) : mL;
        if (ml) {
            last = jbl + 31 - clz32(ml);
        } else {
            for (int32_t b = jbl - kLB; b >= (nb & ~(kLB - 1)); b -= kLB) {
                uint32_t m2 = nonzero_cols(P, b, lane);
                if (b < nb) m2 &= 0xFFu << (nb - b);
                if (m2) {
                    last = b + 31 - clz32(m2);
                    break;
                }
            }
        }
    }
    J.beg = nb;
    J.end = last + 2 < J.qlen ? last + 2 : J.qlen;
}

// All blocks of one row of one lane, in the order the kernel runs them.
// The blocks of one row of one lane as the kernel's warp runs them: kmax (>= nblk) is the most
// blocks any lane of the warp has in this row, and every lane walks the same iterations, doing
// only its own blocks: the first (masked), the middle ones two at a time (one alone when an odd
// number of them is left for the warp), the last (masked).  Returns the first block's and the
// last block's non-zero column masks for row_end in mF, mL.  any_single: some lane of the warp
// has a one-block row (nblk == 1).
template <bool kSym>
G3X_HD void row_blocks(const Planes& P, int lane, RowState& r, const PairConst& pc, const uint4* ge,
                       int nblk, int kmax, bool any_single, uint32_t& mF, uint32_t& mL) {
    mF = mL = 0;
    const int32_t kb0 = r.beg >> 3;                 // block index of the first block
    const int at0 = (kb0 << 5) + lane;              // its uint4 index in the lane-interleaved planes
    if (nblk > 1) mF = block_first<kSym>(P, at0, kb0, r, pc, ge);
    int k = 1, at = at0 + 32;
    for (; k + 1 < kmax - 1; k += 2, at += 64)
        if (k < nblk - 1) block_mid2<kSym>(P, at, kb0 + k, k + 1 < nblk - 1, r, pc);
    if (k < kmax - 1 && k < nblk - 1) block_mid<kSym>(P, at, kb0 + k, r, pc);
    if (nblk > 0)
        mL = block_last<kSym>(P, at0 + ((nblk - 1) << 5), kb0 + nblk - 1, nblk == 1, any_single, r, pc, ge);
}

// Blocks of a row with a non-empty band [beg, end).
G3X_HD int blocks_in_row(const RowState& r) {
    return r.beg < r.end ? ((r.end - 1) >> 3) - (r.beg >> 3) + 1 : 0;
}

// Row -1 of a new job in the lane's row buffer (ksw.cu:317-319), blocks 0 .. (qlen + 1) / 8:
// H(-1, c) = h0 at column 0, then max(v1 - (c - 1) e_ins, 0) with v1 = max(h0 - oe_ins, 0) up to
// column max(qlen, 1), zero beyond; E = 0.  Word p of block b holds columns 8b + p and 8b + p + 4:
// max(base - p e, 0) and max(base - (p + 4) e, 0) with base = v1 - (8b - 1) e, the value of column
// 8b, computed in int32 per block; a non-positive base leaves the block zero, and a positive one is
// below 2^15 with base - 7 e above -2^15, so the int16 steps stay in range.
G3X_HD void init_row(const Planes& P, int lane, int32_t qlen, int32_t h0, const ScoreParams& sp,
                     const PairConst& pc, const uint4* ge) {
    const int32_t v1 = h0 > sp.oe_ins ? h0 - sp.oe_ins : 0;
    const int32_t lim = (qlen > 1 ? qlen : 1) + 1;          // first column that is zero
    const int nb = ((qlen + 1) >> 3) + 1;
    for (int b = 0; b < nb; ++b) {
        const int32_t base = v1 + sp.e_ins - 8 * b * sp.e_ins;   // value of column 8b (when >= 1)
        uint32_t w[4] = {0u, 0u, 0u, 0u};
        if (base > 0) {
            const uint4 keep = ge[lim - 8 * b < 9 ? (lim - 8 * b > 0 ? lim - 8 * b : 0) : 9];
            const uint32_t k2[4] = {~keep.x, ~keep.y, ~keep.z, ~keep.w};
            const uint32_t b2 = rep16(base);
#pragma unroll
            for (int p = 0; p < 4; ++p)
                w[p] = __viaddmax_s16x2(b2, pc.ni[p], 0u) & k2[p];
        }
        if (b == 0) w[0] = (w[0] & 0xFFFF0000u) | ((uint32_t)h0 & 0xFFFFu);
        P.H[(b << 5) + lane] = make_uint4(w[0], w[1], w[2], w[3]);
        P.E[(b << 5) + lane] = make_uint4(0u, 0u, 0u, 0u);
    }
}

}  // namespace l16
}  // namespace g3x

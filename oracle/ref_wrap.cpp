/*
 * ref_wrap.cpp -- host driver around the reference's own ksw_extend2 (bwa/src/ksw.cu:303-401),
 * which build_ref.sh compiles unmodified from the reference tree into oracle/_ref/.
 * Test infrastructure only (parity pin and the timed CPU reference arm); nothing in the
 * product path links it.
 *
 * Exports (C ABI, loaded with ctypes):
 *   g3r_ksw_extend2_batch  -- n jobs over one u8 code buffer, on `threads` host threads
 *                            (dynamic 256-job chunks), outputs {score,qle,tle,gtle,gscore,max_off}.
 */
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

/* The reference's entry point, exactly as declared at bwa/src/ksw.h:33 (C++ linkage). */
int ksw_extend2(int qlen, const uint8_t *query, int tlen, const uint8_t *target, int m,
                const int8_t *mat, int o_del, int e_del, int o_ins, int e_ins, int w,
                int end_bonus, int zdrop, int h0, int *_qle, int *_tle, int *_gtle,
                int *_gscore, int *_max_off, void *d_buffer_ptr);

namespace {
struct Arena {
    char *base;
    size_t used, cap;
};
}  // namespace

/* Bump allocation with 8-byte alignment; the arena is reset per call, like the reference's
   per-batch arena that is never freed inside a batch (bwa/src/gmem_alloc.cu:69-116). */
void *g3r_arena_take(void *arena, size_t bytes, int zero)
{
    Arena *a = static_cast<Arena *>(arena);
    size_t at = (a->used + 7) & ~size_t(7);
    if (at + bytes > a->cap) abort();     /* sized by the caller: cannot happen */
    a->used = at + bytes;
    if (zero) memset(a->base + at, 0, bytes);
    return a->base + at;
}

/* Same record names as ref_seed_head.inc so the C++ symbol of g3r_seed_extend links. */
struct mem_opt_t {
    int a, b, o_del, e_del, o_ins, e_ins, pen_clip5, pen_clip3, w, zdrop;
    int8_t mat[25];
};
struct mem_seed_t { int64_t rbeg; int32_t qbeg, len; };
struct mem_alnreg_t { int64_t rb, re; int qb, qe, score, truesc, w; };
void g3r_seed_extend(const mem_opt_t *opt, int l_query, const uint8_t *query, const uint8_t *rseq,
                     const int64_t *rmax, const mem_seed_t *s, mem_alnreg_t *a, void *d_buffer_ptr);

struct RefJob {              /* same layout as the oracle's g3o_job */
    int64_t q_off, t_off;
    int32_t qlen, tlen, h0, w;
    int32_t flags, pad_;     /* 1: query reversed, 2: target reversed (aux.cu:261-265) */
};
struct RefScore {            /* same layout as the oracle's g3o_score */
    int8_t mat[25];
    int32_t o_del, e_del, o_ins, e_ins, zdrop, end_bonus;
};
struct RefExt {
    int32_t score, qle, tle, gtle, gscore, max_off;
};

/* Seed records as the oracle's g3o_seed; outputs as the oracle's g3o_reg (first 7 fields). */
struct RefSeedRec {
    int64_t read_off, win_off, rmax0, rmax1, rbeg;
    int32_t l_query, qbeg, len, pad_;
};
struct RefRegOut {
    int64_t rb, re;
    int32_t qb, qe, score, truesc, w, pad_[3];
    int64_t cells;
};

extern "C" int g3r_extend_seeds(const mem_opt_t *opt, const uint8_t *codes, const RefSeedRec *seeds,
                                int64_t n, RefRegOut *out)
{
    Arena a;
    a.cap = 1 << 22;
    a.base = static_cast<char *>(malloc(a.cap));
    for (int64_t k = 0; k < n; ++k) {
        const RefSeedRec &sr = seeds[k];
        mem_seed_t s;
        s.rbeg = sr.rbeg; s.qbeg = sr.qbeg; s.len = sr.len;
        int64_t rmax[2] = {sr.rmax0, sr.rmax1};
        mem_alnreg_t r;
        a.used = 0;
        g3r_seed_extend(opt, sr.l_query, codes + sr.read_off, codes + sr.win_off, rmax, &s, &r, &a);
        RefRegOut &o = out[k];
        memset(&o, 0, sizeof(o));
        o.rb = r.rb; o.re = r.re; o.qb = r.qb; o.qe = r.qe; o.score = r.score;
        o.truesc = r.truesc; o.w = r.w;
    }
    free(a.base);
    return 0;
}

extern "C" int g3r_ksw_extend2_batch(const RefJob *jobs, int64_t n, const uint8_t *codes,
                                     const RefScore *sc, RefExt *out, int threads)
{
    std::atomic<int64_t> next(0);
    auto work = [&]() {
        Arena a;
        a.cap = 0;
        a.base = nullptr;
        std::vector<uint8_t> qr, tr;
        for (;;) {
            int64_t b = next.fetch_add(256);
            if (b >= n) break;
            int64_t e = b + 256 < n ? b + 256 : n;
            for (int64_t k = b; k < e; ++k) {
                const RefJob &j = jobs[k];
                size_t need = size_t(j.qlen) * 5 + (size_t(j.qlen) + 2) * 8 + 64;
                if (need > a.cap) {
                    free(a.base);
                    a.cap = need * 2;
                    a.base = static_cast<char *>(malloc(a.cap));
                }
                a.used = 0;
                RefExt &o = out[k];
                const uint8_t *q = codes + j.q_off, *t = codes + j.t_off;
                if (j.flags & 1) {
                    qr.assign(q, q + j.qlen);
                    std::reverse(qr.begin(), qr.end());
                    q = qr.data();
                }
                if (j.flags & 2) {
                    tr.assign(t, t + j.tlen);
                    std::reverse(tr.begin(), tr.end());
                    t = tr.data();
                }
                o.score = ksw_extend2(j.qlen, q, j.tlen, t, 5, sc->mat,
                                      sc->o_del, sc->e_del, sc->o_ins, sc->e_ins, j.w,
                                      sc->end_bonus, sc->zdrop, j.h0, &o.qle, &o.tle, &o.gtle,
                                      &o.gscore, &o.max_off, &a);
            }
        }
        free(a.base);
    };
    if (threads <= 1) {
        work();
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t) pool.emplace_back(work);
        for (auto &t : pool) t.join();
    }
    return 0;
}

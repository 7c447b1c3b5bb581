/*
 * ksw_oracle.c -- CPU restatement of BWA-MEM seed extension, used ONLY as test
 * infrastructure (parity checker and CPU baseline).  Nothing in the product path
 * (g3sa_b200/) links, loads or calls this file.
 *
 * What it restates (paths are relative to the sunwookim028/G3SA tree):
 *   - ksw_extend2:            bwa/src/ksw.cu:299-401   (eh_t + the banded extension)
 *   - band-retry driver:      bwa/src/aux.cu:250-301   (left/right extension of one seed,
 *                                                       MAX_BAND_TRY = 2, aux.cuh:401)
 *   - cal_max_gap:            bwa/src/aux.cu:168-175
 *   - mem_chain2aln:          bwa/src/aux.cu:178-315 with the window fetch of
 *                             bwa/src/bntseq.cu:7-87
 *   - ksw_global2 + NM/MD:    bwa/src/ksw.cu:694-809, bwa/src/aux.cu:2830-2861
 *   - traceback pairs:        bwa/src/aux.cu:506-513, 2698-2745 (FINALIZEALN_preprocessing2)
 *   - ksw_align2 (16-bit):    bwa/src/ksw.cu:18-64, 155-262, 271-292 (ksw_qinit, ksw_i16)
 *   - seed filter:            bwa/src/aux.cu:117-162 (mem_seed_sw, mem_flt_chained_seeds)
 *
 * Parity pin: each restatement is checked against the reference's own lines compiled from
 * its source (oracle/build_ref.sh -> oracle/_ref/libksw_ref.so) on seeded inputs and edge
 * cases (tests/test_oracle.py, test_chain_oracle.py, test_global_oracle.py,
 * test_tbpair_oracle.py, test_sw_oracle.py, test_seedflt_oracle.py), and against the
 * committed golden vectors in tests/golden/ that were generated from that compiled
 * reference.
 *
 * Extra output not present in the reference: the number of DP cells evaluated
 * (the trip count of the inner loop at ksw.cu:346, summed over the executed rows,
 * including the row that breaks), and the number of target rows entered.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <stdio.h>
#include <math.h>

typedef struct { int32_t h, e; } g3o_eh;          /* ksw.cu:299-301 */

typedef struct {
    int32_t score, qle, tle, gtle, gscore, max_off;  /* ksw_extend2 return + out params */
} g3o_ext;

/* Band clamp of ksw.cu:321-329: (int)((double)(qlen*max + end_bonus - o)/e + 1.), >= 1. */
static int g3o_gap_limit(int qlen, int max_sc, int end_bonus, int o, int e)
{
    int v = (int)((double)(qlen * max_sc + end_bonus - o) / e + 1.);
    return v > 1 ? v : 1;
}

/*
 * One banded extension.  Same argument meaning as ksw_extend2 (ksw.h:33); scratch is
 * malloc'd here instead of coming from the device arena.  *cells / *rows receive the
 * work counters (may be NULL).
 */
static int g3o_extend_impl(int qlen, const uint8_t *query, int tlen, const uint8_t *target,
                           int m, const int8_t *mat, int o_del, int e_del, int o_ins, int e_ins,
                           int w, int end_bonus, int zdrop, int h0,
                           int *qle_out, int *tle_out, int *gtle_out, int *gscore_out,
                           int *max_off_out, int64_t *cells_out, int32_t *rows_out,
                           int clean_stale, int32_t *stale_reads)
{
    const int oe_del = o_del + e_del, oe_ins = o_ins + e_ins;
    int8_t *prof = (int8_t *)malloc((size_t)(qlen > 0 ? qlen : 1) * m);
    /* qlen + 2 entries: the reference writes eh[1] even when qlen == 0 (an arena slot
       past its qlen + 1 entries that is never read back); keep that write in bounds. */
    g3o_eh *row = (g3o_eh *)calloc((size_t)qlen + 2, sizeof(g3o_eh));
    int64_t cells = 0;
    int32_t rows = 0;

    /* query profile, ksw.cu:312-315: prof[k*qlen + j] = mat[k*m + query[j]] */
    for (int k = 0; k < m; ++k)
        for (int j = 0; j < qlen; ++j)
            prof[k * qlen + j] = mat[k * m + query[j]];

    /* row "-1", ksw.cu:317-319 */
    row[0].h = h0;
    row[1].h = h0 > oe_ins ? h0 - oe_ins : 0;
    for (int j = 2; j <= qlen && row[j - 1].h > e_ins; ++j)
        row[j].h = row[j - 1].h - e_ins;

    /* band clamp, ksw.cu:321-329 */
    int max_sc = 0;
    for (int k = 0; k < m * m; ++k)
        if (mat[k] > max_sc) max_sc = mat[k];
    {
        int lim = g3o_gap_limit(qlen, max_sc, end_bonus, o_ins, e_ins);
        if (w > lim) w = lim;
        lim = g3o_gap_limit(qlen, max_sc, end_bonus, o_del, e_del);
        if (w > lim) w = lim;
    }

    int best = h0, best_i = -1, best_j = -1;   /* ksw.cu:331 */
    int prev_end = -1;                          /* end of the previous row (-1: row 0) */
    int32_t stale = 0;
    int g_best = -1, g_row = -1;                /* gscore, max_ie */
    int off_max = 0;
    int beg = 0, end = qlen;

    for (int i = 0; i < tlen; ++i) {           /* ksw.cu:334 */
        const int8_t *sc = &prof[target[i] * qlen];
        int f = 0, hleft, rmax = 0, rmax_j = -1, j;
        ++rows;
        if (beg < i - w) beg = i - w;           /* ksw.cu:338-340 */
        if (end > i + w + 1) end = i + w + 1;
        if (end > qlen) end = qlen;
        if (beg == 0) {                         /* ksw.cu:342-345: first column */
            hleft = h0 - (o_del + e_del * (i + 1));
            if (hleft < 0) hleft = 0;
        } else {
            hleft = 0;
        }
        for (j = beg; j < end; ++j) {           /* ksw.cu:346-370 */
            int diag = row[j].h, e = row[j].e, mm, h, t;
            if (prev_end >= 0 && j > prev_end) {
                /* entry not written by the previous row: left over from an older row
                   (the band grew by two columns, ksw.cu:390) */
                if (diag | e) ++stale;
                if (clean_stale) { diag = 0; e = 0; }
            }
            row[j].h = hleft;
            mm = diag ? diag + sc[j] : 0;
            h = mm > e ? mm : e;
            if (f > h) h = f;
            hleft = h;
            if (!(rmax > h)) rmax_j = j;        /* ties move to the later column */
            if (h > rmax) rmax = h;
            t = mm - oe_del; if (t < 0) t = 0;
            e -= e_del;     if (e < t) e = t;
            row[j].e = e;
            t = mm - oe_ins; if (t < 0) t = 0;
            f -= e_ins;     if (f < t) f = t;
        }
        cells += (end > beg) ? (end - beg) : 0;
        row[end].h = hleft;                     /* ksw.cu:371 */
        row[end].e = 0;
        prev_end = end;
        if (j == qlen) {                        /* ksw.cu:372-375: to-end score */
            if (!(g_best > hleft)) g_row = i;
            if (hleft > g_best) g_best = hleft;
        }
        if (rmax == 0) break;                   /* ksw.cu:376 */
        if (rmax > best) {                      /* ksw.cu:377-379 */
            best = rmax; best_i = i; best_j = rmax_j;
            {
                int d = rmax_j - i; if (d < 0) d = -d;
                if (d > off_max) off_max = d;
            }
        } else if (zdrop > 0) {                 /* ksw.cu:380-386 */
            int di = i - best_i, dj = rmax_j - best_j;
            if (di > dj) {
                if (best - rmax - (di - dj) * e_del > zdrop) break;
            } else {
                if (best - rmax - (dj - di) * e_ins > zdrop) break;
            }
        }
        /* ksw.cu:388-391: shrink the band to the non-zero span of this row */
        for (j = beg; j < end && row[j].h == 0 && row[j].e == 0; ++j) ;
        beg = j;
        for (j = end; j >= beg && row[j].h == 0 && row[j].e == 0; --j) ;
        end = j + 2 < qlen ? j + 2 : qlen;
    }
    free(row);
    free(prof);
    if (qle_out) *qle_out = best_j + 1;        /* ksw.cu:395-400 */
    if (tle_out) *tle_out = best_i + 1;
    if (gtle_out) *gtle_out = g_row + 1;
    if (gscore_out) *gscore_out = g_best;
    if (max_off_out) *max_off_out = off_max;
    if (cells_out) *cells_out = cells;
    if (rows_out) *rows_out = rows;
    if (stale_reads) *stale_reads = stale;
    return best;
}

int g3o_ksw_extend2(int qlen, const uint8_t *query, int tlen, const uint8_t *target,
                    int m, const int8_t *mat, int o_del, int e_del, int o_ins, int e_ins,
                    int w, int end_bonus, int zdrop, int h0,
                    int *qle_out, int *tle_out, int *gtle_out, int *gscore_out,
                    int *max_off_out, int64_t *cells_out, int32_t *rows_out)
{
    return g3o_extend_impl(qlen, query, tlen, target, m, mat, o_del, e_del, o_ins, e_ins, w,
                           end_bonus, zdrop, h0, qle_out, tle_out, gtle_out, gscore_out,
                           max_off_out, cells_out, rows_out, 0, NULL);
}

/* Test-only probe: the same extension with stale buffer entries read as zero when
   clean_stale != 0, and the count of non-zero stale reads.  Used to find jobs whose
   result depends on the reference's stale-entry reads (they become known-answer tests). */
int g3o_ksw_extend2_probe(int qlen, const uint8_t *query, int tlen, const uint8_t *target,
                          const int8_t *mat, int o_del, int e_del, int o_ins, int e_ins, int w,
                          int end_bonus, int zdrop, int h0, int clean_stale, int32_t *out6,
                          int32_t *stale_reads)
{
    out6[0] = g3o_extend_impl(qlen, query, tlen, target, 5, mat, o_del, e_del, o_ins, e_ins, w,
                              end_bonus, zdrop, h0, &out6[1], &out6[2], &out6[3], &out6[4],
                              &out6[5], NULL, NULL, clean_stale, stale_reads);
    return out6[0];
}

/* ---------------------------------------------------------------------------------- */
/* Batched form: jobs index into one u8 code buffer.                                    */
/* ---------------------------------------------------------------------------------- */

#define G3O_QREV 1           /* query read backwards from q_off + qlen - 1 */
#define G3O_TREV 2           /* target read backwards */
typedef struct {
    int64_t q_off, t_off;        /* byte offsets into codes[] */
    int32_t qlen, tlen, h0, w;
    int32_t flags, pad_;         /* G3O_QREV / G3O_TREV: the reversed copies mem_chain2aln
                                    makes for the left extension (aux.cu:261-265) */
} g3o_job;

typedef struct {
    int8_t mat[25];
    int32_t o_del, e_del, o_ins, e_ins, zdrop, end_bonus;
} g3o_score;

typedef struct {
    const g3o_job *jobs;
    const uint8_t *codes;
    const g3o_score *sc;
    g3o_ext *out;
    int64_t *cells;
    int32_t *rows;
    int64_t n;
    int64_t next;                /* shared work counter */
    pthread_mutex_t lock;
} g3o_batch_ctx;

static const uint8_t *g3o_view(const uint8_t *src, int32_t len, int rev, uint8_t **buf)
{
    if (!rev) return src;
    *buf = (uint8_t *)malloc((size_t)len + 1);
    for (int32_t k = 0; k < len; ++k) (*buf)[k] = src[len - 1 - k];
    return *buf;
}

static void g3o_run_one(const g3o_batch_ctx *c, int64_t k)
{
    const g3o_job *jb = &c->jobs[k];
    g3o_ext *o = &c->out[k];
    uint8_t *qb = NULL, *tb = NULL;
    const uint8_t *q = g3o_view(c->codes + jb->q_off, jb->qlen, jb->flags & G3O_QREV, &qb);
    const uint8_t *t = g3o_view(c->codes + jb->t_off, jb->tlen, jb->flags & G3O_TREV, &tb);
    o->score = g3o_ksw_extend2(jb->qlen, q, jb->tlen, t,
                               5, c->sc->mat, c->sc->o_del, c->sc->e_del, c->sc->o_ins,
                               c->sc->e_ins, jb->w, c->sc->end_bonus, c->sc->zdrop, jb->h0,
                               &o->qle, &o->tle, &o->gtle, &o->gscore, &o->max_off,
                               c->cells ? &c->cells[k] : NULL, c->rows ? &c->rows[k] : NULL);
    free(qb);
    free(tb);
}

static void *g3o_worker(void *arg)
{
    g3o_batch_ctx *c = (g3o_batch_ctx *)arg;
    for (;;) {
        int64_t b, e;
        pthread_mutex_lock(&c->lock);
        b = c->next;
        c->next += 256;
        pthread_mutex_unlock(&c->lock);
        if (b >= c->n) break;
        e = b + 256 < c->n ? b + 256 : c->n;
        for (int64_t k = b; k < e; ++k) g3o_run_one(c, k);
    }
    return NULL;
}

/* Runs n jobs on `threads` host threads (1 = the calling thread only). */
int g3o_extend_batch(const g3o_job *jobs, int64_t n, const uint8_t *codes, const g3o_score *sc,
                     g3o_ext *out, int64_t *cells, int32_t *rows, int threads)
{
    g3o_batch_ctx c;
    c.jobs = jobs; c.codes = codes; c.sc = sc; c.out = out; c.cells = cells; c.rows = rows;
    c.n = n; c.next = 0;
    pthread_mutex_init(&c.lock, NULL);
    if (threads <= 1) {
        g3o_worker(&c);
    } else {
        pthread_t *tid = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)threads);
        for (int t = 0; t < threads; ++t) pthread_create(&tid[t], NULL, g3o_worker, &c);
        for (int t = 0; t < threads; ++t) pthread_join(tid[t], NULL);
        free(tid);
    }
    pthread_mutex_destroy(&c.lock);
    return 0;
}

/* ---------------------------------------------------------------------------------- */
/* Seed-level driver: left + right extension with band retry, aux.cu:250-301.           */
/* ---------------------------------------------------------------------------------- */

typedef struct {
    int32_t a, o_del, e_del, o_ins, e_ins, w, zdrop, pen_clip5, pen_clip3;
    int8_t mat[25];
} g3o_opt;

typedef struct {
    int64_t read_off;            /* byte offset of the read in codes[] */
    int64_t win_off;             /* byte offset of the reference window rseq[] in codes[] */
    int64_t rmax0, rmax1;        /* window [rmax0, rmax1) in reference coordinates */
    int64_t rbeg;                /* seed start on the reference */
    int32_t l_query, qbeg, len;  /* read length, seed start on the read, seed length */
} g3o_seed;

typedef struct {
    int64_t rb, re;
    int32_t qb, qe, score, truesc, w;
    int32_t tries_left, tries_right;    /* ksw_extend2 calls made on each side */
    int64_t cells;                       /* DP cells over all calls of this seed */
} g3o_reg;

/* aux.cu:168-175 */
int g3o_cal_max_gap(const g3o_opt *opt, int qlen)
{
    int l_del = (int)((double)(qlen * opt->a - opt->o_del) / opt->e_del + 1.);
    int l_ins = (int)((double)(qlen * opt->a - opt->o_ins) / opt->e_ins + 1.);
    int l = l_del > l_ins ? l_del : l_ins;
    l = l > 1 ? l : 1;
    return l < opt->w << 1 ? l : opt->w << 1;
}

void g3o_extend_seed(const g3o_opt *opt, const uint8_t *codes, const g3o_seed *s, g3o_reg *a)
{
    const uint8_t *query = codes + s->read_off;
    const uint8_t *rseq = codes + s->win_off;
    int aw0 = opt->w, aw1 = opt->w;
    int64_t cells = 0, c1;
    memset(a, 0, sizeof(*a));
    a->score = a->truesc = -1;
    if (s->qbeg) {                                          /* aux.cu:258-281 */
        int qle, tle, gtle, gscore, max_off;
        int ql = s->qbeg;
        int64_t tl = s->rbeg - s->rmax0;
        uint8_t *qs = (uint8_t *)malloc((size_t)ql + 1), *rs = (uint8_t *)malloc((size_t)tl + 1);
        for (int i = 0; i < ql; ++i) qs[i] = query[ql - 1 - i];
        for (int64_t i = 0; i < tl; ++i) rs[i] = rseq[tl - 1 - i];
        for (int i = 0; i < 2; ++i) {                       /* MAX_BAND_TRY = 2 */
            int prev = a->score;
            aw0 = opt->w << i;
            a->score = g3o_ksw_extend2(ql, qs, (int)tl, rs, 5, opt->mat, opt->o_del, opt->e_del,
                                       opt->o_ins, opt->e_ins, aw0, opt->pen_clip5, opt->zdrop,
                                       s->len * opt->a, &qle, &tle, &gtle, &gscore, &max_off,
                                       &c1, NULL);
            cells += c1;
            a->tries_left = i + 1;
            if (a->score == prev || max_off < (aw0 >> 1) + (aw0 >> 2)) break;
        }
        if (gscore <= 0 || gscore <= a->score - opt->pen_clip5) {
            a->qb = s->qbeg - qle; a->rb = s->rbeg - tle; a->truesc = a->score;
        } else {
            a->qb = 0; a->rb = s->rbeg - gtle; a->truesc = gscore;
        }
        free(qs); free(rs);
    } else {
        a->score = a->truesc = s->len * opt->a; a->qb = 0; a->rb = s->rbeg;
    }
    if (s->qbeg + s->len != s->l_query) {                   /* aux.cu:283-301 */
        int qle, tle, gtle, gscore, max_off, sc0 = a->score;
        int qe = s->qbeg + s->len;
        int64_t re = s->rbeg + s->len - s->rmax0;
        for (int i = 0; i < 2; ++i) {
            int prev = a->score;
            aw1 = opt->w << i;
            a->score = g3o_ksw_extend2(s->l_query - qe, query + qe,
                                       (int)(s->rmax1 - s->rmax0 - re), rseq + re, 5, opt->mat,
                                       opt->o_del, opt->e_del, opt->o_ins, opt->e_ins, aw1,
                                       opt->pen_clip3, opt->zdrop, sc0, &qle, &tle, &gtle,
                                       &gscore, &max_off, &c1, NULL);
            cells += c1;
            a->tries_right = i + 1;
            if (a->score == prev || max_off < (aw1 >> 1) + (aw1 >> 2)) break;
        }
        if (gscore <= 0 || gscore <= a->score - opt->pen_clip3) {
            a->qe = qe + qle; a->re = s->rmax0 + re + tle; a->truesc += a->score - sc0;
        } else {
            a->qe = s->l_query; a->re = s->rmax0 + re + gtle; a->truesc += gscore - sc0;
        }
    } else {
        a->qe = s->l_query; a->re = s->rbeg + s->len;
    }
    a->w = aw0 > aw1 ? aw0 : aw1;
    a->cells = cells;
}

void g3o_extend_seeds(const g3o_opt *opt, const uint8_t *codes, const g3o_seed *seeds,
                      int64_t n, g3o_reg *out)
{
    for (int64_t k = 0; k < n; ++k) g3o_extend_seed(opt, codes, &seeds[k], &out[k]);
}

/* Test-only: flags[k] = 1 when job k's outputs change if stale buffer entries are read as
   zero, 0 otherwise (stale[k] = number of non-zero stale reads). */
void g3o_stale_scan(const g3o_job *jobs, int64_t n, const uint8_t *codes, const g3o_score *sc,
                    int32_t *flags, int32_t *stale)
{
    for (int64_t k = 0; k < n; ++k) {
        const g3o_job *jb = &jobs[k];
        uint8_t *qb = NULL, *tb = NULL;
        const uint8_t *q = g3o_view(codes + jb->q_off, jb->qlen, jb->flags & G3O_QREV, &qb);
        const uint8_t *t = g3o_view(codes + jb->t_off, jb->tlen, jb->flags & G3O_TREV, &tb);
        int32_t a[6], b[6], st = 0, st2 = 0;
        g3o_ksw_extend2_probe(jb->qlen, q, jb->tlen, t, sc->mat, sc->o_del, sc->e_del, sc->o_ins,
                              sc->e_ins, jb->w, sc->end_bonus, sc->zdrop, jb->h0, 0, a, &st);
        flags[k] = 0;
        stale[k] = st;
        if (st) {
            g3o_ksw_extend2_probe(jb->qlen, q, jb->tlen, t, sc->mat, sc->o_del, sc->e_del, sc->o_ins,
                                  sc->e_ins, jb->w, sc->end_bonus, sc->zdrop, jb->h0, 1, b, &st2);
            flags[k] = memcmp(a, b, sizeof(a)) != 0;
        }
        free(qb);
        free(tb);
    }
}

/* ---------------------------------------------------------------------------------- */
/* Chain level: mem_chain2aln (aux.cu:178-315) with the window fetch of                 */
/* bns_fetch_seq_gpu (bntseq.cu:62-87).  The reference is given as one sequence of      */
/* 2*l_pac codes at codes[ref_off]: the forward strand, then its reverse complement     */
/* (position p >= l_pac holds 3 - forward[2*l_pac - 1 - p], what bns_get_seq_gpu reads  */
/* for the reverse strand, bntseq.cu:39-60), so a window [b, e) is codes[ref_off + b].  */
/* ---------------------------------------------------------------------------------- */

typedef struct { int64_t rbeg; int32_t qbeg, len, score, pad_; } g3o_cseed;      /* mem_seed_t */
typedef struct { int32_t seed_beg, n, rid; float frac_rep; } g3o_chain;           /* mem_chain_t */
typedef struct { int64_t read_off; int32_t l_query, chain_beg, n_chains, pad_; } g3o_read;
typedef struct { int64_t offset; int32_t len, pad_; } g3o_ann;                     /* bntann1_t */
typedef struct {                                                                    /* mem_alnreg_t */
    int64_t rb, re;
    int32_t qb, qe, rid, score, truesc, w, seedcov, seedlen0;
    float frac_rep;
    int32_t pad_;
} g3o_alnreg;

/* The contig holding forward position pos_f: the last one whose offset is <= pos_f
   (bns_pos2rid_gpu, bntseq.cu:7-21). */
static int g3o_pos2rid(const g3o_ann *anns, int n_seqs, int64_t pos_f)
{
    int lo = 0, hi = n_seqs;           /* first index with offset > pos_f, in [lo, hi] */
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (anns[mid].offset <= pos_f) lo = mid + 1; else hi = mid;
    }
    return lo > 0 ? lo - 1 : 0;
}

/* bns_fetch_seq_gpu's clipping of the window [*b, *e) to the contig (and strand) of
   position mid (bntseq.cu:62-80). */
static void g3o_clip_window(const g3o_ann *anns, int n_seqs, int64_t l_pac, int64_t *b,
                            int64_t mid, int64_t *e)
{
    if (*e < *b) { int64_t t = *b; *b = *e; *e = t; }
    const int rev = mid >= l_pac;
    const int rid = g3o_pos2rid(anns, n_seqs, rev ? (l_pac << 1) - 1 - mid : mid);
    int64_t lo = anns[rid].offset, hi = lo + anns[rid].len;
    if (rev) { const int64_t t = lo; lo = (l_pac << 1) - hi; hi = (l_pac << 1) - t; }
    if (*b < lo) *b = lo;
    if (*e > hi) *e = hi;
}

static int g3o_cmp_u64(const void *x, const void *y)
{
    const uint64_t a = *(const uint64_t *)x, b = *(const uint64_t *)y;
    return a < b ? -1 : a > b;
}

/* Is seed s (almost) inside region p: fully contained, not much longer than p's seed, and
   on p's diagonal band ahead of or behind the seed (aux.cu:217-231). */
static int g3o_around(const g3o_opt *opt, int l_query, const g3o_cseed *s, const g3o_alnreg *p)
{
    if (s->rbeg < p->rb || s->rbeg + s->len > p->re || s->qbeg < p->qb || s->qbeg + s->len > p->qe)
        return 0;
    if (s->len - p->seedlen0 > .1 * l_query) return 0;
    int qd = s->qbeg - p->qb;
    int64_t rd = s->rbeg - p->rb;
    int gap = g3o_cal_max_gap(opt, (int)(qd < rd ? qd : rd));
    int w = gap < p->w ? gap : p->w;
    if (qd - rd < w && rd - qd < w) return 1;
    qd = p->qe - (s->qbeg + s->len);
    rd = p->re - (s->rbeg + s->len);
    gap = g3o_cal_max_gap(opt, (int)(qd < rd ? qd : rd));
    w = gap < p->w ? gap : p->w;
    return qd - rd < w && rd - qd < w;
}

/* One chain of a read; av/nav = the read's regions so far, appended to. */
static void g3o_chain2aln_one(const g3o_opt *opt, const uint8_t *codes, int64_t ref_off,
                              int64_t l_pac, const g3o_ann *anns, int n_seqs, int64_t read_off,
                              int l_query, const g3o_chain *c, const g3o_cseed *all_seeds,
                              g3o_alnreg *av, int32_t *nav, int64_t *cells)
{
    const int n = c->n;
    if (n == 0) return;
    const g3o_cseed *cs = all_seeds + c->seed_beg;
    /* the widest span any seed can reach (aux.cu:186-205) */
    int64_t r0 = l_pac << 1, r1 = 0;
    for (int i = 0; i < n; ++i) {
        const g3o_cseed *t = &cs[i];
        const int tail = l_query - t->qbeg - t->len;
        const int64_t b = t->rbeg - (t->qbeg + g3o_cal_max_gap(opt, t->qbeg));
        const int64_t e = t->rbeg + t->len + (tail + g3o_cal_max_gap(opt, tail));
        if (b < r0) r0 = b;
        if (e > r1) r1 = e;
    }
    if (r0 < 0) r0 = 0;
    if (r1 > l_pac << 1) r1 = l_pac << 1;
    if (r0 < l_pac && l_pac < r1) {              /* one strand only: the first seed's */
        if (cs[0].rbeg < l_pac) r1 = l_pac; else r0 = l_pac;
    }
    g3o_clip_window(anns, n_seqs, l_pac, &r0, cs[0].rbeg, &r1);

    /* seeds by decreasing (score, index) (aux.cu:207-212); a key set to 0 marks a skip */
    uint64_t *srt = (uint64_t *)malloc((size_t)n * sizeof(uint64_t));
    for (int i = 0; i < n; ++i) srt[i] = (uint64_t)cs[i].score << 32 | (uint64_t)i;
    qsort(srt, (size_t)n, sizeof(uint64_t), g3o_cmp_u64);

    for (int k = n - 1; k >= 0; --k) {
        const g3o_cseed *s = &cs[(uint32_t)srt[k]];
        int i = 0;
        while (i < *nav && !g3o_around(opt, l_query, s, &av[i])) ++i;
        if (i < *nav) {
            /* contained: extend anyway only when an earlier, long enough seed overlaps it on
               another diagonal (aux.cu:234-244) */
            int j;
            for (j = k + 1; j < n; ++j) {
                if (srt[j] == 0) continue;
                const g3o_cseed *t = &cs[(uint32_t)srt[j]];
                if (t->len < s->len * .95) continue;
                if (s->qbeg <= t->qbeg && s->qbeg + s->len - t->qbeg >= s->len >> 2 &&
                    t->qbeg - s->qbeg != t->rbeg - s->rbeg) break;
                if (t->qbeg <= s->qbeg && t->qbeg + t->len - s->qbeg >= s->len >> 2 &&
                    s->qbeg - t->qbeg != s->rbeg - t->rbeg) break;
            }
            if (j == n) { srt[k] = 0; continue; }
        }
        g3o_alnreg *a = &av[(*nav)++];
        memset(a, 0, sizeof(*a));
        g3o_seed gs;
        gs.read_off = read_off; gs.win_off = ref_off + r0; gs.rmax0 = r0; gs.rmax1 = r1;
        gs.rbeg = s->rbeg; gs.l_query = l_query; gs.qbeg = s->qbeg; gs.len = s->len;
        g3o_reg r;
        g3o_extend_seed(opt, codes, &gs, &r);            /* aux.cu:253-301, 309 */
        if (cells) *cells += r.cells;
        a->rb = r.rb; a->re = r.re; a->qb = r.qb; a->qe = r.qe;
        a->score = r.score; a->truesc = r.truesc; a->w = r.w;
        a->rid = c->rid;
        for (int t = 0; t < n; ++t) {                    /* seedcov, aux.cu:303-307 */
            const g3o_cseed *u = &cs[t];
            if (u->qbeg >= a->qb && u->qbeg + u->len <= a->qe && u->rbeg >= a->rb &&
                u->rbeg + u->len <= a->re)
                a->seedcov += u->len;
        }
        a->seedlen0 = s->len;
        a->frac_rep = c->frac_rep;
    }
    free(srt);
}

/* Every read's chains in order; read r's regions go to regs[chains[chain_beg].seed_beg ...]
   (a read yields at most one region per seed), their number to nregs[r]. */
void g3o_chain2aln_reads(const g3o_opt *opt, const uint8_t *codes, int64_t ref_off, int64_t l_pac,
                         const g3o_ann *anns, int n_seqs, const g3o_read *reads, int64_t n_reads,
                         const g3o_chain *chains, const g3o_cseed *seeds, g3o_alnreg *regs,
                         int32_t *nregs, int64_t *cells)
{
    for (int64_t r = 0; r < n_reads; ++r) {
        const g3o_read *rd = &reads[r];
        int32_t nav = 0;
        if (rd->n_chains > 0) {
            g3o_alnreg *av = regs + chains[rd->chain_beg].seed_beg;
            for (int ch = 0; ch < rd->n_chains; ++ch)
                g3o_chain2aln_one(opt, codes, ref_off, l_pac, anns, n_seqs, rd->read_off, rd->l_query,
                                  &chains[rd->chain_beg + ch], seeds, av, &nav, cells ? cells + r : NULL);
        }
        nregs[r] = nav;
    }
}

/* ---------------------------------------------------------------------------------- */
/* Banded global alignment with backtrack: ksw_global2 (ksw.cu:706-809) and the CIGAR  */
/* run merging of push_cigar (ksw.cu:694-704).  Outside the band the DP holds          */
/* -0x40000000 (ksw.cu:548).                                                            */
/* ---------------------------------------------------------------------------------- */

#define G3O_NEG_INF (-0x40000000)

static void g3o_push_op(uint32_t *cig, int *n, int op, int len)
{
    if (*n > 0 && (int)(cig[*n - 1] & 0xf) == op) cig[*n - 1] += (uint32_t)len << 4;
    else cig[(*n)++] = (uint32_t)len << 4 | (uint32_t)op;
}

/* Score of the best global alignment in the band |i - j| <= w; with cigar != NULL the
   CIGAR (BAM order: len << 4 | op, 0 = M, 1 = I, 2 = D) goes there (room for qlen + tlen + 2
   operations) and its length to *n_cigar, 0 when no alignment in the band reaches the last
   cell (score <= -2^29).  *cells receives the DP cells (may be NULL). */
int g3o_ksw_global2(int qlen, const uint8_t *query, int tlen, const uint8_t *target,
                    const int8_t *mat, int o_del, int e_del, int o_ins, int e_ins, int w,
                    int *n_cigar, uint32_t *cigar, int64_t *cells)
{
    const int oe_del = o_del + e_del, oe_ins = o_ins + e_ins;
    const int ncol = qlen < 2 * w + 1 ? qlen : 2 * w + 1;
    uint8_t *z = cigar && ncol > 0 && tlen > 0 ? (uint8_t *)malloc((size_t)ncol * tlen) : NULL;
    int32_t *H = (int32_t *)malloc(sizeof(int32_t) * ((size_t)qlen + 1));
    int32_t *E = (int32_t *)malloc(sizeof(int32_t) * ((size_t)qlen + 1));
    int64_t nc = 0;
    H[0] = 0; E[0] = G3O_NEG_INF;                           /* the first row */
    for (int j = 1; j <= qlen; ++j) {
        H[j] = j <= w ? -(o_ins + e_ins * j) : G3O_NEG_INF;
        E[j] = G3O_NEG_INF;
    }
    for (int i = 0; i < tlen; ++i) {
        const int beg = i > w ? i - w : 0, end = i + w + 1 < qlen ? i + w + 1 : qlen;
        const int8_t *row = mat + target[i] * 5;
        int32_t f = G3O_NEG_INF;
        int32_t h1 = beg == 0 ? -(o_del + e_del * (i + 1)) : G3O_NEG_INF;
        for (int j = beg; j < end; ++j) {
            /* H[j] = H(i-1, j-1), E[j] = E(i, j), f = F(i, j), h1 = H(i, j-1) */
            const int32_t m = H[j] + row[query[j]];
            int32_t e = E[j];
            H[j] = h1;
            uint8_t d = m >= e ? 0 : 1;
            int32_t h = m >= e ? m : e;
            if (h < f) { d = 2; h = f; }
            h1 = h;
            int32_t t = m - oe_del;
            e -= e_del;
            if (e > t) d |= 1 << 2; else e = t;
            E[j] = e;
            t = m - oe_ins;
            f -= e_ins;
            if (f > t) d |= 2 << 4; else f = t;
            if (z) z[(size_t)i * ncol + (j - beg)] = d;
        }
        nc += end > beg ? end - beg : 0;
        H[end] = h1; E[end] = G3O_NEG_INF;
    }
    const int score = H[qlen];
    if (cigar && score <= G3O_NEG_INF / 2) {
        /* no alignment inside the band reaches the last cell: the reference's backtrack then
           walks direction bytes it never wrote (undefined); here the CIGAR is empty */
        *n_cigar = 0;
    } else if (cigar) {
        int n = 0, which = 0;
        int i = tlen - 1, k = (i + w + 1 < qlen ? i + w + 1 : qlen) - 1;
        while (i >= 0 && k >= 0) {
            which = z[(size_t)i * ncol + (k - (i > w ? i - w : 0))] >> (which << 1) & 3;
            if (which == 0) { g3o_push_op(cigar, &n, 0, 1); --i; --k; }
            else if (which == 1) { g3o_push_op(cigar, &n, 2, 1); --i; }
            else { g3o_push_op(cigar, &n, 1, 1); --k; }
        }
        if (i >= 0) g3o_push_op(cigar, &n, 2, i + 1);
        if (k >= 0) g3o_push_op(cigar, &n, 1, k + 1);
        for (int a = 0; a < n >> 1; ++a) {
            const uint32_t t = cigar[a]; cigar[a] = cigar[n - 1 - a]; cigar[n - 1 - a] = t;
        }
        *n_cigar = n;
    }
    free(z); free(H); free(E);
    if (cells) *cells = nc;
    return score;
}

/* n global alignments over one code buffer (jobs as g3o_job, flags ignored; h0 unused):
   scores, CIGARs at cigar[k * stride] (stride >= qlen + tlen + 2), their lengths. */
void g3o_global_batch(const g3o_job *jobs, int64_t n, const uint8_t *codes, const g3o_score *sc,
                      int32_t *score, uint32_t *cigar, int32_t stride, int32_t *n_cigar, int64_t *cells)
{
    for (int64_t k = 0; k < n; ++k) {
        const g3o_job *j = &jobs[k];
        int nc = 0;
        score[k] = g3o_ksw_global2(j->qlen, codes + j->q_off, j->tlen, codes + j->t_off, sc->mat, sc->o_del,
                                   sc->e_del, sc->o_ins, sc->e_ins, j->w, &nc, cigar + (size_t)k * stride,
                                   cells ? cells + k : NULL);
        n_cigar[k] = nc;
    }
}

/* NM and MD of a global alignment, as the traceback stage computes them after ksw_global2
   (aux.cu:2831-2860): along the CIGAR, a mismatch in an M run adds to NM and writes the run of
   matches before it and the target base; a D that is neither the first nor the last operation
   writes the matches before it, '^' and the deleted target bases, and adds its length to NM;
   an I adds its length to NM only.  Bases print as "ACGTN", or "TGCAN" when rc.  md gets the
   NUL-terminated string (room for 4 * (qlen + tlen) + 16 bytes); returns NM. */
int g3o_nm_md(const uint32_t *cigar, int n_cigar, const uint8_t *query, const uint8_t *target, int rc,
              char *md)
{
    const char *base = rc ? "TGCAN" : "ACGTN";
    int x = 0, y = 0, u = 0, n_mm = 0, n_gap = 0, l = 0;
    for (int k = 0; k < n_cigar; ++k) {
        const int op = cigar[k] & 0xf, len = (int)(cigar[k] >> 4);
        if (op == 0) {
            for (int i = 0; i < len; ++i) {
                if (query[x + i] != target[y + i]) {
                    l += sprintf(md + l, "%d", u);
                    md[l++] = base[target[y + i]];
                    ++n_mm; u = 0;
                } else ++u;
            }
            x += len; y += len;
        } else if (op == 2) {
            if (k > 0 && k < n_cigar - 1) {
                l += sprintf(md + l, "%d", u);
                md[l++] = '^';
                for (int i = 0; i < len; ++i) md[l++] = base[target[y + i]];
                u = 0; n_gap += len;
            }
            y += len;
        } else if (op == 1) {
            x += len; n_gap += len;
        }
    }
    l += sprintf(md + l, "%d", u);
    md[l] = 0;
    return n_mm + n_gap;
}

/* NM and MD for every job of a global batch (flags bit 2 = the "TGCAN" alphabet). */
void g3o_nm_md_batch(const g3o_job *jobs, int64_t n, const uint8_t *codes, const uint32_t *cigar,
                     int32_t stride, const int32_t *n_cigar, int32_t *nm, char *md, int32_t md_stride)
{
    for (int64_t k = 0; k < n; ++k)
        nm[k] = g3o_nm_md(cigar + (size_t)k * stride, n_cigar[k], codes + jobs[k].q_off, codes + jobs[k].t_off,
                          (jobs[k].flags & 4) != 0, md + (size_t)k * md_stride);
}

/* ---------------------------------------------------------------------------------- */
/* Striped local Smith-Waterman with 16-bit cells: ksw_align2 (ksw.cu:271-292) over the  */
/* query profile of ksw_qinit (ksw.cu:18-64, two-byte cells) and the pass of ksw_i16     */
/* (ksw.cu:155-262).  The reference stops ksw_align2 at its first line (ksw.cu:276); this */
/* restates the function as written after that line.                                    */
/* ---------------------------------------------------------------------------------- */

typedef struct { int32_t score, te, qe, score2, te2, tb, qb; } g3o_swr;   /* kswr_t, ksw.h:24-29 */
#define G3O_XSTOP  0x20000
#define G3O_XSUBO  0x40000
#define G3O_XSTART 0x80000

/* The vector helpers of ksw.cu:66-153 act on eight int16 lanes: a plain add whose int result
   is stored back into int16 (wraps), a signed max, and "subtract, 0 if not positive" computed in
   int before the store. */
static int16_t g3o_sub0(int16_t a, int16_t b) { const int v = (int)a - (int)b; return (int16_t)(v > 0 ? v : 0); }

/* One pass of ksw_i16.  Lane k of vector j of the striped profile holds query position
   j + k * slen (score 0 past the query); the row loop, the lazy-F loop of at most 16 rounds
   that leaves E alone, the per-row maximum, the list of row maxima at or above minsc
   (XSUBO) and the stop at endsc (XSTOP) follow ksw.cu:190-239; the end position on the query
   is the smallest position holding the best row's maximum (the scan of ksw.cu:244-248 reads
   the cells as uint16), the second best score comes from the list entries more than
   ceil(score / max(mat)) rows away from te (ksw.cu:249-256). */
static g3o_swr g3o_sw16_pass(int qlen, const uint8_t *query, int tlen, const uint8_t *target,
                             const int8_t *mat, int o_del, int e_del, int o_ins, int e_ins, int xtra,
                             int64_t *cells)
{
    g3o_swr r = { 0, -1, -1, -1, -1, -1, -1 };               /* g_defr, ksw.cu:5 */
    const int slen = (qlen + 7) / 8, np = slen * 8;
    int16_t *prof = (int16_t *)malloc(sizeof(int16_t) * 5 * (size_t)(np > 0 ? np : 1));
    int16_t *H0 = (int16_t *)calloc((size_t)np + 8, sizeof(int16_t));
    int16_t *H1 = (int16_t *)calloc((size_t)np + 8, sizeof(int16_t));
    int16_t *E = (int16_t *)calloc((size_t)np + 8, sizeof(int16_t));
    int16_t *Hmax = (int16_t *)calloc((size_t)np + 8, sizeof(int16_t));
    uint64_t *b = NULL;
    int n_b = 0, m_b = 0, gmax = 0, te = -1, maxmat = 0;
    const int minsc = (xtra & G3O_XSUBO) ? xtra & 0xffff : 0x10000;
    const int endsc = (xtra & G3O_XSTOP) ? xtra & 0xffff : 0x10000;
    const int16_t oed = (int16_t)(o_del + e_del), ed = (int16_t)e_del;
    const int16_t oei = (int16_t)(o_ins + e_ins), ei = (int16_t)e_ins;
    for (int k = 0; k < 25; ++k) if (mat[k] > maxmat) maxmat = mat[k];
    for (int a = 0; a < 5; ++a)
        for (int j = 0; j < slen; ++j)
            for (int k = 0; k < 8; ++k) {
                const int pos = j + k * slen;
                prof[((size_t)a * slen + j) * 8 + k] = pos < qlen ? mat[a * 5 + query[pos]] : 0;
            }
    int64_t nc = 0;
    for (int i = 0; i < tlen; ++i) {
        const int16_t *S = prof + (size_t)target[i] * slen * 8;
        int16_t h[8], f[8], mx[8];
        for (int k = 0; k < 8; ++k) {                        /* the last vector moved up a lane */
            h[k] = k == 0 || slen == 0 ? 0 : H0[(size_t)(slen - 1) * 8 + k - 1];
            f[k] = 0; mx[k] = 0;
        }
        for (int j = 0; j < slen; ++j) {
            for (int k = 0; k < 8; ++k) {
                const size_t at = (size_t)j * 8 + k;
                int16_t v = (int16_t)(h[k] + S[at]);
                if (E[at] > v) v = E[at];
                if (f[k] > v) v = f[k];
                if (v > mx[k]) mx[k] = v;
                H1[at] = v;
                int16_t e = g3o_sub0(E[at], ed), t = g3o_sub0(v, oed);
                E[at] = e > t ? e : t;
                f[k] = g3o_sub0(f[k], ei); t = g3o_sub0(v, oei);
                if (t > f[k]) f[k] = t;
                h[k] = H0[at];
            }
        }
        nc += qlen;
        for (int round = 0; round < 16; ++round) {          /* lazy F */
            for (int k = 7; k > 0; --k) f[k] = f[k - 1];
            f[0] = 0;
            for (int j = 0; j < slen; ++j) {
                int any = 0;
                for (int k = 0; k < 8; ++k) {
                    const size_t at = (size_t)j * 8 + k;
                    int16_t v = H1[at] > f[k] ? H1[at] : f[k];
                    H1[at] = v;
                    v = g3o_sub0(v, oei);
                    f[k] = g3o_sub0(f[k], ei);
                    any |= f[k] > v;
                }
                if (!any) goto lazy_done;
            }
        }
lazy_done:;
        int imax = mx[0];
        for (int k = 1; k < 8; ++k) if (mx[k] > imax) imax = mx[k];
        if (imax >= minsc) {
            if (n_b == 0 || (int32_t)b[n_b - 1] + 1 != i) {
                if (n_b == m_b) {
                    m_b = m_b ? m_b << 1 : 8;
                    b = (uint64_t *)realloc(b, 8 * (size_t)m_b);
                }
                b[n_b++] = (uint64_t)imax << 32 | (uint32_t)i;
            } else if ((int)(b[n_b - 1] >> 32) < imax) {
                b[n_b - 1] = (uint64_t)imax << 32 | (uint32_t)i;
            }
        }
        if (imax > gmax) {
            gmax = imax; te = i;
            memcpy(Hmax, H1, sizeof(int16_t) * (size_t)np);
            if (gmax >= endsc) break;
        }
        int16_t *sw = H0; H0 = H1; H1 = sw;
    }
    r.score = gmax; r.te = te;
    int best = -1;
    for (int x = 0; x < np; ++x) {
        const int v = (uint16_t)Hmax[x], pos = x / 8 + x % 8 * slen;
        if (v > best) { best = v; r.qe = pos; }
        else if (v == best && pos < r.qe) r.qe = pos;
    }
    if (n_b > 0) {
        const int c = (r.score + maxmat - 1) / maxmat, low = te - c, high = te + c;
        for (int x = 0; x < n_b; ++x) {
            const int e = (int32_t)b[x];
            if ((e < low || e > high) && (int)(b[x] >> 32) > r.score2) { r.score2 = (int)(b[x] >> 32); r.te2 = e; }
        }
    }
    free(prof); free(H0); free(H1); free(E); free(Hmax); free(b);
    if (cells) *cells += nc;
    return r;
}

/* ksw_align2 with 16-bit cells (ksw.cu:271-292): the forward pass; with XSTART (and, under
   XSUBO, a score reaching xtra & 0xffff) a second pass over the query prefix 0..qe and the
   target with its prefix 0..te reversed, stopping at the first score, gives the start
   positions when it finds the same score.  qlen >= 1; *cells (may be NULL) receives the cells
   of both passes (query length x target rows entered, padding lanes not counted). */
g3o_swr g3o_ksw_align2(int qlen, const uint8_t *query, int tlen, const uint8_t *target, const int8_t *mat,
                       int o_del, int e_del, int o_ins, int e_ins, int xtra, int64_t *cells)
{
    int64_t nc = 0;
    g3o_swr r = g3o_sw16_pass(qlen, query, tlen, target, mat, o_del, e_del, o_ins, e_ins, xtra, &nc);
    if ((xtra & G3O_XSTART) && !((xtra & G3O_XSUBO) && r.score < (xtra & 0xffff))) {
        const int lq = r.qe + 1, lt = r.te + 1;
        uint8_t *rq = (uint8_t *)malloc((size_t)lq + 1), *rt = (uint8_t *)malloc((size_t)tlen + 1);
        for (int k = 0; k < lq; ++k) rq[k] = query[lq - 1 - k];
        for (int k = 0; k < tlen; ++k) rt[k] = k < lt ? target[lt - 1 - k] : target[k];
        const g3o_swr rr = g3o_sw16_pass(lq, rq, tlen, rt, mat, o_del, e_del, o_ins, e_ins,
                                         G3O_XSTOP | r.score, &nc);
        if (r.score == rr.score) { r.tb = r.te - rr.te; r.qb = r.qe - rr.qe; }
        free(rq); free(rt);
    }
    if (cells) *cells = nc;
    return r;
}

/* n local alignments over one code buffer (jobs as g3o_job: G3O_QREV / G3O_TREV read the
   sequence backwards; h0 and w unused), one xtra for all. */
void g3o_sw_batch(const g3o_job *jobs, int64_t n, const uint8_t *codes, const g3o_score *sc, int xtra,
                  g3o_swr *out, int64_t *cells)
{
    for (int64_t k = 0; k < n; ++k) {
        const g3o_job *jb = &jobs[k];
        uint8_t *qb = NULL, *tb = NULL;
        const uint8_t *q = g3o_view(codes + jb->q_off, jb->qlen, jb->flags & G3O_QREV, &qb);
        const uint8_t *t = g3o_view(codes + jb->t_off, jb->tlen, jb->flags & G3O_TREV, &tb);
        out[k] = g3o_ksw_align2(jb->qlen, q, jb->tlen, t, sc->mat, sc->o_del, sc->e_del, sc->o_ins, sc->e_ins,
                                xtra, cells ? cells + k : NULL);
        free(qb); free(tb);
    }
}

/* ---------------------------------------------------------------------------------- */
/* Pair preparation of the traceback stage: FINALIZEALN_preprocessing2_kernel            */
/* (aux.cu:2698-2745) with infer_bw (aux.cu:506-513) and bns_get_seq_gpu                 */
/* (bntseq.cu:39-60).                                                                    */
/* ---------------------------------------------------------------------------------- */

typedef struct { int32_t a, o_del, e_del, o_ins, e_ins; } g3o_tbopt;

/* Band width a global alignment of l1 and l2 bases with this score needs (aux.cu:506-513):
   0 for equal lengths that leave no room for two gaps, else (min(l1,l2) a - score - q) / r + 2
   (the double truncated), at least |l1 - l2|. */
static int g3o_infer_bw(int l1, int l2, int score, int a, int q, int r)
{
    if (l1 == l2 && l1 * a - score < (q + r - a) << 1) return 0;
    int w = (int)((double)((l1 < l2 ? l1 : l2) * a - score - q) / r + 2.);
    const int d = l1 > l2 ? l1 - l2 : l2 - l1;
    return w < d ? d : w;
}

/* Per record k (read recs[2k], region recs[2k+1]): the query read[qb, qe) (its code-buffer
   offset and length), the reference slice [rb, re) as bns_get_seq_gpu returns it (bounds
   swapped if reversed, clipped to [0, 2 l_pac), empty when it spans the forward/reverse
   boundary) to tgt[k * tstride ...] with its length, and the band width: 0 when the query and
   [rb, re) have equal lengths, else the larger infer_bw of the deletion and insertion costs,
   at most (max_gap + |rlen - lq| + 1) / 2 with max_gap the larger of the insertion and
   deletion gaps half the query can pay for (at least 1), at least |rlen - lq| + 3; stored as
   uint16 (aux.cu:2745).  rb_out[k] = rb (the stage prints the reverse-strand alphabet in MD
   when rb >= l_pac). */
void g3o_tb_pairs(const g3o_tbopt *opt, const uint8_t *codes, int64_t ref_off, int64_t l_pac,
                  const g3o_read *reads, const g3o_alnreg *regs, const int32_t *recs, int64_t n,
                  int64_t *q_off, int32_t *qlen, uint8_t *tgt, int32_t tstride, int32_t *tlen, int32_t *w,
                  int64_t *rb_out)
{
    for (int64_t k = 0; k < n; ++k) {
        const g3o_read *rd = &reads[recs[2 * k]];
        const g3o_alnreg *g = &regs[recs[2 * k + 1]];
        const int lq = g->qe - g->qb;
        int64_t beg = g->rb, end = g->re, rlen = 0;
        if (end < beg) { const int64_t t = beg; beg = end; end = t; }
        if (end > l_pac << 1) end = l_pac << 1;
        if (beg < 0) beg = 0;
        if (beg >= l_pac || end <= l_pac) rlen = end - beg;
        q_off[k] = rd->read_off + g->qb;
        qlen[k] = lq;
        tlen[k] = (int32_t)rlen;
        for (int64_t x = 0; x < rlen && x < tstride; ++x) tgt[k * tstride + x] = codes[ref_off + beg + x];
        int bw = 0;
        if ((int64_t)lq != g->re - g->rb) {
            const int l2 = (int)(g->re - g->rb);
            const int wd = g3o_infer_bw(lq, l2, g->score, opt->a, opt->o_del, opt->e_del);
            const int wi = g3o_infer_bw(lq, l2, g->score, opt->a, opt->o_ins, opt->e_ins);
            bw = wd > wi ? wd : wi;
            const int half = ((lq + 1) >> 1) * opt->a;
            const int max_ins = (int)((double)(half - opt->o_ins) / opt->e_ins + 1.);
            const int max_del = (int)((double)(half - opt->o_del) / opt->e_del + 1.);
            int max_gap = max_ins > max_del ? max_ins : max_del;
            if (max_gap < 1) max_gap = 1;
            const int dl = (int)rlen > lq ? (int)rlen - lq : lq - (int)rlen;
            const int hi = (max_gap + dl + 1) >> 1;
            if (bw > hi) bw = hi;
            if (bw < dl + 3) bw = dl + 3;
        }
        w[k] = (uint16_t)bw;
        rb_out[k] = g->rb;
    }
}

/* ---------------------------------------------------------------------------------- */
/* The seed filter of long reads: mem_seed_sw (aux.cu:117-143) and                      */
/* mem_flt_chained_seeds (aux.cu:144-162, as CHAINFILTERING_flt_chained_seeds_kernel      */
/* runs it per read, aux.cu:1991-2030).                                                  */
/* ---------------------------------------------------------------------------------- */

#define G3O_SHORT_EXT 50            /* MEM_SHORT_EXT, aux.cuh:396 */
#define G3O_SHORT_LEN 200           /* MEM_SHORT_LEN, aux.cuh:397 */

/* The local alignment score of the window around a short seed, or -1 when the seed or its
   window is long enough to skip it (aux.cu:117-143): the seed +-50 bases on the read and on
   the reference (clipped to the read, to [0, 2 l_pac) and to the strand of the seed's middle),
   both below 200 bases, the reference window clipped to the contig of the middle
   (bns_fetch_seq_gpu), then ksw_align2 with KSW_XSTART; only the score is used.  *cells (may
   be NULL) grows by the cells of both passes. */
int g3o_seed_sw(const g3o_opt *opt, const uint8_t *codes, int64_t ref_off, int64_t l_pac, const g3o_ann *anns,
                int n_seqs, int l_query, const uint8_t *query, const g3o_cseed *s, int64_t *cells)
{
    if (s->len >= G3O_SHORT_LEN) return -1;
    int qb = s->qbeg, qe = s->qbeg + s->len;
    int64_t rb = s->rbeg, re = s->rbeg + s->len;
    const int64_t mid = (rb + re) >> 1;
    qb -= G3O_SHORT_EXT; if (qb < 0) qb = 0;
    qe += G3O_SHORT_EXT; if (qe > l_query) qe = l_query;
    rb -= G3O_SHORT_EXT; if (rb < 0) rb = 0;
    re += G3O_SHORT_EXT; if (re > l_pac << 1) re = l_pac << 1;
    if (rb < l_pac && l_pac < re) {
        if (mid < l_pac) re = l_pac; else rb = l_pac;
    }
    if (qe - qb >= G3O_SHORT_LEN || re - rb >= G3O_SHORT_LEN) return -1;
    g3o_clip_window(anns, n_seqs, l_pac, &rb, mid, &re);
    const int tlen = (int)(re - rb);
    int64_t nc = 0;
    const g3o_swr x = g3o_ksw_align2(qe - qb, query + qb, tlen > 0 ? tlen : 0, codes + ref_off + rb, opt->mat,
                                     opt->o_del, opt->e_del, opt->o_ins, opt->e_ins, G3O_XSTART, &nc);
    if (cells) *cells += nc;
    return x.score;
}

/* mem_flt_chained_seeds for every read: reads whose min_l = 1.1 * min_chain_weight (or, with
   no minimum chain weight, 5.5 * logf(l_query)) exceeds 0.05 * l_query are left alone;
   otherwise every seed of every chain gets its window score, and a chain keeps, in order, the
   seeds whose score is -1 (their score becoming len * a) or at least
   (int)(a * min_l + .499).  chains[].n and the seeds are changed in place; sw_score[i]
   receives seed i's window score (-2 for seeds of reads left alone). */
void g3o_flt_chained_seeds(const g3o_opt *opt, int min_chain_weight, const uint8_t *codes, int64_t ref_off,
                           int64_t l_pac, const g3o_ann *anns, int n_seqs, const g3o_read *reads, int64_t n_reads,
                           g3o_chain *chains, g3o_cseed *seeds, int32_t *sw_score, int64_t *cells)
{
    for (int64_t r = 0; r < n_reads; ++r) {
        const g3o_read *rd = &reads[r];
        const int lq = rd->l_query;
        const double min_l = min_chain_weight ? 1.1f * min_chain_weight : 5.5f * logf((float)lq);
        const int min_hsp = (int)(opt->a * min_l + .499);
        if (min_l > 0.05f * lq) continue;
        for (int c = 0; c < rd->n_chains; ++c) {
            g3o_chain *ch = &chains[rd->chain_beg + c];
            g3o_cseed *sd = seeds + ch->seed_beg;
            int k = 0;
            for (int j = 0; j < ch->n; ++j) {
                g3o_cseed s = sd[j];
                s.score = g3o_seed_sw(opt, codes, ref_off, l_pac, anns, n_seqs, lq, codes + rd->read_off, &s, cells);
                if (sw_score) sw_score[ch->seed_beg + j] = s.score;
                if (s.score < 0 || s.score >= min_hsp) {
                    if (s.score < 0) s.score = s.len * opt->a;
                    sd[k++] = s;
                }
            }
            ch->n = k;
        }
    }
}

/*
 * g3x.h -- C ABI of the B200 BWA-MEM seed-extension library (libg3x.so).
 *
 * The library replaces the seed-extension stage of the sunwookim028/G3SA bwa/ pipeline:
 * the per-job device function
 *     int ksw_extend2(int qlen, const uint8_t *query, int tlen, const uint8_t *target,
 *                     int m, const int8_t *mat, int o_del, int e_del, int o_ins, int e_ins,
 *                     int w, int end_bonus, int zdrop, int h0, int *_qle, int *_tle,
 *                     int *_gtle, int *_gscore, int *_max_off, void *d_buffer_ptr)
 *     (bwa/src/ksw.h:33, bwa/src/ksw.cu:303-401)
 * and its callers: the left/right band-retry loop of mem_chain2aln
 * (bwa/src/aux.cu:250-301, MAX_BAND_TRY at bwa/src/aux.cuh:401) and the batch stage kernel
 * localExtending (bwa/src/aux.cuh:208-214, launched at bwa/src/bwamem.cu:276).
 *
 * Every output (score, qle, tle, gtle, gscore, max_off) is bit-identical to the
 * reference's CPU ksw_extend2 on the same inputs.
 *
 * Conventions
 *   - Return value: 0 (G3X_OK) or a negative G3X_ERR_* code; g3x_strerror() names it.
 *     Nothing traps and nothing calls exit().
 *   - d_* pointers are device memory owned by the caller; h_* pointers are host memory.
 *   - A g3x_ctx is bound to one GPU and one host thread at a time (not thread-safe).
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *
 * Sequences travel as two bit planes over one base index space:
 *   codes[b >> 4] bits 2*(b & 15) .. +1   : 2-bit base code (A=0 C=1 G=2 T=3)
 *   nmask[b >> 5] bit  (b & 31)           : 1 = ambiguous base N (code 4)
 * A job names its query and target by their first base index and length.
 */
#ifndef G3X_H
#define G3X_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------------------- */
#define G3X_OK                 0
#define G3X_ERR_INVALID       -1   /* bad argument (null pointer, n < 0, bad option) */
#define G3X_ERR_SCORE         -2   /* scoring the kernels do not support (m != 5, e <= 0) */
#define G3X_ERR_TOO_LONG      -3   /* a job exceeds the length limits (per-job status) */
#define G3X_ERR_CUDA          -4   /* a CUDA runtime call failed */
#define G3X_ERR_TIMEOUT       -5   /* a bounded device wait gave up (per-job status) */
#define G3X_ERR_INTERNAL      -6   /* a device-side consistency check failed (per-job) */
#define G3X_ERR_NOMEM         -7   /* allocation of library-owned scratch failed */
#define G3X_ERR_NOT_TRAINED   -8   /* learned schedule requested before a model was set */
#define G3X_ERR_SCRATCH       -9   /* batch larger than the fixed scratch of a no-alloc call */

/* ---- data records -------------------------------------------------------------------- */

/* Scoring, as mem_opt_t carries it (bwa/src/bwa.h:157-189; defaults bwa/src/fastmap.cpp:77-124:
   a=1 b=4 o=6 e=1 zdrop=100 pen_clip=5, mat from bwa_fill_scmat). mat[t*5 + q] scores target
   code t against query code q, as the query profile at bwa/src/ksw.cu:312-315 indexes it. */
typedef struct {
    int8_t  mat[25];
    int8_t  pad_[3];
    int32_t m;            /* alphabet size; must be 5 */
    int32_t o_del, e_del, o_ins, e_ins;
    int32_t zdrop;
    int32_t end_bonus;    /* only clamps the band, as in bwa/src/ksw.cu:325-329 */
} g3x_score_t;            /* 56 bytes */

/* One extension job = one ksw_extend2 call. */
#define G3X_JOB_QREV 1u   /* read the query backwards: query[k] = base q_off + qlen-1-k */
#define G3X_JOB_TREV 2u   /* read the target backwards */
typedef struct {
    uint32_t q_off;       /* base index of the query's first base in the planes */
    uint32_t t_off;       /* base index of the target's first base */
    uint16_t qlen, tlen;  /* qlen <= 65534 */
    int32_t  h0;          /* score of the seed (ksw_extend2's h0) */
    int32_t  w;           /* band width before clamping */
    uint32_t flags;       /* G3X_JOB_* */
} g3x_job_t;              /* 24 bytes */

/* ksw_extend2's return value and out-parameters, in that order. */
typedef struct {
    int32_t score, qle, tle, gtle, gscore, max_off;
} g3x_ext_t;              /* 24 bytes */

/* ---- context ------------------------------------------------------------------------- */
typedef struct g3x_ctx g3x_ctx;

/* Binds a context to CUDA device `device` (one GPU only). */
int g3x_ctx_create(g3x_ctx **ctx, int device);
int g3x_ctx_destroy(g3x_ctx *ctx);
const char *g3x_strerror(int code);

/* ---- batched ksw_extend2 ------------------------------------------------------------- */

#define G3X_SCHED_PLAIN   0   /* one 32-lane block per job, jobs in the given order */
#define G3X_SCHED_SORTED  1   /* persistent kernel, jobs ordered by length (fallback) */
#define G3X_SCHED_LEARNED 2   /* persistent kernel, jobs ordered by the learned cost model */

#define G3X_KERNEL_AUTO    0  /* rolling for G3X_SCHED_PLAIN, row-parallel otherwise */
#define G3X_KERNEL_ROLLING 1  /* anti-diagonal wavefront: rows on lanes, 4-cell lane steps */
#define G3X_KERNEL_ROWPAR  2  /* one row per step: columns on lanes, F by shuffle scan */
#define G3X_KERNEL_LANE    3  /* one job per lane: the scalar row loop, 8-column blocks */
#define G3X_KERNEL_LANE16  4  /* one job per lane, two cells per int16x2 instruction (jobs whose
                                 scores fit 16 bits) */
#define G3X_KERNEL_LANE2   5  /* one job per lane, rows i and i+1 in flight together */
#define G3X_KERNEL_BAND    6  /* one job per warp, the band's row buffer in registers over a window
                                 of `tile` columns (256, 512 or 1024, 0 = 1024) that slides with
                                 the band; jobs whose band 2w' + 2 exceeds it get TOO_LONG */

typedef struct {
    int32_t schedule;     /* G3X_SCHED_* */
    int32_t max_qlen;     /* upper bound of qlen over the batch (required) */
    int32_t max_tlen;     /* upper bound of tlen over the batch (required) */
    int32_t lanes;        /* lanes per job: 1 (lane kernel), 4 (row-parallel only), 8, 16, 32,
                             or 0 = tuned; raised when a warp of such groups would not fit in
                             shared memory */
    int32_t tile;         /* row-parallel: cells per lane per tile (5, 9 or 13), 0 = tuned */
    int32_t kernel;       /* G3X_KERNEL_* */
    int32_t *d_cells;     /* optional per-job DP cell count (trip count of ksw.cu:346) */
    int64_t n_bases;      /* bases the planes hold (required, 1 .. 2^32): a job or seed reaching
                             past it is refused with a per-job G3X_ERR_INVALID, unread */
    int32_t *d_rows;      /* optional per-job row count: trips of the row loop of ksw.cu:346
                             (the z-drop or an empty band ends it before tlen) */
} g3x_batch_opts_t;       /* 48 bytes */

/* n jobs; outputs to d_out[k] and d_status[k] (G3X_OK or a G3X_ERR_* per job: TOO_LONG for a
   job beyond max_qlen/max_tlen or beyond what a fixed lane kernel holds, INVALID for a seed
   score -max_score < h0 < 0, which callers of ksw_extend2 never pass, or for a job whose query
   or target reaches past opts->n_bases: q_off + qlen or t_off + tlen > n_bases; such a job's
   bases are never read).
   Replaces n calls of ksw_extend2 (bwa/src/ksw.h:33) issued by localExtending
   (bwa/src/aux.cu:2289-2382). Asynchronous on `stream`. */
int g3x_ksw_extend2_batch(g3x_ctx *ctx, const g3x_score_t *score, const g3x_job_t *d_jobs,
                          int32_t n, const uint32_t *d_codes, const uint32_t *d_nmask,
                          g3x_ext_t *d_out, int32_t *d_status, const g3x_batch_opts_t *opts,
                          void *stream);

/* No counterpart in the reference: a variant of g3x_ksw_extend2_batch with G3X_SCHED_SORTED
   (same width classes and kernels, same outputs) that allocates nothing.  For callers that
   must not allocate device memory while they run: a pipeline stage between other stages'
   kernels, where cudaMalloc/cudaFree would synchronise the device; a process that reserved
   the GPU's memory up front (as the reference's device_alloc does); a framework whose
   allocator owns all device memory.  It needs no context: its scratch (sort keys, job order,
   histogram, per-class job counters) is one static device array of the library, 8.13 MiB,
   whose address the first call on a device looks up (cudaGetSymbolAddress).  CUDA loads the
   library's kernels and that array lazily, on first use, and loading may allocate device memory
   and synchronise: make one call with a small batch on each device before the phase in which
   nothing may allocate (n = 0 does the address look-up alone).  The address belongs to the
   device's primary context: no cudaDeviceReset between calls.  At most G3X_NOALLOC_MAX_JOBS
   jobs per call, else G3X_ERR_SCRATCH.  All calls on a device share that array: calls that
   overlap on the GPU (two streams, two host threads) race and corrupt each other's results,
   so serialise them.  n_bases: the bases the planes hold, as g3x_batch_opts_t.n_bases (jobs
   reaching past them get G3X_ERR_INVALID, unread).  Makes `device` current.  Asynchronous on
   `stream`. */
#define G3X_NOALLOC_MAX_JOBS 1048576
int g3x_ksw_extend2_batch_noalloc(int device, const g3x_score_t *score, const g3x_job_t *d_jobs,
                                  int32_t n, const uint32_t *d_codes, const uint32_t *d_nmask,
                                  int64_t n_bases, g3x_ext_t *d_out, int32_t *d_status,
                                  int32_t max_qlen, int32_t max_tlen, void *stream);

/* ---- schedule tuning ----------------------------------------------------------------------- */
/* The persistent schedules split a batch into width classes: a job belongs to the first class
   whose `width` holds its query (qlen bounds the widest row, min(qlen, 2w+1), w after the
   clamp of bwa/src/ksw.cu:321-329); the last class takes every longer job (several tiles per
   row when its rows are wider than one tile).  Each
   class runs the row-parallel kernel with `lanes` lanes per job and `tile` cells per lane;
   `warp_batch` = 1 makes a warp pull one job per group at once and wait for all of them
   (jobs then balance by the schedule's cost order), 0 lets each group refill on its own;
   the lane-per-job kernels (lanes = 1) refill their idle lanes in waves of at least `refill`.
   A lane class with tile = 2 runs its middle blocks in int16x2; the scheduler sends a job whose
   scores do not provably fit a lane class's arithmetic (16-bit fields, h0 >= 0) to the last
   class instead. */
#define G3X_MAX_CLASSES 8
typedef struct {
    int32_t width;        /* widest query of the class (the last class: unbounded) */
    int32_t lanes;        /* 1 = lane-per-job kernel; 4, 8, 16, 32 = row-parallel groups */
    int32_t tile;         /* row-parallel: cells per lane per tile (5, 9, 13); with 32 lanes, 256,
                             512 or 1024 = the band kernel (G3X_KERNEL_BAND) with that window
                             (not the last class: a job whose band exceeds the window goes to
                             the last class); lane kernel: 0 (int32, one job per lane), 2 (int16x2,
                             two cells per instruction) or 4 (int32, one job per lane with two of
                             its rows in flight) */
    int32_t warp_batch;   /* 1: a warp takes its jobs together and waits for all of them */
    int32_t refill;       /* lane kernel: idle lanes that trigger a refill wave (1-32) */
} g3x_tile_t;

/* A new context's classes: the int16x2 lane kernel (lanes 1, tile 2, refill 8) for queries up to
   32, 56, 88, 128, 168, 200 and 256 bases, then 32-lane row-parallel groups (tile 9) for longer
   queries and jobs outside the int16 fit.  g3x_autotune replaces them with classes fitted to a
   batch. */
int g3x_get_tiles(g3x_ctx *ctx, g3x_tile_t *h_tiles, int32_t *n);
int g3x_set_tiles(g3x_ctx *ctx, const g3x_tile_t *h_tiles, int32_t n);
/* Whether the context's width classes may use the int16x2 lane kernel (1, a new context's
   setting) or compute every cell in int32 (0), for workloads that rule the 16-bit path out.
   With 0 the context's int16x2 classes become int32 lane classes (tile 0, same refill),
   g3x_autotune considers int32 kernels only, and g3x_set_tiles refuses tile 2 with
   G3X_ERR_INVALID.  An explicit G3X_KERNEL_LANE16 batch is not affected.  Outputs are the same
   either way. */
int g3x_set_int16(g3x_ctx *ctx, int32_t enable);
/* Fits the width classes to the given jobs (device buffers) and tunes them: the class widths
   become max_qlen x (0.138, 0.241, 0.379, 0.552, 0.724, 0.862, 1) (rounded up to 8 columns,
   duplicates dropped) plus
   the unbounded class; then every candidate configuration of each class is timed on the class's
   jobs and the fastest kept in the context; h_tiles/n receive the table.  n_bases: the bases the
   planes hold, as g3x_batch_opts_t.n_bases.  Blocks.  Outputs of the trial runs are discarded. */
int g3x_autotune(g3x_ctx *ctx, const g3x_score_t *score, const g3x_job_t *d_jobs, int32_t n,
                 const uint32_t *d_codes, const uint32_t *d_nmask, int64_t n_bases, int32_t max_qlen,
                 int32_t max_tlen, g3x_tile_t *h_tiles, int32_t *n_tiles);
/* The same, with the jobs ordered as `schedule` (G3X_SCHED_SORTED or G3X_SCHED_LEARNED, which
   needs a trained model) orders them, so the choices fit that schedule; g3x_autotune is the
   G3X_SCHED_SORTED form. */
int g3x_autotune_schedule(g3x_ctx *ctx, int32_t schedule, const g3x_score_t *score,
                          const g3x_job_t *d_jobs, int32_t n, const uint32_t *d_codes,
                          const uint32_t *d_nmask, int64_t n_bases, int32_t max_qlen,
                          int32_t max_tlen, g3x_tile_t *h_tiles, int32_t *n_tiles);
/* Occupancy counters of the last persistent batch on this context: h_stats[0] = group-rows
   computed, [1] = group-rows a group waited for the other groups of its warp (warp_batch),
   [2] = warp batches.  Synchronises the context's device. */
int g3x_last_stats(g3x_ctx *ctx, uint64_t *h_stats);

/* Per-class kernel timing of the scheduled batches (no counterpart in the reference): with
   timing on (1), every persistent class launch made outside CUDA-graph capture is bracketed by
   CUDA events on the stream it runs on, the classes running side by side as usual; with 2,
   the classes run one after another on the caller's stream, each timed alone; 0 = off.
   g3x_class_times then returns, for the last such batch, each class's launch duration in ms
   (-1: not launched) and job count; n receives the number of classes.  Synchronises the
   context's device. */
int g3x_set_timing(g3x_ctx *ctx, int32_t on);
int g3x_class_times(g3x_ctx *ctx, float *h_ms, int32_t *h_jobs, int32_t *n);

/* ---- seed-level extension with band retry ---------------------------------------------- */

/* Options of the seed-level call: scoring, match score a (the seed scores len * a), the first
   band width w (a retry uses 2w; MAX_BAND_TRY = 2, bwa/src/aux.cuh:401) and the clipping
   penalties that choose local vs to-end extension (mem_opt_t pen_clip5/pen_clip3,
   bwa/src/bwa.h:157-189). */
typedef struct {
    g3x_score_t score;
    int32_t a, w, pen_clip5, pen_clip3;
} g3x_opt_t;              /* 72 bytes */

/* One seed of a chain with its reference window, as mem_chain2aln sees it
   (mem_seed_t, bwa/src/bwa.h:202-210; window [rmax0, rmax1) of bwa/src/aux.cu:187-205). */
typedef struct {
    uint32_t read_off;    /* base index of read[0] in the planes */
    uint32_t win_off;     /* base index of reference position rmax0 in the planes */
    int32_t  l_query;     /* read length */
    int32_t  qbeg, len;   /* seed on the read */
    int32_t  pad_;
    int64_t  rbeg;        /* seed start on the reference */
    int64_t  rmax0, rmax1;
} g3x_seed_t;             /* 48 bytes */

/* The mem_alnreg_t fields the extension block of mem_chain2aln sets
   (bwa/src/bwa.h:229-247, bwa/src/aux.cu:253-309). */
typedef struct {
    int64_t rb, re;       /* [rb, re) on the reference */
    int32_t qb, qe;       /* [qb, qe) on the read */
    int32_t score, truesc;
    int32_t w;            /* band width used: max over the two sides */
    uint8_t tries_left, tries_right;   /* ksw_extend2 calls made on each side (0-2) */
    uint8_t pad_[2];
} g3x_reg_t;              /* 40 bytes */

/* Left then right extension of n seeds with BWA's band retry, replacing the extension block
   of mem_chain2aln (bwa/src/aux.cu:253-310) for one seed per call.  Device buffers;
   asynchronous on `stream`.  opts->max_qlen / max_tlen bound read and window lengths;
   opts->schedule and lanes pick the extension kernel.  The first call with a larger n
   allocates context scratch (synchronously). */
int g3x_extend_seeds(g3x_ctx *ctx, const g3x_opt_t *opt, const g3x_seed_t *d_seeds, int32_t n,
                     const uint32_t *d_codes, const uint32_t *d_nmask, g3x_reg_t *d_regs,
                     int32_t *d_status, const g3x_batch_opts_t *opts, void *stream);

/* The same over n host seeds in chunks of `chunk` seeds: each chunk's seeds and the plane
   words they reference are copied to the GPU while the chunks before it are extended (seven
   chunks in flight, each with its own device buffer set, pinned staging and compute stream,
   beside one copy stream), and the regions come back to h_regs/h_status.  Host planes should
   be pinned for the copies to overlap.  Blocks until all chunks are done.  A chunk with a
   seed that reaches past n_bases ends the call with G3X_ERR_INVALID before anything of that
   chunk is copied (the chunks before it have their results written).  The buffer sets,
   staging and streams stay in the context, grown when a call needs more, so repeated calls
   allocate nothing. */
int g3x_extend_seeds_stream(g3x_ctx *ctx, const g3x_opt_t *opt, const g3x_seed_t *h_seeds,
                            int64_t n, const uint32_t *h_codes, const uint32_t *h_nmask,
                            int64_t n_bases, g3x_reg_t *h_regs, int32_t *h_status,
                            int32_t chunk, const g3x_batch_opts_t *opts);

/* ---- chain-level extension: mem_chain2aln --------------------------------------------- */
/* Records of the chain-level call, with the fields mem_chain2aln reads or sets
   (bwa/src/bwa.h:202-247, bwa/src/bntseq.h:42-65).  The reference sequence lives in the
   code planes as 2*l_pac bases starting at base ref_off: the forward strand of every contig
   (contig k at anns[k].offset, anns[k].len bases), then its reverse complement, so reference
   position p >= l_pac holds 3 - forward[2*l_pac - 1 - p] (what bns_get_seq_gpu returns for
   the reverse strand, bwa/src/bntseq.cu:39-60).  Every base index (reads, reference) must be
   below 2^32. */
typedef struct {
    int64_t rbeg;         /* seed start in [0, 2*l_pac) */
    int32_t qbeg, len, score;
    int32_t pad_;
} g3x_cseed_t;            /* mem_seed_t, 24 bytes */

typedef struct {
    int32_t seed_beg, n;  /* seeds [seed_beg, seed_beg + n) of the seed array */
    int32_t rid;
    float frac_rep;
} g3x_chain_t;            /* mem_chain_t, 16 bytes */

typedef struct {
    int64_t read_off;     /* base index of read[0] in the planes */
    int32_t l_query;
    int32_t chain_beg, n_chains;   /* the read's chains, processed in this order */
    int32_t pad_;
} g3x_read_t;             /* 24 bytes */

typedef struct {
    int64_t offset;       /* first forward position of the contig */
    int32_t len;
    int32_t pad_;
} g3x_ann_t;              /* bntann1_t, 16 bytes */

typedef struct {
    int64_t l_pac;        /* forward length of the reference */
    int64_t ref_off;      /* base index of reference position 0 in the planes */
    int32_t n_seqs;       /* contigs */
    int32_t pad_;
    const g3x_ann_t *d_anns;   /* n_seqs contigs, device memory, increasing offsets */
} g3x_refinfo_t;          /* 32 bytes */

typedef struct {
    int64_t rb, re;       /* [rb, re) on the reference (2*l_pac coordinates) */
    int32_t qb, qe;       /* [qb, qe) on the read */
    int32_t rid, score, truesc, w, seedcov, seedlen0;
    float frac_rep;
    int32_t pad_;
} g3x_alnreg_t;           /* mem_alnreg_t fields mem_chain2aln sets, 56 bytes */

/* mem_chain2aln (bwa/src/aux.cu:178-315) for every chain of n_reads reads.  A read's chains
   run in order on the read's region list: each chain's reference window is the span its seeds
   can reach (cal_max_gap, aux.cu:168-205) clipped to the first seed's contig and strand
   (bns_fetch_seq_gpu, bwa/src/bntseq.cu:62-87); its seeds run by decreasing (score, index)
   (aux.cu:207-212); a seed inside an earlier region of the read, with no long enough
   earlier seed of the chain overlapping it on another diagonal, is skipped (aux.cu:214-245);
   every other seed is extended left and right with band retry (as g3x_extend_seeds) and gives
   one region with its seed coverage (aux.cu:247-314).  A read's chains must be contiguous in
   d_chains and their seeds contiguous in d_seeds, one chain after the other: read r's
   regions go to d_regs[chains[chain_beg].seed_beg ...] (at most one per seed), their number
   to d_nregs[r], a per-read status to d_status[r] (G3X_OK; G3X_ERR_INVALID for a read whose
   records break these rules; G3X_ERR_TOO_LONG when an extension exceeds the job limits, the
   read's processing stopping there).  A seed's extension depends on nothing but the seed,
   its chain's window and the read, so every seed of the batch is extended in one batch
   through the context's schedule (opts->schedule, lanes, tile, kernel as for
   g3x_extend_seeds; max_qlen / max_tlen are taken from the batch) and the reads' decisions
   are replayed on the results: the same regions as the reference, more DP cells (the
   results of the seeds it skips are discarded).  The host waits for `stream` once, after
   the windows are known.  Allocates context scratch for larger calls. */
int g3x_chain2aln(g3x_ctx *ctx, const g3x_opt_t *opt, const g3x_refinfo_t *ref,
                  const g3x_read_t *d_reads, int32_t n_reads, const g3x_chain_t *d_chains,
                  int32_t n_chains, const g3x_cseed_t *d_seeds, int32_t n_seeds,
                  const uint32_t *d_codes, const uint32_t *d_nmask, g3x_alnreg_t *d_regs,
                  int32_t *d_nregs, int32_t *d_status, const g3x_batch_opts_t *opts, void *stream);

/* ---- the stage's inputs from the reference's own data ----------------------------------- */
/* The packed reference (bwa's pac: base k in byte k >> 2, bits ((~k) & 3) << 1,
   bwa/src/bntseq.cu:4-5) as the 2*l_pac bases that g3x_chain2aln and g3x_pair_generate read:
   the forward strand, then its reverse complement (bns_get_seq_gpu, bwa/src/bntseq.cu:39-60),
   written to the planes at base index `base`.  Device buffers; asynchronous on `stream` (the
   current device).  Only the planes' words holding bases [base, base + 2*l_pac) are written,
   and in the first and last of them only those bases. */
int g3x_pac_to_planes(const uint8_t *d_pac, int64_t l_pac, uint32_t *d_codes, uint32_t *d_nmask,
                      int64_t base, void *stream);

/* g3x_pack_codes on device buffers: len u8 codes (0-3 bases, anything else N) to bases
   [base, base + len) of the planes, e.g. the batch's reads (the reference's d_seq) in one
   call; their read_off is then base + d_seq_offset[r].  Same word rule as above. */
int g3x_pack_codes_device(const uint8_t *d_seq, int64_t len, uint32_t *d_codes, uint32_t *d_nmask,
                          int64_t base, void *stream);

/* One seed of one chain of one read, as the reference's seed_record_t names it (seqID,
   chainID, seedID; bwa/src/bwa.h:272-287), with chain and seed absolute indices into the
   chain and seed arrays (seed relative to its chain). */
typedef struct {
    int32_t read, chain, seed;
} g3x_seedrec_t;          /* 12 bytes */

/* ExtendingPairGenerate (bwa/src/aux.cu:2101-2189) for n_recs seed records: the chain's
   reference window (aux.cu:2134-2156, clipped by bns_fetch_seq_gpu to the first seed's contig
   and strand) as a g3x_seed_t for g3x_extend_seeds (which reads the sequences in place and
   reverses the left side itself), and the window's contig id in d_rid (what the reference
   writes to the region's rid).  d_status[i]: G3X_OK, or G3X_ERR_INVALID for a record that
   indexes outside its arrays (its g3x_seed_t then makes no extension jobs).  Asynchronous on
   `stream` (the current device). */
int g3x_pair_generate(const g3x_opt_t *opt, const g3x_refinfo_t *ref, const g3x_read_t *d_reads,
                      int32_t n_reads, const g3x_chain_t *d_chains, int32_t n_chains,
                      const g3x_cseed_t *d_seeds, int32_t n_seeds, const g3x_seedrec_t *d_recs,
                      int32_t n_recs, g3x_seed_t *d_out, int32_t *d_rid, int32_t *d_status,
                      void *stream);

/* One alignment of the traceback stage, as its seed_record_t names it (seqID, regID;
   bwa/src/bwa.h:272-287), with the region as an absolute index into the region array. */
typedef struct {
    int32_t read, reg;
} g3x_alnrec_t;           /* 8 bytes */

/* The pair preparation of the traceback stage for n_recs alignment records:
   FINALIZEALN_preprocessing2_kernel (bwa/src/aux.cu:2698-2745) and the band cap of
   traceback_baseline (aux.cu:2810-2812, GLOBALSW_BANDWITH_CUTOFF = 500, aux.cuh:428).  Record
   i's region (d_regs[reg], e.g. from g3x_chain2aln) becomes the g3x_ksw_global2_batch job
   d_jobs[i]: query = read [qb, qe) at d_reads[read].read_off + qb, target = the reference slice
   [rb, re) as bns_get_seq_gpu returns it (bwa/src/bntseq.cu:39-60: bounds swapped if reversed,
   clipped to [0, 2 l_pac), empty when it spans the forward/reverse boundary) at ref_off + beg;
   w = 0 when qe - qb == re - rb, else the larger infer_bw (aux.cu:506-513) of the deletion and
   insertion costs for the region's score, at most (max_gap + |tlen - qlen| + 1) / 2, at least
   |tlen - qlen| + 3, then kept as the reference's uint16 and capped at 500; G3X_JOB_MDRC when
   rb >= l_pac.  (The reference's reversal kernel FINALIZEALN_reverseSeq_kernel, aux.cu:
   2755-2790, writes reversed copies that nothing reads, so the slices go in as they are.)
   d_status[i]: G3X_OK; G3X_ERR_INVALID for a record outside its arrays, a region with qe < qb
   or one wholly outside [0, 2 l_pac) (empty job); G3X_ERR_TOO_LONG when a slice is longer than 65535 bases.  Asynchronous
   on `stream` (the current device). */
int g3x_traceback_pairs(const g3x_opt_t *opt, const g3x_refinfo_t *ref, const g3x_read_t *d_reads,
                        int32_t n_reads, const g3x_alnreg_t *d_regs, int32_t n_regs,
                        const g3x_alnrec_t *d_recs, int32_t n_recs, g3x_job_t *d_jobs, int32_t *d_status,
                        void *stream);

/* ---- banded global alignment with backtrack ------------------------------------------- */
/* n calls of ksw_global2 (bwa/src/ksw.cu:706-809) as traceback_baseline issues them
   (bwa/src/aux.cu:2794-2830): job k aligns its query (q_off, qlen) globally to its target
   (t_off, tlen) inside the band |i - j| <= w (the job's w; h0 unused; G3X_JOB_QREV/TREV read
   the planes reversed; a job reaching past the planes' n_bases bases gets G3X_ERR_INVALID,
   unread).  d_score[k] = the reference's return value; the CIGAR (BAM order,
   len << 4 | op, 0 = M, 1 = I, 2 = D, runs merged as push_cigar does, ksw.cu:694-704) goes to
   d_cigar[k * cigar_stride ...] and its length to d_n_cigar[k].  When no alignment inside the
   band reaches the last cell (score <= -2^29) the reference's backtrack reads direction bytes
   it never wrote; here the CIGAR is then empty.  d_status[k]: G3X_OK; G3X_ERR_TOO_LONG for a
   job beyond max_qlen / max_tlen / max_w or whose CIGAR exceeds cigar_stride (empty CIGAR;
   qlen + tlen + 2 always suffices).  With d_nm and d_md (both or neither), NM and the MD
   string follow as the traceback stage computes them after ksw_global2 (bwa/src/aux.cu:2831-2860;
   bases as "ACGTN", or "TGCAN" for jobs with G3X_JOB_MDRC): d_nm[k], and the NUL-terminated MD
   at d_md[k * md_stride] (G3X_ERR_TOO_LONG and an empty string when it does not fit;
   4 (qlen + tlen) + 16 bytes always do).  Scratch: max_tlen x min(max_qlen, 2 max_w + 1) bytes
   per resident warp (at most 8 GiB, fewer warps beyond), allocated in the context for larger
   calls; the jobs are ordered by size with the context's scheduling scratch, so calls on one
   context belong on one stream.  Asynchronous on `stream`. */
#define G3X_JOB_MDRC 4u   /* MD prints the reverse-strand alphabet "TGCAN" */
int g3x_ksw_global2_batch(g3x_ctx *ctx, const g3x_score_t *score, const g3x_job_t *d_jobs, int32_t n,
                          const uint32_t *d_codes, const uint32_t *d_nmask, int64_t n_bases, int32_t max_qlen,
                          int32_t max_tlen, int32_t max_w, int32_t *d_score, uint32_t *d_cigar,
                          int32_t cigar_stride, int32_t *d_n_cigar, int32_t *d_nm, char *d_md,
                          int32_t md_stride, int32_t *d_status, void *stream);

/* ---- striped local alignment with 16-bit cells --------------------------------------- */
/* n calls of ksw_align2 (bwa/src/ksw.cu:271-292 with ksw_qinit :18-64 and ksw_i16 :155-262),
   the local alignment mem_seed_sw runs on the window around a short seed (bwa/src/aux.cu:
   117-143); the reference stops ksw_align2 at its first statement (ksw.cu:276), and this is
   the function as written after it, with 16-bit cells (the only kind its ksw_i16 reads).
   Job k aligns its query (q_off, qlen) locally to its target (t_off, tlen) (h0 and w unused;
   G3X_JOB_QREV/TREV read the planes reversed; a job reaching past the planes' n_bases bases gets
   G3X_ERR_INVALID, unread); d_out[k] is the kswr_t: best score, its end on
   the target (te) and query (qe); with G3X_KSW_XSUBO (minimum score in xtra & 0xffff) the
   best row maximum more than ceil(score / max(mat)) rows from te (score2, te2); with
   G3X_KSW_XSTART the start positions (tb, qb) from the reversed pass, when it finds the same
   score; with G3X_KSW_XSTOP (score in xtra & 0xffff) the pass stops once the best score
   reaches it.  Fields not computed are -1 (g_defr, ksw.cu:5).  d_status[k]: G3X_OK;
   G3X_ERR_INVALID for qlen 0 (the reference reads before its buffers); G3X_ERR_TOO_LONG for
   qlen > 256 or, under XSUBO, tlen > max_tlen.  Returns G3X_ERR_INVALID for G3X_KSW_XBYTE (the
   reference fills an 8-bit profile and reads it as 16-bit cells) and G3X_ERR_SCORE for gap
   costs above 32767 or, under XSUBO, a matrix without a positive score.  Scratch in the
   context (the job order; under XSUBO 4 bytes per job and target row); calls on one context
   belong on one stream.  Asynchronous on `stream`. */
typedef struct {
    int32_t score, te, qe, score2, te2, tb, qb;   /* == kswr_t, bwa/src/ksw.h:24-29 */
} g3x_swr_t;
#define G3X_KSW_XBYTE  0x10000   /* bwa/src/ksw.h:7-10 */
#define G3X_KSW_XSTOP  0x20000
#define G3X_KSW_XSUBO  0x40000
#define G3X_KSW_XSTART 0x80000
int g3x_ksw_align2_batch(g3x_ctx *ctx, const g3x_score_t *score, const g3x_job_t *d_jobs, int32_t n,
                         const uint32_t *d_codes, const uint32_t *d_nmask, int64_t n_bases, int32_t xtra,
                         int32_t max_tlen, g3x_swr_t *d_out, int32_t *d_status, void *stream);

/* The seed filter of long reads: mem_flt_chained_seeds (bwa/src/aux.cu:145-162) for every read,
   as CHAINFILTERING_flt_chained_seeds_kernel runs it (aux.cu:1991-2030), with the window score
   of mem_seed_sw (aux.cu:117-143).  A read is left alone when min_l = 1.1 * min_chain_weight
   (5.5 * logf(l_query) when min_chain_weight is 0) exceeds 0.05 * l_query; otherwise each seed
   shorter than 200 bases whose window (the seed +-50 bases on the read and the reference,
   clipped to the read, to [0, 2 l_pac), to the strand and the contig of the seed's middle) is
   below 200 bases on both gets the score of ksw_align2 over that window, and each chain keeps,
   in order, the seeds without a window (their score becoming len * a) and those scoring at least
   (int)(a * min_l + .499).  d_chains[].n and d_seeds are changed in place, as the reference
   changes its chains; the same layout rules as g3x_chain2aln (a read's chains contiguous, their
   seeds within the seed array; n_bases: the bases the planes hold, windows reaching past them
   are not aligned).  d_sw_score (optional): per seed its window score, -1 without a
   window, -2 for seeds of reads left alone.  d_status[r]: G3X_OK, or G3X_ERR_INVALID for a read
   whose records lie outside their arrays (its chains untouched).  Only the score of ksw_align2
   is used, which its first pass alone decides, so the start-position pass is not run.  Scratch
   in the context; asynchronous on `stream`. */
int g3x_flt_chained_seeds(g3x_ctx *ctx, const g3x_opt_t *opt, int32_t min_chain_weight, const g3x_refinfo_t *ref,
                          const g3x_read_t *d_reads, int32_t n_reads, g3x_chain_t *d_chains, int32_t n_chains,
                          g3x_cseed_t *d_seeds, int32_t n_seeds, const uint32_t *d_codes, const uint32_t *d_nmask,
                          int64_t n_bases, int32_t *d_sw_score, int32_t *d_status, void *stream);

/* ---- host-resident batches, pipelined --------------------------------------------------- */
/* No counterpart in the reference (its batches stay on the device between pipeline stages).
   A pipe extends batches of jobs that live in host memory with the context's schedule and
   width classes, overlapping each batch's copies with its neighbours' extension.  It owns two
   device buffer sets of max_jobs jobs, max_code_words code-plane words and max_nmask_words
   N-plane words, and three streams.  g3x_pipe_submit returns at once: the batch's inputs are
   copied to the next set once the work queued on `stream` before the call is done, the batch
   is extended when they arrive (g3x_ksw_extend2_batch with `schedule`, kernel AUTO), and its
   outputs and per-job statuses are copied to h_out / h_status.  Consecutive submits alternate
   sets, so batch k+1's input copies and batch k-1's output copies run while batch k is
   extended.  g3x_pipe_wait makes `stream` wait for every batch submitted so far: host buffers
   of a batch must stay valid and unchanged until then, and pinned host memory is needed for
   the copies to overlap.  Batches run one at a time on the context's scratch; other calls on
   the same context belong after g3x_pipe_wait.  The first submit of a larger batch may
   allocate context scratch.  G3X_ERR_INVALID for a batch beyond the pipe's sizes. */
typedef struct g3x_pipe g3x_pipe;
int g3x_pipe_create(g3x_ctx *ctx, const g3x_score_t *score, int32_t schedule, int32_t max_jobs,
                    int64_t max_code_words, int64_t max_nmask_words, g3x_pipe **out);
int g3x_pipe_submit(g3x_pipe *p, const g3x_job_t *h_jobs, int32_t n, const uint32_t *h_codes,
                    int64_t code_words, const uint32_t *h_nmask, int64_t nmask_words,
                    int32_t max_qlen, int32_t max_tlen, g3x_ext_t *h_out, int32_t *h_status,
                    void *stream);
int g3x_pipe_wait(g3x_pipe *p, void *stream);
/* Waits for the pipe's batches on the host, then frees it. */
int g3x_pipe_destroy(g3x_pipe *p);

/* ---- CUDA graphs ------------------------------------------------------------------------- */
/* Captures one g3x_ksw_extend2_batch call (all of its kernels and memsets, on the
   context's streams) into an executable CUDA graph bound to these buffers and options;
   g3x_graph_launch replays it on `stream`.  The captured batch reads its inputs when it runs,
   so new jobs written into the same buffers are processed by the next replay. */
typedef struct g3x_graph g3x_graph;
int g3x_graph_capture(g3x_ctx *ctx, const g3x_score_t *score, const g3x_job_t *d_jobs,
                      int32_t n, const uint32_t *d_codes, const uint32_t *d_nmask,
                      g3x_ext_t *d_out, int32_t *d_status, const g3x_batch_opts_t *opts,
                      g3x_graph **graph);
int g3x_graph_launch(g3x_graph *graph, void *stream);
int g3x_graph_destroy(g3x_graph *graph);

/* ---- learned cost model ------------------------------------------------------------------ */
/* A 5 -> 64 -> 64 -> 1 ReLU MLP (fp32) per context that predicts a job's work from five
   features: qlen/128, tlen/256, h0/64, and the ungapped extension along the seed's diagonal
   over the first min(qlen, tlen) bases (from h0, +1 per identical base pair, -4 per other pair,
   N counting as other): its best score / 64 and the number of bases at which it is first
   reached / 128.  Its output is a correction to the length bound: log2(1 + rows) less
   log2(1 + tlen), rows the trips of the row loop of ksw.cu:346 (g3x_batch_opts_t.d_rows), 0 for
   a job that runs to its last row.  Trained on the GPU by the library's own
   forward/backward/Adam kernels; G3X_SCHED_LEARNED orders jobs by log2(1 + tlen) plus
   min(0, prediction + 1): only a predicted end before half the rows moves a job.  No counterpart in the reference (its extension stage has no
   scheduler). */
#define G3X_MLP_FEATURES 5
#define G3X_MLP_PARAMS 4609   /* W1[64][5] b1[64] W2[64][64] b2[64] W3[64] b3 */

/* d_feat[k*5 .. k*5+4] = features of job k; a job reaching past the planes' n_bases bases reads
   none of them (its diagonal features are those of an empty overlap). */
int g3x_features(g3x_ctx *ctx, const g3x_job_t *d_jobs, int32_t n, const uint32_t *d_codes,
                 const uint32_t *d_nmask, int64_t n_bases, float *d_feat, void *stream);
/* Fresh He-style parameters from `seed`; clears the optimiser state. */
int g3x_mlp_init(g3x_ctx *ctx, uint64_t seed);
/* Mini-batch Adam on mean squared error over n samples (d_feat n x 5, d_target n); the
   last mini-batch's loss of each epoch goes to h_epoch_loss[epoch] when not NULL. Blocks. */
int g3x_mlp_train(g3x_ctx *ctx, const float *d_feat, const float *d_target, int32_t n,
                  int32_t epochs, int32_t batch, float lr, uint64_t seed, float *h_epoch_loss);
/* Gradient of the mean squared error over the first n samples (host copy) and the loss. */
int g3x_mlp_gradient(g3x_ctx *ctx, const float *d_feat, const float *d_target, int32_t n,
                     float *h_grad, float *h_loss);
/* d_pred[k] = model output for job k. Asynchronous on `stream`. */
int g3x_mlp_predict(g3x_ctx *ctx, const float *d_feat, int32_t n, float *d_pred, void *stream);
/* d_pred[k] = the correction the learned schedule applies to job k's row key: the features, the
   network in bf16 on the tensor cores (fp32 sums) and the sort key in one kernel, as
   G3X_SCHED_LEARNED computes it (within a few hundredths of g3x_mlp_predict's fp32 value), except
   that a job the network calls early-ending (prediction below -1) gets 0 when one of the 16
   diagonals next to the seed's (offsets 1-8 either way) matches at least 18 of its first 32 base
   pairs: such a job continues past an indel and keeps its place in the length order.
   Asynchronous on `stream`. */
int g3x_mlp_predict_jobs(g3x_ctx *ctx, const g3x_job_t *d_jobs, int32_t n, const uint32_t *d_codes,
                         const uint32_t *d_nmask, int64_t n_bases, float *d_pred, void *stream);
/* Whether G3X_SCHED_LEARNED consults the model (1, the default) or falls back to the length order
   without running the feature and network kernels (0): for workloads where the model predicts
   no early ends, its order is the length order and the inference would only cost time.  The
   trainer (g3sa_b200.learn) sets it from its traces. */
int g3x_mlp_set_active(g3x_ctx *ctx, int32_t active);
int g3x_mlp_get_params(g3x_ctx *ctx, float *h_params);
int g3x_mlp_set_params(g3x_ctx *ctx, const float *h_params);

/* ---- diagnostics ------------------------------------------------------------------------ */

/* No counterpart in the reference: the plain kernel (G3X_SCHED_PLAIN) bounds the steps it spends
   on one job (its wavefront protocol advances a row or a lane every step, so a correct run never
   reaches the bound); a job that reaches it ends with the per-job status G3X_ERR_TIMEOUT and the
   batch goes on.  This sets that bound to `limit` steps for later batches of the context (0: the
   kernel's own bound, 8 (tlen + 2)(qlen + 8) + 4096), so tests can make it run out on normal jobs. */
int g3x_set_step_limit(g3x_ctx *ctx, int64_t limit);

/* Measured 32-bit integer ALU throughput of the context's GPU (ops/s): independent chains of
   the 3-input DPX maximum on every SM.  The cells/s roofline is this figure / 8 (ops per DP
   cell).  No counterpart in the reference. */
int g3x_int_peak(g3x_ctx *ctx, double *ops_per_s);

/* ---- host-side packing ----------------------------------------------------------------- */

/* Packs len u8 codes (0-3 bases, anything else = N) into the planes starting at base index
   `base` (codes/nmask must be large enough and zero-initialised where not yet written).
   Replaces the u8 query/target buffers the reference hands ksw_extend2. */
int g3x_pack_codes(const uint8_t *h_seq, int64_t len, uint32_t *h_codes, uint32_t *h_nmask,
                   int64_t base);

#ifdef __cplusplus
}
#endif
#endif /* G3X_H */

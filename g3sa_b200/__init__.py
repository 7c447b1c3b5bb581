"""g3sa_b200 -- B200-native BWA-MEM seed extension (ksw_extend2 + band retry).

The product is the native library ``libg3x.so`` (sm_100a kernels behind the C ABI in
``include/g3x.h``).  This module is the Python host mirror used by the tests and the
benchmark: numpy record types matching the C structs, a ctypes binding of the C ABI, and
helpers that move torch tensors (device memory and streams) through it.  There is no
Python or CPU fallback for the extension itself: if ``libg3x.so`` cannot be loaded, every
call raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libg3x.so")
SYNTH_PATH = os.path.join(HERE, "libg3x_synth.so")

# ---- status codes (include/g3x.h) ------------------------------------------------------
G3X_OK = 0
G3X_ERR_INVALID = -1
G3X_ERR_SCORE = -2
G3X_ERR_TOO_LONG = -3
G3X_ERR_CUDA = -4
G3X_ERR_TIMEOUT = -5
G3X_ERR_INTERNAL = -6
G3X_ERR_NOMEM = -7
G3X_ERR_NOT_TRAINED = -8

SCHED_PLAIN, SCHED_SORTED, SCHED_LEARNED = 0, 1, 2
JOB_QREV, JOB_TREV, JOB_MDRC = 1, 2, 4

# ---- record types (byte-identical to the C structs) -------------------------------------
SCORE_DT = np.dtype([("mat", "i1", 25), ("pad_", "i1", 3), ("m", "<i4"), ("o_del", "<i4"),
                     ("e_del", "<i4"), ("o_ins", "<i4"), ("e_ins", "<i4"), ("zdrop", "<i4"),
                     ("end_bonus", "<i4")])
JOB_DT = np.dtype([("q_off", "<u4"), ("t_off", "<u4"), ("qlen", "<u2"), ("tlen", "<u2"),
                   ("h0", "<i4"), ("w", "<i4"), ("flags", "<u4")])
EXT_DT = np.dtype([("score", "<i4"), ("qle", "<i4"), ("tle", "<i4"), ("gtle", "<i4"),
                   ("gscore", "<i4"), ("max_off", "<i4")])
# g3x_swr_t == kswr_t (bwa/src/ksw.h:24-29)
SWR_DT = np.dtype([("score", "<i4"), ("te", "<i4"), ("qe", "<i4"), ("score2", "<i4"), ("te2", "<i4"),
                   ("tb", "<i4"), ("qb", "<i4")])
KSW_XBYTE, KSW_XSTOP, KSW_XSUBO, KSW_XSTART = 0x10000, 0x20000, 0x40000, 0x80000
SEED_DT = np.dtype([("read_off", "<i8"), ("win_off", "<i8"), ("rmax0", "<i8"), ("rmax1", "<i8"),
                    ("rbeg", "<i8"), ("l_query", "<i4"), ("qbeg", "<i4"), ("len", "<i4"),
                    ("pad_", "<i4")])
OPT_DT = np.dtype([("score", SCORE_DT), ("a", "<i4"), ("w", "<i4"), ("pen_clip5", "<i4"),
                   ("pen_clip3", "<i4")])
DSEED_DT = np.dtype([("read_off", "<u4"), ("win_off", "<u4"), ("l_query", "<i4"), ("qbeg", "<i4"),
                     ("len", "<i4"), ("pad_", "<i4"), ("rbeg", "<i8"), ("rmax0", "<i8"),
                     ("rmax1", "<i8")])
REG_DT = np.dtype([("rb", "<i8"), ("re", "<i8"), ("qb", "<i4"), ("qe", "<i4"), ("score", "<i4"),
                   ("truesc", "<i4"), ("w", "<i4"), ("tries_left", "u1"), ("tries_right", "u1"),
                   ("pad_", "u1", 2)])
BATCH_OPTS_DT = np.dtype([("schedule", "<i4"), ("max_qlen", "<i4"), ("max_tlen", "<i4"),
                          ("lanes", "<i4"), ("tile", "<i4"), ("kernel", "<i4"), ("d_cells", "<u8"),
                          ("n_bases", "<i8"), ("d_rows", "<u8")])
KERNEL_AUTO, KERNEL_ROLLING, KERNEL_ROWPAR, KERNEL_LANE, KERNEL_LANE16, KERNEL_LANE2, KERNEL_BAND = 0, 1, 2, 3, 4, 5, 6
TILE_DT = np.dtype([("width", "<i4"), ("lanes", "<i4"), ("tile", "<i4"), ("warp_batch", "<i4"),
                    ("refill", "<i4")])
MLP_PARAMS, MLP_FEATURES = 4609, 5
SYNTH_PARAMS_DT = np.dtype([("kind", "<i4"), ("n", "<i4"), ("w", "<i4"), ("a", "<i4"),
                            ("o_del", "<i4"), ("e_del", "<i4"), ("o_ins", "<i4"), ("e_ins", "<i4"),
                            ("threads", "<i4"), ("pad_", "<i4"), ("unrelated", "<f8"),
                            ("seed", "<u8")])
assert SCORE_DT.itemsize == 56 and JOB_DT.itemsize == 24 and EXT_DT.itemsize == 24
# g3x_refinfo_t
REFINFO_DT = np.dtype([("l_pac", "<i8"), ("ref_off", "<i8"), ("n_seqs", "<i4"), ("pad_", "<i4"),
                       ("d_anns", "<u8")])
assert REFINFO_DT.itemsize == 32
assert SEED_DT.itemsize == 56 and OPT_DT.itemsize == 72 and DSEED_DT.itemsize == 48
assert REG_DT.itemsize == 40


def default_opt(w=100, a=1, pen_clip5=5, pen_clip3=5, **score_kw):
    """g3x_opt_t with mem_opt_init defaults (bwa/src/fastmap.cpp:77-113)."""
    o = np.zeros(1, OPT_DT)
    o["score"] = default_score(a=a, **score_kw)
    o["a"], o["w"], o["pen_clip5"], o["pen_clip3"] = a, w, pen_clip5, pen_clip3
    return o


def device_seeds(seeds):
    """SEED_DT records (the generator's / oracle's layout) as g3x_seed_t records."""
    d = np.zeros(len(seeds), DSEED_DT)
    for f in ("read_off", "win_off", "l_query", "qbeg", "len", "rbeg", "rmax0", "rmax1"):
        d[f] = seeds[f]
    return d


def bwa_matrix(a=1, b=4):
    """bwa_fill_scmat (bwa/src/fastmap.cpp:115-124): match a, mismatch -b, N row/column -1."""
    m = np.full((5, 5), -1, np.int8)
    for i in range(4):
        for j in range(4):
            m[i, j] = a if i == j else -b
    return m.ravel()


def default_score(a=1, b=4, o_del=6, e_del=1, o_ins=6, e_ins=1, zdrop=100, end_bonus=5):
    """mem_opt_init defaults (bwa/src/fastmap.cpp:77-113); end_bonus = pen_clip5/3."""
    s = np.zeros(1, SCORE_DT)
    s["mat"][0] = bwa_matrix(a, b)
    s["m"] = 5
    s["o_del"], s["e_del"], s["o_ins"], s["e_ins"] = o_del, e_del, o_ins, e_ins
    s["zdrop"], s["end_bonus"] = zdrop, end_bonus
    return s


# ---- native libraries ------------------------------------------------------------------
_lib = None
_synth = None


def lib():
    """The product library.  Raises if it is missing: there is no fallback."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libg3x.so is not built (python -m g3sa_b200.build)")
        L = ctypes.CDLL(LIB_PATH)
        P, I32 = ctypes.c_void_p, ctypes.c_int32
        L.g3x_ctx_create.argtypes = [ctypes.POINTER(P), ctypes.c_int]
        L.g3x_ctx_create.restype = ctypes.c_int
        L.g3x_ctx_destroy.argtypes = [P]
        L.g3x_ctx_destroy.restype = ctypes.c_int
        L.g3x_strerror.argtypes = [ctypes.c_int]
        L.g3x_strerror.restype = ctypes.c_char_p
        L.g3x_ksw_extend2_batch.argtypes = [P, P, P, I32, P, P, P, P, P, P]
        L.g3x_ksw_extend2_batch.restype = ctypes.c_int
        L.g3x_extend_seeds.argtypes = [P, P, P, I32, P, P, P, P, P, P]
        L.g3x_extend_seeds.restype = ctypes.c_int
        L.g3x_extend_seeds_stream.argtypes = [P, P, P, ctypes.c_int64, P, P, ctypes.c_int64, P, P,
                                              I32, P]
        L.g3x_extend_seeds_stream.restype = ctypes.c_int
        L.g3x_features.argtypes = [P, P, I32, P, P, ctypes.c_int64, P, P]
        L.g3x_mlp_init.argtypes = [P, ctypes.c_uint64]
        L.g3x_mlp_train.argtypes = [P, P, P, I32, I32, I32, ctypes.c_float, ctypes.c_uint64, P]
        L.g3x_mlp_gradient.argtypes = [P, P, P, I32, P, P]
        L.g3x_mlp_predict.argtypes = [P, P, I32, P, P]
        L.g3x_mlp_get_params.argtypes = [P, P]
        L.g3x_mlp_set_params.argtypes = [P, P]
        L.g3x_mlp_set_active.argtypes = [P, I32]
        L.g3x_mlp_predict_jobs.argtypes = [P, P, I32, P, P, ctypes.c_int64, P, P]
        L.g3x_get_tiles.argtypes = [P, P, P]
        L.g3x_set_tiles.argtypes = [P, P, I32]
        L.g3x_autotune.argtypes = [P, P, P, I32, P, P, ctypes.c_int64, I32, I32, P, P]
        L.g3x_autotune_schedule.argtypes = [P, I32, P, P, I32, P, P, ctypes.c_int64, I32, I32, P, P]
        L.g3x_last_stats.argtypes = [P, P]
        L.g3x_set_timing.argtypes = [P, I32]
        L.g3x_set_step_limit.argtypes = [P, ctypes.c_int64]
        L.g3x_set_int16.argtypes = [P, I32]
        L.g3x_class_times.argtypes = [P, P, P, P]
        L.g3x_graph_capture.argtypes = [P, P, P, I32, P, P, P, P, P, ctypes.POINTER(P)]
        L.g3x_graph_launch.argtypes = [P, P]
        L.g3x_graph_destroy.argtypes = [P]
        I64 = ctypes.c_int64
        L.g3x_chain2aln.argtypes = [P, P, P, P, I32, P, I32, P, I32, P, P, P, P, P, P, P]
        L.g3x_chain2aln.restype = ctypes.c_int
        L.g3x_ksw_global2_batch.argtypes = [P, P, P, I32, P, P, I64, I32, I32, I32, P, P, I32, P, P, P, I32, P, P]
        L.g3x_ksw_global2_batch.restype = ctypes.c_int
        L.g3x_ksw_align2_batch.argtypes = [P, P, P, I32, P, P, I64, I32, I32, P, P, P]
        L.g3x_ksw_align2_batch.restype = ctypes.c_int
        L.g3x_flt_chained_seeds.argtypes = [P, P, I32, P, P, I32, P, I32, P, I32, P, P, I64, P, P, P]
        L.g3x_flt_chained_seeds.restype = ctypes.c_int
        L.g3x_pac_to_planes.argtypes = [P, I64, P, P, I64, P]
        L.g3x_pac_to_planes.restype = ctypes.c_int
        L.g3x_pack_codes_device.argtypes = [P, I64, P, P, I64, P]
        L.g3x_pack_codes_device.restype = ctypes.c_int
        L.g3x_pair_generate.argtypes = [P, P, P, I32, P, I32, P, I32, P, I32, P, P, P, P]
        L.g3x_pair_generate.restype = ctypes.c_int
        L.g3x_traceback_pairs.argtypes = [P, P, P, I32, P, I32, P, I32, P, P, P]
        L.g3x_traceback_pairs.restype = ctypes.c_int
        L.g3x_pipe_create.argtypes = [P, P, I32, I32, I64, I64, ctypes.POINTER(P)]
        L.g3x_pipe_create.restype = ctypes.c_int
        L.g3x_pipe_submit.argtypes = [P, P, I32, P, I64, P, I64, I32, I32, P, P, P]
        L.g3x_pipe_submit.restype = ctypes.c_int
        L.g3x_pipe_wait.argtypes = [P, P]
        L.g3x_pipe_wait.restype = ctypes.c_int
        L.g3x_pipe_destroy.argtypes = [P]
        L.g3x_pipe_destroy.restype = ctypes.c_int
        L.g3x_int_peak.argtypes = [P, ctypes.POINTER(ctypes.c_double)]
        L.g3x_int_peak.restype = ctypes.c_int
        L.g3x_pack_codes.argtypes = [P, ctypes.c_int64, P, P, ctypes.c_int64]
        L.g3x_pack_codes.restype = ctypes.c_int
        _lib = L
    return _lib


def synth_lib():
    global _synth
    if _synth is None:
        if not os.path.exists(SYNTH_PATH):
            raise RuntimeError("libg3x_synth.so is not built (python -m g3sa_b200.build)")
        L = ctypes.CDLL(SYNTH_PATH)
        P = ctypes.c_void_p
        L.g3x_synth_create.argtypes = [P]
        L.g3x_synth_create.restype = P
        L.g3x_synth_count.argtypes = [P, ctypes.c_int]
        L.g3x_synth_count.restype = ctypes.c_int64
        L.g3x_synth_copy.argtypes = [P, P, P, P]
        L.g3x_synth_copy.restype = ctypes.c_int
        L.g3x_synth_free.argtypes = [P]
        L.g3x_synth_free.restype = None
        L.g3x_synth_pack.argtypes = [P, ctypes.c_int64, P, P, ctypes.c_int]
        L.g3x_synth_pack.restype = ctypes.c_int
        _synth = L
    return _synth


def strerror(code):
    return lib().g3x_strerror(int(code)).decode()


class G3xError(RuntimeError):
    def __init__(self, code, what=""):
        super().__init__(f"{what}: {strerror(code)} ({code})" if what else f"{strerror(code)} ({code})")
        self.code = code


def _check(rc, what):
    if rc != G3X_OK:
        raise G3xError(rc, what)


# ---- synthetic workloads ---------------------------------------------------------------
class Workload:
    """A generated job set: u8 codes (one byte per base), jobs (JOB_DT) indexing it, seeds."""

    def __init__(self, u8, jobs, seeds):
        self.u8, self.jobs, self.seeds = u8, jobs, seeds
        self._planes = None

    @property
    def n(self):
        return len(self.jobs)

    def planes(self, threads=0):
        """2-bit codes and N-mask planes (uint32) of the whole u8 buffer, base index = byte."""
        if self._planes is None:
            self._planes = pack_planes(self.u8, threads)
        return self._planes

    def cells_upper(self):
        return int((self.jobs["qlen"].astype(np.int64) * self.jobs["tlen"]).sum())


def synth(kind, n, seed, w=100, unrelated=0.2, threads=0, a=1, o_del=6, e_del=1, o_ins=6, e_ins=1):
    """Seeded synthetic jobs; kinds 1 (right extensions), 2 (seeds -> left/right), 4 (long)."""
    L = synth_lib()
    p = np.zeros(1, SYNTH_PARAMS_DT)
    p["kind"], p["n"], p["w"], p["a"] = kind, n, w, a
    p["o_del"], p["e_del"], p["o_ins"], p["e_ins"] = o_del, e_del, o_ins, e_ins
    p["threads"], p["unrelated"], p["seed"] = threads, unrelated, seed
    h = L.g3x_synth_create(p.ctypes.data)
    if not h:
        raise ValueError("bad synth parameters")
    try:
        nj, nb, ns = (L.g3x_synth_count(h, k) for k in range(3))
        jobs = np.zeros(nj, JOB_DT)
        u8 = np.zeros(max(nb, 1), np.uint8)
        seeds = np.zeros(ns, SEED_DT)
        L.g3x_synth_copy(h, jobs.ctypes.data, u8.ctypes.data, seeds.ctypes.data)
    finally:
        L.g3x_synth_free(h)
    return Workload(u8[:nb] if nb else u8[:0], jobs, seeds)


def pack_planes(u8, threads=0):
    n = len(u8)
    codes = np.zeros((n + 31) // 32 * 2 + 2, np.uint32)
    nmask = np.zeros((n + 31) // 32 + 1, np.uint32)
    u8 = np.ascontiguousarray(u8, np.uint8)
    synth_lib().g3x_synth_pack(u8.ctypes.data, n, codes.ctypes.data, nmask.ctypes.data, threads)
    return codes, nmask


# ---- device-side API -------------------------------------------------------------------
class Context:
    """A g3x_ctx bound to one CUDA device."""

    def __init__(self, device=0):
        self._h = ctypes.c_void_p()
        _check(lib().g3x_ctx_create(ctypes.byref(self._h), int(device)), "g3x_ctx_create")
        self.device = device

    def close(self):
        if self._h:
            lib().g3x_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def capture_batch(self, score, d_jobs, n, d_codes, d_nmask, d_out, d_status, max_qlen,
                      max_tlen, schedule=SCHED_SORTED, lanes=0, d_cells=None, tile=0,
                      kernel=KERNEL_AUTO, n_bases=None, d_rows=None):
        """g3x_graph_capture of one batch; returns a Graph whose launch() replays it."""
        opts = np.zeros(1, BATCH_OPTS_DT)
        opts["schedule"], opts["max_qlen"], opts["max_tlen"], opts["lanes"] = (
            schedule, max_qlen, max_tlen, lanes)
        opts["tile"], opts["kernel"] = tile, kernel
        opts["d_cells"] = _ptr(d_cells) if d_cells is not None else 0
        opts["n_bases"] = plane_bases(d_codes, d_nmask, n_bases)
        opts["d_rows"] = _ptr(d_rows) if d_rows is not None else 0
        h = ctypes.c_void_p()
        _check(lib().g3x_graph_capture(self._h, score.ctypes.data, _ptr(d_jobs), int(n), _ptr(d_codes),
                                       _ptr(d_nmask), _ptr(d_out), _ptr(d_status), opts.ctypes.data,
                                       ctypes.byref(h)), "g3x_graph_capture")
        return Graph(h)

    # ---- learned cost model ----
    def features(self, d_jobs, n, d_codes, d_nmask, d_feat, stream=None, n_bases=None):
        _check(lib().g3x_features(self._h, _ptr(d_jobs), int(n), _ptr(d_codes), _ptr(d_nmask),
                                  plane_bases(d_codes, d_nmask, n_bases), _ptr(d_feat), _stream(stream)),
               "g3x_features")

    def mlp_predict_jobs(self, d_jobs, n, d_codes, d_nmask, d_pred, stream=None, n_bases=None):
        """g3x_mlp_predict_jobs: the correction the learned schedule applies per job (its bf16
        tensor-core prediction, or 0 where the near-diagonal check keeps an early call in the
        length order)."""
        _check(lib().g3x_mlp_predict_jobs(self._h, _ptr(d_jobs), int(n), _ptr(d_codes), _ptr(d_nmask),
                                          plane_bases(d_codes, d_nmask, n_bases), _ptr(d_pred), _stream(stream)),
               "g3x_mlp_predict_jobs")

    def mlp_set_active(self, active):
        """g3x_mlp_set_active: 0 makes the learned schedule use the length order, no inference."""
        _check(lib().g3x_mlp_set_active(self._h, int(bool(active))), "g3x_mlp_set_active")

    def mlp_init(self, seed):
        _check(lib().g3x_mlp_init(self._h, int(seed)), "g3x_mlp_init")

    def mlp_train(self, d_feat, d_target, n, epochs, batch, lr, seed=0):
        losses = np.zeros(max(epochs, 1), np.float32)
        _check(lib().g3x_mlp_train(self._h, _ptr(d_feat), _ptr(d_target), int(n), int(epochs),
                                   int(batch), float(lr), int(seed), losses.ctypes.data),
               "g3x_mlp_train")
        return losses[:epochs]

    def mlp_gradient(self, d_feat, d_target, n):
        grad = np.zeros(MLP_PARAMS, np.float32)
        loss = ctypes.c_float()
        _check(lib().g3x_mlp_gradient(self._h, _ptr(d_feat), _ptr(d_target), int(n),
                                      grad.ctypes.data, ctypes.addressof(loss)), "g3x_mlp_gradient")
        return grad, loss.value

    def mlp_predict(self, d_feat, n, d_pred, stream=None):
        _check(lib().g3x_mlp_predict(self._h, _ptr(d_feat), int(n), _ptr(d_pred), _stream(stream)),
               "g3x_mlp_predict")

    def mlp_params(self):
        p = np.zeros(MLP_PARAMS, np.float32)
        _check(lib().g3x_mlp_get_params(self._h, p.ctypes.data), "g3x_mlp_get_params")
        return p

    def mlp_set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        _check(lib().g3x_mlp_set_params(self._h, p.ctypes.data), "g3x_mlp_set_params")

    # ---- width classes / autotuning ----
    def get_tiles(self):
        t = np.zeros(8, TILE_DT)
        n = ctypes.c_int32()
        _check(lib().g3x_get_tiles(self._h, t.ctypes.data, ctypes.addressof(n)), "g3x_get_tiles")
        return [tuple(int(v) for v in row) for row in t[:n.value]]

    def set_tiles(self, tiles):
        t = np.array([tuple(x) for x in tiles], TILE_DT)
        _check(lib().g3x_set_tiles(self._h, t.ctypes.data, len(t)), "g3x_set_tiles")

    def autotune(self, score, d_jobs, n, d_codes, d_nmask, max_qlen, max_tlen, schedule=SCHED_SORTED,
                 n_bases=None):
        t = np.zeros(8, TILE_DT)
        k = ctypes.c_int32()
        _check(lib().g3x_autotune_schedule(self._h, int(schedule), score.ctypes.data, _ptr(d_jobs), int(n),
                                           _ptr(d_codes), _ptr(d_nmask), plane_bases(d_codes, d_nmask, n_bases),
                                           int(max_qlen), int(max_tlen),
                                           t.ctypes.data, ctypes.addressof(k)), "g3x_autotune_schedule")
        return [tuple(int(v) for v in row) for row in t[:k.value]]

    def last_stats(self):
        s = np.zeros(3, np.uint64)
        _check(lib().g3x_last_stats(self._h, s.ctypes.data), "g3x_last_stats")
        return [int(v) for v in s]

    def set_int16(self, enable):
        """g3x_set_int16: False keeps the width classes (and the autotuner) to int32 kernels."""
        _check(lib().g3x_set_int16(self._h, int(bool(enable))), "g3x_set_int16")

    def set_step_limit(self, limit):
        """g3x_set_step_limit: the plain kernel's per-job step bound (0: its own bound)."""
        _check(lib().g3x_set_step_limit(self._h, ctypes.c_int64(int(limit))), "g3x_set_step_limit")

    def set_timing(self, mode):
        """0 off; 1: CUDA events around every class launch of later scheduled batches (classes
        side by side); 2: classes one after another on the caller's stream, each timed alone."""
        _check(lib().g3x_set_timing(self._h, int(mode)), "g3x_set_timing")

    def class_times(self):
        """[(ms, jobs)] per width class of the last timed scheduled batch (ms -1: not run)."""
        ms = np.zeros(8, np.float32)
        jobs = np.zeros(8, np.int32)
        n = ctypes.c_int32()
        _check(lib().g3x_class_times(self._h, ms.ctypes.data, jobs.ctypes.data, ctypes.addressof(n)),
               "g3x_class_times")
        return [(float(ms[k]), int(jobs[k])) for k in range(n.value)]

    def int_peak(self):
        """Measured 32-bit integer ALU ops/s of this GPU (g3x_int_peak)."""
        v = ctypes.c_double()
        _check(lib().g3x_int_peak(self._h, ctypes.byref(v)), "g3x_int_peak")
        return v.value

    def extend_batch(self, score, d_jobs, n, d_codes, d_nmask, d_out, d_status, max_qlen,
                     max_tlen, schedule=SCHED_PLAIN, lanes=0, d_cells=None, stream=None,
                     tile=0, kernel=KERNEL_AUTO, n_bases=None, d_rows=None):
        """g3x_ksw_extend2_batch on torch device tensors (or raw device pointers)."""
        opts = np.zeros(1, BATCH_OPTS_DT)
        opts["schedule"], opts["max_qlen"], opts["max_tlen"], opts["lanes"] = (
            schedule, max_qlen, max_tlen, lanes)
        opts["tile"], opts["kernel"] = tile, kernel
        opts["d_cells"] = _ptr(d_cells) if d_cells is not None else 0
        opts["n_bases"] = plane_bases(d_codes, d_nmask, n_bases)
        opts["d_rows"] = _ptr(d_rows) if d_rows is not None else 0
        rc = lib().g3x_ksw_extend2_batch(self._h, score.ctypes.data, _ptr(d_jobs), int(n),
                                         _ptr(d_codes), _ptr(d_nmask), _ptr(d_out),
                                         _ptr(d_status), opts.ctypes.data, _stream(stream))
        _check(rc, "g3x_ksw_extend2_batch")


    def extend_seeds(self, opt, d_seeds, n, d_codes, d_nmask, d_regs, d_status, max_qlen,
                     max_tlen, schedule=SCHED_SORTED, lanes=0, stream=None, tile=0,
                     kernel=KERNEL_AUTO, n_bases=None):
        """g3x_extend_seeds: left + right extension with band retry on device buffers."""
        opts = np.zeros(1, BATCH_OPTS_DT)
        opts["schedule"], opts["max_qlen"], opts["max_tlen"], opts["lanes"] = (
            schedule, max_qlen, max_tlen, lanes)
        opts["tile"], opts["kernel"] = tile, kernel
        opts["n_bases"] = plane_bases(d_codes, d_nmask, n_bases)
        rc = lib().g3x_extend_seeds(self._h, opt.ctypes.data, _ptr(d_seeds), int(n), _ptr(d_codes),
                                    _ptr(d_nmask), _ptr(d_regs), _ptr(d_status), opts.ctypes.data,
                                    _stream(stream))
        _check(rc, "g3x_extend_seeds")

    def chain2aln(self, opt, l_pac, ref_off, d_anns, n_seqs, d_reads, n_reads, d_chains, n_chains,
                  d_seeds, n_seeds, d_codes, d_nmask, d_regs, d_nregs, d_status,
                  schedule=SCHED_SORTED, lanes=0, tile=0, kernel=KERNEL_AUTO, stream=None, n_bases=None):
        """g3x_chain2aln on device buffers (records of g3sa_b200.chains: READ_DT, CHAIN_DT,
        CSEED_DT, ANN_DT in; ALNREG_DT per seed slot, nregs and status per read out)."""
        ri = np.zeros(1, REFINFO_DT)
        ri["l_pac"], ri["ref_off"], ri["n_seqs"], ri["d_anns"] = l_pac, ref_off, n_seqs, _ptr(d_anns)
        opts = np.zeros(1, BATCH_OPTS_DT)
        opts["schedule"], opts["lanes"], opts["tile"], opts["kernel"] = schedule, lanes, tile, kernel
        opts["n_bases"] = plane_bases(d_codes, d_nmask, n_bases)
        rc = lib().g3x_chain2aln(self._h, opt.ctypes.data, ri.ctypes.data, _ptr(d_reads), int(n_reads),
                                 _ptr(d_chains), int(n_chains), _ptr(d_seeds), int(n_seeds), _ptr(d_codes),
                                 _ptr(d_nmask), _ptr(d_regs), _ptr(d_nregs), _ptr(d_status), opts.ctypes.data,
                                 _stream(stream))
        _check(rc, "g3x_chain2aln")

    def global_batch(self, score, d_jobs, n, d_codes, d_nmask, max_qlen, max_tlen, max_w, d_score, d_cigar,
                     cigar_stride, d_n_cigar, d_status, d_nm=None, d_md=None, md_stride=0, stream=None,
                     n_bases=None):
        """g3x_ksw_global2_batch on device buffers (JOB_DT jobs; the job's w is the band; NM/MD
        when d_nm and d_md are given)."""
        _check(lib().g3x_ksw_global2_batch(self._h, score.ctypes.data, _ptr(d_jobs), int(n), _ptr(d_codes),
                                           _ptr(d_nmask), plane_bases(d_codes, d_nmask, n_bases), int(max_qlen),
                                           int(max_tlen), int(max_w), _ptr(d_score),
                                           _ptr(d_cigar), int(cigar_stride), _ptr(d_n_cigar), _ptr(d_nm),
                                           _ptr(d_md), int(md_stride), _ptr(d_status), _stream(stream)),
               "g3x_ksw_global2_batch")

    def align2_batch(self, score, d_jobs, n, d_codes, d_nmask, xtra, max_tlen, d_out, d_status, stream=None,
                     n_bases=None):
        """g3x_ksw_align2_batch on device buffers: JOB_DT jobs, SWR_DT results (kswr_t), the
        KSW_X* flags in xtra."""
        _check(lib().g3x_ksw_align2_batch(self._h, score.ctypes.data, _ptr(d_jobs), int(n), _ptr(d_codes),
                                          _ptr(d_nmask), plane_bases(d_codes, d_nmask, n_bases), int(xtra),
                                          int(max_tlen), _ptr(d_out), _ptr(d_status),
                                          _stream(stream)),
               "g3x_ksw_align2_batch")

    def flt_chained_seeds(self, opt, min_chain_weight, l_pac, ref_off, d_anns, n_seqs, d_reads, n_reads, d_chains,
                          n_chains, d_seeds, n_seeds, d_codes, d_nmask, d_status, d_sw_score=None, stream=None,
                          n_bases=None):
        """g3x_flt_chained_seeds on device buffers (the chain and seed arrays change in place)."""
        ri = np.zeros(1, REFINFO_DT)
        ri["l_pac"], ri["ref_off"], ri["n_seqs"], ri["d_anns"] = l_pac, ref_off, n_seqs, _ptr(d_anns)
        _check(lib().g3x_flt_chained_seeds(self._h, opt.ctypes.data, int(min_chain_weight), ri.ctypes.data,
                                           _ptr(d_reads), int(n_reads), _ptr(d_chains), int(n_chains), _ptr(d_seeds),
                                           int(n_seeds), _ptr(d_codes), _ptr(d_nmask),
                                           plane_bases(d_codes, d_nmask, n_bases), _ptr(d_sw_score),
                                           _ptr(d_status), _stream(stream)),
               "g3x_flt_chained_seeds")

    def extend_seeds_stream(self, opt, seeds, codes, nmask, n_bases, regs, status, max_qlen,
                            max_tlen, chunk=65536, schedule=SCHED_SORTED, lanes=0, tile=0,
                            kernel=KERNEL_AUTO):
        """g3x_extend_seeds_stream on host arrays: numpy DSEED_DT records, or a pinned torch
        tensor holding them (any dtype: the seed count is its byte size / 48)."""
        if isinstance(seeds, np.ndarray):
            if seeds.dtype != DSEED_DT:
                raise ValueError("seeds must be DSEED_DT records (device_seeds())")
            n_seeds = len(seeds)
        elif hasattr(seeds, "element_size"):
            nbytes = seeds.numel() * seeds.element_size()
            if nbytes % DSEED_DT.itemsize:
                raise ValueError("seed tensor size is not a whole number of g3x_seed_t records")
            n_seeds = nbytes // DSEED_DT.itemsize
        else:
            n_seeds = len(seeds)
        opts = np.zeros(1, BATCH_OPTS_DT)
        opts["schedule"], opts["max_qlen"], opts["max_tlen"], opts["lanes"] = (
            schedule, max_qlen, max_tlen, lanes)
        opts["tile"], opts["kernel"] = tile, kernel
        opts["n_bases"] = n_bases
        hp = lambda a: a.ctypes.data if isinstance(a, np.ndarray) else a.data_ptr()  # noqa: E731
        rc = lib().g3x_extend_seeds_stream(self._h, opt.ctypes.data, hp(seeds), n_seeds, hp(codes),
                                           hp(nmask), int(n_bases), hp(regs), hp(status), int(chunk),
                                           opts.ctypes.data)
        _check(rc, "g3x_extend_seeds_stream")


def _host_ptr(a):
    return a.ctypes.data if isinstance(a, np.ndarray) else a.data_ptr()


def _nbytes(a):
    return a.nbytes if isinstance(a, np.ndarray) else a.numel() * a.element_size()


def pac_to_planes(d_pac, l_pac, d_codes, d_nmask, base, stream=None):
    """g3x_pac_to_planes: bwa's packed reference (device bytes) to forward + reverse-complement
    planes at base index `base`."""
    _check(lib().g3x_pac_to_planes(_ptr(d_pac), int(l_pac), _ptr(d_codes), _ptr(d_nmask), int(base),
                                   _stream(stream)), "g3x_pac_to_planes")


def pack_codes_device(d_seq, n, d_codes, d_nmask, base, stream=None):
    """g3x_pack_codes_device: n u8 codes (device) to the planes at base index `base`."""
    _check(lib().g3x_pack_codes_device(_ptr(d_seq), int(n), _ptr(d_codes), _ptr(d_nmask), int(base),
                                       _stream(stream)), "g3x_pack_codes_device")


def pair_generate(opt, l_pac, ref_off, d_anns, n_seqs, d_reads, n_reads, d_chains, n_chains, d_seeds,
                  n_seeds, d_recs, n_recs, d_out, d_rid, d_status, stream=None):
    """g3x_pair_generate: per seed record (SEEDREC_DT) its g3x_seed_t (DSEED_DT) and contig id."""
    ri = np.zeros(1, REFINFO_DT)
    ri["l_pac"], ri["ref_off"], ri["n_seqs"], ri["d_anns"] = l_pac, ref_off, n_seqs, _ptr(d_anns)
    _check(lib().g3x_pair_generate(opt.ctypes.data, ri.ctypes.data, _ptr(d_reads), int(n_reads), _ptr(d_chains),
                                   int(n_chains), _ptr(d_seeds), int(n_seeds), _ptr(d_recs), int(n_recs),
                                   _ptr(d_out), _ptr(d_rid), _ptr(d_status), _stream(stream)), "g3x_pair_generate")


SEEDREC_DT = np.dtype([("read", "<i4"), ("chain", "<i4"), ("seed", "<i4")])
# g3x_alnrec_t: one alignment of the traceback stage (read, absolute region index)
ALNREC_DT = np.dtype([("read", "<i4"), ("reg", "<i4")])


def traceback_pairs(opt, l_pac, ref_off, d_reads, n_reads, d_regs, n_regs, d_recs, n_recs, d_jobs, d_status,
                    stream=None):
    """g3x_traceback_pairs: per alignment record (ALNREC_DT) the ksw_global2 job (JOB_DT) of its
    region, as the traceback stage prepares it."""
    ri = np.zeros(1, REFINFO_DT)
    ri["l_pac"], ri["ref_off"] = l_pac, ref_off
    _check(lib().g3x_traceback_pairs(opt.ctypes.data, ri.ctypes.data, _ptr(d_reads), int(n_reads), _ptr(d_regs),
                                     int(n_regs), _ptr(d_recs), int(n_recs), _ptr(d_jobs), _ptr(d_status),
                                     _stream(stream)), "g3x_traceback_pairs")


class Pipe:
    """g3x_pipe: batches in host memory (numpy arrays or pinned torch tensors), extended with
    the context's schedule while the neighbouring batches' copies run.  submit() returns at
    once; wait(stream) makes `stream` wait for every submitted batch, after which the output
    buffers hold the results.  Host buffers must stay alive and unchanged until then."""

    def __init__(self, ctx, score, schedule, max_jobs, max_code_words, max_nmask_words):
        self._score = np.ascontiguousarray(score)
        self._ctx = ctx
        h = ctypes.c_void_p()
        _check(lib().g3x_pipe_create(ctx._h, self._score.ctypes.data, int(schedule), int(max_jobs),
                                     int(max_code_words), int(max_nmask_words), ctypes.byref(h)),
               "g3x_pipe_create")
        self._h = h.value

    def submit(self, jobs, n, codes, nmask, max_qlen, max_tlen, out, status, stream=None):
        """jobs: JOB_DT records (or their bytes); codes/nmask: the uint32 planes (or their
        bytes); out: n x 6 int32 (g3x_ext_t); status: n int32."""
        rc = lib().g3x_pipe_submit(self._h, _host_ptr(jobs), int(n), _host_ptr(codes), _nbytes(codes) // 4,
                                   _host_ptr(nmask), _nbytes(nmask) // 4, int(max_qlen), int(max_tlen),
                                   _host_ptr(out), _host_ptr(status), _stream(stream))
        _check(rc, "g3x_pipe_submit")

    def wait(self, stream=None):
        _check(lib().g3x_pipe_wait(self._h, _stream(stream)), "g3x_pipe_wait")

    def close(self):
        if self._h:
            lib().g3x_pipe_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Graph:
    """An executable CUDA graph of one captured batch (g3x_graph)."""

    def __init__(self, h):
        self._h = h

    def launch(self, stream=None):
        _check(lib().g3x_graph_launch(self._h, _stream(stream)), "g3x_graph_launch")

    def close(self):
        if self._h:
            lib().g3x_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def plane_bases(d_codes, d_nmask, n_bases=None):
    """The bases a pair of planes holds: n_bases when given, else what the two buffers' sizes
    cover (16 bases per code word, 32 per N-mask word); raw pointers need n_bases."""
    if n_bases is not None:
        return int(n_bases)
    if isinstance(d_codes, int) or isinstance(d_nmask, int):
        raise ValueError("n_bases is needed for planes given as raw pointers")
    return min(_nbytes(d_codes) // 4 * 16, _nbytes(d_nmask) // 4 * 32, 1 << 32)


def _ptr(t):
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return t.data_ptr()


def _stream(s):
    if s is None:
        return None
    return s.cuda_stream if hasattr(s, "cuda_stream") else int(s)

"""What ordering by the job's true cost buys the row-synchronous lane kernel, on a CPU model:
a warp takes 32 consecutive jobs of a width class and runs until the longest is done, each row
costing the widest row's blocks, so its work is max(rows) x max(blocks per row) per batch of
32.  Ordering by the cost the learned model predicts (here: the true cells, the model's
target) leaves less of that work idle than the length-sorted fallback (tlen), because jobs
that z-drop early (unrelated targets) no longer share warps with full-length ones."""
import numpy as np

import g3sa_b200 as g
from tests import native as nat

WIDTHS = np.array([16, 40, 72, 104, 144, 184, 232, 1 << 30])


def warp_efficiency(order_key, rows, blocks, cls):
    useful = total = 0
    for k in range(len(WIDTHS)):
        idx = np.nonzero(cls == k)[0]
        if idx.size < 32:
            continue
        o = idx[np.lexsort(order_key(idx))]
        n = len(o) // 32 * 32
        r = rows[o[:n]].reshape(-1, 32).astype(np.int64)
        b = blocks[o[:n]].reshape(-1, 32).astype(np.int64)
        total += (r.max(1) * b.max(1)).sum() * 32
        useful += (r * b).sum()
    return useful / total


def test_cost_order_beats_length_order():
    wl = g.synth(2, 20000, seed=0x5C4ED, w=100, unrelated=0.2)
    _, cells, rows = nat.oracle_extend(wl.jobs, wl.u8, g.default_score())
    q = wl.jobs["qlen"].astype(np.int64)
    t = wl.jobs["tlen"].astype(np.int64)
    wide = np.minimum(q, 201)
    blocks = np.maximum(1, (wide + 7) // 8)
    cls = np.searchsorted(WIDTHS, q, side="left")
    wbin = lambda idx: 31 - np.minimum((wide[idx] + 7) >> 3, 31)            # noqa: E731
    rbin = lambda lr: np.clip(((16 - lr) * 4).astype(int), 0, 63)           # noqa: E731
    sorted_key = lambda idx: (wbin(idx), rbin(np.log2(1 + t[idx])))       # noqa: E731
    cost_key = lambda idx: (wbin(idx), rbin(np.log2(1 + cells[idx]) - np.log2(np.maximum(wide[idx], 1))))  # noqa: E731
    e_sorted = warp_efficiency(sorted_key, rows, blocks, cls)
    e_cost = warp_efficiency(cost_key, rows, blocks, cls)
    assert e_cost > e_sorted + 0.08, (e_cost, e_sorted)
    assert e_cost > 0.9


def test_learned_target_is_a_correction_below_the_length_bound():
    """The cost model's training target, log2(1 + rows) less log2(1 + tlen), is never positive
    (the row loop of ksw.cu:346 runs at most tlen times), exactly 0 for the jobs that run to
    their last row, and clearly negative where the z-drop ends a job early (unrelated
    targets)."""
    from g3sa_b200 import learn
    sc = g.default_score()
    wl = g.synth(2, 4000, seed=0x7A26, w=100, unrelated=0.2)
    _, _, rows = nat.oracle_extend(wl.jobs, wl.u8, sc)
    tlen = wl.jobs["tlen"]
    tgt = learn.row_target(np.asarray(rows), tlen)
    assert tgt.dtype == np.float32 and (tgt <= 0).all()
    full = rows == tlen
    assert full.mean() > 0.5 and (tgt[full] == 0).all()
    assert np.percentile(tgt[~full], 25) < -1.0      # a quarter of them end before half their rows

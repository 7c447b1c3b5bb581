"""The kernels' warp protocol (g3x_core.h), run on the CPU lane by lane by libg3x_emu.so,
against the oracle.  Also checks the two properties the kernels rely on: no two lanes touch
the same row-buffer slot in one step, and at most one row ends per step."""
import numpy as np
import pytest

import g3sa_b200 as g
from tests import golden_io, native as nat


@pytest.mark.parametrize("G", [2, 3, 8, 16, 32])
@pytest.mark.parametrize("name", ["cfg1", "cfg2", "edge", "stale", "score2", "nozdrop", "cfg4_w100"])
def test_emu_matches_golden(name, G):
    u8, jobs, score, ext = golden_io.load_jobs(name)
    codes, nmask = g.pack_planes(u8)
    out, status, cells, stats = nat.emu_extend(jobs, codes, nmask, score, G)
    assert (status == 0).all()
    bad = np.nonzero((out != ext).any(1))[0]
    assert bad.size == 0, f"{name} G={G}: jobs {bad[:5]}"
    assert stats[:, 3].sum() == 0, "two lanes touched one slot in a step"
    assert stats[:, 2].max() <= 1, "more than one row ended in a step"


@pytest.mark.parametrize("G", [8, 16])
def test_emu_cells_match_oracle(G):
    wl = g.synth(2, 1500, seed=31, w=100)
    sc = g.default_score()
    ref, cells, rows = nat.oracle_extend(wl.jobs, wl.u8, sc)
    codes, nmask = wl.planes()
    out, status, c, stats = nat.emu_extend(wl.jobs, codes, nmask, sc, G)
    assert (out == ref).all()
    assert (c == cells).all()
    # speculative rows computed past the row that ends the extension stay rare
    assert stats[:, 1].sum() <= 1.01 * cells.sum()


def test_emu_w_variants():
    sc = g.default_score()
    for w in (1, 3, 10, 40):
        wl = g.synth(1, 400, seed=40 + w, w=w, unrelated=0.2)
        ref, _, _ = nat.oracle_extend(wl.jobs, wl.u8, sc)
        codes, nmask = wl.planes()
        out, status, _, _ = nat.emu_extend(wl.jobs, codes, nmask, sc, 8)
        assert (out == ref).all(), w

"""The per-lane logic of the int16x2 lane kernel (g3sa_b200/csrc/g3x_lane16.cuh), run on the
CPU by its model (libg3x_emu16.so), against the golden vectors made by the reference's own
ksw_extend2 and against the oracle on fresh seeded workloads: all six outputs and the per-job
cell counts, for every job inside the kernel's int16 fit.  The model starts each job on a row
buffer of stale words (checking the closed-form row -1 against init_h; status -6 otherwise) and
walks each row with a varying number of warp iterations, as the kernel's lanes do."""
import numpy as np
import pytest

import g3sa_b200 as g
from tests import golden_io, native as nat


@pytest.mark.parametrize("name", golden_io.job_sets())
def test_lane16_model_matches_golden(name):
    u8, jobs, score, ext = golden_io.load_jobs(name)
    out, cells, status = nat.emu16_extend(jobs, u8, score)
    assert set(np.unique(status)) <= {0, -3}       # ok, or outside the int16 fit
    ok = status == 0
    assert ok.any() or name.startswith("cfg4")
    bad = np.nonzero((out[ok] != ext[ok]).any(1))[0]
    assert bad.size == 0, f"{name}: first mismatching jobs {np.nonzero(ok)[0][bad[:5]]}"
    _, ocells, _ = nat.oracle_extend(jobs, u8, score)
    assert (cells[ok] == ocells[ok]).all()


@pytest.mark.parametrize("kind,n,w,unrel", [(2, 6000, 100, 0.2), (1, 8000, 100, 0.0), (2, 4000, 7, 0.2),
                                            (2, 3000, 30, 0.5)])
def test_lane16_model_matches_oracle_fresh(kind, n, w, unrel):
    wl = g.synth(kind, n, seed=4242 + kind + w, w=w, unrelated=unrel)
    sc = g.default_score()
    out, cells, status = nat.emu16_extend(wl.jobs, wl.u8, sc)
    ref, rcells, _ = nat.oracle_extend(wl.jobs, wl.u8, sc)
    assert set(np.unique(status)) <= {0, -3}
    ok = status == 0
    assert ok.mean() > 0.95
    bad = np.nonzero((out[ok] != ref[ok]).any(1))[0]
    assert bad.size == 0, f"first mismatching jobs {np.nonzero(ok)[0][bad[:5]]}"
    assert (cells[ok] == rcells[ok]).all()


def test_lane16_model_asymmetric_gaps():
    """o_del != o_ins: the E step takes its own max(M - oe_del, 0)."""
    wl = g.synth(2, 3000, seed=515, w=100, unrelated=0.2)
    sc = g.default_score(o_del=5, e_del=2, o_ins=7, e_ins=1)
    out, cells, status = nat.emu16_extend(wl.jobs, wl.u8, sc)
    ref, rcells, _ = nat.oracle_extend(wl.jobs, wl.u8, sc)
    assert set(np.unique(status)) <= {0, -3}
    ok = status == 0
    assert ok.mean() > 0.9
    assert (out[ok] == ref[ok]).all() and (cells[ok] == rcells[ok]).all()

"""g3x_ksw_extend2_batch_noalloc: the sorted-schedule batch whose scratch is the library's
static device array.  Its outputs must equal the oracle's (and g3x_ksw_extend2_batch's with
G3X_SCHED_SORTED) on the same jobs, on two calls in a row -- the second call reuses the array
the first one left behind, and leaves the device's free memory as it found it.  This file is
collected last so that it also runs after every other test in one process."""
import ctypes

import numpy as np
import pytest

import g3sa_b200 as g

G3X_ERR_SCRATCH = -9
G3X_NOALLOC_MAX_JOBS = 1048576


def _bind():
    lib = g.lib()
    fn = lib.g3x_ksw_extend2_batch_noalloc
    P, I32 = ctypes.c_void_p, ctypes.c_int32
    fn.argtypes = [ctypes.c_int, P, P, I32, P, P, ctypes.c_int64, P, P, I32, I32, P]
    fn.restype = ctypes.c_int
    return fn


def test_noalloc_rejects_batches_beyond_its_scratch():
    # Checked on the host before any device work, so this runs without a GPU.
    fn = _bind()
    sc = g.default_score()
    dummy = ctypes.c_void_p(16)
    rc = fn(0, sc.ctypes.data, dummy, G3X_NOALLOC_MAX_JOBS + 1, dummy, dummy, 1 << 20, dummy, dummy,
            100, 300, None)
    assert rc == G3X_ERR_SCRATCH
    assert b"1048576" in g.lib().g3x_strerror(rc)


@pytest.mark.gpu
def test_noalloc_matches_oracle_and_sorted_batch_on_two_calls():
    import torch
    from tests import native as nat
    from tests.gpu_util import run_batch, to_dev

    fn = _bind()
    sc = g.default_score()
    # set-up call: looks the scratch array's address up on this device
    assert fn(0, sc.ctypes.data, None, 0, None, None, 0, None, None, 0, 0, None) == 0
    batches = [g.synth(2, 1500, seed=0x5EED1, w=100, unrelated=0.2),
               g.synth(1, 2500, seed=0x5EED2, w=100, unrelated=0.2)]
    for call, wl in enumerate(batches):
        n = wl.n
        mq, mt = int(wl.jobs["qlen"].max()), int(wl.jobs["tlen"].max())
        ref, _, _ = nat.oracle_extend(wl.jobs, wl.u8, sc)
        want, want_status, _ = run_batch(wl.u8, wl.jobs, sc, schedule=g.SCHED_SORTED)
        assert (want_status == 0).all()
        np.testing.assert_array_equal(want, ref)

        codes, nmask = wl.planes()
        d_jobs, d_codes, d_nmask = to_dev(wl.jobs), to_dev(codes), to_dev(nmask)
        out = torch.full((n, 6), -777, dtype=torch.int32, device="cuda")
        status = torch.full((n,), 99, dtype=torch.int32, device="cuda")
        stream = torch.cuda.current_stream()
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc = fn(0, sc.ctypes.data, d_jobs.data_ptr(), n, d_codes.data_ptr(), d_nmask.data_ptr(),
                g.plane_bases(d_codes, d_nmask), out.data_ptr(), status.data_ptr(), mq, mt,
                ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, g.lib().g3x_strerror(rc)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        if call > 0:
            # the first call may load the library's kernels; the second allocates nothing
            assert free1 == free0, f"device memory changed by {free0 - free1} bytes"
        assert (status.cpu().numpy() == 0).all()
        np.testing.assert_array_equal(out.cpu().numpy(), ref)

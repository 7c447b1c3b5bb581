"""C-ABI surface checks that need no GPU: every function include/g3x.h declares is exported
by libg3x.so, the record layouts match, host-side packing is exact, and calls fail with
status codes (not crashes) when no GPU is present or arguments are bad."""
import ctypes
import os
import re

import numpy as np
import pytest

import g3sa_b200 as g

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ \*]*?\b(g3x_[a-z0-9_]+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from g3sa_b200 import build
    build.build_lib()
    return g.lib()


def test_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert "g3x_ksw_extend2_batch" in names and len(names) >= 5
    for n in names:
        assert hasattr(lib, n), n


def test_record_sizes():
    assert g.SCORE_DT.itemsize == 56
    assert g.JOB_DT.itemsize == 24
    assert g.EXT_DT.itemsize == 24
    assert g.BATCH_OPTS_DT.itemsize == 48


def test_batch_opts_layout_matches_header(tmp_path):
    """The options record the bindings build has the C struct's size and field offsets."""
    import subprocess
    src = tmp_path / "opts.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "g3x.h"\nint main(void) {\n'
                   '  printf("%zu %zu %zu %zu %zu\\n", sizeof(g3x_batch_opts_t), offsetof(g3x_batch_opts_t, kernel),\n'
                   '         offsetof(g3x_batch_opts_t, d_cells), offsetof(g3x_batch_opts_t, n_bases),\n'
                   '         offsetof(g3x_batch_opts_t, d_rows));\n'
                   '  return 0;\n}\n')
    exe = tmp_path / "opts"
    subprocess.check_call(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    size, kern, cells, nb, rows = (int(v) for v in subprocess.check_output([str(exe)]).split())
    dt = g.BATCH_OPTS_DT
    assert (size, kern, cells, nb, rows) == (dt.itemsize, dt.fields["kernel"][1], dt.fields["d_cells"][1],
                                             dt.fields["n_bases"][1], dt.fields["d_rows"][1])


def test_noalloc_rejects_a_missing_plane_length(lib):
    fn = lib.g3x_ksw_extend2_batch_noalloc
    fn.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                   ctypes.c_int32, ctypes.c_void_p]
    dummy = ctypes.c_void_p(16)
    sc = g.default_score()
    for nb in (0, -5, (1 << 32) + 1):
        assert fn(0, sc.ctypes.data, dummy, 10, dummy, dummy, nb, dummy, dummy, 100, 300, None) == g.G3X_ERR_INVALID


def test_pack_codes_roundtrip(lib):
    rng = np.random.default_rng(0)
    seq = rng.integers(0, 6, 1000).astype(np.uint8)
    codes = np.zeros(80, np.uint32)
    nmask = np.zeros(40, np.uint32)
    base = 37
    assert lib.g3x_pack_codes(seq.ctypes.data, len(seq), codes.ctypes.data, nmask.ctypes.data, base) == 0
    b = np.arange(base, base + len(seq))
    got = (codes[b >> 4] >> ((b & 15) * 2)) & 3
    nb = (nmask[b >> 5] >> (b & 31)) & 1
    dec = np.where(nb == 1, 4, got)
    assert (dec == np.minimum(seq, 4)).all()
    # the threaded packer used for bulk streams agrees
    u8 = np.zeros(base + len(seq), np.uint8)
    u8[base:] = np.minimum(seq, 4)
    c2, n2 = g.pack_planes(u8)
    nb2 = (n2[b >> 5] >> (b & 31)) & 1
    dec2 = np.where(nb2 == 1, 4, (c2[b >> 4] >> ((b & 15) * 2)) & 3)
    assert (nb2 == nb).all() and (dec2 == dec).all()


def test_strerror(lib):
    for code in range(0, -9, -1):
        assert g.strerror(code) != "unknown error"
    assert g.strerror(-99) == "unknown error"


def test_bad_arguments_return_codes(lib):
    assert lib.g3x_ctx_destroy(None) == g.G3X_ERR_INVALID
    assert lib.g3x_ksw_extend2_batch(None, None, None, 1, None, None, None, None, None, None) == g.G3X_ERR_INVALID
    assert lib.g3x_pack_codes(None, 5, None, None, 0) == g.G3X_ERR_INVALID


def test_widened_entry_points_reject_bad_arguments(lib):
    """The entry points of the rows around the extension check their arguments before any CUDA
    call: no context, negative counts, missing buffers and refused flags return codes."""
    sc = g.default_score()
    assert lib.g3x_ksw_global2_batch(None, sc.ctypes.data, None, 1, None, None, 1000, 10, 10, 5, None, None, 4,
                                     None, None, None, 0, None, None) == g.G3X_ERR_INVALID
    assert lib.g3x_ksw_align2_batch(None, sc.ctypes.data, None, 1, None, None, 1000, 0, 0, None, None, None) == \
        g.G3X_ERR_INVALID
    opt = g.default_opt()
    ri = np.zeros(1, g.REFINFO_DT)
    ri["l_pac"], ri["ref_off"] = 1000, 0
    assert lib.g3x_traceback_pairs(opt.ctypes.data, ri.ctypes.data, None, 1, None, 1, None, -1, None, None,
                                   None) == g.G3X_ERR_INVALID
    assert lib.g3x_traceback_pairs(opt.ctypes.data, ri.ctypes.data, None, 1, None, 1, None, 0, None, None,
                                   None) == g.G3X_OK   # nothing to do
    assert lib.g3x_traceback_pairs(opt.ctypes.data, ri.ctypes.data, None, 1, None, 1, None, 3, None, None,
                                   None) == g.G3X_ERR_INVALID
    assert lib.g3x_flt_chained_seeds(None, opt.ctypes.data, 0, ri.ctypes.data, None, 1, None, 0, None, 0, None,
                                     None, 1000, None, None, None) == g.G3X_ERR_INVALID
    assert lib.g3x_chain2aln(None, opt.ctypes.data, ri.ctypes.data, None, 1, None, 0, None, 0, None, None, None,
                             None, None, None, None) == g.G3X_ERR_INVALID
    assert lib.g3x_pair_generate(opt.ctypes.data, ri.ctypes.data, None, 1, None, 1, None, 1, None, -2, None, None,
                                 None, None) == g.G3X_ERR_INVALID
    assert lib.g3x_pac_to_planes(None, 10, None, None, 0, None) == g.G3X_ERR_INVALID


def test_ctx_without_gpu_is_an_error_not_a_crash(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    h = ctypes.c_void_p()
    assert lib.g3x_ctx_create(ctypes.byref(h), 0) == g.G3X_ERR_CUDA


@pytest.mark.parametrize("compiler,std", [("gcc", "-std=c99"), ("g++", "-std=c++11")])
def test_header_compiles_as_c_and_cpp(tmp_path, compiler, std):
    """include/g3x.h is a plain C header (the boundary a cgo / JNI / ctypes stub binds): it
    compiles on its own as C99 and as C++11, without CUDA or torch headers."""
    import shutil
    import subprocess
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} not installed")
    src = tmp_path / ("probe.c" if compiler == "gcc" else "probe.cpp")
    src.write_text('#include "g3x.h"\nint probe(void) { return G3X_OK + (int)sizeof(g3x_job_t); }\n')
    subprocess.check_call([compiler, std, "-Wall", "-Werror", "-fsyntax-only",
                           "-I", os.path.join(ROOT, "include"), str(src)])

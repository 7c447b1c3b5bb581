"""Builds the native libraries in-tree.

    libg3x.so      product library: sm_100a kernels + C-ABI host code (nvcc)
    libg3x_emu.so  CPU model of the kernels' warp protocol, loaded by tests only (g++)
    libg3x_emu16.so CPU model of the int16x2 lane kernel's per-lane logic, tests only (nvcc)
    libg3x_phase.so the product library with phase clocks in the int16x2 lane kernel
                   (python -m g3sa_b200.build --phase-clocks; profile_case --phase-clocks)
    libg3x_synth.so seeded synthetic workload generator + multi-threaded plane packer (g++)

Run as ``python -m g3sa_b200.build``.  The oracle libraries are built by oracle/Makefile
(and oracle/build_ref.sh where the reference tree exists); __graft_entry__.build() drives
all of them.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["g3x_kernels.cu", "g3x_api.cu", "g3x_peak.cu", "g3x_seeds.cu", "g3x_stream.cu", "g3x_rowpar.cu", "g3x_model.cu", "g3x_sched.cu", "g3x_lane.cu", "g3x_lane16.cu", "g3x_lane2.cu", "g3x_band.cu", "g3x_noalloc.cu", "g3x_pipe.cu", "g3x_chain.cu", "g3x_produce.cu", "g3x_global.cu", "g3x_sw.cu", "g3x_seedflt.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_lib(force=False, verbose_ptxas=False):
    out = os.path.join(HERE, "libg3x.so")
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "g3x.h"))
    if not force and not _stale(out, deps):
        return out
    cmd = [NVCC] + ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
                           "-o", out] + [os.path.join(CSRC, f) for f in CU_SOURCES]
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    _run(cmd)
    return out


def build_phase_lib(force=False):
    """libg3x_phase.so: the product library with the int16x2 lane kernel's phase clocks compiled
    in (-DG3X_PHASE_CLOCKS), for profile_case --phase-clocks only."""
    out = os.path.join(HERE, "libg3x_phase.so")
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "g3x.h"))
    if not force and not _stale(out, deps):
        return out
    _run([NVCC] + ARCH + ["-lineinfo", "-O3", "-std=c++17", "-DG3X_PHASE_CLOCKS", "-Xcompiler", "-fPIC", "-shared",
                          "-o", out] + [os.path.join(CSRC, f) for f in CU_SOURCES])
    return out


def build_emu(force=False):
    out = os.path.join(HERE, "libg3x_emu.so")
    deps = [os.path.join(CSRC, "g3x_emu.cpp"), os.path.join(CSRC, "g3x_core.h")]
    if not force and not _stale(out, deps):
        return out
    _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", out,
          os.path.join(CSRC, "g3x_emu.cpp")])
    return out


def build_emu16(force=False):
    """CPU model of the int16x2 lane kernel's per-lane logic (host code built by nvcc, whose
    headers give the DPX intrinsics host versions)."""
    out = os.path.join(HERE, "libg3x_emu16.so")
    deps = [os.path.join(CSRC, f) for f in ("g3x_emu16.cu", "g3x_lane16.cuh", "g3x_core.h", "g3x_internal.h")]
    if not force and not _stale(out, deps):
        return out
    _run([NVCC] + ARCH + ["-O2", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-o", out,
                          os.path.join(CSRC, "g3x_emu16.cu")])
    return out


def build_synth(force=False):
    out = os.path.join(HERE, "libg3x_synth.so")
    deps = [os.path.join(CSRC, "g3x_synth.cpp"), os.path.join(HERE, "..", "include", "g3x.h")]
    if not force and not _stale(out, deps):
        return out
    _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", out,
          os.path.join(CSRC, "g3x_synth.cpp"), "-lpthread"])
    return out


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    force = "--force" in argv
    build_lib(force=force, verbose_ptxas="--ptxas-v" in argv)
    if "--phase-clocks" in argv:
        build_phase_lib(force=force)
    build_emu(force=force)
    build_emu16(force=force)
    build_synth(force=force)


if __name__ == "__main__":
    main()

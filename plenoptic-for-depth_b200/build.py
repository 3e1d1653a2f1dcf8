"""Build recipe of the engine's shared library (libpfd.so, sm_100a) and of the
test helper libraries, in-tree under plenoptic-for-depth_b200/_build/.

Compiled with -fmad=false: every fused multiply-add in the kernels is written
out as __fmaf_rn, so the arithmetic is exactly the one the CPU oracle states.
"""
from __future__ import annotations

import concurrent.futures
import os
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG_DIR)
CSRC = os.path.join(PKG_DIR, "csrc")
OUT = os.path.join(PKG_DIR, "_build")
LIB = os.path.join(OUT, "libpfd.so")

NVCC = os.environ.get("PFD_NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-O2,-ffp-contract=off", "-ccbin", "/usr/bin/g++",
]

CU_SOURCES = ["pm_kernels.cu", "pm_sweep.cu", "check_kernels.cu", "refocus_kernels.cu", "vdrd_kernels.cu", "fuse_kernels.cu", "mla_kernels.cu", "select_kernels.cu", "blur_kernels.cu", "pfd_abi.cu"]
CPP_SOURCES = ["neighbors.cpp", "server.cpp", "calib_xml.cpp"]
SYNTH_LIB = os.path.join(OUT, "libpfd_synth.so")
HOST_DIR = os.path.join(PKG_DIR, "host")
HOST_LIB = os.path.join(OUT, "libpfd_host.so")
HOST_SOURCES = ["lf_types.cpp", "frame_views.cpp", "AdaptMIPMFrame.cpp", "AdaptMIPMFrameACMM.cpp", "MIDisparityFilter.cpp", "MICycleCheck.cpp"]
GXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-parameter",
             "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include"]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps() -> list[str]:
    files = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for dirpath, _, names in os.walk(d):
            for n in names:
                if n.endswith((".cu", ".cuh", ".h", ".hpp", ".cpp", ".c")):
                    files.append(os.path.join(dirpath, n))
    return files


def build_lib(force: bool = False, verbose: bool = False) -> str:
    """Compile libpfd.so for sm_100a (cross-compiles without a GPU)."""
    os.makedirs(OUT, exist_ok=True)
    deps = _deps() + [__file__]
    if not force and not _stale(LIB, deps):
        return LIB
    objs, cmds = [], []
    for src in CU_SOURCES:
        obj = os.path.join(OUT, src.replace(".cu", ".o"))
        cmd = [NVCC, *ARCH, *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        cmds.append(cmd)
        objs.append(obj)
    for src in CPP_SOURCES:
        obj = os.path.join(OUT, src.replace(".cpp", ".o"))
        cmds.append(["/usr/bin/g++", "-std=c++17", "-O2", "-fPIC", "-I", os.path.join(ROOT, "include"),
                     "-I", "/usr/local/cuda/include", "-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    # the translation units are independent: compile them side by side, the
    # largest (the sweep's kernel variants) first
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_run, c) for c in sorted(cmds, key=lambda c: "pm_sweep" not in c[-3])]:
            f.result()
    tmp = LIB + ".tmp"
    _run([NVCC, *ARCH, "-shared", "-Xlinker", "-soname=libpfd.so", "-o", tmp, *objs, "-ccbin", "/usr/bin/g++"])
    os.replace(tmp, LIB)
    return LIB


def build_host(force: bool = False) -> str:
    """Compile libpfd_host.so: the C++ classes with the reference's interface
    (include/pfd/) over libpfd.so.  Plain g++; no device code."""
    lib = build_lib()
    srcs = [os.path.join(HOST_DIR, s) for s in HOST_SOURCES]
    deps = srcs + [os.path.join(HOST_DIR, "frame_views.h"), lib, __file__] + _deps()
    if not force and not _stale(HOST_LIB, deps):
        return HOST_LIB
    tmp = HOST_LIB + ".tmp"
    _run(["/usr/bin/g++", *GXX_FLAGS, "-shared", "-Wl,-soname,libpfd_host.so", "-o", tmp, *srcs,
          "-L", OUT, "-l:libpfd.so", "-Wl,-rpath,$ORIGIN"])
    os.replace(tmp, HOST_LIB)
    return HOST_LIB


def build_synth(force: bool = False) -> str:
    """Compile the synthetic-frame generator (plain C, OpenMP)."""
    os.makedirs(OUT, exist_ok=True)
    src = os.path.join(CSRC, "synth.c")
    if force or _stale(SYNTH_LIB, [src, __file__]):
        tmp = SYNTH_LIB + ".tmp"
        _run(["/usr/bin/gcc", "-std=gnu11", "-O2", "-fPIC", "-shared", "-fopenmp", src, "-o", tmp, "-lm"])
        os.replace(tmp, SYNTH_LIB)
    return SYNTH_LIB


TEST_OUT = os.path.join(ROOT, "tests", "_build")
TEX_PROBE = os.path.join(TEST_OUT, "libtexprobe.so")
FMA_PROBE = os.path.join(TEST_OUT, "libfmaprobe.so")
SHIM_PROBE = os.path.join(TEST_OUT, "libshimprobe.so")


def build_test_helpers(force: bool = False) -> str:
    """Compile the device probes the tests and bench.py use (the texture
    probe, the FP32 throughput probe) and the C++ drop-in probe."""
    os.makedirs(TEST_OUT, exist_ok=True)
    for name, lib_path in (("tex_probe.cu", TEX_PROBE), ("fma_probe.cu", FMA_PROBE)):
        src = os.path.join(ROOT, "tests", "csrc", name)
        if force or _stale(lib_path, [src, __file__]):
            tmp = lib_path + ".tmp"
            _run([NVCC, *ARCH, "-O2", "-shared", "-Xcompiler", "-fPIC", "-ccbin", "/usr/bin/g++", src, "-o", tmp])
            os.replace(tmp, lib_path)
    host = build_host()
    src = os.path.join(ROOT, "tests", "csrc", "shim_probe.cpp")
    if force or _stale(SHIM_PROBE, [src, host, __file__] + _deps()):
        tmp = SHIM_PROBE + ".tmp"
        rel = os.path.relpath(OUT, TEST_OUT)
        _run(["/usr/bin/g++", *GXX_FLAGS, "-shared", "-o", tmp, src, "-L", OUT, "-l:libpfd_host.so", "-l:libpfd.so",
              "-Wl,-rpath,$ORIGIN/" + rel])
        os.replace(tmp, SHIM_PROBE)
    return TEX_PROBE


def build_all(force: bool = False, verbose: bool = False) -> list[str]:
    return [build_lib(force, verbose), build_host(force), build_synth(force), build_test_helpers(force)]


if __name__ == "__main__":
    print(build_all(force="--force" in sys.argv, verbose="-v" in sys.argv))

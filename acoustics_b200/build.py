"""Build libfdtd_b200.so in-tree (acoustics_b200/_lib/) with nvcc for sm_100a.

Both device translation units are compiled with -fmad=false and the host
sources with -ffp-contract=off: FP64 results and cell classification are then
reproducible against a CPU evaluation of the same expressions, and FP32 results
(whose kernels request their FMAs explicitly) do not depend on how the compiler
contracts one template instantiation or another, so every tile shape, the
single-solve and the batched kernels produce the same bits.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libfdtd_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_FP64 = ["fdtd_fp64.cu", "fdtd_noalloc.cu", "fdtd_fp32.cu", "fdtd_fetch.cu"]  # all compiled with -fmad=false
CU_FAST = []
CPP = ["fdtd_api.cpp", "fdtd_step.cpp", "fdtd_xml.cpp", "fdtd_batch.cpp", "fdtd_server.cpp", "fdtd_io.cpp", "fdtd_coupled.cpp",
       "fdtd_mesh.cpp", "fdtd_tma.cpp", "fdtd_kinematics.cpp"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def sources():
    return [os.path.join(CSRC, f) for f in CU_FP64 + CU_FAST + CPP if os.path.exists(os.path.join(CSRC, f))]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "fdtd_c.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, lineinfo: bool = True, defines=(), lib: str = LIB) -> str:
    """Compile and link the library.  `defines` (e.g. ["FDTD_SHELL_PLANES=4"])
    and `lib` build another variant of the same ABI elsewhere; load it with
    FDTD_B200_LIB=<path>."""
    if not force and lib == LIB and not defines and not _stale():
        return LIB
    out_dir = os.path.dirname(os.path.abspath(lib))
    os.makedirs(out_dir, exist_ok=True)
    obj_dir = os.path.join(out_dir, "obj" if lib == LIB else "obj_" + os.path.basename(lib).replace(".so", ""))
    os.makedirs(obj_dir, exist_ok=True)
    nvcc = _nvcc()
    cxx = _host_cxx()
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-ccbin", cxx]
    if lineinfo:
        common.append("-lineinfo")
    common += ["-D" + d for d in defines]
    objs = []
    jobs = []
    for f in CU_FP64 + CU_FAST + CPP:
        src = os.path.join(CSRC, f)
        if not os.path.exists(src):
            continue
        obj = os.path.join(obj_dir, f + ".o")
        flags = list(common)
        if f in CU_FP64:
            flags += ["-fmad=false"]
        if f.endswith(".cu"):
            cmd = [nvcc] + ARCH + flags + ["-c", src, "-o", obj]
        else:
            cmd = [nvcc] + flags + ["-x", "cu", "-c", src, "-o", obj] if False else \
                  [nvcc] + ARCH + flags + ["-c", src, "-o", obj]
        objs.append(obj)
        jobs.append(cmd)
    procs = [subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT) for cmd in jobs]
    failed = False
    for cmd, p in zip(jobs, procs):
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stderr.write(" ".join(cmd) + "\n" + out.decode(errors="replace"))
        if p.returncode != 0:
            failed = True
    if failed:
        raise RuntimeError("building libfdtd_b200.so failed")
    tmp = lib + ".tmp"
    link = [nvcc] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs + ["-lpthread"]
    r = subprocess.run(link, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        sys.stderr.write(" ".join(link) + "\n" + r.stdout.decode(errors="replace"))
        raise RuntimeError("linking libfdtd_b200.so failed")
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))

"""Build recipe for the CUDA library (sm_100a) and the drop-in host driver.

``python -m pawsim_b200.build`` (or ``pawsim_b200.build.build()``) compiles every
``csrc/*.cu`` into ``pawsim_b200/libpawsim_b200.so`` with nvcc for sm_100a. The tendency
and pressure kernels are compiled with ``-fmad=false`` so that no multiply-add is fused,
as in the reference's x86-64 build; this is what makes the FP64 path bit-identical.
It then links the C host driver ``host/pawsim_main.c`` against the library into
``pawsim_b200/bin/PAWSIM_B200.exe`` (the drop-in for the reference's ``PAWSIM.exe``).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libpawsim_b200.so")
OBJDIR = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC,-O3",
         "-Xcompiler", "-fvisibility=hidden"]
SOURCES = ["api.cu", "tendency.cu", "pressure.cu", "mg.cu", "noalloc.cu", "nn.cu", "warmstart.cu", "dmg.cu",
           "tracer.cu"]
# (object name, source, extra flags): the fused tendency kernel is built for two tile heights
UNITS = [(s.replace(".cu", ""), s, []) for s in SOURCES] + [
    # one unit per tile height and momentum scheme, so that they compile in parallel
    *[(f"tendency_ty{ty}_m{ms}", "tendency_tile.cu", [f"-DPAWSIM_TEND_TY={ty}", f"-DPAWSIM_TEND_MS={ms}"])
      for ty in (8, 16) for ms in range(4)],
    # 32 x 12 tiles of 384 threads, three CTAs per SM
    *[(f"tendency_ty12_m{ms}", "tendency_tile.cu", ["-DPAWSIM_TEND_TY=12", f"-DPAWSIM_TEND_MS={ms}",
                                                     "-DPAWSIM_TEND_MINB=3"]) for ms in range(4)],
    ("tendency_budget", "tendency_tile.cu", ["-DPAWSIM_TEND_TY=8", "-DPAWSIM_TEND_BUD=1", "-DPAWSIM_TEND_MINB=2"]),
]
DRIVER_SRC = os.path.join(HERE, "host", "pawsim_main.c")
DRIVER = os.path.join(HERE, "bin", "PAWSIM_B200.exe")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_driver(force: bool = False, verbose: bool = False) -> str:
    """gcc the host driver against the library (rpath to the library's directory)."""
    deps = [DRIVER_SRC, LIB, os.path.join(INCLUDE, "pawsim_b200.h")]
    if not force and not _stale(DRIVER, deps):
        return DRIVER
    os.makedirs(os.path.dirname(DRIVER), exist_ok=True)
    cmd = ["gcc", "-O2", "-std=gnu11", "-Wall", "-Wextra", "-I", INCLUDE, DRIVER_SRC, "-o", DRIVER,
           "-L", HERE, "-lpawsim_b200", "-Wl,-rpath,$ORIGIN/..", "-lm", "-pthread"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return DRIVER


def build(force: bool = False, verbose: bool = False) -> str:
    lib = build_lib(force, verbose)
    build_driver(force, verbose)
    return lib


def build_lib(force: bool = False, verbose: bool = False) -> str:
    srcs = sorted({os.path.join(CSRC, u[1]) for u in UNITS})
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "pawsim_b200.h"))
    if not force and not _stale(LIB, deps):
        return LIB
    # objects are kept in _build/ and a unit recompiles only when its source, a header or the
    # build flags changed since its object was written (every header counts for every unit)
    os.makedirs(OBJDIR, exist_ok=True)
    headers = [d for d in deps if not d.endswith(".cu")] + [os.path.abspath(__file__)]
    cmds, objs = [], []
    for name, src, extra in UNITS:
        o = os.path.join(OBJDIR, name + ".o")
        objs.append(o)
        if force or _stale(o, [os.path.join(CSRC, src), *headers]):
            # written under a temporary name and renamed when the compiler succeeds, so that an
            # interrupted build leaves no object that looks up to date
            cmds.append([NVCC, *ARCH, *FLAGS, *extra, "-c", os.path.join(CSRC, src), "-o", o + ".tmp"])
    # translation units compile in parallel (the tendency kernels dominate the build time)
    procs = []
    for cmd in cmds:
        if verbose:
            print(" ".join(cmd))
        procs.append(subprocess.Popen(cmd))
    failed = [c for c, p in zip(cmds, procs) if p.wait() != 0]
    for c in cmds:
        if c in failed:
            if os.path.exists(c[-1]):
                os.remove(c[-1])
        else:
            os.replace(c[-1], c[-1][: -len(".tmp")])
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

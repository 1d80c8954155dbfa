"""Build recipe for the snuqs_b200 native code (in-tree, sm_100a).

Produces, next to this file:

* ``libsnuqs_b200.so`` -- the engine: CUDA kernels + planner + the C ABI of
  ``include/snuqs_b200.h``;
* ``_C.<abi>.so``       -- the pybind11 module with the reference's ``_C``
  surface, linked against ``libsnuqs_b200.so`` (rpath ``$ORIGIN``).

nvcc cross-compiles for ``sm_100a`` without a GPU.  Run as
``python -m snuqs_b200.build`` or through ``__graft_entry__.build()``.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
BUILD = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ENGINE_CU = ["engine.cu", "noalloc.cu", "batch.cu", "jit.cu", "results.cu"]
ENGINE_CC = ["gates.cc", "planner.cc", "adjoint_plan.cc"]
# Fused-sweep kernel instantiations: (precision, tile bits, CTAs per SM).
# Tile sizes must match kTileBitsC128 / kTileBitsC64 in csrc/sq_plan.h; the
# CTA counts keep registers <= 65536 / (CTAs x threads).
SWEEP_INSTANCES = [
    ("double", 4, 1), ("double", 7, 1), ("double", 10, 6), ("double", 11, 3), ("double", 12, 1),
    ("float", 4, 1), ("float", 7, 1), ("float", 10, 8), ("float", 12, 2),
]
# Two-state adjoint kernels: (precision, tile bits); must match kAdjTileBits*.
ADJOINT_INSTANCES = [("double", 4), ("double", 7), ("double", 10),
                     ("float", 4), ("float", 7), ("float", 11)]
# Batched-circuit energy kernels: (precision, tile bits) for every tile size the
# batch autotuner tries.
BATCH_INSTANCES = [("double", 10), ("double", 11), ("double", 12),
                   ("float", 10), ("float", 11), ("float", 12)]
# Batched adjoint-gradient kernels: (precision, tile bits); must match kBatchTileBits*.
BATCH_ADJ_INSTANCES = [("double", 10), ("double", 11), ("float", 11), ("float", 12)]
LIB = os.path.join(HERE, "libsnuqs_b200.so")


def _ext_suffix() -> str:
    return sysconfig.get_config_var("EXT_SUFFIX") or ".so"


PYEXT = os.path.join(HERE, "_C" + _ext_suffix())


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} ... {cmd[-1]}")


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    return hs + [os.path.join(INCLUDE, "snuqs_b200.h")]


def _write_jit_sources() -> None:
    """Embeds the sweep headers in the library (NVRTC compiles them at run time)."""
    out = os.path.join(BUILD, "jit_sources.inc")
    parts = []
    for var, fname in (("kJitPlanSource", "sq_plan.h"), ("kJitSweepSource", "sweep_kernels.cuh"),
                       ("kJitKernelsSource", "jit_kernels.cuh"),
                       ("kJitReduceSource", "reduce_kernels.cuh"), ("kJitBatchSource", "jit_batch.cuh")):
        text = open(os.path.join(CSRC, fname)).read()
        assert ")SQJIT\"" not in text
        parts.append(f'static const char {var}[] = R"SQJIT({text})SQJIT";\n')
    data = "".join(parts)
    if not os.path.exists(out) or open(out).read() != data:
        with open(out, "w") as f:
            f.write(data)


def build(force: bool = False, verbose: bool = False) -> None:
    os.makedirs(BUILD, exist_ok=True)
    _write_jit_sources()
    common = ["-O3", "-std=c++17", "-I", CSRC, "-I", INCLUDE, "-I", BUILD]
    objs = []
    hdrs = _headers()
    for f in ENGINE_CU:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        if force or _stale(obj, [src] + hdrs):
            _run([NVCC, *ARCH, "-lineinfo", *common, "-Xcompiler", "-fPIC",
                  "-Xptxas", "-warn-spills", "-c", src, "-o", obj])
        objs.append(obj)
    jobs = []
    inst_src = os.path.join(CSRC, "sweep_inst.cu")
    inst_deps = [inst_src] + [os.path.join(CSRC, f) for f in
                              ("sweep_kernels.cuh", "sq_plan.h", "sweep_registry.h")]
    for real, m, minb in SWEEP_INSTANCES:
        obj = os.path.join(BUILD, f"sweep_{real}_{m}.o")
        if force or _stale(obj, inst_deps):
            cmd = [NVCC, *ARCH, "-lineinfo", *common, "-Xcompiler", "-fPIC",
                   f"-DSQ_REAL={real}", f"-DSQ_M={m}", f"-DSQ_MINB={minb}",
                   "-Xptxas", "-warn-spills", "-c", inst_src, "-o", obj]
            jobs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                               stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    adj_src = os.path.join(CSRC, "adjoint_inst.cu")
    adj_deps = inst_deps + [adj_src, os.path.join(CSRC, "adjoint_kernels.cuh"),
                            os.path.join(CSRC, "reduce_kernels.cuh")]
    for real, m in ADJOINT_INSTANCES:
        obj = os.path.join(BUILD, f"adjoint_{real}_{m}.o")
        if force or _stale(obj, adj_deps):
            cmd = [NVCC, *ARCH, "-lineinfo", *common, "-Xcompiler", "-fPIC",
                   f"-DSQ_REAL={real}", f"-DSQ_M={m}",
                   "-Xptxas", "-warn-spills", "-c", adj_src, "-o", obj]
            jobs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                               stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    bat_src = os.path.join(CSRC, "batch_inst.cu")
    bat_deps = inst_deps + [bat_src, os.path.join(CSRC, "batch_kernels.cuh"),
                            os.path.join(CSRC, "reduce_kernels.cuh"),
                            os.path.join(CSRC, "adjoint_kernels.cuh")]
    for real, m in BATCH_INSTANCES:
        obj = os.path.join(BUILD, f"batch_{real}_{m}.o")
        if force or _stale(obj, bat_deps):
            cmd = [NVCC, *ARCH, "-lineinfo", *common, "-Xcompiler", "-fPIC",
                   f"-DSQ_REAL={real}", f"-DSQ_M={m}",
                   "-Xptxas", "-warn-spills", "-c", bat_src, "-o", obj]
            jobs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                               stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    badj_src = os.path.join(CSRC, "batch_adj_inst.cu")
    badj_deps = bat_deps + [badj_src]
    for real, m in BATCH_ADJ_INSTANCES:
        obj = os.path.join(BUILD, f"batch_adj_{real}_{m}.o")
        if force or _stale(obj, badj_deps):
            cmd = [NVCC, *ARCH, "-lineinfo", *common, "-Xcompiler", "-fPIC",
                   f"-DSQ_REAL={real}", f"-DSQ_M={m}",
                   "-Xptxas", "-warn-spills", "-c", badj_src, "-o", obj]
            jobs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                               stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    for cmd, proc in jobs:
        out, _ = proc.communicate()
        if proc.returncode != 0:
            sys.stderr.write(" ".join(cmd) + "\n" + out)
            raise RuntimeError("build step failed: " + cmd[-1])
        if verbose and out.strip():
            print(out.strip())
    for f in ENGINE_CC:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        if force or _stale(obj, [src] + hdrs):
            _run(["g++", *common, "-fPIC", "-Wall", "-c", src, "-o", obj])
        objs.append(obj)
    if force or _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static",
              "-ldl", "-Xlinker", "--no-undefined"])
    import pybind11

    pysrc = os.path.join(CSRC, "pymodule.cc")
    if force or _stale(PYEXT, [pysrc, LIB] + hdrs):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fvisibility=hidden",
              "-I", pybind11.get_include(), "-I", sysconfig.get_paths()["include"],
              "-I", INCLUDE, pysrc, "-o", PYEXT, "-L", HERE, "-lsnuqs_b200",
              "-Wl,-rpath,$ORIGIN"])
    if verbose:
        print("built", LIB, PYEXT)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)

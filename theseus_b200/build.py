"""Build the sm_100a shared library theseus_b200/libtheseus_b200.so.

Every kernel translation unit is compiled by nvcc for sm_100a
(-gencode arch=compute_100a,code=sm_100a) into theseus_b200/_build/, in
parallel, and linked into one shared object exporting the C ABI of
include/theseus_b200.h.  Re-running only rebuilds stale objects.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtheseus_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "-Xptxas", "-O3",
         "--expt-relaxed-constexpr", "-I", SRC, "-I", INCLUDE]
ORDERS = (3, 4, 5, 6)


def units():
    """(object name, source, extra defines) of every translation unit."""
    u = [("thx_api.o", "thx_api.cu", []), ("thx_host.o", "thx_host.cpp", []),
         ("thx_lte_host.o", "thx_lte_host.cpp", []), ("thx_engine.o", "thx_engine.cu", []),
         ("thx_noalloc.o", "thx_noalloc.cu", []), ("thx_checkpoint.o", "thx_checkpoint.cpp", []),
         ("thx_geometry.o", "thx_geometry.cu", []), ("thx_peak.o", "thx_peak.cu", []),
         ("thx_trials.o", "thx_trials.cu", ["-DTHX_TRIAL_FMA"])]
    for dim in (2, 3):
        u.append((f"lte_face_{dim}.o", "thx_inst_lte.cu", [f"-DTHX_DIM={dim}"]))
        for n in ORDERS:
            u.append((f"lte_{dim}_{n}.o", "thx_inst_lte.cu", [f"-DTHX_DIM={dim}", f"-DTHX_N={n}"]))
    for prec in (0, 1):
        for dim in (2, 3):
            u.append((f"face_{prec}_{dim}.o", "thx_inst_face.cu", [f"-DTHX_PREC={prec}", f"-DTHX_DIM={dim}"]))
            for n in ORDERS:
                u.append((f"order_{prec}_{dim}_{n}.o", "thx_inst_order.cu",
                          [f"-DTHX_PREC={prec}", f"-DTHX_DIM={dim}", f"-DTHX_N={n}"]))
    return u


def _headers():
    return [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".cuh", ".h"))] + \
        [os.path.join(INCLUDE, "theseus_b200.h")]


def _stale(obj, src):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + _headers())


def _compile(job):
    obj, src, defs = job
    # The FP64 path keeps every multiply and add separately rounded, like the
    # reference's CPU builds (-ffp-contract=off), so that it reproduces the CPU
    # right-hand side to round-off even where the result cancels strongly.
    # The FP32-mixed units may contract to FMA.
    # The tensor-core trial keeps contraction on: its SIMT form is the
    # strongest (fused) baseline.
    if "-DTHX_PREC=1" not in defs and "-DTHX_TRIAL_FMA" not in defs:
        defs = defs + ["--fmad=false"]
    cmd = [NVCC] + ARCH + FLAGS + defs + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC] + FLAGS + defs + ["-x", "cu", "-c", src, "-o", obj] + ARCH
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(obj)}:\n{r.stderr[-4000:]}")
    return obj


def build(verbose=False, jobs=None):
    os.makedirs(OUT, exist_ok=True)
    todo, objs = [], []
    for name, src, defs in units():
        obj = os.path.join(OUT, name)
        objs.append(obj)
        if _stale(obj, os.path.join(SRC, src)):
            todo.append((obj, os.path.join(SRC, src), defs))
    if todo:
        jobs = jobs or max(1, min(len(todo), os.cpu_count() or 4))
        if verbose:
            print(f"[theseus_b200] compiling {len(todo)} units with {jobs} jobs", flush=True)
        with ThreadPoolExecutor(jobs) as ex:
            list(ex.map(_compile, todo))
    if todo or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        # link beside the library and rename: a reader never sees a partial file
        tmp = LIB + ".partial"
        cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
    print(LIB)
    sys.exit(0)

"""Build libtrackpad_b200.so in-tree with nvcc for sm_100a.

The tracking kernel is compiled three times: with FMA contraction (the fast
build), with -fmad=false (the strict build, whose arithmetic matches the
reference operation for operation) and strict with bounds checks (the checked
build, selected per call by tp_opts.bounds_check).  Host code is compiled without FMA
contraction so that hoisted element constants are bit-identical to the values
the reference computes per particle.
"""
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libtrackpad_b200.so")
BUILD = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd):
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        sys.stderr.write(p.stdout + p.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return p.stdout + p.stderr


def build(verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    base = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
            "-I", os.path.join(HERE, "..", "include"), "-I", CSRC, "--expt-relaxed-constexpr"]
    if ptxas_info:
        base += ["-Xptxas", "-v"]
    units = [
        ("tp_track_fast.o", "tp_track.cu", ["-DTP_NS=fast", "-fmad=true"]),
        ("tp_track_strict.o", "tp_track.cu", ["-DTP_NS=strict", "-fmad=false", "-DTP_OCC_VARIANTS"]),
        ("tp_track_strict_low.o", "tp_track.cu", ["-DTP_NS=strict_low", "-fmad=false", "-DTP_OCC_LOW"]),
        ("tp_track_checked.o", "tp_track.cu", ["-DTP_NS=checked", "-fmad=false", "-DTP_BOUNDS_CHECK"]),
        ("tp_runtime.o", "tp_runtime.cu", ["-fmad=false"]),
        ("tp_adjoint.o", "tp_adjoint.cu", ["-fmad=false"]),
        ("tp_compile.o", "tp_compile.cpp", ["-fmad=false", "-x", "cu"]),
        ("tp_noalloc.o", "tp_noalloc.cu", ["-fmad=false"]),
        ("tp_tpsa.o", "tp_tpsa.cu", ["-fmad=false"]),
    ]
    objs = []
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(HERE, "..", "include", "trackpad_b200.h"))
    newest_dep = max(os.path.getmtime(d) for d in deps)
    jobs = []
    for obj, src, extra in units:
        o = os.path.join(BUILD, obj)
        s = os.path.join(CSRC, src)
        stale = (not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), newest_dep)
                 or os.environ.get("TP_REBUILD") or ptxas_info)
        if stale:
            jobs.append(base + extra + ["-c", s, "-o", o])
        objs.append(o)
    # the translation units are independent: compile them concurrently
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        log = list(ex.map(_run, jobs))
    relinked = bool(jobs)
    if relinked or not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(o) for o in objs):
        _run([nvcc(), *ARCH, "-shared", "-o", OUT, *objs, "-Xcompiler", "-fPIC", "-cudart", "static"])
    if verbose:
        print("\n".join(log))
    return OUT


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv)
    print("built", OUT)

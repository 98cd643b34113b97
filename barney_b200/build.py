"""Build recipe for libbarney_b200.so (in-tree, sm_100a only).

    python -m barney_b200.build          # or barney_b200.build.build()
    python -m barney_b200.build --bounds-check   # libbarney_b200_bc.so, every access checked

Device code: --fmad=false with IEEE division and square root, so the kernels
evaluate every FP32 expression exactly as written (bit-identical to the CPU
restatement in oracle/); bn_kernels.cu is compiled a second time with
-DBNB_FAST_MATH, FMA contraction and approximate division and square root into
the fast-math object (the renderer parameter bnx.fastMath).  Host code: -ffp-contract=off for the same reason
(camera set-up).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libbarney_b200.so")
LIB_BC = os.path.join(HERE, "libbarney_b200_bc.so")  # bounds-checked build (-DBNB_BOUNDS_CHECK)
SOURCES = ["bn_kernels.cu", "bn_api.cpp", "bn_server.cpp"]
# the fast-math object (renderer parameter bnx.fastMath): bn_kernels.cu again,
# with FMA contraction and approximate division and square root
FAST_SOURCE = "bn_kernels.cu"
FAST_FLAGS = ["-DBNB_FAST_MATH", "--fmad=true", "-prec-div=false", "-prec-sqrt=false"]
HEADERS = ["bn_device.h", "bn_objects.h", os.path.join("..", "..", "include", "bn_volume.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden,-O3",
    "-Xptxas", "-v",
]


def nvcc():
    for p in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if p and (os.path.isabs(p) and os.path.exists(p) or not os.path.isabs(p)):
            return p
    return "nvcc"


def _digest(bounds_check=False):
    """Content hash of every input of the build (sources, headers, flags)."""
    import hashlib
    h = hashlib.sha1((" ".join(NVCC_FLAGS + FAST_FLAGS) + (" -DBNB_BOUNDS_CHECK" if bounds_check else "")).encode())
    for s in SOURCES + HEADERS:
        with open(os.path.join(CSRC, s), "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def _stale(bounds_check=False):
    """True unless the library was built from the current sources (content
    hash, so copies that reset file times do not force a rebuild)."""
    lib = LIB_BC if bounds_check else LIB
    if not os.path.exists(lib) or not os.path.exists(lib + ".sha1"):
        return True
    with open(lib + ".sha1") as f:
        return f.read().strip() != _digest(bounds_check)


def build(force=False, verbose=False, bounds_check=False):
    """Compile every source for sm_100a into barney_b200/libbarney_b200.so
    (bounds_check: libbarney_b200_bc.so with -DBNB_BOUNDS_CHECK).
    Processes that find the library stale at the same time (ranks of one job)
    build it once: the build holds an exclusive lock, and whoever gets the
    lock next sees the fresh library."""
    lib = LIB_BC if bounds_check else LIB
    if not force and not _stale(bounds_check):
        return lib
    import fcntl
    with open(lib + ".lock", "w") as lock:
        fcntl.flock(lock, fcntl.LOCK_EX)
        if not force and not _stale(bounds_check):
            return lib
        return _build_locked(verbose, bounds_check)


def _build_locked(verbose, bounds_check=False):
    LIB_OUT = LIB_BC if bounds_check else LIB
    flags = NVCC_FLAGS + (["-DBNB_BOUNDS_CHECK"] if bounds_check else [])
    objs = []
    logs = []
    units = [(src, os.path.splitext(src)[0], flags) for src in SOURCES]
    exact = {"--fmad=false", "-prec-div=true", "-prec-sqrt=true"}
    units.append((FAST_SOURCE, "bn_kernels_fast", [f for f in flags if f not in exact] + FAST_FLAGS))
    # the objects compile in parallel (the two kernel objects dominate)
    procs = []
    for src, stem, fl in units:
        obj = os.path.join(CSRC, stem + ("_bc.o" if bounds_check else ".o"))
        cmd = [nvcc(), *fl, "-c", os.path.join(CSRC, src), "-o", obj]
        procs.append((src, obj, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    for src, obj, p in procs:
        out, _ = p.communicate()
        logs.append(f"== {os.path.basename(obj)}\n" + out)
        if p.returncode != 0:
            sys.stderr.write(out)
            raise RuntimeError("nvcc failed on " + src)
        objs.append(obj)
    tmp = LIB_OUT + ".tmp"
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp, *objs,
           "-Xcompiler", "-fPIC"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, LIB_OUT)
    with open(LIB_OUT + ".sha1", "w") as f:
        f.write(_digest(bounds_check))
    for o in objs:
        os.remove(o)
    if not bounds_check:
        with open(os.path.join(CSRC, "ptxas.log"), "w") as f:
            f.write("\n".join(logs))
    if verbose:
        print("\n".join(logs))
    return LIB_OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, bounds_check="--bounds-check" in sys.argv))

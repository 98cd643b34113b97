"""Build recipe for libbarney_b200.so (in-tree, sm_100a only).

    python -m barney_b200.build          # or barney_b200.build.build()

Device code: --fmad=false with IEEE division and square root, so the kernels
evaluate every FP32 expression exactly as written (bit-identical to the CPU
restatement in oracle/).  Host code: -ffp-contract=off for the same reason
(camera set-up).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libbarney_b200.so")
SOURCES = ["bn_kernels.cu", "bn_api.cpp", "bn_server.cpp"]
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


def _digest():
    """Content hash of every input of the build (sources, headers, flags)."""
    import hashlib
    h = hashlib.sha1(" ".join(NVCC_FLAGS).encode())
    for s in SOURCES + HEADERS:
        with open(os.path.join(CSRC, s), "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def _stale():
    """True unless libbarney_b200.so was built from the current sources
    (content hash, so copies that reset file times do not force a rebuild)."""
    if not os.path.exists(LIB) or not os.path.exists(LIB + ".sha1"):
        return True
    with open(LIB + ".sha1") as f:
        return f.read().strip() != _digest()


def build(force=False, verbose=False):
    """Compile every source for sm_100a into barney_b200/libbarney_b200.so.
    Processes that find the library stale at the same time (ranks of one job)
    build it once: the build holds an exclusive lock, and whoever gets the
    lock next sees the fresh library."""
    if not force and not _stale():
        return LIB
    import fcntl
    with open(LIB + ".lock", "w") as lock:
        fcntl.flock(lock, fcntl.LOCK_EX)
        if not force and not _stale():
            return LIB
        return _build_locked(verbose)


def _build_locked(verbose):
    objs = []
    logs = []
    for src in SOURCES:
        obj = os.path.join(CSRC, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc(), *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        logs.append(r.stdout + r.stderr)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc failed on " + src)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp, *objs,
           "-Xcompiler", "-fPIC"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, LIB)
    with open(LIB + ".sha1", "w") as f:
        f.write(_digest())
    for o in objs:
        os.remove(o)
    with open(os.path.join(CSRC, "ptxas.log"), "w") as f:
        f.write("\n".join(logs))
    if verbose:
        print("\n".join(logs))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

"""Build the B200 runtime library (libphysis_rt_b200.so) in-tree with nvcc.

Every .cu file under csrc/ is compiled for sm_100a only and linked into one
shared library at physis_b200/lib/libphysis_rt_b200.so, which is the C ABI
that user programs, generated code and the Python mirror load.
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(OUT_DIR, "libphysis_rt_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
    "-fmad=false", "--expt-relaxed-constexpr", "-I" + os.path.join(HERE, "..", "include"),
]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _needs_build(obj, src):
    if not os.path.exists(obj):
        return True
    deps = [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC)
                    if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(HERE, "..", "include", "physis_b200.h"))
    deps.append(os.path.abspath(__file__))
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, extra):
    obj = os.path.join(OUT_DIR, "obj", os.path.basename(src) + ".o")
    if not _needs_build(obj, src):
        return obj, None
    cmd = [NVCC] + FLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, "FAILED: " + " ".join(cmd) + "\n" + r.stdout + r.stderr
    return obj, r.stderr if "warning" in r.stderr else None


def build(verbose=False, extra=None):
    """Compile (incrementally) and link the runtime; returns the .so path."""
    extra = list(extra or [])
    os.makedirs(os.path.join(OUT_DIR, "obj"), exist_ok=True)
    srcs = sources()
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, extra), srcs))
    errors = [m for _, m in results if m and m.startswith("FAILED")]
    if errors:
        raise RuntimeError("\n".join(errors))
    if verbose:
        for _, m in results:
            if m:
                print(m, file=sys.stderr)
    objs = [o for o, _ in results]
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl",
                                                              "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))

"""Build ``libfv3core_b200.so`` in-tree with nvcc for sm_100a.

Usage: ``python -m fv3core_b200.build`` (also called by ``__graft_entry__.build``).
Compiles every ``csrc/*.cu`` to an object (in parallel) and links one shared
library next to this file.  Rebuilds only what changed.
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfv3core_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + [
    "-O3",
    # no a*b+c contraction: every FP64 operation rounds on its own, as in the
    # reference's numpy execution, so results agree to the last bits
    "--fmad=false",
    "-lineinfo",
    "-std=c++17",
    "--extended-lambda",
    "-Xcompiler",
    "-fPIC",
    "-I" + INCLUDE,
]


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src, extra):
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    hm = _headers_mtime()
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hm):
        return obj, None
    cmd = [NVCC] + FLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, r.stderr + r.stdout
    return obj, (r.stderr if "warning" in r.stderr.lower() else None)


def build(verbose=False, extra=()):
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources()
    objs = []
    errors = []
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for obj, msg in ex.map(lambda s: _compile(s, list(extra)), srcs):
            objs.append(obj)
            if msg:
                if "error" in msg.lower():
                    errors.append(msg)
                elif verbose:
                    print(msg, file=sys.stderr)
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stderr + r.stdout)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))

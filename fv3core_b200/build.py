"""Build the two libraries in-tree with nvcc for sm_100a.

Usage: ``python -m fv3core_b200.build`` (also called by ``__graft_entry__.build``).
Compiles every ``csrc/*.cu`` twice (in parallel) and links two shared
libraries next to this file:

* ``libfv3core_b200.so``: FP64 fields, no a*b+c contraction, so results
  agree with the numpy oracle to the last bit;
* ``libfv3core_b200_f32.so``: the mixed-precision build of the same sources
  (``FV3B_REAL_T=float``): FP32 fields and bulk arithmetic, FP64 column
  solves; fused multiply-add allowed.

Rebuilds only what changed.
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
LIB_F32 = os.path.join(HERE, "libfv3core_b200_f32.so")
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
    hs.append(os.path.abspath(__file__))  # the flags live here
    return max((os.path.getmtime(h) for h in hs), default=0.0)


VARIANTS = {
    "f64": (LIB, []),
    # mixed precision: FP32 fields, CUDA's FP64 exp/log/pow in the column solves
    "f32": (LIB_F32, ["-DFV3B_REAL_T=float", "-DFV3B_FAST_TRANSCENDENTALS"]),
}


def _flags(variant):
    if variant == "f32":
        return [f for f in FLAGS if f != "--fmad=false"] + ["--fmad=true"] + VARIANTS[variant][1]
    return FLAGS


def _compile(src, extra, variant="f64"):
    obj = os.path.join(BUILD, variant, os.path.basename(src)[:-3] + ".o")
    hm = _headers_mtime()
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hm):
        return obj, None
    cmd = [NVCC] + _flags(variant) + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, r.stderr + r.stdout
    return obj, (r.stderr if "warning" in r.stderr.lower() else None)


def build(verbose=False, extra=(), variants=("f64", "f32")):
    srcs = _sources()
    jobs = [(src, v) for v in variants for src in srcs]
    for v in variants:
        os.makedirs(os.path.join(BUILD, v), exist_ok=True)
    objs = {v: [] for v in variants}
    errors = []
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for (src, v), (obj, msg) in zip(jobs, ex.map(lambda j: _compile(j[0], list(extra), j[1]), jobs)):
            objs[v].append(obj)
            if msg:
                if "error" in msg.lower():
                    errors.append(msg)
                elif verbose:
                    print(msg, file=sys.stderr)
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    for v in variants:
        lib = VARIANTS[v][0]
        newest = max(os.path.getmtime(o) for o in objs[v])
        if not os.path.exists(lib) or os.path.getmtime(lib) < newest:
            cmd = [NVCC] + ARCH + ["-shared", "-o", lib] + objs[v] + ["-lcudart"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError("link failed:\n" + r.stderr + r.stdout)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))

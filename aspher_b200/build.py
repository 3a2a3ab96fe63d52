"""Build recipe of libaspher_b200.so (sm_100a), in-tree.

``python -m aspher_b200.build`` compiles every ``csrc/*.cu`` with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` into ``_build/`` objects (in
parallel) and links ``aspher_b200/libaspher_b200.so``.  Objects are rebuilt
only when a source or header is newer.
"""

import concurrent.futures as cf
import glob
import os
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libaspher_b200.so")
BUILD = os.path.join(ROOT, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max(os.path.getmtime(h) for h in hs) if hs else 0.0


def _compile(src, verbose=False):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    hdr = _newest_header()
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr):
        return obj, ""
    cmd = [NVCC] + ARCH + FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-c", src, "-o", obj]
    t0 = time.time()
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s" % (src, p.stderr))
    # date the object at the start of its compile: a source or header edited
    # while it compiled is newer than it, so the next build recompiles
    os.utime(obj, (t0, t0))
    return obj, p.stderr


def build(verbose=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    jobs = jobs or min(len(srcs), os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(jobs) as ex:
        res = list(ex.map(lambda s: _compile(s, verbose), srcs))
    objs = [o for o, _ in res]
    if verbose:
        for _, log in res:
            if log:
                sys.stderr.write(log)
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart",
                                                              "-Xlinker", "--no-undefined"]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("link failed:\n" + p.stderr)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))

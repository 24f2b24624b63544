"""Build libvlxb.so (sm_100a) in-tree.

    python -m vlxb.build [-j N]      (run from vlx-twoe-ints_b200/)

Steps: run the two code generators (csrc/gen_quartets.py, csrc/gen_abi.py),
compile every translation unit with nvcc for sm_100a in parallel, link the
shared library next to this file.  Objects go to vlx-twoe-ints_b200/_build/;
ptxas register/spill reports go to _build/ptxas/<unit>.txt.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys
import time

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REPO_ROOT = os.path.dirname(PKG_ROOT)
CSRC = os.path.join(PKG_ROOT, "csrc")
GEN = os.path.join(CSRC, "generated")
BUILD = os.path.join(PKG_ROOT, "_build")
LIB = os.path.join(PKG_ROOT, "vlxb", "libvlxb.so")
NVCC = os.environ.get("NVCC", "nvcc")

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v", "-I", CSRC] + ARCH_FLAGS

COMMON_HEADERS = ["common.cuh", "engine.cuh", "jk_kernels.cuh", "prep.cuh", "classes.cuh", "col_kernels.cuh",
                  "md.cuh", "md_kernels.cuh", "jgrad_kernels.cuh", "kgrad_kernels.cuh", "tma.cuh", "jtma_kernels.cuh"]


def _run_generators():
    subprocess.run([sys.executable, os.path.join(CSRC, "gen_quartets.py"), GEN], check=True)
    subprocess.run([sys.executable, os.path.join(CSRC, "gen_column.py"), GEN], check=True)
    subprocess.run([sys.executable, os.path.join(CSRC, "gen_abi.py")], check=True)


def _sources():
    srcs = [os.path.join(CSRC, "prep.cu"), os.path.join(CSRC, "api.cu"), os.path.join(CSRC, "schwarz.cu"),
            os.path.join(CSRC, "noalloc.cu"), os.path.join(CSRC, "aomap.cu"),
            os.path.join(CSRC, "listbuild.cu"), os.path.join(CSRC, "fshell.cu"), os.path.join(GEN, "abi.cu")]
    srcs += sorted(glob.glob(os.path.join(GEN, "cls_*.cu")))
    return srcs


def _deps(src):
    deps = [src] + [os.path.join(CSRC, h) for h in COMMON_HEADERS] + [os.path.join(GEN, "hrr_pairs.cuh"),
                                                                     os.path.join(REPO_ROOT, "include", "vlxb.h")]
    base = os.path.basename(src)
    if base.startswith("cls_"):
        deps.append(os.path.join(GEN, f"col_{base.split('_')[1]}.cuh"))
        with open(src) as fh:  # every generated quartet header the unit includes (its class first)
            deps += [os.path.join(GEN, ln.split('"')[1]) for ln in fh if ln.startswith('#include "q_')]
    if base == "prep.cu":
        deps.append(os.path.join(GEN, "schedule_default.inc"))
    return deps


def _obj(src):
    return os.path.join(BUILD, "obj", os.path.basename(src)[:-3] + ".o")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def _compile(src):
    obj = _obj(src)
    cmd = [NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj]
    t0 = time.time()
    r = subprocess.run(cmd, capture_output=True, text=True)
    rep = os.path.join(BUILD, "ptxas", os.path.basename(src)[:-3] + ".txt")
    with open(rep, "w") as fh:
        fh.write(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr[-4000:]}")
    return src, time.time() - t0


def build(jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(os.path.join(BUILD, "obj"), exist_ok=True)
    os.makedirs(os.path.join(BUILD, "ptxas"), exist_ok=True)
    _run_generators()
    srcs = _sources()
    todo = [s for s in srcs if _stale(_obj(s), _deps(s))]
    # heaviest units first (d-rich classes) for a shorter critical path
    todo.sort(key=lambda s: -sum(os.path.getsize(d) for d in _deps(s) if os.path.basename(d).startswith("q_")))
    jobs = jobs or max(1, os.cpu_count() or 1)
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            for src, dt in ex.map(_compile, todo):
                if verbose:
                    print(f"  {os.path.basename(src)}: {dt:.1f}s", flush=True)
    objs = [_obj(s) for s in srcs]
    if _stale(LIB, objs):
        cmd = [NVCC, "-shared", "-o", LIB] + objs + ARCH_FLAGS + ["-cudart", "static"]
        subprocess.run(cmd, check=True)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    args = ap.parse_args()
    t0 = time.time()
    lib = build(args.j, verbose=True)
    print(f"built {lib} in {time.time() - t0:.1f}s")


if __name__ == "__main__":
    main()

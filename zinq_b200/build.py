"""Build the CUDA library libzinq_qd.so in-tree for sm_100a with nvcc.

The translation units are compiled in parallel (one nvcc per .cu file) and
linked into zinq_b200/libzinq_qd.so with the CUDA runtime linked statically,
so the library has no dependency beyond the NVIDIA driver.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libzinq_qd.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-ccbin", "g++"]

SOURCES = ["options.cu", "expr.cpp", "job.cu", "result.cu", "fft_seam.cu", "spectrum.cu", "serve.cu", "tune.cu", "service.cu", "measure.cu", "tma_map.cu"]
# line_inst.cu is compiled once per (precision, number of electronic states)
VARIANTS = [("line_inst.cu", f"line_{t[0]}{s}", [f"-DZQD_T={t}", f"-DZQD_S={s}", f"-DZQD_LAUNCH=launch_line_{t[0]}{s}",
                                                   f"-DZQD_SERVICE=launch_service_{t[0]}{s}"])
            for t in ("double", "float") for s in (1, 2, 3, 4)]
# nd_inst.cu likewise: the 2-D / 3-D driver
VARIANTS += [("nd_inst.cu", f"nd_{t[0]}{s}", [f"-DZQD_T={t}", f"-DZQD_S={s}", f"-DZQD_ND_CREATE=nd_create_{t[0]}{s}",
                                               f"-DZQD_ND_RUN=nd_run_{t[0]}{s}", f"-DZQD_ND_STEP=nd_step_{t[0]}{s}"])
             for t in ("double", "float") for s in (1, 2, 3, 4)]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers(src):
    """Local headers `src` includes, followed transitively (quoted includes only)."""
    inc_dirs = [CSRC, os.path.join(os.path.dirname(HERE), "include")]
    seen, todo = set(), [src]
    while todo:
        f = todo.pop()
        with open(f) as fh:
            for line in fh:
                line = line.strip()
                if not line.startswith("#include \""):
                    continue
                name = line.split('"')[1]
                for d in [os.path.dirname(f)] + inc_dirs:
                    h = os.path.join(d, name)
                    if os.path.exists(h):
                        if h not in seen:
                            seen.add(h)
                            todo.append(h)
                        break
    return sorted(seen)


def _compile(item, verbose=False):
    src, stem, defines = item
    obj = os.path.join(BUILD, stem + ".o")
    deps = [src] + _headers(src)
    if not _stale(obj, deps):
        return obj
    lang = ["-x", "cu"] if src.endswith(".cpp") else []
    cmd = [NVCC, *ARCH, *FLAGS, *defines, *lang, "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    items = [(os.path.join(CSRC, s), os.path.splitext(s)[0], []) for s in SOURCES]
    items += [(os.path.join(CSRC, s), stem, d) for s, stem, d in VARIANTS]
    # the heaviest units first so they overlap with the rest
    items.sort(key=lambda it: 0 if it[1].startswith("line_") else 1)
    with cf.ThreadPoolExecutor(max_workers=jobs or min(12, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda it: _compile(it, verbose), items))
    if _stale(OUT, objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", OUT, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    print(build(verbose=True))

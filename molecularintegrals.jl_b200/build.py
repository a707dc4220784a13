"""Build libmolints_cuda.so in-tree: generate the class kernels, nvcc for sm_100a, link.

    python build.py [--force] [-j N]

Every translation unit is compiled with
    nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3 -std=c++17 -Xptxas -v
and the ptxas resource report (registers, spills, shared memory) is kept in
_build/ptxas.log.  The library lands next to this file, where the loader looks for it.
"""
from __future__ import annotations

import argparse
import os
import re
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libmolints_cuda.so"
INCLUDE = HERE.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
                     "--expt-relaxed-constexpr"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found")
    return path


def sources():
    sys.path.insert(0, str(CSRC))
    try:
        import gen_eri
    finally:
        sys.path.pop(0)
    gen = gen_eri.generate()
    return ([CSRC / "molints.cu", CSRC / "plan_build.cu", CSRC / "noalloc.cu", CSRC / "serve.cu", CSRC / "one_e.cu",
             CSRC / "eri_generic.cu", CSRC / "generated" / "rys_tables.cu"] +
            sorted(gen))


_INCLUDE_RE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _deps(src: Path):
    """src and every project header it includes, directly or through other headers (quoted
    includes, resolved against the including file's folder, then csrc/ and include/)."""
    seen, todo = [], [src]
    while todo:
        f = todo.pop()
        if f in seen or not f.exists():
            continue
        seen.append(f)
        for name in _INCLUDE_RE.findall(f.read_text(errors="replace")):
            for base in (f.parent, CSRC, INCLUDE):
                cand = (base / name).resolve()
                if cand.exists():
                    todo.append(cand)
                    break
    return seen


def _compile(src: Path, force: bool):
    obj = BUILD / (src.stem + ".o")
    log = BUILD / (src.stem + ".ptxas")
    if (not force and obj.exists() and
            all(obj.stat().st_mtime >= d.stat().st_mtime for d in _deps(src) if d.exists())):
        return obj, None
    cmd = [nvcc()] + NVCC_FLAGS + ["-I", str(CSRC), "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    log.write_text(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stderr[-4000:]}")
    return obj, r.stderr


def build(force: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sources()
    jobs = jobs or max(1, min(len(srcs), os.cpu_count() or 4))
    with ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(lambda s: _compile(s, force), srcs))
    objs = [r[0] for r in results]
    (BUILD / "ptxas.log").write_text("\n".join((BUILD / (s.stem + ".ptxas")).read_text()
                                               for s in srcs if (BUILD / (s.stem + ".ptxas")).exists()))
    if force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(f".{os.getpid()}.tmp")
        cmd = [nvcc()] + ARCH + ["-shared", "-o", str(tmp)] + [str(o) for o in objs] + ["-lcudart"]
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    a = ap.parse_args()
    print(build(a.force, a.j))

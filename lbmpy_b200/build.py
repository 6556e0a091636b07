"""Builds liblbmb200.so in place: nvcc for sm_100a, one object per kernel family, in parallel.

Usage: ``python -m lbmpy_b200.build [--verbose]``.  The library lands next to this file, so the
package loads it from the source tree (``lbmpy_b200/liblbmb200.so``).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblbmb200.so")
SOURCES = ["lbm_abi.cu", "lbm_q19_pop.cu", "lbm_q19_mrt.cu", "lbm_q27_pop.cu", "lbm_q27_mrt.cu",
           "lbm_q27_cum.cu", "lbm_q27_cum1.cu", "lbm_q27_cm.cu", "lbm_q27_closure.cu", "lbm_mlp.cu",
           "lbm_halo.cu", "lbm_q19_pop_b.cu", "lbm_q19_mrt_b.cu", "lbm_q27_pop_b.cu", "lbm_q27_cum_b.cu",
           "lbm_q27_cum1_b.cu", "lbm_q27_mrt_b.cu", "lbm_q27_cm_b.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build liblbmb200.so")


def host_compiler() -> list:
    # the system g++ (the environment's CC/CXX may point at a toolchain without libgomp/libstdc++ headers)
    gxx = "/usr/bin/g++"
    return ["-ccbin", gxx] if os.path.exists(gxx) else []


def flags(verbose=False) -> list:
    f = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-DNDEBUG",
         "-I" + os.path.join(HERE, "..", "include")] + ARCH + host_compiler()
    if verbose:
        f += ["-Xptxas", "-v"]
    return f


def _includes(name: str, seen: set) -> None:
    """Quoted includes of a csrc file, transitively."""
    if name in seen:
        return
    path = os.path.join(CSRC, name)
    if not os.path.exists(path):
        return
    seen.add(name)
    with open(path) as fh:
        for line in fh:
            line = line.strip()
            if line.startswith("#include \""):
                inc = line.split('"')[1]
                if "/" not in inc:
                    _includes(inc, seen)


def _digest(source: str = None) -> str:
    """Hash of the compiler flags, the public header and the given source with every csrc header
    it includes (or of all sources and headers)."""
    h = hashlib.sha256()
    if source is None:
        names = sorted(n for n in os.listdir(CSRC) if n.endswith((".cuh", ".h", ".cu")))
    else:
        seen = set()
        _includes(source, seen)
        names = sorted(seen)
    for name in names:
        with open(os.path.join(CSRC, name), "rb") as fh:
            h.update(name.encode() + fh.read())
    with open(os.path.join(HERE, "..", "include", "lbm_b200.h"), "rb") as fh:
        h.update(fh.read())
    h.update(" ".join(flags()).encode())
    return h.hexdigest()


def build(verbose: bool = False, force: bool = False) -> str:
    from .csrc import gen_tables
    gen_tables.write()
    stamp = os.path.join(BUILD, "stamp")
    digest = _digest()
    if not force and os.path.exists(LIB) and os.path.exists(stamp) and open(stamp).read() == digest:
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()

    def compile_one(src):
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        ostamp = obj + ".stamp"
        d = _digest(src)
        if not force and not verbose and os.path.exists(obj) and os.path.exists(ostamp) and open(ostamp).read() == d:
            return obj, ""
        cmd = [cc, "-c", os.path.join(CSRC, src), "-o", obj] + flags(verbose)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
        with open(ostamp, "w") as fh:
            fh.write(d)
        return obj, r.stderr

    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    if verbose:
        for obj, err in results:
            sys.stderr.write(err)
    objs = [o for o, _ in results]
    tmp = LIB + ".tmp"
    cmd = [cc, "-shared", "-o", tmp] + objs + ARCH + host_compiler()
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    with open(stamp, "w") as fh:
        fh.write(digest)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    print(build(verbose=args.verbose, force=args.force))

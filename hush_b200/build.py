"""Builds the in-tree native libraries.

* ``hush_b200/libhush_b200.so``: the CUDA kernels for sm_100a and the C ABI declared in ``include/hush.h``
  (nvcc, one object per ``csrc/*.cu`` in parallel, static CUDA runtime).
* ``oracle/liboracle_hush.so``: the CPU oracle (test infrastructure; built here so tests can load it).

Usage: ``python -m hush_b200.build [--force] [-v]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libhush_b200.so")
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "liboracle_hush.so")
WEIGHTS = os.path.join(PKG, "data", "hush-weights.bin")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --use_fast_math: exp / log / division / sqrt as the hardware approximations. WGSL itself only promises that
# accuracy (exp 3 + 2|x| ULP, log 2^-21 absolute on [0.5, 2], division 2.5 ULP, inverseSqrt 2 ULP), so the kernels
# stay inside the reference's own numerical contract; the parity tests bound the effect against the exact oracle.
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", "--use_fast_math", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-fopenmp",
    "-I", os.path.join(ROOT, "include"), "-I", BUILD, "-I", CSRC,
] + ARCH
# SVGF's temporal pass compares a weighted-average history length stored with round-toward-zero against 4
# (svgf.js:94, 121): an ulp of difference flips the branch, so that file keeps IEEE arithmetic throughout.
PER_FILE_DROP = {"svgf.cu": {"--use_fast_math"}}


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _gen_weights_inc() -> str:
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(BUILD, "weights_builtin.inc")
    blob = open(WEIGHTS, "rb").read()
    vals = [int.from_bytes(blob[i:i + 2], "little") for i in range(0, len(blob), 2)]
    body = ",".join(f"0x{v:04x}" for v in vals)
    text = (
        "// generated by hush_b200/build.py from hush_b200/data/hush-weights.bin\n"
        f"static const unsigned short HUSH_BUILTIN_WEIGHTS[{len(vals)}] = {{{body}}};\n"
        f"static const unsigned long HUSH_BUILTIN_WEIGHT_COUNT = {len(vals)};\n"
    )
    if not os.path.exists(out) or open(out).read() != text:
        with open(out, "w") as f:
            f.write(text)
    return out


def _newest(paths) -> float:
    return max((os.path.getmtime(p) for p in paths if os.path.exists(p)), default=0.0)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def build_oracle(force: bool = False, verbose: bool = False) -> str:
    src = [os.path.join(ORACLE_DIR, f) for f in os.listdir(ORACLE_DIR) if f.endswith((".cpp", ".h"))]
    src += [os.path.join(ORACLE_DIR, "Makefile"), os.path.join(CSRC, "scene.h")]
    if force or not os.path.exists(ORACLE_LIB) or _newest(src) > os.path.getmtime(ORACLE_LIB):
        _run(["make", "-C", ORACLE_DIR, "-B" if force else "-s", "liboracle_hush.so"], verbose)
    return ORACLE_LIB


def build_cuda(force: bool = False, verbose: bool = False, extra_flags=None) -> str:
    inc = _gen_weights_inc()
    nvcc = _nvcc()
    sources = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh", ".inc"))]
    headers += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    headers.append(inc)
    header_time = _newest(headers)
    flags = NVCC_FLAGS + list(extra_flags or [])
    objs = []
    jobs = []
    for s in sources:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s[:-3] + ".o")
        objs.append(obj)
        if force or not os.path.exists(obj) or max(os.path.getmtime(src), header_time) > os.path.getmtime(obj):
            drop = PER_FILE_DROP.get(s, set())
            jobs.append([nvcc, "-c", src, "-o", obj] + [x for x in flags if x not in drop])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            list(ex.map(lambda c: _run(c, verbose), jobs))
    if force or jobs or not os.path.exists(LIB) or _newest(objs) > os.path.getmtime(LIB):
        tmp = LIB + ".tmp"
        _run([nvcc, "-shared", "-o", tmp] + objs + ARCH + ["-Xcompiler", "-fopenmp", "-lgomp"], verbose)
        os.replace(tmp, LIB)
    return LIB


def build(force: bool = False, verbose: bool = False) -> None:
    build_oracle(force, verbose)
    build_cuda(force, verbose)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    build(a.force, a.verbose)
    print(LIB)
    return 0


if __name__ == "__main__":
    sys.exit(main())

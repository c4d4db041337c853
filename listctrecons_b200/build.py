"""Build liblct.so (the CUDA kernels + C ABI) in-tree for sm_100a.

    python -m listctrecons_b200.build [--force] [-j N]

Every csrc/*.cu and csrc/*.cpp is compiled by nvcc (host code by the system g++), objects go
to listctrecons_b200/_build/, and the shared library to listctrecons_b200/liblct.so.  The CUDA
runtime is linked statically so the library does not depend on the runtime copy another
library in the process (for example torch) loaded.  Only the ``lct_*`` C entry points are
exported.

probe/probe.cu becomes listctrecons_b200/liblctprobe.so: measurement probes (the texture unit's
sampling rule, the L1 load bandwidth) that tests and the benchmark load; nothing in liblct.so
uses it.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "liblct.so"
PROBE_SRC = PKG / "probe" / "probe.cu"
PROBE_LIB = PKG / "liblctprobe.so"
NVCC = os.environ.get("LCT_NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "--extended-lambda",
    "-I",
    str(ROOT / "include"),
    "-I",
    str(CSRC),
    "-Xcompiler",
    "-fPIC,-fvisibility=hidden,-ffp-contract=off,-fno-fast-math",
    # host-side float expressions must round like the reference's (no FMA contraction)
    "-ccbin",
    "g++",
]


def _sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "lct.h"]
    return max(h.stat().st_mtime for h in hs)


def _compile(src: Path, force: bool, verbose: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    if not force and obj.exists():
        if obj.stat().st_mtime >= max(src.stat().st_mtime, _headers_mtime()):
            return obj
    cmd = [NVCC, *ARCH, *COMMON, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cu":
        cmd[1:1] = ["-Xptxas", "-warn-spills"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
    if verbose and (res.stdout.strip() or res.stderr.strip()):
        print(res.stdout + res.stderr, file=sys.stderr)
    return obj


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    # relink also when the set of sources changed (a removed file leaves a newer library behind)
    stamp = BUILD / "liblct.objects"
    names = "\n".join(o.name for o in objs)
    same_set = stamp.exists() and stamp.read_text() == names
    if force or not same_set or not LIB.exists() or LIB.stat().st_mtime < newest:
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
        os.replace(tmp, LIB)
        stamp.write_text(names)
    build_probe(force)
    return LIB


def build_probe(force: bool = False) -> Path:
    if force or not PROBE_LIB.exists() or PROBE_LIB.stat().st_mtime < PROBE_SRC.stat().st_mtime:
        tmp = PROBE_LIB.with_suffix(".so.tmp")
        cmd = [NVCC, *ARCH, "-O3", "-std=c++17", "-lineinfo", "-Xcompiler",
               "-fPIC,-fvisibility=hidden", "-shared", "-cudart", "static", str(PROBE_SRC),
               "-o", str(tmp)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed for {PROBE_SRC.name}:\n{res.stdout}\n{res.stderr}")
        os.replace(tmp, PROBE_LIB)
    return PROBE_LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.j, verbose=a.v))


if __name__ == "__main__":
    main()

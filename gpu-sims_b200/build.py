"""Builds liblbm_b200.so (CUDA sm_100a kernels + C++ host runtime) in-tree.

    python gpu-sims_b200/build.py [--force]

Objects go to gpu-sims_b200/_build/, the library to gpu-sims_b200/lbm/.
nvcc cross-compiles for sm_100a without a GPU.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
OUT = PKG / "lbm" / "liblbm_b200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "-I", str(INCLUDE)] + ARCH
# The voxeliser must round every float op like the reference's host C++.
HOST_EXTRA = {"host_tools.cpp": ["-Xcompiler", "-ffp-contract=off"]}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src] + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    return any(d.stat().st_mtime > obj.stat().st_mtime for d in deps)


def build(force: bool = False, verbose: bool = False, out: Path | None = None,
          build_dir: Path | None = None, defines: list[str] | None = None) -> Path:
    """Compiles every source in csrc/ and links the shared library.  `out`,
    `build_dir` and `defines` (-D flags) allow variant builds elsewhere."""
    global BUILD, OUT
    BUILD = build_dir or BUILD
    OUT = out or OUT
    extra = [f"-D{d}" for d in (defines or [])]
    BUILD.mkdir(parents=True, exist_ok=True)
    OUT.parent.mkdir(parents=True, exist_ok=True)
    cc = nvcc()
    objs, cmds = [], []
    for src in sources():
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if not force and not _stale(obj, src):
            continue
        lang = ["-x", "cu"] if src.suffix == ".cpp" else []
        cmds.append([cc] + lang + ["-c", str(src), "-o", str(obj)] + CUDA_FLAGS + extra +
                    HOST_EXTRA.get(src.name, []))
    # translation units compile in parallel (the step kernels dominate)
    with concurrent.futures.ThreadPoolExecutor(max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for cmd in cmds:
            if verbose:
                print(" ".join(cmd), flush=True)
        for r in ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds):
            if r.returncode:
                sys.stderr.write(r.stdout + r.stderr)
                raise subprocess.CalledProcessError(r.returncode, r.args)
    if force or not OUT.exists() or any(o.stat().st_mtime > OUT.stat().st_mtime for o in objs):
        cmd = [cc, "-shared", "-o", str(OUT)] + [str(o) for o in objs] + ARCH
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return OUT


HOST_SRC = PKG / "host" / "lbm_frame_loop.cpp"


def build_host(lib: Path | None = None, out: Path | None = None) -> Path:
    """Compiles the headless C++ host program (host/lbm_frame_loop.cpp)
    against include/ and the library, with the library's directory as its
    run path."""
    lib = lib or OUT
    out = out or HOST_SRC.with_suffix("")
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-std=c++17", "-O2", "-Wall", "-I", str(INCLUDE), str(HOST_SRC), "-o", str(out),
           "-L", str(lib.parent), "-l:" + lib.name, "-Wl,-rpath," + str(lib.parent)]
    subprocess.run(cmd, check=True)
    return out


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
    print(build_host())
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""Build libcalculator.so (the C-ABI + sm_100a kernels) in-tree with nvcc,
and the C host: librover_host.so (bundle loader) and the `Rover` executable.

    python -m rover_b200.build          # -> rover_b200/lib/libcalculator.so,
                                        #    rover_b200/lib/librover_host.so,
                                        #    rover_b200/bin/Rover

Compiled for sm_100a only.  -fmad=false keeps every floating-point multiply
and add separately rounded, as the reference's host build does; the kernels
also spell those steps with _rn intrinsics.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB_DIR = HERE / "lib"
LIB = LIB_DIR / "libcalculator.so"
HOST_DIR = HERE / "host"
HOST_LIB = LIB_DIR / "librover_host.so"
BIN_DIR = HERE / "bin"
ROVER = BIN_DIR / "Rover"
HOST_SOURCES = ["sha256.c", "json.c", "bundle.c", "artifacts.c"]
HOST_CXX_SOURCES = ["layout.cpp"]

SOURCES = ["calculator.cu", "pq_search.cu", "pq_decoded.cu", "pq_batched.cu", "gate_train.cu", "plan.cu", "sq_search.cu", "distance.cu", "sessions.cu", "seed_rank_tc.cu", "pq_train.cu", "rpcmem_compat.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    LIB_DIR.mkdir(exist_ok=True)
    obj_dir = HERE / "_build"
    obj_dir.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((HERE.parent / "include").glob("*.h"))
    objs, jobs = [], []
    for src in SOURCES:
        s = CSRC / src
        o = obj_dir / (s.stem + ".o")
        objs.append(o)
        if not force and not _stale(o, [s, *headers]):
            continue
        cmd = [nvcc(), *ARCH, "-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-O2",
               "--expt-relaxed-constexpr", "-I", str(CSRC), "-I", str(HERE.parent / "include"), "-c", str(s),
               "-o", str(o)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        jobs.append(cmd)
    # translation units compile independently: run them side by side
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        for f in [pool.submit(subprocess.run, cmd, check=True) for cmd in jobs]:
            f.result()
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-Xlinker", "-Bsymbolic",
               "-lcudart_static", "-lpthread", "-ldl", "-lrt"]
        subprocess.run(cmd, check=True)
    build_host(force)
    return LIB


def cc() -> str:
    for cand in (os.environ.get("CC"), shutil.which("gcc"), shutil.which("cc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("no C compiler found")


def build_host(force: bool = False) -> Path:
    """librover_host.so and bin/Rover (gcc; no CUDA needed to build them)."""
    LIB_DIR.mkdir(exist_ok=True)
    BIN_DIR.mkdir(exist_ok=True)
    include = HERE.parent / "include"
    headers = list(HOST_DIR.glob("*.h")) + list(include.glob("*.h"))
    srcs = [HOST_DIR / s for s in HOST_SOURCES]
    cxx_srcs = [HOST_DIR / s for s in HOST_CXX_SOURCES]
    flags = ["-std=c11", "-O2", "-Wall", "-Wextra", "-Wno-unused-parameter", "-I", str(include), "-I", str(HOST_DIR)]
    if force or _stale(HOST_LIB, [*srcs, *cxx_srcs, *headers]):
        objs = []
        for s_ in cxx_srcs:   # C++ parts (the layout tool) compiled apart, linked into the same library
            o = LIB_DIR / (s_.stem + ".host.o")
            subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-fPIC", "-c", str(s_), "-o", str(o)], check=True)
            objs.append(str(o))
        subprocess.run([cc(), *flags, "-fPIC", "-shared", "-o", str(HOST_LIB), *map(str, srcs), *objs, "-lm",
                        "-lstdc++", "-lpthread"], check=True)
        for o in objs:
            Path(o).unlink()
    cli = HOST_DIR / "rover_cli.c"
    if force or _stale(ROVER, [cli, HOST_LIB, LIB, *headers]):
        subprocess.run([cc(), *flags, "-o", str(ROVER), str(cli), "-L", str(LIB_DIR), "-lrover_host", "-lcalculator",
                        "-lm", "-Wl,-rpath,$ORIGIN/../lib"], check=True)
    return ROVER


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)

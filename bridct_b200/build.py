"""Builds libbridct_b200.so in-tree for sm_100a.

    python -m bridct_b200.build          # or __graft_entry__.build()

Steps: regenerate csrc/sj_generated.cuh from csrc/gen_sj.py when the generator changed,
compile each CUDA translation unit with nvcc (-gencode arch=compute_100a,code=sm_100a), the
plain-form instantiations once per array height in parallel, and link one shared library
with the CUDA runtime linked statically; then build the pipe runner against it.  Objects go to _build/ at the repository root.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = ROOT / "_build"
LIB = PKG / "libbridct_b200.so"
RUNNER = PKG / "bridct_runner"
HEIGHTS = (8, 16, 32, 64, 128, 256, 512, 1024)
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
              "--expt-relaxed-constexpr", "-I", str(ROOT / "include")] + ARCH


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libbridct_b200.so")


def _newer(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed:\n" + " ".join(map(str, cmd)) + "\n" + r.stdout + r.stderr)


def generate() -> None:
    gen = CSRC / "gen_sj.py"
    hdr = CSRC / "sj_generated.cuh"
    if _newer(hdr, [gen]):
        r = subprocess.run([sys.executable, str(gen)], capture_output=True, text=True, check=True)
        hdr.write_text(r.stdout)


def build(verbose: bool = False) -> Path:
    generate()
    OUT.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((ROOT / "include").glob("*.h"))
    jobs = []
    for h in HEIGHTS:
        obj = OUT / f"plain_h{h}.o"
        src = CSRC / "plain_inst.cu"
        jobs.append((obj, [nvcc()] + NVCC_FLAGS + [f"-DBRIDCT_H={h}", "-c", str(src), "-o", str(obj)],
                     [src] + headers))
    for src in sorted(CSRC.glob("*.cu")):
        if src.name == "plain_inst.cu":
            continue
        obj = OUT / (src.stem + ".o")
        jobs.append((obj, [nvcc()] + NVCC_FLAGS + ["-c", str(src), "-o", str(obj)], [src] + headers))
    todo = [(o, c) for o, c, d in jobs if _newer(o, d)]
    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 4))) as ex:
        for fut in [ex.submit(_run, c) for _, c in todo]:
            fut.result()
    objs = [o for o, _, _ in jobs]
    if _newer(LIB, objs):
        _run([nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", str(LIB)] + [str(o) for o in objs])
    # the pipe runner (wire protocol of the reference's test runner) next to the library
    runner_src = PKG / "runner" / "bridct_runner.c"
    if _newer(RUNNER, [runner_src, LIB, ROOT / "include" / "bridct.h"]):
        cc = os.environ.get("CC") or shutil.which("gcc") or "cc"
        _run([cc, "-std=c11", "-O2", "-Wall", "-I", str(ROOT / "include"), str(runner_src), "-L", str(PKG),
              "-l:libbridct_b200.so", "-Wl,-rpath,$ORIGIN", "-o", str(RUNNER)])
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(verbose=True)

"""Build libfclaw_b200.so (sm_100a) in-tree with nvcc.

Usage: python -m forestclaw_b200.build [--force]

The FP64 kernels are compiled with -fmad=false: every multiply and add is
rounded separately, as the reference Fortran is on x86-64 without FMA, so the
FP64 results match the reference's arithmetic operation by operation.  The
mixed-precision step (fcb_step_mixed.cu) is compiled with --use_fast_math:
its FP32 solves use the fast division and square root.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libfclaw_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "-I", str(PKG.parent / "include")]



def _nccl_include() -> str:
    """nccl.h of the NCCL that PyTorch ships (the library the process loads), else the system one."""
    try:
        import nvidia.nccl as n  # noqa: PLC0415
        for root in n.__path__:
            if (Path(root) / "include" / "nccl.h").exists():
                return str(Path(root) / "include")
    except ImportError:
        pass
    return "/usr/include"


# per-source extra flags
SOURCES = {
    "fcb_step.cu": ["-fmad=false"],
    "fcb_step_warp.cu": ["-fmad=false"],
    "fcb_step_pipe.cu": ["-fmad=false"],
    "fcb_step_mixed.cu": ["--use_fast_math"],
    "fcb_step_fused.cu": ["-fmad=false"],
    "fcb_step_fused_mixed.cu": ["--use_fast_math"],
    "fcb_ghost.cu": ["-fmad=false"],
    "fcb_amr.cu": ["-fmad=false"],
    "fcb_runtime.cu": [],
    "fcb_serve.cu": [],
    "fcb_capi.cu": ["-Xcompiler", "-fvisibility=default"],
    "fcb_noalloc.cu": ["-fmad=false"],
    "fcb_src.cu": ["-fmad=false"],
    "fcb_probe.cu": ["-fmad=false"],
    "fcb_timesync.cu": ["-fmad=false"],
    "fcb_output.cpp": [],
    "fcb_comm.cu": ["-I", _nccl_include()],
}


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _includes(path: Path, seen=None) -> set:
    """Project headers a source includes, directly or through other headers."""
    seen = set() if seen is None else seen
    for line in path.read_text().splitlines():
        line = line.strip()
        if line.startswith("#include \""):
            name = line.split("\"")[1]
            for d in (CSRC, PKG.parent / "include"):
                h = d / name
                if h.exists() and h not in seen:
                    seen.add(h)
                    _includes(h, seen)
    return seen


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    objs = []
    jobs = []
    for src, flags in SOURCES.items():
        obj = BUILD / (src + ".o")
        objs.append(obj)
        deps = [CSRC / src, Path(__file__), *sorted(_includes(CSRC / src))]
        if force or _stale(obj, deps):
            cmd = [NVCC, *ARCH, *COMMON, *flags, "-c", str(CSRC / src), "-o", str(obj)]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    if force or jobs or _stale(LIB, objs):
        run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs)])
    return LIB


if __name__ == "__main__":
    p = build(force="--force" in sys.argv, verbose=True)
    print(p)

"""Builds libfeelmri_b200.so in-tree with nvcc for sm_100a.

The library is a plain shared object exporting the C ABI declared in
include/feelmri_b200.h; Python reaches it through ctypes (feelmri_b200._lib).
"""
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libfeelmri_b200.so"
BUILD = ROOT / "_build"

SOURCES = [
    "context.cu",
    "pod.cu",
    "pod_build.cu",
    "bloch.cu",
    "signal_common.cu",
    "signal_plain.cu",
    "signal_tc.cu",
    "signal.cu",
    "mass.cu",
]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    return "nvcc"


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src, *CSRC.glob("*.cuh"), ROOT / "include" / "feelmri_b200.h", Path(__file__)]
    return any(d.stat().st_mtime > obj.stat().st_mtime for d in deps)


def build(verbose: bool = False, extra_flags=None, jobs: int = 8) -> Path:
    """Compiles every .cu under csrc/ and links libfeelmri_b200.so."""
    BUILD.mkdir(exist_ok=True)
    flags = NVCC_FLAGS + list(extra_flags or [])
    procs = []
    objs = []
    for name in SOURCES:
        src = CSRC / name
        obj = BUILD / (name + ".o")
        objs.append(obj)
        if not _stale(obj, src):
            continue
        cmd = [nvcc(), *ARCH, *flags, "-I", str(ROOT / "include"), "-dc", "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((name, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        if len(procs) >= jobs:
            _drain(procs)
    _drain(procs)
    link = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(LIB), *map(str, objs)]
    if verbose:
        print(" ".join(link), flush=True)
    out = subprocess.run(link, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if out.returncode != 0:
        raise RuntimeError("link failed:\n" + out.stdout)
    return LIB


def build_host(verbose: bool = False) -> Path:
    """Compiles the CPython extension _hostconv (host-side argument
    conversion, csrc/hostconv.cpp) with g++ next to the package."""
    import sysconfig
    import numpy as np
    src = CSRC / "hostconv.cpp"
    out = PKG / ("_hostconv" + sysconfig.get_config_var("EXT_SUFFIX"))
    if out.exists() and out.stat().st_mtime > max(src.stat().st_mtime, Path(__file__).stat().st_mtime):
        return out
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden", "-pthread",
           "-I", sysconfig.get_paths()["include"], "-I", np.get_include(), str(src), "-o", str(out)]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if res.returncode != 0:
        raise RuntimeError("g++ failed on hostconv.cpp:\n" + res.stdout)
    return out


def _drain(procs):
    failed = []
    for name, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((name, out))
        elif out.strip() and "warning" in out:
            sys.stderr.write(out)
    procs.clear()
    if failed:
        raise RuntimeError("\n".join(f"nvcc failed on {n}:\n{o}" for n, o in failed))


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
    print(build_host(verbose="-v" in sys.argv))

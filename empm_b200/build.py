"""Build libempm_b200.so in-tree with nvcc for sm_100a.

    python -m empm_b200.build [--verbose]

Every ``csrc/*.cu`` is compiled to an object and linked into
``empm_b200/_lib/libempm_b200.so`` (cudart linked statically). Objects are
rebuilt when the hash of their sources, the headers and the flags changes.
"""
from __future__ import annotations

import argparse
import glob
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
BUILD_DIR = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                     "-Xptxas", "-warn-spills"]
# extra nvcc arguments, e.g. launch-shape macros for a sweep:
#   EMPM_NVCC_EXTRA="-DEMPM_FUSED_MIN_CTAS=3" python -m empm_b200.build
NVCC_FLAGS += os.environ.get("EMPM_NVCC_EXTRA", "").split()


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _digest(paths, extra) -> str:
    h = hashlib.sha256()
    for p in paths:
        h.update(os.path.basename(p).encode())
        with open(p, "rb") as f:
            h.update(f.read())
    h.update(" ".join(extra).encode())
    return h.hexdigest()


def _stamp_path(target: str) -> str:
    return target + ".sha256"


def _up_to_date(target: str, digest: str) -> bool:
    """True when target exists and was built from sources with this digest
    (content hashes, not modification times: a stale object copied in with a
    newer time stamp is rebuilt all the same)."""
    stamp = _stamp_path(target)
    if not (os.path.exists(target) and os.path.exists(stamp)):
        return False
    with open(stamp) as f:
        return f.read().strip() == digest


def _write_stamp(target: str, digest: str) -> None:
    with open(_stamp_path(target), "w") as f:
        f.write(digest + "\n")


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(BUILD_DIR, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) +
                     glob.glob(os.path.join(os.path.dirname(HERE), "include", "*.h")))
    objs, obj_digests = [], []
    for src in sources:
        obj = os.path.join(BUILD_DIR, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        digest = _digest([src] + headers, NVCC_FLAGS)
        obj_digests.append(digest)
        if force or not _up_to_date(obj, digest):
            cmd = [nvcc()] + NVCC_FLAGS + ["-c", src, "-o", obj]
            if verbose:
                cmd += ["-Xptxas", "-v"]
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
            _write_stamp(obj, digest)
    target = os.path.join(OUT_DIR, "libempm_b200.so")
    link_digest = hashlib.sha256("".join(obj_digests).encode()).hexdigest()
    if force or not _up_to_date(target, link_digest):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", target] + objs + ["-cudart", "static"]
        subprocess.run(cmd, check=True)
        _write_stamp(target, link_digest)
    return target


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(verbose=a.verbose, force=a.force))
    sys.exit(0)

"""Build libatom3d_b200.so (sm_100a) in-tree with nvcc.

The library is a plain C-ABI shared object: no torch headers, no pybind.
Run ``python -m atom3d_b200.build`` or call :func:`build`.
"""

from __future__ import annotations

import hashlib
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG_DIR, "csrc")
INCLUDE = os.path.join(os.path.dirname(PKG_DIR), "include")
OUT_DIR = os.path.join(PKG_DIR, "_lib")
LIB_NAME = "libatom3d_b200.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON_FLAGS = [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC",
    "--expt-relaxed-constexpr",
    "-I" + INCLUDE,
]


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h", ".inc"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return sorted(hs)


def _digest(paths: list[str], extra: str) -> str:
    h = hashlib.sha256(extra.encode())
    for p in paths:
        with open(p, "rb") as f:
            h.update(p.encode())
            h.update(f.read())
    return h.hexdigest()


def lib_path() -> str:
    return os.path.join(OUT_DIR, LIB_NAME)


def build(force: bool = False, verbose: bool = False, extra_flags: list[str] | None = None) -> str:
    """Compile every .cu under csrc/ and link the shared library.

    Objects are cached by a content hash of the sources, headers and flags.
    """
    os.makedirs(OUT_DIR, exist_ok=True)
    flags = ARCH_FLAGS + COMMON_FLAGS + list(extra_flags or [])
    headers = _headers()
    stamp_path = os.path.join(OUT_DIR, "build.stamp")
    srcs = sources()
    digest = _digest(srcs + headers, " ".join(flags))
    out = lib_path()
    if not force and os.path.exists(out) and os.path.exists(stamp_path):
        with open(stamp_path) as f:
            if f.read().strip() == digest:
                return out
    hdr_digest = _digest(headers, " ".join(flags))

    def compile_one(src: str) -> str:
        base = os.path.splitext(os.path.basename(src))[0]
        obj = os.path.join(OUT_DIR, base + ".o")
        ostamp = obj + ".stamp"
        d = _digest([src], hdr_digest)
        if not force and os.path.exists(obj) and os.path.exists(ostamp):
            with open(ostamp) as f:
                if f.read().strip() == d:
                    return obj
        cmd = [NVCC, *flags, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr:
            print(r.stderr, file=sys.stderr)
        with open(ostamp, "w") as f:
            f.write(d)
        return obj

    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(compile_one, srcs))
    cmd = [NVCC, *ARCH_FLAGS, "-shared", "-cudart", "static", "-o", out, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    with open(stamp_path, "w") as f:
        f.write(digest)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

"""Build recipe for the native library libdcvc_b200.so (sm_100a only).

Compiles every .cu/.cpp under dcvc_b200/csrc with nvcc into one shared library placed next to
this file, so it ships with the source tree.  Objects are cached under dcvc_b200/_build and
rebuilt when a source or any header in csrc/ or include/ changes.
"""
import hashlib
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdcvc_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-pthread",
          "-I" + CSRC, "-I" + INCLUDE]


def _sources():
    out = []
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cu", ".cpp")):
            out.append(os.path.join(CSRC, name))
    return out


def _headers_digest():
    h = hashlib.sha1()
    for d in (CSRC, INCLUDE):
        for name in sorted(os.listdir(d)):
            if name.endswith((".h", ".cuh", ".hpp")):
                with open(os.path.join(d, name), "rb") as f:
                    h.update(name.encode())
                    h.update(f.read())
    return h.hexdigest()


def _compile(src, hdr_digest, verbose):
    with open(src, "rb") as f:
        key = hashlib.sha1(f.read() + hdr_digest.encode() + " ".join(COMMON + ARCH).encode()).hexdigest()[:16]
    obj = os.path.join(BUILD, os.path.basename(src) + "." + key + ".o")
    if os.path.exists(obj):
        return obj
    cmd = [NVCC] + ARCH + COMMON + ["-c", src, "-o", obj + ".tmp"]
    if src.endswith(".cpp"):
        cmd = [NVCC] + COMMON + ["-x", "c++", "-c", src, "-o", obj + ".tmp"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    os.replace(obj + ".tmp", obj)
    return obj


def build(verbose=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    digest = _headers_digest()
    srcs = _sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, digest, verbose), srcs))
    link_flags = ["-shared", "-cudart", "static", "-lpthread"]
    link_key = hashlib.sha1(("".join(sorted(objs)) + " ".join(link_flags)).encode()).hexdigest()[:16]
    stamp = os.path.join(BUILD, "link." + link_key)
    if os.path.exists(LIB) and os.path.exists(stamp):
        return LIB
    cmd = [NVCC] + ARCH + ["-o", LIB + ".tmp"] + objs + link_flags
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(LIB + ".tmp", LIB)
    for name in os.listdir(BUILD):
        if name.startswith("link."):
            os.remove(os.path.join(BUILD, name))
    open(stamp, "w").close()
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))

"""Builds libfinb200.so in-tree with nvcc for sm_100a (no GPU needed).

Each translation unit compiles to its own object in parallel (one nvcc per
source), and the objects link into the shared library.  An object is rebuilt
when its source or any header is newer than it.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib", "libfinb200.so")
OBJ = os.path.join(HERE, "_lib", "obj")

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC",
    "-Xptxas", "-v",
]
SOURCES = ["finess_b200.cu", "fin_ini.cpp", "fin_noalloc.cu", "fin_mlp.cu", "fin_batch.cu", "fin_mhd.cu",
           "fin_output.cu"]


def _walk_sources(exts):
    for d in (CSRC, os.path.join(ROOT, "include")):
        for dirpath, _, files in os.walk(d):
            if os.path.basename(dirpath) == "shim":   # compiled into applications, not this library
                continue
            for f in files:
                if f.endswith(exts):
                    yield os.path.join(dirpath, f)


def _newest(exts):
    return max((os.path.getmtime(f) for f in _walk_sources(exts)), default=0.0)


def _compile(nvcc, src, obj, verbose):
    cmd = [nvcc] + NVCC_FLAGS + ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "-c", src, "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    return src, res


def build(force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    headers = _newest((".cuh", ".h"))
    nvcc = os.environ.get("NVCC", "nvcc")
    jobs = []
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJ, s + ".o")
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(headers, os.path.getmtime(src)):
            jobs.append((src, obj))
    if not jobs and os.path.exists(OUT) and os.path.getmtime(OUT) >= max(os.path.getmtime(o) for o in objs):
        return OUT
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda j: _compile(nvcc, j[0], j[1], verbose), jobs))
    failed = False
    for src, res in results:
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            failed = True
        elif verbose:
            sys.stdout.write(res.stderr)
    if failed:
        raise RuntimeError("nvcc failed")
    res = subprocess.run([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", OUT] + objs,
                         capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("link failed")
    return OUT


def build_app(src, out, force=False):
    """An application's own .cu file (its physics policy and hooks, its
    extern "C" entry points) compiled against this library's device headers
    (fin_physics.cuh, fin_physics_host.h, fin_sample.cuh) into a shared
    library, as an application links its callbacks."""
    headers = _newest((".cuh", ".h"))
    if not force and os.path.exists(out) and os.path.getmtime(out) >= max(headers, os.path.getmtime(src)):
        return out
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + ["-shared", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "-o", out, src]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed on " + src)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

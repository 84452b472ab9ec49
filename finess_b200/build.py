"""Builds libfinb200.so in-tree with nvcc for sm_100a (no GPU needed)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib", "libfinb200.so")

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-shared",
    "-Xptxas", "-v",
]
SOURCES = ["finess_b200.cu", "fin_ini.cpp", "fin_noalloc.cu", "fin_mlp.cu", "fin_batch.cu", "fin_mhd.cu", "fin_output.cu"]


def _newest_source():
    newest = 0.0
    for d in (CSRC, os.path.join(ROOT, "include")):
        for dirpath, _, files in os.walk(d):
            if os.path.basename(dirpath) == "shim":   # compiled into applications, not this library
                continue
            for f in files:
                if f.endswith((".cu", ".cuh", ".h", ".cpp")):
                    newest = max(newest, os.path.getmtime(os.path.join(dirpath, f)))
    return newest


def build(force=False, verbose=False):
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= _newest_source():
        return OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "-o", OUT] + \
        [os.path.join(CSRC, s) for s in SOURCES]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed")
    if verbose:
        sys.stdout.write(res.stderr)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

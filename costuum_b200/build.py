"""Build the CUDA library libtmx.so in-tree for sm_100a (B200).

The table kernels (tmx_tables.cu) are compiled with --fmad=false so their
recurrences round like the reference's x86-64 build; the block, observable
and probe kernels use fused multiply-add.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtmx.so")

SOURCES = [
    ("tmx_tables.cu", ["--fmad=false"]),
    ("tmx_blocks.cu", []),
    ("tmx_tangent.cu", []),
    ("tmx_observables.cu", ["--fmad=false"]),
    ("tmx_probe.cu", []),
    ("tmx_host.cu", []),
    ("tmx_table.cu", []),
    ("tmx_noalloc.cu", []),
    ("tmx_plain.cu", []),
    ("tmx_graph.cu", []),
]

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
         "-I", os.path.join(HERE, "..", "include")]


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build failed: " + " ".join(cmd))
    return r.stdout


def build(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    newest = 0.0
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC)
               if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "tmx.h"))
    hdr_time = max(os.path.getmtime(h) for h in headers)
    for src, extra in SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(obj)
        stale = (not os.path.exists(obj)
                 or os.path.getmtime(obj) < max(os.path.getmtime(path), hdr_time))
        if stale:
            out = _run([NVCC] + ARCH + FLAGS + extra + ["-c", path, "-o", obj])
            if verbose and out:
                print(out)
        newest = max(newest, os.path.getmtime(obj))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))

"""Build the in-tree sm_100a shared library gexs_b200/libgexs_b200.so.

nvcc cross-compiles for sm_100a without a GPU.  Objects go to
gexs_b200/_build/ (git-ignored); the .so lands beside this file so it
travels with the repository snapshot.

    python -m gexs_b200.build [--ptxas-verbose]
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
          "-I" + os.path.join(ROOT, "include")]
SOURCES = [
    "csrc/gexs_kernels.cu",
    "csrc/gexs_tiles_voigt.cu",
    "csrc/gexs_tiles_erf.cu",
    "csrc/gexs_tiles_gh16.cu",
    "csrc/gexs_tiles_gh32.cu",
    "csrc/gexs_capi.cu",
    "csrc/gexs_calib.cu",
    "csrc/gexs_noalloc.cu",
    "csrc/gexs_ingest.cu",
    "host/B200Manager.cpp",
    "host/gexs_server.cpp",
    "host/B200ExomolReader.cpp",
    "host/gexs_output.cpp",
    "host/gexs_tips.cpp",
    "host/gexs_shard.cpp",
    "host/B200MultiManager.cpp",
]
LIB = os.path.join(HERE, "libgexs_b200.so")


def _run(cmd):
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("command failed: %s\n%s%s" % (" ".join(cmd), p.stdout, p.stderr))
    return p.stdout + p.stderr


def build(ptxas_verbose=False, force=False):
    bdir = os.path.join(HERE, "_build")
    os.makedirs(bdir, exist_ok=True)
    deps = []
    for root, _, files in os.walk(os.path.join(HERE, "csrc")):
        deps += [os.path.join(root, f) for f in files]
    for root, _, files in os.walk(os.path.join(HERE, "host")):
        deps += [os.path.join(root, f) for f in files]
    deps.append(os.path.join(ROOT, "include", "gexs_b200.h"))
    deps.append(os.path.join(ROOT, "include", "gexs_serve.h"))
    deps.append(os.path.join(ROOT, "include", "gexs_reader.h"))
    newest = max(os.path.getmtime(d) for d in deps)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB

    def compile_one(src):
        obj = os.path.join(bdir, os.path.basename(src) + ".o")
        cmd = [NVCC] + ARCH + COMMON + ["-c", os.path.join(HERE, src), "-o", obj]
        if ptxas_verbose and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        return obj, _run(cmd)

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    log = "".join(r[1] for r in results)
    objs = [r[0] for r in results]
    tmp = LIB + ".tmp"
    _run([NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart_static", "-lpthread", "-ldl", "-lrt"])
    os.replace(tmp, LIB)
    if ptxas_verbose:
        sys.stderr.write(log)
    return LIB


if __name__ == "__main__":
    build(ptxas_verbose="--ptxas-verbose" in sys.argv, force=True)
    print(LIB)

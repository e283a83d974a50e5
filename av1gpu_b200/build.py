"""Build of the CUDA library (sm_100a) and of the CPU oracle.

    python -m av1gpu_b200.build          # libisearch.so in-tree (+ oracle/_ref/liboracle.so when the reference exists)

The library includes av1core's public headers (the DecisionRecord ABI, the AV1 spec tables and the default CDFs) from
AV1CORE_INCLUDE (default: the reference checkout's av1core/include); nothing else of the reference is compiled into it.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libisearch.so")
REF = os.environ.get("AV1GPU_REF", "/root/reference")
AV1CORE_INCLUDE = os.environ.get("AV1CORE_INCLUDE", os.path.join(REF, "av1core", "include"))
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
# every source of the library (a change to any of them rebuilds it)
SOURCES = sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".py")))


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def gen_txfm():
    out = os.path.join(CSRC, "txfm_gen.cuh")
    gen = os.path.join(CSRC, "gen_txfm.py")
    if _newer(out, [gen]):
        code = subprocess.run([sys.executable, gen], check=True, capture_output=True, text=True).stdout
        with open(out, "w") as f:
            f.write(code)


def build_lib(verbose=False):
    gen_txfm()
    deps = [os.path.join(CSRC, s) for s in SOURCES] + [os.path.join(ROOT, "include", "is_api.h")]
    if not _newer(LIB, deps):
        return LIB
    if not os.path.isdir(AV1CORE_INCLUDE):
        if os.path.exists(LIB):
            return LIB
        raise RuntimeError("av1core headers not found at %s (set AV1CORE_INCLUDE)" % AV1CORE_INCLUDE)
    cmd = [NVCC, "-std=c++17", "-O3", "-lineinfo", "-gencode", "arch=compute_100a,code=sm_100a",
           "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills",
           "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "-I" + AV1CORE_INCLUDE,
           os.path.join(CSRC, "is_api.cu"), "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def build_oracle():
    if not os.path.isdir(REF):
        return None   # the GPU host has no reference checkout: the prebuilt oracle/_ref travels with the tree
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "REF=" + REF], check=True)
    return os.path.join(ROOT, "oracle", "_ref", "liboracle.so")


def build_all(verbose=False):
    build_lib(verbose)
    build_oracle()


if __name__ == "__main__":
    build_all(verbose=True)

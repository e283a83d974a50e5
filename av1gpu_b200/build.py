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
# the reference checkout (its av1core headers and sources); set AV1GPU_REF, or AV1CORE_INCLUDE for the headers only.
# Without it the prebuilt libisearch.so / oracle/_ref are used as they are.
REF = os.environ.get("AV1GPU_REF", "")
AV1CORE_INCLUDE = os.environ.get("AV1CORE_INCLUDE", os.path.join(REF, "av1core", "include") if REF else "")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


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


# compilation units: (source, object, defines).  The analysis unit is compiled once per bit depth and kernel pair, the
# closed loop once per format, the entropy coder and the post-filters once; the units build in parallel and are linked into one library.
UNITS = [("is_api.cu", "is_api.o", []),
         ("is_k_an.cu", "is_k_an8w.o", ["-DIS_BD=8", "-DIS_AN_PART=0"]), ("is_k_an.cu", "is_k_an8t.o", ["-DIS_BD=8", "-DIS_AN_PART=1"]),
         ("is_k_an.cu", "is_k_an10w.o", ["-DIS_BD=10", "-DIS_AN_PART=0"]), ("is_k_an.cu", "is_k_an10t.o", ["-DIS_BD=10", "-DIS_AN_PART=1"]),
         ("is_k_rc.cu", "is_k_rc8_420.o", ["-DIS_BD=8", "-DIS_SS=1"]), ("is_k_rc.cu", "is_k_rc8_444.o", ["-DIS_BD=8", "-DIS_SS=0"]),
         ("is_k_rc.cu", "is_k_rc10_420.o", ["-DIS_BD=10", "-DIS_SS=1"]), ("is_k_rc.cu", "is_k_rc10_444.o", ["-DIS_BD=10", "-DIS_SS=0"]),
         ("is_k_ent.cu", "is_k_ent.o", []), ("is_k_pf.cu", "is_k_pf.o", [])]
BUILD_DIR = os.path.join(HERE, "_build")
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC",
              "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def _local_deps(src, seen=None):
    """src and every header of csrc/ or include/ it includes, recursively."""
    import re
    seen = set() if seen is None else seen
    if src in seen or not os.path.exists(src):
        return seen
    seen.add(src)
    with open(src) as f:
        for m in re.finditer(r'^\s*#\s*include\s+"([^"]+)"', f.read(), re.M):
            for d in (CSRC, os.path.join(ROOT, "include")):
                cand = os.path.join(d, m.group(1))
                if os.path.exists(cand):
                    _local_deps(cand, seen)
                    break
    return seen


def build_lib(verbose=False, jobs=None):
    gen_txfm()
    if not os.path.isdir(AV1CORE_INCLUDE):
        if os.path.exists(LIB):
            return LIB
        raise RuntimeError("av1core headers not found at %s (set AV1GPU_REF or AV1CORE_INCLUDE)" % AV1CORE_INCLUDE)
    os.makedirs(BUILD_DIR, exist_ok=True)
    incs = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "-I" + AV1CORE_INCLUDE]
    todo = []
    for src, obj, defs in UNITS:
        o = os.path.join(BUILD_DIR, obj)
        if _newer(o, sorted(_local_deps(os.path.join(CSRC, src)))):
            todo.append([NVCC] + NVCC_FLAGS + defs + incs + ["-c", os.path.join(CSRC, src), "-o", o + ".tmp"])
    if todo:
        from concurrent.futures import ThreadPoolExecutor

        def run(cmd):
            if verbose:
                print(" ".join(cmd), flush=True)
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode:
                raise RuntimeError("compile failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
            if verbose and (r.stdout or r.stderr):
                print(r.stdout + r.stderr, flush=True)
            os.replace(cmd[-1], cmd[-1][:-4])
        with ThreadPoolExecutor(max_workers=jobs or min(len(todo), os.cpu_count() or 1)) as ex:
            list(ex.map(run, todo))
    objs = [os.path.join(BUILD_DIR, o) for _, o, _ in UNITS]
    if todo or _newer(LIB, objs):
        subprocess.run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC"] + objs +
                       ["-o", LIB + ".tmp"], check=True)
        os.replace(LIB + ".tmp", LIB)
    return LIB


def build_oracle():
    if not REF or not os.path.isdir(REF):
        return None   # the GPU host has no reference checkout: the prebuilt oracle/_ref travels with the tree
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "REF=" + REF], check=True)
    # the reference's own GPU search (measurement only: the speed bar and its decisions for BD-rate comparisons); a
    # failure here leaves the comparison out, not the build
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "-f", "refgpu.mk", "REF=" + REF, "-j%d" % (os.cpu_count() or 1)],
                       capture_output=True, text=True)
    if r.returncode:
        print("note: the reference GPU search was not built (oracle/refgpu.mk):", (r.stderr or r.stdout)[-400:], file=sys.stderr)
    return os.path.join(ROOT, "oracle", "_ref", "liboracle.so")


def build_all(verbose=False):
    build_lib(verbose)
    build_oracle()


if __name__ == "__main__":
    build_all(verbose=True)

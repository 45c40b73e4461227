"""Build libflsp_dg.so (sm_100a) in-tree with nvcc.

    python -m felspa_b200.build [--verbose] [--force]

Kernel families live in separate translation units (felspa_b200/csrc/
flsp_k_*.cu, each with its own constant-memory tables) that compile in
parallel; flsp_api.cu holds the C ABI.  The library links the static CUDA
runtime, so the .so built here runs unchanged on a B200 host.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libflsp_dg.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
UNITS = ["flsp_api.cu", "flsp_k_adv.cu", "flsp_k_sep2.cu", "flsp_k_sep3.cu", "flsp_k_hj.cu", "flsp_k_misc.cu", "flsp_mlp.cu", "flsp_k_batch.cu", "flsp_io.cu"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def deps(path, seen=None):
    """the file and every local header it includes, recursively"""
    seen = set() if seen is None else seen
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    with open(path) as f:
        for line in f:
            line = line.strip()
            if line.startswith("#include \""):
                name = line.split('"')[1]
                for d in (CSRC, os.path.join(ROOT, "include")):
                    cand = os.path.join(d, name)
                    if os.path.exists(cand):
                        deps(cand, seen)
                        break
    return seen


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(unit, verbose):
    src = os.path.join(CSRC, unit)
    obj = os.path.join(OBJ, unit.replace(".cu", ".o"))
    if not _stale(obj, sorted(deps(src))):
        return obj, ""
    cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj + ".tmp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {unit}:\n{r.stdout}{r.stderr}")
    os.replace(obj + ".tmp", obj)
    return obj, r.stderr


def build(verbose=False, force=False):
    os.makedirs(OBJ, exist_ok=True)
    if force:
        for f in os.listdir(OBJ):
            os.remove(os.path.join(OBJ, f))
    with cf.ThreadPoolExecutor(len(UNITS)) as ex:
        res = list(ex.map(lambda u: _compile(u, verbose), UNITS))
    objs = [o for o, _ in res]
    if verbose:
        for _, log in res:
            sys.stderr.write(log)
    if _stale(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", *objs, "-o", LIB + ".tmp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc link failed:\n{r.stdout}{r.stderr}")
        os.replace(LIB + ".tmp", LIB)
    build_examples()
    return LIB


EXAMPLES = os.path.join(HERE, "examples")


def build_examples():
    """C++ drivers written against include/flsp_dg.hpp, linked to the library"""
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    for f in sorted(os.listdir(EXAMPLES)):
        if not f.endswith(".cpp"):
            continue
        src = os.path.join(EXAMPLES, f)
        exe = os.path.join(EXAMPLES, f[:-4] + ".bin")
        hdrs = [os.path.join(ROOT, "include", h) for h in ("flsp_dg.h", "flsp_dg.hpp")]
        if not _stale(exe, [src, LIB] + hdrs):
            continue
        cmd = [cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), src, "-o", exe,
               "-L", HERE, "-lflsp_dg", "-Wl,-rpath,$ORIGIN/.."]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"building {f} failed:\n{r.stdout}{r.stderr}")


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv)
    print(LIB)

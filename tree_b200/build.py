"""Builds tree_b200/libtree_b200.so from tree_b200/csrc/ with nvcc for sm_100a.

Run as ``python -m tree_b200.build``.  The parity kernels (octree build, FP64
walk, integrator, direct sum) are compiled with -fmad=false so that no
multiply-add contraction changes their rounding; the mixed-precision kernels
keep FMA.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtree_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
          "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]
NOFMA = {"build.cu", "walk64.cu", "kdk.cu", "direct.cu"}


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else shutil.which("nvcc")


def _version_define():
    try:
        rev = subprocess.run(["git", "-C", HERE, "describe", "--always", "--dirty"],
                             capture_output=True, text=True, timeout=10).stdout.strip()
    except Exception:  # noqa: BLE001 - version string only
        rev = "unknown"
    return f'-DTREE_GPU_VERSION_STR="tree_b200 sm_100a {rev or "unknown"}"'


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _compile(src, verbose):
    nvcc = _nvcc()
    obj = os.path.join(OUT_DIR, src.replace(".cu", ".o"))
    flags = list(COMMON)
    if src in NOFMA:
        flags.append("-fmad=false")
    cmd = [nvcc, *ARCH, *flags, _version_define(), "-c",
           os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose=False):
    nvcc = _nvcc()
    if nvcc is None:
        raise RuntimeError("nvcc not found")
    os.makedirs(OUT_DIR, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for (o, log), s in zip(results, srcs):
            print(f"== {s}\n{log}")
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-o", tmp, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    build_driver()
    return LIB


DRIVER = os.path.join(HERE, "tree_run")


def build_driver():
    """The host driver tree_b200/tree_run (control.prm / input.xyz in,
    ener / rdf / res files out), linked against the library next to it."""
    cxx = shutil.which("g++") or "g++"
    src = os.path.join(HERE, "host", "tree_run.cpp")
    cmd = [cxx, "-O2", "-std=c++17", src, "-o", DRIVER + ".tmp", "-L" + HERE,
           "-ltree_b200", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"driver build failed:\n{r.stdout}\n{r.stderr}")
    os.replace(DRIVER + ".tmp", DRIVER)
    return DRIVER


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))

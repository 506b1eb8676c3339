"""Builds tinker-hp_b200/libthp.so from csrc/ with nvcc for sm_100a.

Each translation unit is compiled separately (in parallel) into _build/ and
linked into an in-tree shared library against cuFFT; the CUDA runtime is
linked statically so the library does not depend on the runtime version of
other libraries in the process.
"""
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libthp.so")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def nvcc():
    p = os.path.join(CUDA_HOME, "bin", "nvcc")
    return p if os.path.exists(p) else shutil.which("nvcc")


def flags(extra=()):
    return ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"),
                   "--expt-relaxed-constexpr", *extra]


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _compile(src, verbose=False, extra=()):
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    cmd = [nvcc(), *flags(extra), "-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "thp.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    if not force and not _stale():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    with concurrent.futures.ThreadPoolExecutor(max_workers=8) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose, extra), sources()))
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcufft", "-cudart", "static",
           "-Xlinker", "-rpath=" + os.path.join(CUDA_HOME, "lib64")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

"""Builds libns_b200.so (all CUDA sources, sm_100a) in-tree: 3dnssolver_b200/lib/.

    python -m 3dnssolver_b200.build   (or importlib; __graft_entry__.build() calls build())
"""
import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libns_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                     "--expt-relaxed-constexpr", "-I", INCLUDE]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


DRIVER_SRC = os.path.join(HERE, "driver", "ns_driver.cpp")
DRIVER = os.path.join(LIBDIR, "ns_b200_driver")


def _digest():
    h = hashlib.sha256()
    for f in sorted(os.listdir(CSRC)) + [os.path.join(INCLUDE, "ns_b200.h"), DRIVER_SRC]:
        p = f if os.path.isabs(f) else os.path.join(CSRC, f)
        with open(p, "rb") as fh:
            h.update(p.encode() + fh.read())
    h.update(" ".join(NVCC_FLAGS).encode())
    return h.hexdigest()


def build(force=False, verbose=False):
    os.makedirs(LIBDIR, exist_ok=True)
    stamp = os.path.join(LIBDIR, ".digest")
    dig = _digest()
    if (not force and os.path.exists(LIB) and os.path.exists(DRIVER) and os.path.exists(stamp)
            and open(stamp).read() == dig):
        return LIB
    objdir = os.path.join(LIBDIR, "_obj")
    os.makedirs(objdir, exist_ok=True)
    cc = nvcc()

    def compile_one(src):
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [cc] + NVCC_FLAGS + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr:
            sys.stderr.write(r.stderr)
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(compile_one, sources()))
    tmp = LIB + ".tmp"
    r = subprocess.run([cc] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart_static", "-lrt", "-ldl",
                                                                       "-lpthread"],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    build_driver()
    with open(stamp, "w") as fh:
        fh.write(dig)
    return LIB


def build_driver():
    """The input.xml-driven executable (the reference's main/Driver) over the C ABI."""
    cxx = next((c for c in ("/usr/bin/g++", shutil.which("g++")) if c and os.path.exists(c)), None)
    if cxx is None:
        raise RuntimeError("g++ not found")
    cmd = [cxx, "-O2", "-std=c++17", "-Wall", "-I", INCLUDE, DRIVER_SRC, "-L", LIBDIR, "-lns_b200",
           "-Wl,-rpath,$ORIGIN", "-o", DRIVER]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"driver build failed:\n{r.stdout}\n{r.stderr}")
    return DRIVER


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

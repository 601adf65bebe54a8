"""Build libhosono_gpu.so in-tree for sm_100a (nvcc; no GPU needed).

kernels.cu is compiled twice: strict (--fmad=false, every FP64 operation
rounded on its own; bit-identical to the oracle) and fast (--fmad=true).
The CUDA runtime is linked statically so the library does not depend on
which libcudart another module of the process loaded.
"""
import concurrent.futures
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libhosono_gpu.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", INCLUDE, "-I", CSRC,
               "--expt-relaxed-constexpr"] + ARCH


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_cxx():
    # the environment may point CXX at a g++ build without libquadmath
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _sources():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def jobs(verbose=False):
    nv = nvcc()
    ccbin = ["-ccbin", host_cxx()]
    hdrs = [p for p in _sources() if p.endswith((".h", ".cuh"))] + [os.path.join(INCLUDE, "hosono_gpu.h")]
    out = []
    k = os.path.join(CSRC, "kernels.cu")
    out.append((os.path.join(BUILD, "kernels_strict.o"), [k] + hdrs,
                [nv, "-c", k, "-DHOSONO_FAST=0", "--fmad=false", "-Xptxas", "-v" if verbose else "-O3"] + ccbin
                + NVCC_COMMON + ["-o", os.path.join(BUILD, "kernels_strict.o")]))
    out.append((os.path.join(BUILD, "kernels_fast.o"), [k] + hdrs,
                [nv, "-c", k, "-DHOSONO_FAST=1", "--fmad=true", "-Xptxas", "-v" if verbose else "-O3"] + ccbin
                + NVCC_COMMON + ["-o", os.path.join(BUILD, "kernels_fast.o")]))
    for name in ("hosono_gpu.cu", "engine.cu", "layout.cu", "noalloc.cu", "server.cu", "diagnostics.cu", "ic.cu"):
        src = os.path.join(CSRC, name)
        obj = os.path.join(BUILD, name.replace(".cu", ".o"))
        out.append((obj, [src] + hdrs, [nv, "-c", src, "--fmad=false"] + ccbin + NVCC_COMMON + ["-o", obj]))
    for name in ("gp_setup.cpp", "setup.cpp"):
        src = os.path.join(CSRC, name)
        obj = os.path.join(BUILD, name.replace(".cpp", ".o"))
        out.append((obj, [src] + hdrs,
                    [host_cxx(), "-c", src, "-std=gnu++17", "-O2", "-fPIC", "-ffp-contract=off", "-I", INCLUDE,
                     "-o", obj]))
    return out


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    todo = [j for j in jobs(verbose) if force or _newer(j[0], j[1])]

    def run(job):
        r = subprocess.run(job[2], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("build failed:\n" + " ".join(job[2]) + "\n" + r.stdout + r.stderr)
        return r.stdout + r.stderr

    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for log in ex.map(run, todo):
            if verbose and log:
                sys.stderr.write(log)
    objs = [j[0] for j in jobs()]
    if force or todo or _newer(LIB, objs):
        cmd = [nvcc(), "-shared", "-ccbin", host_cxx()] + ARCH + objs + ["-o", LIB, "-lquadmath", "-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))

"""Builds libgsplat_ffi_c.so (the CUDA SortedAlpha renderer) in-tree.

    python gsplat-rs_b200/build.py [--force] [-j N] [--out LIB] [-D NAME=VALUE ...]

CUDA sources are compiled for sm_100a only. The two kernels whose results
must match the CPU restatement bit for bit (preprocess, raster) are built
with --fmad=false; host C++ is built with -ffp-contract=off for the same
reason (the reference's f32 arithmetic rounds after every operation).
Output: gsplat-rs_b200/lib/libgsplat_ffi_c.so, or --out (objects then go to a
build folder beside it, so variants with other -D tuning values do not mix).
"""

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libgsplat_ffi_c.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler",
              "-ffp-contract=off", "-I", CSRC, "-I", INCLUDE] + ARCH
EXACT_FP = {"k_preprocess.cu", "k_raster.cu", "ply_device.cu"}
CXX = os.environ.get("CXX", "g++")
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra",
             "-Wno-unused-parameter", "-I", CSRC, "-I", INCLUDE,
             "-I", os.path.join(CUDA_HOME, "include")]


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return max(os.path.getmtime(h) for h in hs)


def compile_one(src, force, hdr_mtime, extra, build_dir, defines):
    path = os.path.join(CSRC, src)
    obj = os.path.join(build_dir, src + ".o")
    if (not force and os.path.exists(obj)
            and os.path.getmtime(obj) >= max(os.path.getmtime(path), hdr_mtime)):
        return obj, None
    dflags = ["-D" + d for d in defines]
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + dflags + extra + (["--fmad=false"] if src in EXACT_FP else []) + [
            "-c", path, "-o", obj]
    else:
        cmd = [CXX] + CXX_FLAGS + dflags + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    return obj, (r.stderr.strip() or None) and ("warnings:\n" + r.stderr if "warning" in r.stderr else None)


def build(force=False, jobs=8, verbose_ptxas=False, out=None, defines=()):
    lib = os.path.abspath(out) if out else LIB
    build_dir = BUILD if not out else os.path.splitext(lib)[0] + "_build"
    os.makedirs(build_dir, exist_ok=True)
    os.makedirs(os.path.dirname(lib), exist_ok=True)
    hdr = headers_mtime()
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    objs, errors, notes = [], [], []
    with concurrent.futures.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(compile_one, s, force, hdr, extra, build_dir, list(defines))
                for s in sources()]
        for f in futs:
            obj, msg = f.result()
            objs.append(obj)
            if msg and msg.startswith("warnings:"):
                notes.append(msg)
            elif msg:
                errors.append(msg)
    if errors:
        raise RuntimeError("compile failed:\n" + "\n\n".join(errors))
    for n in notes:
        print(n, file=sys.stderr)
    if force or not os.path.exists(lib) or any(os.path.getmtime(o) > os.path.getmtime(lib) for o in objs):
        tmp = lib + ".tmp"
        cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        shutil.move(tmp, lib)
    return lib


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("--ptxas-v", action="store_true", help="print register/smem usage")
    ap.add_argument("--out", help="library path (default gsplat-rs_b200/lib/libgsplat_ffi_c.so)")
    ap.add_argument("-D", dest="defines", action="append", default=[],
                    help="NAME=VALUE tuning define passed to every compile")
    a = ap.parse_args()
    print(build(a.force or a.ptxas_v, a.j, a.ptxas_v, a.out, a.defines))


if __name__ == "__main__":
    main()

"""Build libfhb200.so (sm_100a) in-tree with nvcc.

    python -m fhelium_b200.csrc.build [--verbose]

Objects are compiled in parallel and linked into fhelium_b200/lib/libfhb200.so.
The build is skipped when the library is newer than every source.
"""

from __future__ import annotations

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
LIB_DIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIB_DIR, "libfhb200.so")
# (source, object name, extra defines): the cluster kernels are instantiated
# once per ring degree so that nvcc can compile them in parallel.
SOURCES = [("fhb_context.cu", "fhb_context.o", []), ("fhb_capi.cu", "fhb_capi.o", []), ("fhb_ops.cu", "fhb_ops.o", []),
           ("fhb_noalloc.cu", "fhb_noalloc.o", []), ("fhb_tc_ntt.cu", "fhb_tc_ntt.o", []), ("fhb_tc_basis.cu", "fhb_tc_basis.o", []),
           ("fhb_items.cu", "fhb_items.o", [])] + [
    ("fhb_inst_logn.cu", f"fhb_inst_logn{k}.o", [f"-DFHB_LOGN={k}"]) for k in range(12, 18)]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; set NVCC")
    return cand


def _deps() -> list[str]:
    files = [os.path.join(HERE, f) for f in os.listdir(HERE) if f.endswith((".cu", ".cuh", ".h"))]
    files.append(os.path.join(ROOT, "include", "fhb200.h"))
    return files


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _deps())


def build(verbose: bool = False, force: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    nvcc = _nvcc()
    obj_dir = os.path.join(PKG, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                    "-I", os.path.join(ROOT, "include")]
    if verbose:
        flags += ["-Xptxas", "-v"]

    def compile_one(item) -> str:
        src, obj_name, defines = item
        obj = os.path.join(obj_dir, obj_name)
        cmd = [nvcc, *flags, *defines, "-c", os.path.join(HERE, src), "-o", obj]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{res.stderr[-6000:]}")
        if verbose:
            sys.stderr.write(res.stderr)
        return obj

    with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as pool:
        objs = list(pool.map(compile_one, SOURCES))
    tmp = LIB + f".{os.getpid()}.tmp"
    subprocess.run([nvcc, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs], check=True)
    os.replace(tmp, LIB)
    return LIB


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    print(build(verbose=args.verbose, force=args.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())

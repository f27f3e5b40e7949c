"""In-tree build of the engine's shared library for sm_100a.

``python -m bine_trees_fugaku_b200.build`` (or ``build()``) compiles the
engine's sources with nvcc into lib/libbine_b200.so next to this file, so the
library travels with the source tree.  ``--mpicxx mpicxx`` (or
``--mpi-include DIR [--mpi-lib-dir DIR]``) also builds the PMPI layer,
lib/libbine_mpi.so, against that MPI (build_mpi).
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libbine_b200.so")

SOURCES = ["bine_capi.cu", "bine_plan.cc", "bine_mlp.cu", "bine_fuse.cc"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale():
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    for d in (CSRC, os.path.join(HERE, "..", "include")):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".cc", ".h")) and os.path.getmtime(os.path.join(d, f)) > t:
                return True
    return False


def build(force=False, verbose=False):
    """Compiles lib/libbine_b200.so if it is missing or older than its sources."""
    if not force and not _stale():
        return LIB_PATH
    os.makedirs(LIB_DIR, exist_ok=True)
    tmp = LIB_PATH + ".tmp"
    cmd = [nvcc_path(), *NVCC_FLAGS, "-o", tmp] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd))
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{p.stdout}\n{p.stderr}")
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


MPI_LIB_PATH = os.path.join(LIB_DIR, "libbine_mpi.so")


def build_mpi(mpicxx=None, include=None, lib_dir=None, libs=("mpi",), verbose=False):
    """Compiles the PMPI layer (csrc/bine_mpi.cc) against an MPI
    installation into lib/libbine_mpi.so, either with the MPI's compiler
    wrapper (`mpicxx`) or with its include directory and libraries.  Link
    an MPI program with -lbine_mpi ahead of the MPI library (or preload it)
    and its MPI_Allreduce ... MPI_Reduce run on the GPU.  This image has no
    MPI: the tests build the layer against the oracle's MPI shim instead
    (make -C oracle dropin)."""
    build()
    cuda = os.path.dirname(os.path.dirname(nvcc_path()))
    cxx = [mpicxx] if mpicxx else ["g++"] + ([f"-I{include}"] if include else [])
    cmd = cxx + ["-std=c++17", "-O2", "-fPIC", "-shared", f"-I{cuda}/include", "-o", MPI_LIB_PATH,
                 os.path.join(CSRC, "bine_mpi.cc"), f"-L{LIB_DIR}", "-lbine_b200", f"-L{cuda}/lib64", "-lcudart",
                 "-lrt", "-Wl,-rpath,$ORIGIN", f"-Wl,-rpath,{cuda}/lib64"]
    if not mpicxx:
        cmd += ([f"-L{lib_dir}"] if lib_dir else []) + [f"-l{n}" for n in libs]
    if verbose:
        print(" ".join(cmd))
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"building the PMPI layer failed:\n{p.stdout}\n{p.stderr}")
    return MPI_LIB_PATH


if __name__ == "__main__":
    args = sys.argv[1:]
    if "--mpicxx" in args or "--mpi-include" in args:
        def opt(k):
            return args[args.index(k) + 1] if k in args else None
        print(build_mpi(mpicxx=opt("--mpicxx"), include=opt("--mpi-include"), lib_dir=opt("--mpi-lib-dir"),
                        verbose=True))
    else:
        print(build(force="--force" in args, verbose=True))

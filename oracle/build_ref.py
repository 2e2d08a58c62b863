"""ORACLE recipe: build the reference's ERI kernels for the CPU into oracle/_ref/.

Runs only where the reference checkout exists; its path is an argument
(``build(ref_root)``, or the first command-line argument, or ``REF_ROOT``):
there is no default location.  It imports the reference's kernel-source modules
(ccsd_gpu/cuda/int2e_ip1_module.py, ccsd_gpu/cuda/int2e_module.py) with a
stand-in for ``cupy`` (only ``_build_cuda_source`` and the Rys data loader are
called, no CuPy object is touched), writes the generated kernel source to
oracle/_ref/*.inc and compiles oracle/ref_eri_shim.cpp against it with g++ and
OpenMP into oracle/_ref/libref_eri.so, and oracle/ref_eri_gpu.cu with nvcc for
sm_100a into oracle/_ref/libref_eri_gpu.so (the reference's kernels on the
GPU, as a comparator).  Nothing here is copied into the
repository: oracle/_ref/ is git-ignored and only travels with the working
tree.
"""
import importlib.util
import os
import subprocess
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def generate_sources(ref_root):
    cuda_dir = os.path.join(ref_root, "ccsd_gpu", "cuda")
    saved = {k: sys.modules.get(k) for k in ("cupy", "ccsd_gpu", "ccsd_gpu.cuda")}
    sys.modules["cupy"] = types.ModuleType("cupy")
    pkg = types.ModuleType("ccsd_gpu")
    pkg.__path__ = []
    sub = types.ModuleType("ccsd_gpu.cuda")
    sub.__path__ = []
    sys.modules["ccsd_gpu"] = pkg
    sys.modules["ccsd_gpu.cuda"] = sub
    try:
        ip1 = _load("ccsd_gpu.cuda.int2e_ip1_module", os.path.join(cuda_dir, "int2e_ip1_module.py"))
        eri = _load("ccsd_gpu.cuda.int2e_module", os.path.join(cuda_dir, "int2e_module.py"))
        data = ip1._load_or_extract_rys_data()
        return eri._build_cuda_source(data), ip1._build_cuda_source(data)
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
        for k in ("ccsd_gpu.cuda.int2e_ip1_module", "ccsd_gpu.cuda.int2e_module"):
            sys.modules.pop(k, None)


def build(ref_root=None, verbose=False):
    """Build oracle/_ref/libref_eri.so from the checkout at ``ref_root``
    (``REF_ROOT`` if None).  Returns None when no checkout is given or it has
    no ccsd_gpu/cuda directory (the prebuilt library, if any, is kept)."""
    ref_root = ref_root or os.environ.get("REF_ROOT")
    if not ref_root or not os.path.isdir(os.path.join(ref_root, "ccsd_gpu", "cuda")):
        return None
    os.makedirs(OUT, exist_ok=True)
    src_eri, src_ip1 = generate_sources(ref_root)
    with open(os.path.join(OUT, "int2e_src.inc"), "w") as f:
        f.write(src_eri)
    with open(os.path.join(OUT, "int2e_ip1_src.inc"), "w") as f:
        f.write(src_ip1)
    so = os.path.join(OUT, "libref_eri.so")
    cmd = ["g++", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=c++17", "-w",
           "-I", OUT, os.path.join(HERE, "ref_eri_shim.cpp"), "-o", so]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    build_gpu(verbose=verbose)
    return so


def build_gpu(verbose=False):
    """Build oracle/_ref/libref_eri_gpu.so (oracle/ref_eri_gpu.cu: the
    reference's kernels for sm_100a behind a launcher of the reference's launch
    loop) from the kernel sources already generated into oracle/_ref/.
    Returns None when the sources or nvcc are missing."""
    import shutil
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not (os.path.exists(os.path.join(OUT, "int2e_src.inc")) and os.path.exists(nvcc)):
        return None
    so = os.path.join(OUT, "libref_eri_gpu.so")
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
           "-shared", "-w", "-I", OUT, os.path.join(HERE, "ref_eri_gpu.cu"), "-o", so]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return so


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REF_ROOT")
    if not root:
        sys.exit("usage: python oracle/build_ref.py <reference checkout>   (or set REF_ROOT)")
    print(build(root, verbose=True))

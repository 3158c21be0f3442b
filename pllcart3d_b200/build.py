"""Build recipe for the in-tree native libraries (sm_100a only).

* ``libpllgpu.so``          - CUDA kernels + runtime + the ``pllgpu_`` C ABI;
  the exact FP64 form is compiled with ``--fmad=false`` so that no
  multiply-add is contracted (the reference's own arithmetic has none), the
  FP64 form and the precision form's FP32 kernels with contraction;
* ``libpllnn.so``            - the learned surrogate's BF16 tensor-core kernels
  (tcgen05 and mma.sync convolutions, pooling, upsampling, Adam);
* ``libpllcart3d_dropin.so`` - the reference-signature drop-in layer (plain C,
  compiled with gcc because the reference's structures name a member ``new``).

Run ``python -m pllcart3d_b200.build`` or call :func:`build`.
"""

from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libpllgpu.so")
NNLIB = os.path.join(HERE, "libpllnn.so")
DROPIN = os.path.join(HERE, "libpllcart3d_dropin.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xptxas", "-warn-spills"]

# per-source contraction: the exact FP64 form (form_f64x.cu) and everything
# the drop-in layer's primitives run reproduce the reference's operation
# order, so no multiply-add is contracted there; the FP64 forms (form_f64.cu,
# form_f64m.cu) are free to contract.  The precision form's FP32 kernels
# (form_f32.cu) fuse only where the source asks (fma, the paired FP32x2
# intrinsics): a contraction the compiler chooses may differ between a
# kernel and its member-batched copy, whose results must be the same bits.
CU_SOURCES = {"runtime.cu": "--fmad=false", "form_f64.cu": "--fmad=true", "form_f64x.cu": "--fmad=false",
              "form_f64m.cu": "--fmad=true",
              "form_f32.cu": "--fmad=false", "primitives.cu": "--fmad=false",
              "noalloc.cu": "--fmad=false", "io.cu": "--fmad=false",
              "wave.cu": "--fmad=false", "ensemble.cu": "--fmad=false"}
HEADERS = ["common.cuh", "step_kernels.cuh", "aux_kernels.cuh", "dct_kernels.cuh", "host_util.h",
           "ctx.cuh", "host_common.cuh", "orchestrate.cuh", "forms.h", "umma_dct.cuh", "fft_dct.cuh", "explicit_tma.cuh",
           "batch.cuh"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise FileNotFoundError("nvcc not found")
    return cand


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    deps = [os.path.join(CSRC, f) for f in [*CU_SOURCES, *HEADERS]]
    deps.append(os.path.join(INC, "pllcart3d_gpu.h"))
    deps.append(__file__)
    if force or _stale(LIB, deps):
        # the translation units compile in parallel (the form units dominate)
        cmds, objs = [], []
        for src, fmad in CU_SOURCES.items():
            obj = os.path.join(CSRC, src.replace(".cu", ".o"))
            cmds.append([_nvcc(), *ARCH, *NVCC_FLAGS, *fmad.split(), "-I", INC, "-c", os.path.join(CSRC, src), "-o", obj])
            objs.append(obj)
        if verbose:
            for cmd in cmds:
                print(" ".join(cmd))
        workers = max(1, min(len(cmds), os.cpu_count() or 1))
        with concurrent.futures.ThreadPoolExecutor(workers) as ex:
            for r in list(ex.map(lambda c: subprocess.run(c), cmds)):
                if r.returncode != 0:
                    raise subprocess.CalledProcessError(r.returncode, r.args)
        cmd = [_nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
        subprocess.run(cmd, check=True)
        for o in objs:
            os.remove(o)
    nsrc = os.path.join(CSRC, "nn.cu")
    if os.path.exists(nsrc) and (force or _stale(NNLIB, [nsrc, os.path.join(CSRC, "nn_umma.cuh"), __file__])):
        cmd = [_nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas",
               "-warn-spills", "-shared", "-cudart", "static", nsrc, "-o", NNLIB]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    dsrc = os.path.join(CSRC, "dropin.c")
    if os.path.exists(dsrc) and (force or _stale(DROPIN, [dsrc, LIB, os.path.join(INC, "pllcart3d_gpu.h")])):
        cmd = ["gcc", "-O2", "-fPIC", "-shared", "-std=gnu99", "-Wall", "-I", INC,
               dsrc, "-o", DROPIN, f"-L{HERE}", "-lpllgpu",
               "-Wl,-rpath,$ORIGIN"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)

"""In-tree build of the CUDA library (sm_100a), the drop-in shims and the CPU checker.

Outputs (git-ignored, shipped with the tree):
  imaging2d_wlsq_b200/libimaging2d_wlsq_b200.so     CUDA kernels + C ABI
  imaging2d_wlsq_b200/dropin/*.so                    reference-named drop-in shims
  oracle/liboracle.so                                CPU restatement (test checker only)
  oracle/_ref/extrapolation_cpu.so                   the reference's own CPU library (when its
                                                     sources are present on this machine)
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
# read-only mount of the reference sources on the build machine (oracle/_ref recipe input)
REFERENCE_TREE = "/root/reference"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
LIB = os.path.join(PKG, "libimaging2d_wlsq_b200.so")
SOURCES = [os.path.join(PKG, "csrc", "wlsq_capi.cu")]
HEADERS = [os.path.join(PKG, "csrc", "wlsq_kernels.cuh"), os.path.join(ROOT, "include", "imaging2d_wlsq_b200.h")]
DROPINS = {
    "extrapolation_cpu.so": ["-DIMG2D_DROPIN_HOST"],
    "extrapolation_gpu.so": ["-DIMG2D_DROPIN_DEVICE=0"],
    "extrapolation_revOp_gpu.so": ["-DIMG2D_DROPIN_DEVICE=1"],
    "extrapolation_sh_revOp_gpu.so": ["-DIMG2D_DROPIN_DEVICE=1"],
}


def _run(cmd):
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_cuda(force=False, verbose_ptxas=False):
    if force or _stale(LIB, SOURCES + HEADERS):
        cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
               "-o", LIB, *SOURCES, "-lcufft"]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
        _run(cmd)
    src = os.path.join(PKG, "csrc", "dropin.c")
    os.makedirs(os.path.join(PKG, "dropin"), exist_ok=True)
    for name, defs in DROPINS.items():
        out = os.path.join(PKG, "dropin", name)
        if force or _stale(out, [src, LIB]):
            _run(["gcc", "-O2", "-shared", "-fPIC", *defs, "-o", out, src, "-L" + PKG, "-limaging2d_wlsq_b200",
                  "-Wl,-rpath,$ORIGIN/.."])


def build_oracle(force=False):
    src = os.path.join(ROOT, "oracle", "wlsq_oracle.c")
    out = os.path.join(ROOT, "oracle", "liboracle.so")
    if force or _stale(out, [src]):
        _run(["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-shared", "-fPIC", "-o", out, src, "-lm"])
    ref = os.path.join(ROOT, "oracle", "build_ref.sh")
    ref_out = os.path.join(ROOT, "oracle", "_ref", "extrapolation_cpu.so")
    if force or not os.path.exists(ref_out):
        # the reference sources, where the build machine mounts them (absent on machines that
        # only run the prebuilt files; the recipe then skips)
        env = dict(os.environ)
        env.setdefault("IMG2D_REFERENCE", REFERENCE_TREE)
        print("+ bash", ref, flush=True)
        subprocess.run(["bash", ref], check=True, env=env)


def build_all(force=False):
    build_cuda(force=force)
    build_oracle(force=force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)

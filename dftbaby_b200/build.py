"""In-tree build of the CUDA library (sm_100a) and of the CPU oracle."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "lib", "libdftbaby_b200.so")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]


def _nvcc():
    for cand in (os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc"), "nvcc"):
        if os.path.sep not in cand or os.path.exists(cand):
            return cand
    return "nvcc"


def build_native(force=False, verbose=False):
    """Compile csrc/*.cu into lib/libdftbaby_b200.so when sources are newer."""
    csrc = os.path.join(HERE, "csrc")
    srcs = [os.path.join(csrc, f) for f in os.listdir(csrc) if f.endswith(".cu")]
    deps = [os.path.join(csrc, f) for f in os.listdir(csrc) if f.endswith(".cuh")]
    hdr = os.path.join(ROOT, "include", "dftbaby_b200.h")
    if not force and os.path.exists(LIB):
        newest = max(os.path.getmtime(p) for p in srcs + deps + [hdr])
        if os.path.getmtime(LIB) >= newest:
            return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    cmd = [_nvcc()] + NVCC_FLAGS + ["-I" + os.path.join(ROOT, "include"), "-o", LIB] + sorted(srcs) + ["-ldl"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return LIB


def build_oracle():
    """Build oracle/lib/liboracle.so (CPU restatement used by tests and the CPU baseline)."""
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])


if __name__ == "__main__":
    print(build_native(force=True, verbose=True))
    build_oracle()

"""Build of the engine's native library (libpwa_b200.so) with nvcc.

The device headers are embedded into the library as text (they are compiled
at plan-creation time by NVRTC together with the generated model code), the
host runtime is compiled for sm_100a, linked against NVRTC and the static
CUDA runtime so that the library loads on machines without a GPU driver."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libpwa_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_LIB = "/usr/local/cuda/lib64"


def _embed():
    out = ["// generated by build_ext.py from the device headers; do not edit"]
    for var, fn in (("kDeviceHeader", "pwa_device.cuh"), ("kKernelsHeader", "pwa_kernels.cuh")):
        txt = open(os.path.join(CSRC, fn)).read()
        # raw string literals are limited in length by some compilers: split
        chunks = [txt[i:i + 8000] for i in range(0, len(txt), 8000)]
        body = "\n".join(f'R"PWA({c})PWA"' for c in chunks)
        out.append(f"static const char {var}[] =\n{body};")
    path = os.path.join(CSRC, "_embedded.inc")
    new = "\n".join(out) + "\n"
    if not os.path.exists(path) or open(path).read() != new:
        with open(path, "w") as f:
            f.write(new)


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    srcs = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(HERE, "..", "include", "pwa_b200.h"), __file__]
    return any(os.path.getmtime(s) > t for s in srcs if os.path.exists(s))


def build(force=False, verbose=False):
    _embed()
    if not force and not _stale():
        return LIB
    cmd = [NVCC, "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
           os.path.join(CSRC, "pwa_runtime.cu"), os.path.join(CSRC, "pwa_hostprog.cpp"),
           "-Xcompiler", "-ffp-contract=off", "-o", LIB + ".tmp",
           "-L" + CUDA_LIB, "-lnvrtc", "-Xlinker", "-rpath," + CUDA_LIB,
           "-cudart", "static"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)

"""Build the CUDA extension in-tree: ``labinius_b200/liblabinius_gpu.so`` for sm_100a.

One nvcc invocation over the C ABI (api.cu), the kernels (kernels.cu) and the host tables,
BLAKE3 and transcript (.cpp). The library exports only the C ABI of include/labinius_gpu.h.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "liblabinius_gpu.so")
SOURCES = ["api.cu", "kernels.cu", "fold_static.cu", "batch.cu", "transcript_dev.cu", "ntt_api.cu", "switch.cu", "wire.cu", "wire_pack.cu", "ring_tables.cpp", "blake3_host.cpp", "transcript.cpp"]
HEADERS = ["kernels.cuh", "tcgen05.cuh", "gf2_dev.cuh", "prime_structs.h", "hasher_state.h", "blake3_dev.cuh", "transcript_dev.h", "switch.h", "upload.h", "error.h", "handles.h", "launch.h", "ring_tables.h", "blake3_host.h", "transcript.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def deps():
    return sources() + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "labinius_gpu.h")]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    return os.path.getmtime(LIB) >= max(os.path.getmtime(p) for p in deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-fvisibility=hidden",
           "-I", INCLUDE, "-o", LIB + ".tmp", *sources()]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    import sys
    print(build(force=True, verbose="-v" in sys.argv))

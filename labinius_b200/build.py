"""Build the CUDA extension in-tree: ``labinius_b200/liblabinius_gpu.so`` for sm_100a.

One nvcc invocation per source (the C ABI, the kernels, the host tables, BLAKE3 and transcript),
run in parallel, then one link. The library exports only the C ABI of include/labinius_gpu.h.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "liblabinius_gpu.so")
SOURCES = ["api.cu", "kernels.cu", "fold_static.cu", "batch.cu", "transcript_dev.cu", "ntt_api.cu", "switch.cu", "wire.cu", "wire_pack.cu", "ring_tables.cpp", "blake3_host.cpp", "transcript.cpp"]
HEADERS = ["kernels.cuh", "copy_pool.h", "tcgen05.cuh", "gf2_dev.cuh", "prime_structs.h", "hasher_state.h", "blake3_dev.cuh", "transcript_dev.h", "switch.h", "upload.h", "error.h", "handles.h", "launch.h", "ring_tables.h", "blake3_host.h", "transcript.h"]
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
    """Compile every source to an object (in parallel, one nvcc per source) under _build/, then link
    the shared library."""
    if not force and up_to_date():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    flags = [*ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
             "-Xcompiler", "-fvisibility=hidden", "-I", INCLUDE]
    if verbose:
        flags.insert(0, "-Xptxas=-v")

    def compile_one(src):
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        subprocess.check_call([nvcc(), *flags, "-c", "-o", obj, src])
        return obj

    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 4)) as ex:
        objs = list(ex.map(compile_one, sources()))
    subprocess.check_call([nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lpthread"])
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    import sys
    print(build(force=True, verbose="-v" in sys.argv))

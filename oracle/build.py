"""Build recipe for the CPU oracle (test infrastructure): one g++ call, output ``oracle/liboracle.so``.

``-ffp-contract=off`` keeps the challenge sampler's f64 norm test free of fused multiply-adds,
matching the reference's separate multiply and add (crates/pcs/src/challenge.rs:382-387).
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
SOURCES = [os.path.join(HERE, "oracle.cpp")]
DEPS = SOURCES + [os.path.join(HERE, "blake3_oracle.h")]


def build(force: bool = False) -> str:
    if not force and os.path.exists(LIB):
        newest = max(os.path.getmtime(p) for p in DEPS)
        if os.path.getmtime(LIB) >= newest:
            return LIB
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-pthread",
           "-Wall", "-Wno-unused-function", *SOURCES, "-o", LIB + ".tmp"]
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True))

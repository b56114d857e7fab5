#!/usr/bin/env python3
"""Build the CPU restatement oracle (test infrastructure) into oracle/_build/liboracle_port.so.

Needs only g++; runs here and on any GPU host (no reference tree needed)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "port", "oracle_port.cpp")
OUT = os.path.join(HERE, "_build", "liboracle_port.so")


def build(force=False):
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) > max(os.path.getmtime(SRC), os.path.getmtime(__file__)):
        return OUT
    r = subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", SRC, "-o", OUT],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle port build failed:\n" + r.stdout + r.stderr)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
    sys.exit(0)

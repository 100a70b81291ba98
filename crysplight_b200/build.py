"""Build the in-tree sm_100a CUDA library (and, for tests, the CPU oracle).

``build()`` compiles ``crysplight_b200/lib/libcrysplight_cuda.so`` with nvcc
for ``sm_100a`` (cross-compiles without a GPU).
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)


def _make(dirpath: str, env=None) -> None:
    r = subprocess.run(["make", "-C", dirpath], capture_output=True, text=True, env=env)
    sys.stdout.write(r.stdout)
    if r.returncode != 0:
        sys.stderr.write(r.stderr)
        raise RuntimeError(f"build failed in {dirpath}")


def build_cuda() -> str:
    _make(os.path.join(PKG, "csrc"))
    return os.path.join(PKG, "lib", "libcrysplight_cuda.so")


def build() -> str:
    return build_cuda()


if __name__ == "__main__":
    print(build())

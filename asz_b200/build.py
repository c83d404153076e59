"""Build steps for the in-tree CUDA library and CLI front ends (make -C asz_b200/csrc)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8) -> None:
    """Compile libasz_b200.so and bin/s1_{compress,decompress} for sm_100a."""
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", os.path.join(HERE, "csrc")], check=True)

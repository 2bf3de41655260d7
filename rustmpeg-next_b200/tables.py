"""Read the normative tables of csrc/vvc_tables.h into numpy (host-side use:
synthetic APS generation and tests)."""
from __future__ import annotations

import functools
import os
import re

import numpy as np

_HDR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "vvc_tables.h")


@functools.lru_cache(maxsize=None)
def table(name: str) -> np.ndarray:
    src = open(_HDR).read()
    m = re.search(r"\b" + re.escape(name) + r"\s*\[[^\]]*\]\s*=\s*\{(.*?)\};", src, re.S)
    if not m:
        raise KeyError(name)
    return np.array([int(v) for v in re.findall(r"-?\d+", m.group(1))], dtype=np.int32)


def alf_fixed_coeff() -> np.ndarray:
    return table("kAlfFixedCoeff").reshape(64, 13)


def dct2(n: int) -> np.ndarray:
    return table(f"kDct2N{n}").reshape(n, n)

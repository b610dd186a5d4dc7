"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device and call the
library through its C-ABI; everything else runs on the CPU.  GPU tests never
skip for a missing library or device: they fail, so a silent fallback cannot
pass."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libfullermd_cuda.so")


@pytest.fixture(scope="session")
def golden():
    cache = {}

    def load(name: str):
        if name not in cache:
            with np.load(GOLDEN / f"{name}.npz") as z:
                cache[name] = {k: z[k] for k in z.files}
        return cache[name]

    return load


@pytest.fixture(scope="session")
def oracle():
    from oracle.fmd_oracle import Oracle, ORACLE_SO
    if not ORACLE_SO.exists():
        import subprocess
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "oracle"], check=True, capture_output=True)
    return Oracle()


@pytest.fixture(scope="session")
def ctx():
    """A context on cuda:0.  Raises (never skips) if the library or device is missing."""
    from fuller_md_en_b200 import Context
    c = Context(0)
    yield c
    c.close()


def rows(cnt, lst, cap):
    """Reference list rows as a list of arrays (entries past cnt ignored)."""
    return [np.asarray(lst[k * cap:k * cap + cnt[k]]) for k in range(len(cnt))]


def csr_rows(cnt, csr):
    out, o = [], 0
    for c in cnt:
        out.append(np.asarray(csr[o:o + c]))
        o += c
    return out


def same_rows(a, b) -> bool:
    return len(a) == len(b) and all(np.array_equal(x, y) for x, y in zip(a, b))


def rel(a, b, floor=1e-30):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), floor))

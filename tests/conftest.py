"""Shared test setup: import paths, the `gpu` marker, and in-tree builds.

GPU parity tests call the product through the C ABI (cuda_b200.api, a ctypes
binding of liblucasntt.so) and check it against the CPU oracle (oracle/).
"""
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on a B200)")


def _make(target_dir: Path, artefact: str) -> None:
    if not (target_dir / artefact).exists():
        subprocess.run(["make", "-C", str(target_dir), "-j8"], check=True,
                       stdout=subprocess.DEVNULL)


_make(ROOT / "oracle", "liblntoracle.so")
_make(ROOT / "cuda_b200", "liblucasntt.so")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    return oracle


@pytest.fixture(scope="session")
def lnt():
    import cuda_b200
    return cuda_b200

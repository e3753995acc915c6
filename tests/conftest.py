"""Shared test set-up: import paths, the `gpu` marker, common fixtures."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT / "strata-k_b200", ROOT / "oracle", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def engine():
    """One engine context for the GPU tests (the CUDA library must be built)."""
    from strata_b200 import Engine
    eng = Engine(0)
    yield eng
    eng.close()


class Lcg:
    """The reference tests' LCG (strata-gpu/tests/tc_diff.rs:32-44)."""

    def __init__(self, seed: int):
        self.s = seed & 0xFFFFFFFFFFFFFFFF

    def next(self) -> int:
        self.s = (self.s * 6364136223846793005 + 1442695040888963407) & 0xFFFFFFFFFFFFFFFF
        return self.s >> 33

    def upto(self, n: int) -> int:
        return self.next() % n


@pytest.fixture
def lcg():
    return Lcg


@pytest.fixture(params=[0, 1], ids=["auto", "sortmerge"])
def peng(request, engine):
    """The engine with plan 0 (automatic: direct-addressed where it applies)
    and plan 1 (sort-merge forced); both must give identical results."""
    engine.set_plan(request.param)
    yield engine
    engine.set_plan(0)


@pytest.fixture(params=[0, 1, 2], ids=["auto-bitrows", "sortmerge", "dense"])
def tceng(request, engine):
    """Bool closure under every plan that applies to it: automatic (bit rows at
    these sizes), sort-merge and direct-addressed; results must be identical."""
    engine.set_plan(request.param)
    yield engine
    engine.set_plan(0)

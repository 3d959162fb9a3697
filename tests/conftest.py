"""Shared test set-up: import paths, the `gpu` marker, native builds."""

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT / "pdf-raster_b200", ROOT / "oracle", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


@pytest.fixture(scope="session")
def oracle():
    import rr_oracle

    rr_oracle.build()
    return rr_oracle


@pytest.fixture(scope="session")
def rrb_lib():
    from rrb import build as rrb_build

    rrb_build.build()
    import rrb

    return rrb


@pytest.fixture(scope="session")
def backend(rrb_lib):
    b = rrb_lib.B200Backend(0)
    yield b
    b.close()

"""GpuBackend::record_scan (crates/gpu/src/backend/mod.rs:340-353): the three
phases of the in-place exclusive u32 scan, checked against NumPy's cumulative
sum (wrapping mod 2^32), and ScanParams::validate's invariants
(crates/gpu/src/backend/params.rs:338-372)."""

import numpy as np
import pytest

TILE = 1024  # 2 * SCAN_WORKGROUP_SIZE


def _scan(backend, values):
    n = values.size
    blocks = (n + TILE - 1) // TILE
    data = backend.alloc_device(4 * n)
    sums = backend.alloc_device(4 * max(1, blocks))
    try:
        backend.wait_transfer(backend.upload_async(data, values.view(np.uint8)))
        backend.begin_page()
        for phase in (0, 1, 2):
            backend.record_scan(data, sums, n, phase)
        backend.wait_page(backend.submit_page())
        out = np.empty(n, np.uint32)
        backend.wait_download(backend.download_async(data, out))
        return out
    finally:
        backend.free_device(data)
        backend.free_device(sums)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2, 511, 1023, 1024, 1025, 4097, 65536 + 3, TILE * 1024])
def test_exclusive_scan_matches_numpy(backend, n):
    rng = np.random.default_rng(n)
    values = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)  # sums wrap
    exp = np.zeros(n, np.uint64)
    exp[1:] = np.cumsum(values[:-1], dtype=np.uint64)  # < 2^52: exact in 64 bits
    exp = (exp & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    assert np.array_equal(_scan(backend, values), exp)


@pytest.mark.gpu
def test_scan_invariants_are_rejected(backend, rrb_lib):
    data = backend.alloc_device(4 * 4096)
    small = backend.alloc_device(4)
    big_data = backend.alloc_device(4 * (TILE * 1024 + 1))
    sums = backend.alloc_device(4 * 1025)
    try:
        backend.begin_page()
        cases = [(data, sums, 0, 0),               # len_elems must be > 0
                 (data, sums, 4097, 0),            # data smaller than len_elems * 4
                 (data, small, 4096, 0),           # block_sums smaller than 4 tiles
                 (big_data, sums, TILE * 1024 + 1, 0),  # more than SCAN_MAX_BLOCKS tiles
                 (data, sums, 4096, 3)]            # unknown phase
        for d, s, n, ph in cases:
            with pytest.raises(rrb_lib.BackendError) as e:
                backend.record_scan(d, s, n, ph)
            assert e.value.kind == "InvariantViolation", (n, ph)
        backend.wait_page(backend.submit_page())
    finally:
        for b in (data, small, big_data, sums):
            backend.free_device(b)

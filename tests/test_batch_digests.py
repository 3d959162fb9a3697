"""Whole-batch parity by pinned page digests.

The CPU oracle rendered every page of the 64-page mixed batch (generator kind
2, seed 0) and every page that serving requests 0..127 ask for (kind 2, seed
= request id, one page each); tests/golden/make_batch_digests.py wrote one
SHA-256 per page, together with a SHA-256 of the page's generated inputs.

On the CPU these tests check that the generator still produces those inputs.
On the B200 they render the whole batch once per tile shape, and every
request through the continuous-batching server, and compare every page with
the oracle's digest: bit-exact on all 64 pages and all 128 requests.
"""

import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
MIXED = GOLDEN / "mixed_batch_digests.json"
SERVING = GOLDEN / "serving_request_digests.json"


def _load(path):
    if not path.exists():
        pytest.fail(f"{path.name} is missing: run tests/golden/make_batch_digests.py")
    return json.loads(path.read_text())


def _sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _input_sha(s) -> str:
    from golden.make_batch_digests import input_digest
    return input_digest(s)


def _page_sha(arena, s, pg=0) -> str:
    o, w, h = int(s.page_offset[pg]), int(s.page_width[pg]), int(s.page_height[pg])
    return _sha(arena[o:o + w * h])


@pytest.fixture(scope="module")
def mixed_scene(rrb_lib):
    return rrb_lib.Scene(kind=2, seed=0)


def test_mixed_batch_digests_pin_the_generated_inputs(rrb_lib, mixed_scene):
    from rrb.shard import SceneShard
    doc = _load(MIXED)
    assert doc["pages"] == mixed_scene.n_pages == len(doc["records"]) == 64
    for rec in doc["records"]:
        sub = SceneShard(mixed_scene, pages=(rec["page"], rec["page"] + 1))
        assert (rec["width"], rec["height"], rec["paths"]) == (int(sub.page_width[0]), int(sub.page_height[0]),
                                                               sub.n_paths)
        assert rec["input_sha256"] == _input_sha(sub), rec["page"]
        assert rec["nonterminating_rows"] == 0


def test_serving_digests_pin_the_generated_inputs(rrb_lib):
    doc = _load(SERVING)
    assert doc["requests"] == len(doc["records"]) >= 128
    for rec in doc["records"][:: 8]:  # every 8th request: generation dominates this check
        s = rrb_lib.Scene(kind=2, seed=rec["request"], n_pages=1)
        assert rec["input_sha256"] == _input_sha(s), rec["request"]


@pytest.mark.gpu
@pytest.mark.parametrize("tile", [(64, 16), (128, 16), (128, 32), (32, 32), (16, 16)])
def test_mixed_batch_every_page_bit_exact(backend, mixed_scene, tile):
    """All 64 pages of the 1.17-Gpixel mixed batch, rendered in one submission,
    equal the oracle's pages (by digest) under each tile shape."""
    doc = _load(MIXED)
    s = mixed_scene
    pages = backend.alloc_device(s.arena_bytes)
    backend.set_tuning(*tile)
    try:
        s.view.pages = None
        batch = backend.batch_upload(s.view)
        try:
            backend.begin_page()
            backend.record_fill_buffer(pages, 255)
            batch.record(pages)
            backend.wait_page(backend.submit_page())
        finally:
            batch.free()
        got = np.empty(s.arena_bytes, np.uint8)
        backend.wait_download(backend.download_async(pages, got))
    finally:
        backend.set_tuning(64, 16, auto_tile=True)
        backend.free_device(pages)
    bad = [rec["page"] for rec in doc["records"] if _page_sha(got, s, rec["page"]) != rec["page_sha256"]]
    assert not bad, f"pages differing from the oracle: {bad}"


@pytest.mark.gpu
def test_every_serving_request_bit_exact(rrb_lib):
    """All 128 pinned requests through the continuous-batching server (two
    workers, submitted at once so they share batches): each request's page
    equals the oracle's page for its seed."""
    doc = _load(SERVING)
    recs = doc["records"]
    burst = 32  # bounds the host memory held by queued requests
    with rrb_lib.Server(workers=2, max_batch_pages=16) as srv:
        for b0 in range(0, len(recs), burst):
            # Generate a burst's scenes first, then submit them back to back:
            # generating between submits would leave the workers idle, and
            # every request would go out alone.
            group = []
            for rec in recs[b0:b0 + burst]:
                sc = rrb_lib.Scene(kind=2, seed=rec["request"], n_pages=1)
                sc.view.pages = None
                group.append((rec, sc, sc.blank_arena(0)))
            pending = [(rec, sc, out, srv.submit(sc.view, out, init=255, keep=sc)) for rec, sc, out in group]
            for rec, sc, out, t in pending:
                srv.wait(t)
                assert _page_sha(out, sc) == rec["page_sha256"], rec["request"]
        st = srv.stats()
    assert st["completed"] == len(recs) and st["batches"] < len(recs)

"""Golden fixtures (tests/golden, made by tests/golden/make_golden.py).

CPU: the seeded generator still produces the same inputs and the oracle the
same pages (guards both against drift). GPU: the B200 path reproduces every
fixture byte for byte through the C ABI.
"""

import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent / "golden"
MANIFEST = json.loads((HERE / "manifest.json").read_text())


def _scene(rrb_lib, key):
    import sys
    sys.path.insert(0, str(HERE))
    from make_golden import scene_hash
    m = MANIFEST[key]
    s = rrb_lib.Scene(**m["params"])
    assert scene_hash(s) == m["input_sha256"], "generator output changed"
    return s


SCENE_KEYS = [k for k in MANIFEST if not k.startswith("handmade")]
HAND_KEYS = [k for k in MANIFEST if k.startswith("handmade")]


@pytest.mark.parametrize("key", SCENE_KEYS)
def test_oracle_reproduces_scene_fixture(oracle, rrb_lib, key):
    s = _scene(rrb_lib, key)
    a = s.blank_arena()
    st = oracle.render_scene(s, a, rowmap=MANIFEST[key]["rowmap"])
    assert hashlib.sha256(a.tobytes()).hexdigest() == MANIFEST[key]["expected_sha256"]
    assert st == MANIFEST[key]["oracle"]


def _hand(key):
    return dict(np.load(HERE / f"{key}.npz"))


@pytest.mark.parametrize("key", HAND_KEYS)
def test_oracle_reproduces_handmade_fixture(oracle, key):
    d, m = _hand(key), MANIFEST[key]
    a = d["init"].copy()
    W, H = m["params"]["width"], m["params"]["height"]
    oracle.render_arrays(a, [0], [W], [H], d["pts"], d["flags"], d["path_pt_off"], d["fill_rule"], d["gray"],
                         d["alpha"], np.zeros(len(d["gray"]), np.uint32), rowmap=m["rowmap"])
    assert np.array_equal(a, d["expected"])


@pytest.mark.gpu
@pytest.mark.parametrize("key", SCENE_KEYS)
def test_gpu_reproduces_scene_fixture(backend, rrb_lib, key):
    s = _scene(rrb_lib, key)
    a = s.blank_arena()
    backend.render_scene(s, a, rowmap=MANIFEST[key]["rowmap"])
    assert np.array_equal(a, np.load(HERE / f"{key}.npz")["expected"])


@pytest.mark.gpu
@pytest.mark.parametrize("key", HAND_KEYS)
def test_gpu_reproduces_handmade_fixture(backend, rrb_lib, key):
    d, m = _hand(key), MANIFEST[key]
    W, H = m["params"]["width"], m["params"]["height"]
    keep = []
    n = len(d["gray"])
    buf = backend.alloc_device(W * H)
    try:
        p = rrb_lib.batch_params(d["pts"], d["flags"], d["path_pt_off"], d["fill_rule"], d["gray"], d["alpha"],
                                 np.zeros(n, np.uint32), [W], [H], [0], buf, rowmap=m["rowmap"], keep=keep)
        a = d["init"].copy()
        backend.render_pages_host(p, a)
    finally:
        backend.free_device(buf)
    assert np.array_equal(a, d["expected"])

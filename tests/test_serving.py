"""Continuous-batching server: every request's pages are the same rendered
alone, in a mixed batch, and by the oracle; admission respects the budget."""

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests(rrb, n, seed0=100):
    out = []
    for i in range(n):
        s = rrb.Scene(kind=2, seed=seed0 + i, n_pages=1 + (i % 2), page_scale=0.1, paths_scale=0.02)
        out.append(s)
    return out


def _run(server, scenes, stagger_s=0.0):
    pages, tickets, res = [], [], []
    for s in scenes:
        s.view.pages = None
        a = s.blank_arena(0)  # overwritten: the server fills pages with `init`
        pages.append(a)
        tickets.append(server.submit(s.view, a, init=255, keep=s))
        if stagger_s:
            time.sleep(stagger_s)
    for t in tickets:
        res.append(server.wait(t))
    return pages, res


def test_same_alone_and_in_the_mix(rrb_lib, oracle):
    scenes = _requests(rrb_lib, 10)
    # A large first request keeps the single worker busy while the small ones
    # queue up behind it, so they are batched together whatever the timing.
    blocker = rrb_lib.Scene(kind=2, seed=7, n_pages=4)
    with rrb_lib.Server(workers=1, max_batch_pages=8) as srv:
        mixed, _ = _run(srv, [blocker] + scenes)
        st = srv.stats()
    mixed = mixed[1:]
    assert st["completed"] == 11 and st["batches"] < 11  # requests shared batches
    with rrb_lib.Server(workers=1, max_batch_pages=1) as srv:
        alone, _ = _run(srv, scenes)
    for i, s in enumerate(scenes):
        assert np.array_equal(mixed[i], alone[i]), i
        if i < 4:
            exp = s.blank_arena()
            oracle.render_scene(s, exp)
            assert np.array_equal(mixed[i], exp), i


def test_admission_under_a_small_budget(rrb_lib):
    scenes = _requests(rrb_lib, 6, seed0=300)
    budget = 64 << 20
    with rrb_lib.Server(workers=2, mem_budget=budget, max_batch_pages=16) as srv:
        pages, res = _run(srv, scenes)
        st = srv.stats()
    assert st["completed"] == 6 and st["in_use_bytes"] == 0
    assert all(r["latency_ns"] > 0 for r in res)


def test_cost_model_policies_keep_the_pixels(rrb_lib, oracle):
    """Shortest-first admission and per-batch tile shapes reorder and retile
    the work but never change a request's pages."""
    from rrb.autotune import CostModel

    scenes = _requests(rrb_lib, 6, seed0=500)
    m = rrb_lib.MLP(0, seed=1)
    params = m.params()
    m.close()
    model = CostModel(params, np.zeros(24, np.float32), np.ones(24, np.float32), 0.0, 1.0,
                      np.tile(np.array([0, 1, 2, 0], np.int32), 4))
    with rrb_lib.Server(workers=2, max_batch_pages=4) as srv:
        srv.set_cost_model(model)
        by_model, _ = _run(srv, scenes)
        st = srv.stats()
    assert st["completed"] == 6 and sum(st["tile_batches"]) == st["batches"]
    with rrb_lib.Server(workers=1, max_batch_pages=4) as srv:
        srv.set_cost_model(table=np.full(16, 1, np.int32), shortest_first=False)
        by_table, _ = _run(srv, scenes)
        st = srv.stats()
    assert st["tile_batches"] == [0, st["batches"], 0]  # every batch took the table's 32x32
    for i, s in enumerate(scenes):
        assert np.array_equal(by_model[i], by_table[i]), i
        if i < 3:
            exp = s.blank_arena()
            oracle.render_scene(s, exp)
            assert np.array_equal(by_model[i], exp), i

"""The benchmark's line contract, checked on the CPU: the B200 line and the
reference line of one workload carry the same `config` (the workload alone),
and workloads whose inputs fit in L2 are timed after an L2 flush."""

import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def test_config_is_the_workload_alone_and_states_the_l2_rule(rrb_lib):
    import bench
    big = rrb_lib.Scene(kind=1, seed=0)                            # the glyph page: 566 MB of points and page
    small = rrb_lib.Scene(kind=0, seed=4, n_paths=300, page_w=640, page_h=480)
    assert not bench.needs_l2_flush(big) and bench.needs_l2_flush(small)
    for sc in (big, small):
        a = bench.workload_config("w", sc, 0)
        b = bench.workload_config("w", sc, 0)
        assert a == b and set(a) == {"workload", "paths", "pages", "rowmap", "l2"}
        assert ("flushed" in a["l2"]) == bench.needs_l2_flush(sc)
        assert (a["paths"], a["pages"]) == (sc.n_paths, sc.n_pages)


def test_every_row_stage_shape_has_a_name():
    import bench
    assert len(bench.ROW_STAGES) == 5

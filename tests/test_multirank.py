"""Multi-rank page sharding on CPU: two gloo ranks split a multi-page batch,
each renders its shard (with the oracle, as no GPU is here), and together
they reproduce the single-process render; the timing reduction is the max."""

import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    sys.path[:0] = [str(root / "pdf-raster_b200"), str(root / "oracle")]
    import torch.distributed as dist

    import rr_oracle
    import rrb
    from rrb.shard import max_over_ranks, shard_arrays

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        scene = rrb.Scene(2, 9, n_pages=5, page_scale=0.05, paths_scale=0.004)
        sh = shard_arrays(scene, rank, world)
        arena = np.full(max(1, sh["arena_bytes"]), 255, np.uint8)
        if sh["arena_bytes"]:
            rr_oracle.render_arrays(arena, sh["page_offset"], sh["page_width"], sh["page_height"], sh["pts"],
                                    sh["flags"], sh["path_pt_off"], sh["fill_rule"], sh["gray"], sh["alpha"],
                                    sh["path_page"])
        np.save(Path(out_dir) / f"rank{rank}.npy", arena[: sh["arena_bytes"]])
        np.save(Path(out_dir) / f"rank{rank}_meta.npy", np.array([sh["arena_base"], *sh["pages"]], np.int64))
        m = max_over_ranks(10.0 + rank, dist)
        np.save(Path(out_dir) / f"rank{rank}_max.npy", np.array([m]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_page_shards_partition_the_batch():
    import sys
    from pathlib import Path

    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "pdf-raster_b200"))
    from rrb.shard import page_shard

    for n in (0, 1, 5, 64):
        for world in (1, 2, 3, 8):
            spans = [page_shard(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [e - b for b, e in spans]
            assert max(sizes) - min(sizes) <= 1


def test_two_gloo_ranks_reproduce_the_single_process_render(tmp_path, oracle, rrb_lib):
    import torch.multiprocessing as mp

    world, port = 2, _free_port()
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, start_method="spawn")
    scene = rrb_lib.Scene(2, 9, n_pages=5, page_scale=0.05, paths_scale=0.004)
    full = scene.blank_arena()
    oracle.render_scene(scene, full)
    got = np.full_like(full, 7)  # bytes between pages keep their value; page bytes must come from a rank
    gaps = np.ones(full.size, bool)
    for pg in range(scene.n_pages):
        o, n = int(scene.page_offset[pg]), int(scene.page_width[pg]) * int(scene.page_height[pg])
        gaps[o:o + n] = False
    covered = 0
    for r in range(world):
        base, p0, p1 = np.load(tmp_path / f"rank{r}_meta.npy")
        part = np.load(tmp_path / f"rank{r}.npy")
        got[base:base + part.size] = part
        covered += p1 - p0
        assert np.load(tmp_path / f"rank{r}_max.npy")[0] == 10.0 + world - 1
    assert covered == scene.n_pages
    assert np.array_equal(got[~gaps], full[~gaps]) and (full[~gaps] != 255).any()

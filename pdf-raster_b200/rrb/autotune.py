"""Autotuner and learned cost model for the composite tile shape.

The composite stage can run with 16x16, 32x32 or 64x16 page tiles; which is
fastest depends on the page (its size, how many paths overlap each tile, how
much of it is covered by rectangles). This module

* sweeps pages of the mixed-page generator (A4/Letter/A3 sizes at several
  scales, log-normal path counts, glyphs / polygons / rectangles) through the
  resident batch path once per tile shape and records (features, device
  time) pairs — the features are rrb_page_features, computed on the host
  before a page is rendered;
* builds the autotuner table: the fastest shape per (page size, edge
  density) bin of the sweep;
* trains the MLP (rrb_mlp_*: CUDA forward / backward / Adam kernels) on the
  log device time;
* chooses a tile shape per page with the model, falling back to the table
  (and to 64x16) when there is no model.

    python -m rrb.autotune sweep --pages 200 --seed 1000 --out tune.npz
    python -m rrb.autotune train --data tune.npz --out cost_model.npz
"""

from __future__ import annotations

import argparse
import json
import sys
import time
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import B200Backend, MLP, Scene, TILE_SHAPES, page_features_all

DEFAULT_SHAPE = 2  # 64x16
N_SHAPES = len(TILE_SHAPES)


def page_scene(seed: int) -> Scene:
    """One page of the mixed-page generator at a seeded scale: page size
    from {A4, Letter, A3} x {150, 300, 600} dpi times 0.15..1, paths
    log-normal (median 5,000) times 0.02..1."""
    rng = np.random.default_rng(seed)
    page_scale = float(rng.choice([0.25, 0.5, 1.0]) * rng.uniform(0.6, 1.0))
    paths_scale = float(np.exp(rng.uniform(np.log(0.02), 0.0)))
    return Scene(2, seed, n_pages=1, page_scale=page_scale, paths_scale=paths_scale)


def features(scene: Scene, page: int = 0) -> np.ndarray:
    """[N_SHAPES, 24] features of one page, one row per tile shape."""
    return page_features_all(scene.view, page)


def time_page(backend: B200Backend, scene: Scene, pages, reps: int = 2) -> np.ndarray:
    """Device milliseconds of rendering the scene with each tile shape (the
    sum of the pipeline's stage times; min over `reps` after one warm-up)."""
    batch = backend.batch_upload(scene.view)
    out = np.zeros(N_SHAPES)
    try:
        for i, (tw, th) in enumerate(TILE_SHAPES):
            backend.set_tuning(tw, th)
            best = np.inf
            for r in range(reps + 1):
                backend.begin_page()
                backend.record_fill_buffer(pages, 255, 0, scene.arena_bytes)
                batch.record(pages)
                backend.wait_page(backend.submit_page())
                if r:
                    best = min(best, sum(ms for ms, _ in backend.stage_times().values()))
            out[i] = best
    finally:
        batch.free()
    return out


def sweep(n_pages: int, seed0: int, device: int = 0, reps: int = 2, log_every: int = 500,
          out_path: str | None = None, save_every: int = 2000) -> dict:
    """(features, ms) of n_pages generated pages x every tile shape; saved to
    out_path every save_every pages (so a cut-off run keeps what it did)."""
    be = B200Backend(device)
    be.set_profiling(True)
    X = np.zeros((n_pages, N_SHAPES, 24), np.float32)
    T = np.zeros((n_pages, N_SHAPES), np.float64)
    pix = np.zeros(n_pages, np.int64)
    cap, pages = 0, None
    t0 = time.time()

    def result(n):
        return {"X": X[:n], "ms": T[:n], "pixels": pix[:n], "seeds": np.arange(seed0, seed0 + n)}

    try:
        for i in range(n_pages):
            sc = page_scene(seed0 + i)
            if sc.arena_bytes > cap:
                if pages is not None:
                    be.free_device(pages)
                cap = int(sc.arena_bytes * 1.25) + 4096
                pages = be.alloc_device(cap)
            X[i] = features(sc)
            T[i] = time_page(be, sc, pages, reps)
            pix[i] = sc.pixels
            if log_every and (i + 1) % log_every == 0:
                print(f"sweep: {i + 1}/{n_pages} pages, {time.time() - t0:.0f} s", file=sys.stderr, flush=True)
            if out_path and (i + 1) % save_every == 0:
                np.savez_compressed(out_path, **result(i + 1))
    finally:
        if pages is not None:
            be.free_device(pages)
        be.close()
    return result(n_pages)


# ---- the autotuner table ---------------------------------------------------------

def bins(X: np.ndarray) -> np.ndarray:
    """Table key of each page (features of any shape): page-size bin x edges-per-pixel bin (4 x 4)."""
    lp = X[..., 0]                       # log1p(pixels)
    dens = X[..., 5] - X[..., 0]         # log(edges / pixels), about
    b0 = np.clip(((lp - 13.0) / 1.0).astype(int), 0, 3)
    b1 = np.clip(((dens + 6.0) / 1.5).astype(int), 0, 3)
    return b0 * 4 + b1


def build_table(X: np.ndarray, T: np.ndarray) -> np.ndarray:
    """Fastest shape per bin (by total time over the bin's pages); 64x16 where empty."""
    keys = bins(X[:, 0])
    table = np.full(16, DEFAULT_SHAPE, np.int32)
    for k in range(16):
        sel = keys == k
        if sel.any():
            table[k] = int(np.argmin(T[sel].sum(0)))
    return table


# ---- the learned model -------------------------------------------------------------

@dataclass
class CostModel:
    params: np.ndarray      # MLP parameters (RRB_MLP_PARAMS floats)
    x_mean: np.ndarray
    x_std: np.ndarray
    y_mean: float
    y_std: float
    table: np.ndarray       # autotuner fallback

    def save(self, path):
        np.savez(path, params=self.params, x_mean=self.x_mean, x_std=self.x_std, y_mean=self.y_mean,
                 y_std=self.y_std, table=self.table)

    @classmethod
    def load(cls, path) -> "CostModel":
        d = np.load(path)
        return cls(d["params"], d["x_mean"], d["x_std"], float(d["y_mean"]), float(d["y_std"]), d["table"])

    def norm(self, X: np.ndarray) -> np.ndarray:
        return ((X - self.x_mean) / self.x_std).astype(np.float32)

    def predict_ms(self, X: np.ndarray, mlp: MLP | None = None) -> np.ndarray:
        """Predicted device ms for feature rows X [..., 24] (on the device kernels)."""
        own = mlp is None
        mlp = mlp or MLP(0)
        try:
            mlp.set_params(self.params)
            z = mlp.predict(self.norm(X.reshape(-1, 24)))
        finally:
            if own:
                mlp.close()
        return np.exp(z.astype(np.float64) * self.y_std + self.y_mean).reshape(X.shape[:-1])

    def choose(self, X: np.ndarray, mlp: MLP | None = None) -> np.ndarray:
        """Tile shape index per page from [pages, N_SHAPES, 24] features."""
        return np.argmin(self.predict_ms(X, mlp), axis=-1)

    def choose_table(self, X: np.ndarray) -> np.ndarray:
        return self.table[bins(X[:, 0])]


def train(X: np.ndarray, T: np.ndarray, epochs: int = 60, batch: int = 2048, lr: float = 2e-3, seed: int = 0,
          device: int = 0) -> CostModel:
    """Fit the MLP to log(ms) of every (page, shape) pair."""
    Xf = X.reshape(-1, 24).astype(np.float64)
    y = np.log(T.reshape(-1))
    x_mean, x_std = Xf.mean(0), Xf.std(0)
    x_std[x_std < 1e-6] = 1.0
    y_mean, y_std = float(y.mean()), float(y.std() or 1.0)
    mlp = MLP(device, seed=seed)
    try:
        Xn = ((Xf - x_mean) / x_std).astype(np.float32)
        yn = ((y - y_mean) / y_std).astype(np.float32)
        # Two phases: a larger step, then a finer one.
        mlp.train(Xn, yn, epochs=epochs, batch=batch, lr=lr, seed=seed)
        mlp.train(Xn, yn, epochs=max(1, epochs // 3), batch=batch, lr=lr / 5, seed=seed + 1)
        params = mlp.params()
    finally:
        mlp.close()
    return CostModel(params, x_mean.astype(np.float32), x_std.astype(np.float32), y_mean, y_std,
                     build_table(X, T))


def evaluate(model: CostModel, X: np.ndarray, T: np.ndarray) -> dict:
    """Held-out pages: total measured device time of each tile policy, and the model's error."""
    n = len(T)
    pred = model.predict_ms(X)
    choice = {"default_64x16": np.full(n, DEFAULT_SHAPE), "table": model.choose_table(X),
              "model": np.argmin(pred, 1), "best": np.argmin(T, 1)}
    totals = {k: float(T[np.arange(n), c].sum()) for k, c in choice.items()}
    for k in range(N_SHAPES):
        totals[f"fixed_{TILE_SHAPES[k][0]}x{TILE_SHAPES[k][1]}"] = float(T[:, k].sum())
    ape = np.abs(pred - T) / T
    return {
        "pages": n,
        "total_ms": totals,
        "model_vs_default": totals["default_64x16"] / totals["model"],
        "model_vs_table": totals["table"] / totals["model"],
        "best_vs_default": totals["default_64x16"] / totals["best"],
        "model_picks_best": float(np.mean(choice["model"] == choice["best"])),
        "mape": float(ape.mean()),
        "median_ape": float(np.median(ape)),
    }


def main(argv=None):
    ap = argparse.ArgumentParser(prog="rrb.autotune")
    sub = ap.add_subparsers(dest="cmd", required=True)
    s = sub.add_parser("sweep")
    s.add_argument("--pages", type=int, default=200)
    s.add_argument("--seed", type=int, default=1000)
    s.add_argument("--reps", type=int, default=2)
    s.add_argument("--out", required=True)
    t = sub.add_parser("train")
    t.add_argument("--data", required=True, nargs="+")
    t.add_argument("--holdout", type=int, default=5000, help="last N pages held out for evaluation")
    t.add_argument("--epochs", type=int, default=60)
    t.add_argument("--out", required=True)
    t.add_argument("--holdout-out", help="write the held-out pages (features, ms) here")
    t.add_argument("--report")
    a = ap.parse_args(argv)
    if a.cmd == "sweep":
        d = sweep(a.pages, a.seed, reps=a.reps, out_path=a.out)
        np.savez_compressed(a.out, **d)
        return
    parts = [np.load(p) for p in a.data]
    X = np.concatenate([p["X"] for p in parts])
    T = np.concatenate([p["ms"] for p in parts])
    h = min(a.holdout, len(T) // 2)
    model = train(X[:-h], T[:-h], epochs=a.epochs)
    model.save(a.out)
    if a.holdout_out:
        np.savez_compressed(a.holdout_out, X=X[-h:], ms=T[-h:])
    rep = {"train_pages": int(len(T) - h), "train_pairs": int((len(T) - h) * N_SHAPES), "holdout_pages": h,
           **evaluate(model, X[-h:], T[-h:])}
    print(json.dumps(rep))
    if a.report:
        Path(a.report).write_text(json.dumps(rep, indent=1) + "\n")


if __name__ == "__main__":
    main()

"""The workload generator is built twice from one source: into the package
(pdf-raster_b200/scenes/librrb_scenes.so, used by the B200 side) and into
oracle/_build/librr_scenes.so (used by the timed CPU reference, so that
process maps oracle/ libraries only). Both builds must give the same inputs."""

import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

SCENES = [dict(kind=0, seed=5, n_paths=300, page_w=640, page_h=480),
          dict(kind=1, seed=6, n_paths=800, page_w=900, page_h=700),
          dict(kind=2, seed=7, n_pages=3, page_scale=0.2, paths_scale=0.05)]

_PRINT = r'''
import sys, json
sys.path[:0] = [{pkg!r}, {tests!r}, {oracle!r}]
from rrb import scenes
if {use_oracle}:
    import rr_oracle
    rr_oracle.build()
    scenes.use_library(rr_oracle.SCENES_LIB_PATH)
from golden.make_batch_digests import input_digest
print(json.dumps([input_digest(scenes.Scene(**kw)) for kw in {scenes!r}]))
'''


def _digests(use_oracle: bool):
    code = _PRINT.format(pkg=str(ROOT / "pdf-raster_b200"), tests=str(ROOT / "tests"), oracle=str(ROOT / "oracle"),
                         use_oracle=use_oracle, scenes=SCENES)
    out = subprocess.run([sys.executable, "-c", code], check=True, capture_output=True, text=True, timeout=600)
    return out.stdout.strip().splitlines()[-1]


def test_oracle_build_of_the_generator_gives_the_same_inputs():
    assert _digests(False) == _digests(True)

"""Generates tests/golden/config1_frame.json: digests of the oracle's config-1 frame.

The reference has no golden images (it cannot run without a graphics stack),
so this fixture freezes the oracle itself: any change to the restated shader
math shows up as a digest change and must be explained.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
for p in (str(REPO / "voxel-engine-v0_b200"), str(REPO)):
    if p not in sys.path:
        sys.path.insert(0, p)


def config1_digest() -> dict:
    from oracle import oracle as O
    from vxe import scenes
    from vxe.scenes import FrameDriver

    sc = scenes.config1()
    drv = FrameDriver(sc)
    drv.initial_uploads()
    _, _, _, cam = drv.step()
    r = O.OracleFrameRunner(drv.world, sc.internal, sc.present, None, sc.clip_res)
    r.render(cam, drv.empty_clip(), threads=4)
    out = r.outputs()
    hits = out["hits"]
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
    idx = np.arange(0, hits.size, 997)
    return {
        "scene": "config1 (seed 12345, 256x144, cold frame)",
        "hits_sha256": sha(hits),
        "depth_sha256": sha(out["depth"]),
        "output_sha256": sha(out["output"]),
        "hit_counts": np.bincount(hits["mat"], minlength=7).tolist(),
        "samples": [[float(hits["t"][i]), int(hits["node"][i]), *map(int, hits["voxel"][i]), int(hits["face"][i]),
                     int(hits["mat"][i])] for i in idx],
    }


if __name__ == "__main__":
    (HERE / "config1_frame.json").write_text(json.dumps(config1_digest(), indent=1) + "\n")
    print("wrote", HERE / "config1_frame.json")

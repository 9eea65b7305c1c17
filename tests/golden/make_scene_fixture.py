"""Makes the scene fixtures of the reference's example scenes (examples/scenes/*.json): for each, its parameters
(<name>_scene.json, the mesh path pointed at the welded mesh below) and its mesh, read, scaled and welded as the
reference reads it (<name>_mesh.npz: V [3 nV], F [3 nF]).  Run where a checkout of the reference is present, naming it
by argument or by the environment variable WEAVESIM_REFERENCE:
    python tests/golden/make_scene_fixture.py /path/to/weave-sim
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
import weavesim_b200 as ws  # noqa: E402
from weavesim_b200 import scenefile  # noqa: E402

# the example scenes: the small dome, the reference's GPU-parity scene (web/tests/selftest.html:38) and its variants,
# the dual domes with a per-area load and with lath groups, the tree
SCENES = ("dome_basic", "v5dome_cm", "v5dome_BugTest", "v5dome_failure", "dualv5dome_cm", "dualv5dome_cm_hybrid", "tree_cm")


def make(ref, name):
    src = os.path.join(ref, "examples", "scenes", name + ".json")
    with open(src) as f:
        d = json.load(f)
    mesh = d["mesh"]
    V, F = scenefile.read_mesh(os.path.join(os.path.dirname(src), mesh["path"]), float(mesh.get("scale", 1.0)))
    np.savez_compressed(os.path.join(HERE, name + "_mesh.npz"), V=V, F=F)
    d["mesh"] = {"path": name + "_mesh.npz", "scale": 1.0}
    with open(os.path.join(HERE, name + "_scene.json"), "w") as f:
        json.dump(d, f, indent=1)
    md = ws.load_scene(os.path.join(HERE, name + "_scene.json"))
    print(f"{name}: {len(V) // 3} vertices, {len(F) // 3} faces -> n {md.n}, m {md.m}, K {md.K}")


def main(ref):
    for name in SCENES:
        make(ref, name)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("WEAVESIM_REFERENCE")
    if not ref:
        sys.exit("usage: make_scene_fixture.py <checkout of the reference> (or set WEAVESIM_REFERENCE)")
    main(ref)

"""Writes the scene-loader fixtures of tests/golden/ from the reference.

    python tests/golden/make_scene_golden.py      (needs oracle/_ref/libref.so and the reference checkout)

* mock_scene.json: the reference's only scene fixture (scenes/mock_scene.json), copied.
* tricky_scene.json: a hand-made scene exercising the JSON forms the loader
  must accept (integer and exponent numbers, -0, key order, unknown keys,
  escapes, whitespace), written by this script.
* *_ref.json: what the reference's own LoadSceneJSON (src/scene_loader.cpp)
  and BuildBVH (src/bvh.cpp) produce for each, as float bit patterns.
"""
import json
import os
import pathlib
import shutil
import struct
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
REF = pathlib.Path(os.environ.get("REF", "/root/reference"))
sys.path.insert(0, str(ROOT / "oracle"))
import oracle as O  # noqa: E402

TRICKY = r"""
{ "lights": [ {"intensity": 2, "type": "point", "radius": 1e1, "color": [1, 0.5, 0.25], "pos": [0, 0, 3.5E0]},
              {"type": "directional", "direction": [-0, 1e-3, -1], "color": [1,1,1], "intensity": 0.5},
              {"type": "area", "whatever": [1, 2, 3]} ],
  "version": 1,
  "comment": "unknown keys are ignored é \"quoted\"",
  "sun": {"color": [1.0, 0.9, 0.8], "direction": [0.3, -0.2, -1], "intensity": 1.25},
  "camera": {"camera_to_world": [1,0,0,0, 0,1,0,0, 0,0,1,0, -4,0,1.5,1], "pos": [-4, 0, 1.5], "fov_y_deg": 45,
             "aspect": 2, "near": 1e-1, "far": 100, "image_width": 64, "image_height": 32, "extra": null},
  "materials": [ {"albedo": [0.5, 0.5, 0.5], "emissive": [0, 0, 0]},
                 {"emissive": [0.1, 0, 0], "albedo": [0.9, 0.1, 0.1], "diffuse_tex": "tex\\stone \"a\".png"} ],
  "triangles": [
    {"v": [[-1, -1, 0], [1, -1, 0], [0, 1, 0]], "n": [[0,0,1],[0,0,1],[0,0,1]], "uv": [[0,0],[1,0],[0.5,1]], "mat": 0},
    {"mat": 1, "uv": [[0,0],[1,0],[0,1]], "n": [[0,0,-1],[0,0,-1],[0,0,-1]],
     "v": [[-0.0, 2.5e-1, 1.0000001], [3.3333333, -1.5e0, 1], [0.1, 0.2, -0.3]]},
    {"v": [[2, 2, 2], [3, 2, 2], [2, 3, 2]], "n": [[1,0,0],[0,1,0],[0,0,1]], "uv": [[0.25,0.75],[1e-2,0],[0,1]], "mat": 1}
  ]
}
"""


def bits(a):
    return [struct.unpack("<I", struct.pack("<f", float(x)))[0] for x in np.asarray(a, np.float32).ravel()]


def record(path):
    s = O.ref_load_scene(str(path))
    assert s is not None
    cam = s["camera"]
    nodes, _ = O.ref_build_bvh(s["tris"])
    return {
        "camera": {"pos": bits(cam.pos[:]), "m": bits(cam.m[:]), "fov": bits([cam.fov]), "aspect": bits([cam.aspect]),
                   "near": bits([cam.near]), "far": bits([cam.far]), "w": cam.w, "h": cam.h},
        "sun": bits(list(s["sun"]["dir"]) + list(s["sun"]["color"]) + [s["sun"]["intensity"]]),
        "tris": bits(s["tris"].view(np.float32).reshape(len(s["tris"]), 25)[:, :24]),
        "mats": [int(m) for m in s["tris"]["material"]],
        "albedo": bits(s["albedo"]), "emissive": bits(s["emissive"]),
        "points": bits(s["points"].view(np.float32)), "n_points": len(s["points"]),
        "directionals": bits(s["directionals"].view(np.float32)), "n_directionals": len(s["directionals"]),
        "bvh_nodes": nodes.view(np.uint32).ravel().tolist(), "n_nodes": len(nodes),
    }


def main():
    shutil.copyfile(REF / "scenes" / "mock_scene.json", HERE / "mock_scene.json")
    (HERE / "tricky_scene.json").write_text(TRICKY)
    for name in ("mock_scene", "tricky_scene"):
        (HERE / f"{name}_ref.json").write_text(json.dumps(record(HERE / f"{name}.json")))
        print("wrote", HERE / f"{name}_ref.json")


if __name__ == "__main__":
    main()

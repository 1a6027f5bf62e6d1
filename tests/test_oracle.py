"""The CPU oracle (oracle/lgoracle.c) pinned against the reference's own
sources compiled in oracle/_ref/libref.so: BVH nodes and triangle order
bit-identical, FP32 accumulators bit-identical."""
import numpy as np
import pytest

import oracle as O
import lumina
from lumina.scene import TRI_DTYPE

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref/libref.so not built")


def soup(n, seed=0, dup=0):
    rng = np.random.default_rng(seed)
    t = np.zeros(n, TRI_DTYPE)
    c = rng.uniform(-5, 5, (n, 1, 3))
    t["v"] = (c + rng.normal(0, 0.3, (n, 3, 3))).astype(np.float32)
    if dup:
        t["v"][:dup] = t["v"][0]  # identical triangles -> identical Morton codes
    t["n"] = np.array([0, 0, 1], np.float32)
    return t


def runs_equal_up_to_permutation(a, b, codes):
    """Triangle arrays equal except for the order inside runs of equal codes."""
    if a.tobytes() == b.tobytes():
        return True
    starts = np.flatnonzero(np.r_[True, codes[1:] != codes[:-1]])
    ends = np.r_[starts[1:], len(codes)]
    for s, e in zip(starts, ends):
        ka = sorted(bytes(x) for x in a[s:e].view(np.uint8).reshape(e - s, -1))
        kb = sorted(bytes(x) for x in b[s:e].view(np.uint8).reshape(e - s, -1))
        if ka != kb:
            return False
    return True


@needs_ref
@pytest.mark.parametrize("case", ["box", "engine_small", "soup", "dups", "tiny1", "tiny3", "tiny5", "allsame"])
def test_bvh_restatement_matches_reference(case, box_scene, small_engine_scene):
    tris = {"box": lambda: box_scene.tris, "engine_small": lambda: small_engine_scene.tris,
            "soup": lambda: soup(3000, 1), "dups": lambda: soup(500, 2, dup=37),
            "tiny1": lambda: soup(1, 3), "tiny3": lambda: soup(3, 4), "tiny5": lambda: soup(5, 5),
            "allsame": lambda: soup(40, 6, dup=40)}[case]()
    rn, rt = O.ref_build_bvh(tris)
    on, ot, perm, codes = O.oracle_build_bvh(tris)
    assert rn.tobytes() == on.tobytes()
    assert runs_equal_up_to_permutation(rt, ot, codes)
    assert ot.tobytes() == tris[perm].tobytes()


@needs_ref
def test_bvh_signed_zero_first_occurrence_wins():
    # -0.0 and +0.0 in one leaf: the reference keeps the first one met (strict <).
    t = soup(3, 9)
    t["v"][0, 0, 0] = -0.0
    t["v"][1, 0, 0] = 0.0
    t["v"][2, :, 0] = np.abs(t["v"][2, :, 0]) + 1
    t["v"][0, 1:, 0] = 1.0
    t["v"][1, 1:, 0] = 1.0
    rn, _ = O.ref_build_bvh(t)
    on, _, _, _ = O.oracle_build_bvh(t)
    assert rn.tobytes() == on.tobytes()


@needs_ref
@pytest.mark.parametrize("spp,bounces", [(1, 0), (9, 2), (16, 3)])
def test_trace_restatement_matches_reference(box_scene, spp, bounces):
    nodes, tris, _, _ = O.oracle_build_bvh(box_scene.tris)
    cam = box_scene.camera.copy()
    cam.width, cam.height = 48, 24
    ra = O.ref_trace_cpu(box_scene, nodes, tris, spp, bounces, camera=cam)
    oa, cnt = O.oracle_render(box_scene, nodes, tris, spp, bounces, camera=cam)
    assert ra.tobytes() == oa.tobytes()
    assert cnt["closest_rays"] > 0


@needs_ref
def test_trace_restatement_engine_scene(small_engine_scene):
    sc = small_engine_scene
    nodes, tris, _, _ = O.oracle_build_bvh(sc.tris)
    ra = O.ref_trace_cpu(sc, nodes, tris, 8, 2, row_start=3, row_step=7)
    oa, _ = O.oracle_render(sc, nodes, tris, 8, 2, row_start=3, row_step=7)
    assert ra.tobytes() == oa.tobytes()
    assert float(oa.sum()) > 0


def test_oracle_tonemap_truncates():
    acc = np.array([[[0.0, 0.25, 4.0]], [[-1.0, 1.0, 0.5]]], np.float32)
    out = O.oracle_tonemap(acc, 4)
    # sqrt(clamp(acc/4)) * 255 truncated
    exp = (np.sqrt(np.clip(acc / np.float32(4), 0, 1)) * np.float32(255)).astype(np.uint8)
    assert (out == exp).all()

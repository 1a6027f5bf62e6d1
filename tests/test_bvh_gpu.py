"""Device LBVH (lg_build_bvh) against the oracle and the reference BuildBVH:
node arrays bit-identical; triangle order identical to the oracle's (ties in
Morton code broken by input index) and to the reference's up to the order
inside runs of equal codes."""
import numpy as np
import pytest

import lumina
import oracle as O
from test_oracle import runs_equal_up_to_permutation, soup

pytestmark = pytest.mark.gpu


CASES = {
    "tiny1": lambda b, e: soup(1, 3),
    "tiny2": lambda b, e: soup(2, 13),
    "tiny3": lambda b, e: soup(3, 4),
    "tiny4": lambda b, e: soup(4, 14),
    "tiny5": lambda b, e: soup(5, 5),
    "tiny17": lambda b, e: soup(17, 15),
    "allsame": lambda b, e: soup(40, 6, dup=40),
    "dups": lambda b, e: soup(500, 2, dup=37),
    "soup": lambda b, e: soup(30000, 1),
    "box": lambda b, e: b.tris,
    "engine_small": lambda b, e: e.tris,
}


@pytest.mark.parametrize("case", list(CASES))
def test_device_bvh_matches_oracle_and_reference(case, box_scene, small_engine_scene):
    tris = CASES[case](box_scene, small_engine_scene)
    nodes, out, perm = lumina.build_bvh(tris)
    on, ot, operm, codes = O.oracle_build_bvh(tris)
    assert len(nodes) == len(on)
    assert nodes.tobytes() == on.tobytes()
    assert out.tobytes() == ot.tobytes()
    assert (perm == operm).all()
    if O.ref_available():
        rn, rt = O.ref_build_bvh(tris)
        assert nodes.tobytes() == rn.tobytes()
        assert runs_equal_up_to_permutation(out, rt, codes)


def test_device_bvh_empty():
    nodes, out, perm = lumina.build_bvh(np.zeros(0, lumina.scene.TRI_DTYPE))
    assert len(nodes) == 0


def test_device_bvh_signed_zero():
    t = soup(3, 9)
    t["v"][0, 0, 0] = -0.0
    t["v"][1, 0, 0] = 0.0
    t["v"][2, :, 0] = np.abs(t["v"][2, :, 0]) + 1
    t["v"][0, 1:, 0] = 1.0
    t["v"][1, 1:, 0] = 1.0
    nodes, _, _ = lumina.build_bvh(t)
    on, _, _, _ = O.oracle_build_bvh(t)
    assert nodes.tobytes() == on.tobytes()


def test_device_bvh_engine_full_size():
    """The 1,050,972-triangle engine-scale scene."""
    sc = lumina.engine_scene(seed=7)
    assert sc.n_tris == 1050972
    nodes, out, perm = lumina.build_bvh(sc.tris)
    on, ot, operm, codes = O.oracle_build_bvh(sc.tris)
    assert nodes.tobytes() == on.tobytes()
    assert out.tobytes() == ot.tobytes()
    if O.ref_available():
        rn, rt = O.ref_build_bvh(sc.tris)
        assert nodes.tobytes() == rn.tobytes()


def test_renderer_builds_same_bvh(box_scene):
    with lumina.Renderer(0) as r:
        r.set_scene(box_scene)
        gn, gt = r.get_bvh()
    on, ot, _, _ = O.oracle_build_bvh(box_scene.tris)
    assert gn.tobytes() == on.tobytes() and gt.tobytes() == ot.tobytes()

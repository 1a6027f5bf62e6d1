"""Traversal-stack overflow is an error, never a silently incomplete image.

The reference's traversal drops pushes past its 64-entry stack without a word
(src/pathtracer.cu:142, :184).  Here every dropped push sets a fault word that
the renderer reports as LG_ERR_DEVICE.  The test builds a caller BVH that is a
chain of 120 binary levels (each node: one leaf, one deeper subtree), keeps
its topology as the render tree, and aims the camera down the chain so that
every box is entered before any triangle is hit; the traversal then needs
about one stack entry per binary level (2-wide records) or three per 4-wide
record, past the 96-entry stack.  The renderer's stack bound says so, so the
frame runs on the checked kernel, which tests the stack depth before every
push: no access goes out of bounds."""
import numpy as np
import pytest

import lumina
from lumina._ffi import NODE_DTYPE, POINT_DTYPE, DIR_DTYPE, TRI_DTYPE, LG_ERR_DEVICE, LuminaError

pytestmark = pytest.mark.gpu

N_CHAIN = 120


def chain_scene(n=N_CHAIN, reverse=True):
    """n triangles facing a camera on the -x side, stacked along +x; triangle
    i sits farther away than triangle i+1 when `reverse`, so the nearest one
    is the deepest leaf of the chain."""
    tris = np.zeros(n, TRI_DTYPE)
    for i in range(n):
        x = 1.0 + 0.05 * ((n - 1 - i) if reverse else i)
        tris[i]["v"] = [[x, -1.0, -1.0], [x, 1.0, -1.0], [x, 0.0, 1.5]]
        tris[i]["n"] = [[-1.0, 0.0, 0.0]] * 3
        tris[i]["material"] = 0
    # Chain in BFS order: internal node 2k has leaf 2k+1 (triangle k) on the
    # left and node 2k+2 on the right; the last internal node has two leaves.
    n_nodes = 2 * n - 1
    nodes = np.zeros(n_nodes, NODE_DTYPE)
    vmin = tris["v"].min(axis=1)
    vmax = tris["v"].max(axis=1)
    for k in range(n - 1):
        i = 2 * k
        nodes[i]["left"], nodes[i]["right"] = i + 1, i + 2
        nodes[i]["firstTri"], nodes[i]["triCount"] = -1, 0
        nodes[i]["bbMin"] = vmin[k:].min(axis=0)
        nodes[i]["bbMax"] = vmax[k:].max(axis=0)
        nodes[i + 1]["firstTri"], nodes[i + 1]["triCount"] = k, 1
        nodes[i + 1]["left"] = nodes[i + 1]["right"] = -1
        nodes[i + 1]["bbMin"], nodes[i + 1]["bbMax"] = vmin[k], vmax[k]
    last = n_nodes - 1
    nodes[last]["firstTri"], nodes[last]["triCount"] = n - 1, 1
    nodes[last]["left"] = nodes[last]["right"] = -1
    nodes[last]["bbMin"], nodes[last]["bbMax"] = vmin[n - 1], vmax[n - 1]
    cam = lumina.Camera(np.zeros(3, np.float32),
                        np.array([1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1], np.float32),
                        fov_y_deg=20.0, aspect=2.0, width=32, height=16)
    sun = np.zeros((), DIR_DTYPE)
    sun["dir"], sun["color"], sun["intensity"] = [1.0, 0.0, 0.0], [1.0, 1.0, 1.0], 1.0
    sc = lumina.Scene(cam, sun, tris, np.array([[0.5, 0.5, 0.5]], np.float32), np.zeros((1, 3), np.float32),
                      np.zeros(0, POINT_DTYPE))
    return sc, nodes


@pytest.mark.parametrize("width", [2, 4])
def test_deep_chain_reports_overflow(width):
    sc, nodes = chain_scene()
    with lumina.Renderer(0) as r:
        r.set_render_tree("buildbvh")
        r.set_scene_bvh(sc, nodes)
        assert r.render_tree() == "buildbvh"
        r.set_bvh_width(width)
        bound, cap = r.stack_bound()
        assert bound > cap, (bound, cap)
        with pytest.raises(LuminaError) as ei:
            r.render(spp=1, bounces=0)
        assert ei.value.code == LG_ERR_DEVICE and "stack overflow" in str(ei.value)
        with pytest.raises(LuminaError) as ei:
            r.gbuffer()
        assert ei.value.code == LG_ERR_DEVICE
        # The error is reported once; the renderer stays usable: a chain whose
        # nearest triangle is tested first never grows the stack.
        sc2, nodes2 = chain_scene(reverse=False)
        r.set_scene_bvh(sc2, nodes2)
        out = r.render(spp=1, bounces=0)
        assert out["rgb"][8, 16].any(), "the centre pixel sees the nearest triangle"


def test_stack_bound_of_ordinary_trees_fits(box_scene, small_engine_scene):
    """Ordinary scenes' render trees have a stack bound within the stack, so
    their frames run on the kernel without per-push checks."""
    for sc in (box_scene, small_engine_scene):
        with lumina.Renderer(0) as r:
            r.set_scene(sc)
            for width in (4, 2):
                r.set_bvh_width(width)
                bound, cap = r.stack_bound()
                assert 0 < bound <= cap, (width, bound, cap)


def test_shallow_chain_renders_same_as_balanced_tree():
    """The same triangles with the default render tree (PLOC) and with the
    nearest-first chain give the same image: the fault word stays clear."""
    sc, nodes = chain_scene(reverse=False)
    with lumina.Renderer(0) as r:
        r.set_render_tree("buildbvh")
        r.set_scene_bvh(sc, nodes)
        a = r.render(spp=1, bounces=0)["accum"]
        r.set_render_tree("ploc_tris")
        b = r.render(spp=1, bounces=0)["accum"]
    assert np.array_equal(a, b)

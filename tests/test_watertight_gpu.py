"""Watertight ray/triangle mode (Woop, Benthin, Wald 2013) beside the
reference's Moller-Trumbore test: no ray may escape a closed mesh, and away
from edges both tests see the same hits."""
import numpy as np
import pytest

import lumina
from lumina import scene as S

pytestmark = pytest.mark.gpu
REL, ABS = 1e-3, 1e-6


def _inside_sphere(subdiv, target, w=320, h=320):
    v, f = S.icosphere(subdiv)
    uv = S._sphere_uv(v)
    tris = S._indexed(v * 10.0 + np.array([0.37, -0.21, 0.13]), v, uv, f, 0)
    cam = S.look_at_camera([0.0, 0.0, 0.0], target, w, h, fov=100.0, aspect=1.0)
    sun = np.zeros((), _ffi_dir())
    return lumina.Scene(cam, sun, tris, np.full((1, 3), 0.5, np.float32), np.zeros((1, 3), np.float32),
                        np.zeros(0, lumina._ffi.POINT_DTYPE))


def _ffi_dir():
    return lumina._ffi.DIR_DTYPE


@pytest.mark.parametrize("target", [[1.0, 0.3, 0.2], [-0.4, 1.0, -0.7], [0.1, -0.2, 1.0]])
def test_no_ray_escapes_a_closed_mesh(target):
    sc = _inside_sphere(6, target)
    misses = {}
    with lumina.Renderer(0) as r:
        r.set_scene(sc)
        for mode in ("mt", "watertight"):
            r.set_intersection(mode)
            alb, _, _ = r.gbuffer()
            misses[mode] = int((alb == 0).all(axis=2).sum())
    print("rays escaping a closed 81,920-triangle sphere (of 102,400):", misses)
    assert misses["watertight"] == 0


def test_watertight_matches_mt_away_from_edges(box_scene):
    with lumina.Renderer(0) as r:
        r.set_scene(box_scene)
        mt = r.render(spp=8, bounces=2)
        gb_mt = r.gbuffer()
        r.set_intersection("watertight")
        wt = r.render(spp=8, bounces=2)
        gb_wt = r.gbuffer()
        r.set_intersection("mt")
        again = r.render(spp=8, bounces=2)
    assert np.array_equal(again["accum"], mt["accum"])  # switching back restores the parity records
    close = np.abs(wt["accum"] - mt["accum"]) <= REL * np.maximum(np.abs(wt["accum"]), np.abs(mt["accum"])) + ABS
    frac = float(close.all(axis=2).mean())
    # t, u, v come from different arithmetic, so 8-bit normals and positions may differ by one step
    same_hit = float(np.mean([(np.abs(a.astype(int) - b.astype(int)) <= 1).all(axis=2).mean()
                              for a, b in zip(gb_mt, gb_wt)]))
    print(f"watertight vs Moller-Trumbore: {frac:.5f} of pixels within 1e-3 (8 spp, 2 bounces); "
          f"{same_hit:.5f} of primary-hit G-buffer pixels within one 8-bit step")
    assert frac >= 0.95 and same_hit >= 0.999

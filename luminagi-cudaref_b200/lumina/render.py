"""BVH build and rendering through liblumina (C ABI), for Python callers."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._ffi import (LG_RENDER_ACCUM64, LG_RENDER_NO_RAY_SORT, NODE_DTYPE, TRI_DTYPE, LgCamera, LgRenderOpts,
                   LgRenderStats, check, lib, ptr)
from .scene import Camera, Scene


def build_bvh(tris: np.ndarray):
    """BuildBVH on the GPU (reference bvh.cpp:164-211).

    Returns (nodes NODE_DTYPE[n_nodes], reordered triangles, perm) where
    perm[i] is the input index of the triangle placed at i."""
    tris = np.ascontiguousarray(tris, TRI_DTYPE)
    n = len(tris)
    nodes = np.zeros(max(2 * n - 1, 1), NODE_DTYPE)
    perm = np.zeros(max(n, 1), np.int32)
    out = np.zeros_like(tris)
    count = C.c_int32(0)
    check(lib().lg_build_bvh(ptr(tris), n, ptr(nodes), C.byref(count), ptr(perm), ptr(out)))
    return nodes[:count.value].copy(), out, perm[:n].copy()


class Renderer:
    """Device-resident scene + frame buffers (one CUDA device)."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        check(lib().lg_renderer_create(device, C.byref(self._h)))
        self.scene: Scene | None = None

    def close(self):
        if self._h:
            lib().lg_renderer_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_scene(self, scene: Scene) -> None:
        """Uploads the scene and builds its BVH on the device."""
        self.scene = scene
        d = scene.desc()
        check(lib().lg_renderer_set_scene(self._h, C.byref(d)))

    def set_scene_bvh(self, scene: Scene, nodes: np.ndarray) -> None:
        """Uploads a scene whose triangles are already in BVH order, with its nodes."""
        self.scene = scene
        nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
        d = scene.desc()
        check(lib().lg_renderer_set_scene_bvh(self._h, C.byref(d), ptr(nodes), len(nodes)))

    def get_bvh(self):
        n = C.c_int32(0)
        check(lib().lg_renderer_get_bvh(self._h, None, C.byref(n), None))
        nodes = np.zeros(n.value, NODE_DTYPE)
        tris = np.zeros(self.scene.n_tris if self.scene is not None else 0, TRI_DTYPE)
        check(lib().lg_renderer_get_bvh(self._h, ptr(nodes), C.byref(n), ptr(tris)))
        return nodes, tris

    def set_bvh_width(self, width: int) -> None:
        """Traversal records: 4-wide (default) or 2-wide; same BVH, same hits."""
        check(lib().lg_renderer_set_bvh_width(self._h, int(width)))

    def set_texture(self, material: int, rgba) -> None:
        """Diffuse texture of one material: (H,W,4) u8 RGBA, or None to remove it."""
        if rgba is None:
            check(lib().lg_renderer_set_texture(self._h, int(material), None, 0, 0))
            return
        rgba = np.ascontiguousarray(rgba, np.uint8)
        assert rgba.ndim == 3 and rgba.shape[2] == 4, "texture must be (H, W, 4) uint8"
        check(lib().lg_renderer_set_texture(self._h, int(material), ptr(rgba), rgba.shape[1], rgba.shape[0]))

    def load_textures(self, asset_root: str):
        """Loads the scene's textures from asset_root/<diffuse_tex>; returns (loaded, missing)."""
        from .image import load_image
        loaded = missing = 0
        for m, rel in enumerate(self.scene.textures if self.scene is not None else []):
            if not rel:
                continue
            try:
                self.set_texture(m, load_image(f"{asset_root}/{rel}"))
                loaded += 1
            except OSError:
                missing += 1
        return loaded, missing

    def set_intersection(self, mode: str) -> None:
        """'mt' (Moller-Trumbore, the reference's test; default) or 'watertight'."""
        modes = {"mt": 0, "watertight": 1}
        check(lib().lg_renderer_set_intersection(self._h, modes[mode]))

    def autotune(self, camera: Camera | None = None, spp: int = 8, bounces: int = 2):
        """Picks the persistent trace grid (resident blocks per SM) by timing; returns (blocks_per_sm, ms)."""
        cam = (camera if camera is not None else self.scene.camera).to_c()
        b, ms = C.c_int32(0), C.c_float(0)
        check(lib().lg_renderer_autotune(self._h, C.byref(cam), spp, bounces, C.byref(b), C.byref(ms)))
        return int(b.value), float(ms.value)

    def autotune_schedule(self, camera: Camera | None = None, spp: int = 8, bounces: int = 2):
        """Picks the refill threshold and leaf quorum by timing; returns (refill, quorum, ms)."""
        cam = (camera if camera is not None else self.scene.camera).to_c()
        f, q, ms = C.c_int32(0), C.c_int32(0), C.c_float(0)
        check(lib().lg_renderer_autotune_schedule(self._h, C.byref(cam), spp, bounces, C.byref(f), C.byref(q),
                                                  C.byref(ms)))
        return int(f.value), int(q.value), float(ms.value)

    def set_refill_threshold(self, threshold: int) -> None:
        """Finished rays per warp (1..32) after which those lanes shade and start their next ray."""
        check(lib().lg_renderer_set_refill_threshold(self._h, int(threshold)))

    def refill_threshold(self) -> int:
        return int(lib().lg_renderer_get_refill_threshold(self._h))

    def set_leaf_quorum(self, quorum: int) -> None:
        """Lanes still looking for a BVH leaf (0..31) below which a warp tests the leaves its lanes hold."""
        check(lib().lg_renderer_set_leaf_quorum(self._h, int(quorum)))

    def leaf_quorum(self) -> int:
        return int(lib().lg_renderer_get_leaf_quorum(self._h))

    def stack_bound(self):
        """(most traversal-stack entries a ray can need over the current records, stack capacity)."""
        b, c = C.c_int32(0), C.c_int32(0)
        check(lib().lg_renderer_get_stack_bound(self._h, C.byref(b), C.byref(c)))
        return int(b.value), int(c.value)

    def set_l2_window(self, enable: bool) -> None:
        """Persisting-L2 access window over the 4-wide BVH records (the reference's CUDAREF_L2_PIN)."""
        check(lib().lg_renderer_set_l2_window(self._h, 1 if enable else 0))

    def set_top_records(self, n: int) -> None:
        """4-wide BVH records (the top of the tree) each trace block keeps in shared memory; 0 = off."""
        check(lib().lg_renderer_set_top_records(self._h, int(n)))

    def top_records(self) -> int:
        return int(lib().lg_renderer_get_top_records(self._h))

    def set_render_tree(self, mode: str) -> None:
        """Tree the traversal records come from: 'ploc_tris' (default; PLOC over the triangles, one per
        leaf), 'ploc' (PLOC over BuildBVH's leaves) or 'buildbvh' (its own topology)."""
        check(lib().lg_renderer_set_render_tree(self._h, {"buildbvh": 0, "ploc": 1, "ploc_tris": 2}[mode]))

    def render_tree(self) -> str:
        m = C.c_int32(-1)
        check(lib().lg_renderer_get_render_tree(self._h, C.byref(m)))
        return {0: "buildbvh", 1: "ploc", 2: "ploc_tris"}.get(m.value, "none")

    def set_counting(self, on: bool) -> None:
        check(lib().lg_renderer_set_counting(self._h, 1 if on else 0))

    def render(self, camera: Camera | None = None, spp: int = 1, bounces: int = 0, sample_base: int = 0,
               accum: bool = True, accum64: bool = False, rgb: bool = True):
        """Renders one frame; returns dict(rgb (H,W,3) u8, accum (H,W,3) f32,
        accum64, kernel_ms, closest_rays, shadow_rays)."""
        cam = camera if camera is not None else self.scene.camera
        c = cam.to_c()
        W, H = int(cam.width), int(cam.height)
        o = LgRenderOpts(spp, bounces, sample_base, LG_RENDER_ACCUM64 if accum64 else 0)
        out_rgb = np.zeros((H, W, 3), np.uint8) if rgb else None
        out_acc = np.zeros((H, W, 3), np.float32) if accum else None
        out_acc64 = np.zeros((H, W, 3), np.float64) if accum64 else None
        st = LgRenderStats()
        check(lib().lg_render(self._h, C.byref(c), C.byref(o), ptr(out_rgb), ptr(out_acc), ptr(out_acc64),
                              C.byref(st)))
        return {"rgb": out_rgb, "accum": out_acc, "accum64": out_acc64, "kernel_ms": st.kernel_ms,
                "closest_rays": int(st.closest_rays), "shadow_rays": int(st.shadow_rays),
                "node_fetches": int(st.node_fetches), "tri_tests": int(st.tri_tests),
                "leaf_fetches": int(st.leaf_fetches)}

    def render_sorted(self, camera: Camera | None = None, spp: int = 1, bounces: int = 0, sample_base: int = 0,
                      sort: bool = True):
        """The reference's ray-sorted render (RenderSceneCUDASorted; cuda_ref --sort): per-sample
        seeding, rays sorted by direction between bounces, no Russian roulette.  sort=False keeps the
        rays in pixel order (same launches without the sorts).  Returns dict(rgb, accum, kernel_ms,
        closest_rays, shadow_rays, ...) as render()."""
        cam = camera if camera is not None else self.scene.camera
        c = cam.to_c()
        W, H = int(cam.width), int(cam.height)
        o = LgRenderOpts(spp, bounces, sample_base, 0 if sort else LG_RENDER_NO_RAY_SORT)
        out_rgb = np.zeros((H, W, 3), np.uint8)
        out_acc = np.zeros((H, W, 3), np.float32)
        st = LgRenderStats()
        check(lib().lg_render_sorted(self._h, C.byref(c), C.byref(o), ptr(out_rgb), ptr(out_acc), C.byref(st)))
        return {"rgb": out_rgb, "accum": out_acc, "kernel_ms": st.kernel_ms,
                "closest_rays": int(st.closest_rays), "shadow_rays": int(st.shadow_rays),
                "node_fetches": int(st.node_fetches), "tri_tests": int(st.tri_tests),
                "leaf_fetches": int(st.leaf_fetches)}

    def gbuffer(self, camera: Camera | None = None):
        """Primary-hit (albedo, normal, worldpos) 8-bit images (reference gbuffer_kernel)."""
        cam = camera if camera is not None else self.scene.camera
        c = cam.to_c()
        H, W = int(cam.height), int(cam.width)
        out = [np.zeros((H, W, 3), np.uint8) for _ in range(3)]
        check(lib().lg_render_gbuffer(self._h, C.byref(c), ptr(out[0]), ptr(out[1]), ptr(out[2])))
        return tuple(out)

    def render_batch(self, cameras, spps, bounces):
        """Renders several frames (per-job camera/spp/bounces); returns (rgb (J,H,W,3), ms per job)."""
        J = len(cameras)
        cams = (LgCamera * J)(*[c.to_c() for c in cameras])
        opts = (LgRenderOpts * J)(*[LgRenderOpts(int(s), int(b), 0, 0) for s, b in zip(spps, bounces)])
        H, W = int(cameras[0].height), int(cameras[0].width)
        assert all(int(c.height) == H and int(c.width) == W for c in cameras), "batch frames share one size"
        out = np.zeros((J, H, W, 3), np.uint8)
        ms = np.zeros(J, np.float32)
        check(lib().lg_render_batch(self._h, cams, opts, J, ptr(out), ptr(ms)))
        return out, ms

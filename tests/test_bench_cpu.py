"""Host logic of bench.py's batched-pose leg, run on the CPU with a stand-in
renderer (the GPU form runs in the benchmark itself)."""
import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "luminagi-cudaref_b200"))


class _Cam:
    def __init__(self, pos=None, tgt=None):
        self.pos, self.tgt = pos, tgt

    def look_at(self, pos, tgt):
        return _Cam(pos, tgt)


class _Scene:
    camera = _Cam()


class _Renderer:
    """Batched frames cost 2 ms per spp, a launch per pose 2.5 ms per spp."""

    def __init__(self):
        self.batch_calls, self.single = [], []

    def render_batch(self, cams, spps, bounces):
        assert len(cams) == len(spps) == len(bounces)
        self.batch_calls.append((len(cams), spps[0], bounces[0], [c.pos for c in cams]))
        return np.zeros((len(cams), 1, 1, 3), np.uint8), np.full(len(cams), 2.0 * spps[0], np.float32)

    def render(self, camera, spp, bounces, accum, rgb):
        assert not accum and not rgb
        self.single.append((camera.pos, spp, bounces))
        return {"kernel_ms": 2.5 * spp}


def test_batched_poses_leg():
    import bench
    from lumina.scene import ENGINE_CENTER, orbit_poses

    r = _Renderer()
    out = bench.batched_poses(r, _Scene(), 2)
    poses = [p for p, _ in orbit_poses(50, seed=11, center=ENGINE_CENTER)]
    # each configuration: a capturing call, then the timed replay, over the same poses
    assert [(n, spp, b) for n, spp, b, _ in r.batch_calls] == [(50, 8, 2), (50, 8, 2), (4, 256, 2), (4, 256, 2)]
    assert r.batch_calls[0][3] == poses and r.batch_calls[2][3] == poses[:4]
    assert [s[1] for s in r.single] == [8] * 50 + [256] * 4
    assert out["spp8"] == {"poses": 50, "bounces": 2, "batch_ms_per_frame": 16.0, "separate_ms_per_frame": 20.0,
                           "speedup": 1.25}
    assert out["spp256"]["poses"] == 4 and abs(out["spp256"]["speedup"] - 1.25) < 1e-12

"""lg_build_bvh_device_noalloc: the BVH build for callers that may not
allocate device memory (its scratch is a fixed array inside liblumina).

Checked through the C ABI against lg_build_bvh_device on the same device
inputs: node arrays, permutation and reordered triangles must be identical
(the BVH tests' tolerance is bit-exactness), for two calls in a row with
different inputs, so a stale scratch state from the first call would show in
the second.  This file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

import lumina
from lumina import _ffi
from lumina._ffi import NODE_DTYPE, TRI_DTYPE

pytestmark = pytest.mark.gpu

LG_NOALLOC_MAX_TRIS = 65536


def _soup(n, seed):
    rng = np.random.default_rng(seed)
    t = np.zeros(n, TRI_DTYPE)
    c = rng.uniform(-5, 5, (n, 1, 3))
    t["v"] = (c + rng.normal(0, 0.3, (n, 3, 3))).astype(np.float32)
    t["v"][: n // 10] = t["v"][0]  # a run of equal Morton codes
    t["n"] = np.array([0, 0, 1], np.float32)
    return t


def _build(fn_name, d_tris, n, torch, out="separate"):
    """Calls fn_name through the C ABI; out selects where the reordered
    triangles go: a separate buffer, nowhere (NULL), or back into d_tris."""
    d_nodes = torch.zeros(max(2 * n - 1, 1) * NODE_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    d_perm = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
    d_out = torch.zeros(max(n, 1) * TRI_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    out_ptr = {"separate": C.c_void_p(d_out.data_ptr()), "none": None,
               "inplace": C.c_void_p(d_tris.data_ptr())}[out]
    count = C.c_int32(-1)
    stream = torch.cuda.current_stream().cuda_stream
    fn = getattr(_ffi.lib(), fn_name)
    _ffi.check(fn(C.c_void_p(d_tris.data_ptr()), n, C.c_void_p(d_nodes.data_ptr()), C.byref(count),
                  C.c_void_p(d_perm.data_ptr()), out_ptr, C.c_void_p(stream)))
    torch.cuda.synchronize()
    nodes = d_nodes.cpu().numpy().view(NODE_DTYPE)[: count.value]
    tris_out = {"separate": d_out, "none": None, "inplace": d_tris}[out]
    tris_np = tris_out.cpu().numpy().view(TRI_DTYPE)[:n] if tris_out is not None else None
    return nodes, d_perm.cpu().numpy()[:n], tris_np


def test_noalloc_build_matches_allocating_build_twice():
    torch = pytest.importorskip("torch")
    box = lumina.box_scene(1).tris
    inputs = [box, _soup(30011, 5)]
    assert all(len(t) <= LG_NOALLOC_MAX_TRIS for t in inputs)
    for tris in inputs:  # two calls in a row, different inputs
        n = len(tris)
        d_tris = torch.from_numpy(tris.view(np.uint8).copy()).cuda()
        ref = _build("lg_build_bvh_device", d_tris, n, torch)
        got = _build("lg_build_bvh_device_noalloc", d_tris, n, torch)
        assert len(got[0]) == len(ref[0]) > 0
        assert got[0].tobytes() == ref[0].tobytes()
        assert (got[1] == ref[1]).all()
        assert got[2].tobytes() == ref[2].tobytes()


def test_noalloc_build_rejects_oversize_input():
    torch = pytest.importorskip("torch")
    n = LG_NOALLOC_MAX_TRIS + 1
    d_tris = torch.zeros(n * TRI_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    d_nodes = torch.zeros(8, dtype=torch.uint8, device="cuda")
    count = C.c_int32(-1)
    rc = _ffi.lib().lg_build_bvh_device_noalloc(C.c_void_p(d_tris.data_ptr()), n, C.c_void_p(d_nodes.data_ptr()),
                                                C.byref(count), None, None, None)
    assert rc == _ffi.LG_ERR_CAPACITY
    assert b"limit" in _ffi.lib().lg_last_error()


def test_noalloc_build_at_the_limit_in_every_output_layout():
    """LG_NOALLOC_MAX_TRIS triangles, with the reordered triangles written to a
    separate buffer, not written (NULL), and written back over the input: the
    last two stage the sorted triangles inside the fixed array, its largest
    layout.  Nodes and permutation must equal the allocating build's, and the
    in-place triangles its separate output."""
    torch = pytest.importorskip("torch")
    n = LG_NOALLOC_MAX_TRIS
    tris = _soup(n, 11)
    src = torch.from_numpy(tris.view(np.uint8).copy()).cuda()
    ref = _build("lg_build_bvh_device", src.clone(), n, torch)
    for out in ("none", "inplace", "separate"):
        got = _build("lg_build_bvh_device_noalloc", src.clone(), n, torch, out=out)
        assert got[0].tobytes() == ref[0].tobytes(), out
        assert (got[1] == ref[1]).all(), out
        if got[2] is not None:
            assert got[2].tobytes() == ref[2].tobytes(), out

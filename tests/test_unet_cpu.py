"""The PyTorch restatement of the reference UNet (oracle/unet_ref.py) pinned to
the reference module's own output (tests/golden/unet_golden.npz, made by
tests/golden/make_unet_golden.py from ml/train.py)."""
import pathlib

import numpy as np
import torch

import unet_ref
from lumina import unet as lunet

GOLD = pathlib.Path(__file__).resolve().parent / "golden" / "unet_golden.npz"


def test_restatement_matches_reference_module():
    g = np.load(GOLD)
    m = unet_ref.UNetRef().eval()
    flat = unet_ref.make_params(int(g["seed"]), m)
    assert len(flat) == int(g["n_params"]) == 1946947
    assert abs(float(flat.astype(np.float64).sum()) - float(g["param_sum"])) < 1e-9
    unet_ref.load_flat(m, flat)
    with torch.no_grad():
        y = m(torch.from_numpy(g["x"])).numpy()
    assert np.abs(y - g["y"]).max() < 1e-6


def test_param_layout_matches_reference_keys():
    m = unet_ref.UNetRef()
    assert [(k, s) for k, s in unet_ref.param_shapes(m)] == lunet.PARAM_SHAPES
    assert lunet.N_PARAMS == 1946947
    m12 = unet_ref.UNetRef(in_ch=12)
    assert [(k, s) for k, s in unet_ref.param_shapes(m12)] == lunet.param_shapes(12)


def test_restatement_matches_reference_module_12ch():
    """The 12-channel (--gbuffer) variant: residual on the first 3 channels."""
    g = np.load(GOLD.parent / "unet12_golden.npz")
    m = unet_ref.UNetRef(in_ch=12).eval()
    flat = unet_ref.make_params(int(g["seed"]), m)
    assert len(flat) == int(g["n_params"]) == 1949539
    assert abs(float(flat.astype(np.float64).sum()) - float(g["param_sum"])) < 1e-9
    unet_ref.load_flat(m, flat)
    with torch.no_grad():
        y = m(torch.from_numpy(g["x"])).numpy()
    assert np.abs(y - g["y"]).max() < 1e-6


def test_bf16_emulation_is_close_to_fp32():
    g = np.load(GOLD)
    m = unet_ref.load_flat(unet_ref.UNetRef().eval(), unet_ref.make_params(int(g["seed"])))
    with torch.no_grad():
        a = m(torch.from_numpy(g["x"]))
        b = unet_ref.forward_bf16(m, torch.from_numpy(g["x"]))
    assert float((a - b).abs().max()) < 0.1


def test_packaged_denoiser_weights():
    """The trained weights shipped in the package (FP16, state_dict order)
    match the 3-channel network's parameter count, are finite, and name the
    orbit poses held out of their training."""
    import pathlib
    z = np.load(pathlib.Path(__file__).resolve().parent.parent / "luminagi-cudaref_b200" / "lumina" / "data" /
                "unet_engine_long.npz")
    p = z["params"].astype(np.float32)
    assert p.shape == (1946947,) and np.isfinite(p).all() and np.abs(p).max() > 0
    assert len(z["val_idx"]) == 5 and (0 <= z["val_idx"]).all() and (z["val_idx"] < int(z["poses"])).all()
    assert int(z["in_ch"]) == 3 and bytes(z["variant"]) == b"ref"

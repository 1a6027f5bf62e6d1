"""Writes tests/golden/unet_golden.npz and unet12_golden.npz from the reference's own UNet module.

Run in a checkout that has the reference at REF (default /root/reference):
    python tests/golden/make_unet_golden.py
It imports LuminaGI-CudaRef ml/train.py, loads the seeded parameters from
oracle/unet_ref.make_params(seed) into the reference UNet and records its
output on a seeded input, so the test suite can pin oracle/unet_ref.UNetRef
to the reference module without the reference checkout.
"""
import os
import pathlib
import sys

import numpy as np
import torch

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
REF = pathlib.Path(os.environ.get("REF", "/root/reference"))
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(REF / "ml"))

import unet_ref  # noqa: E402
from train import UNet  # noqa: E402  (the reference module)

SEED = 1234
torch.manual_seed(0)
ref = UNet(base=32, in_ch=3).eval()
assert [k for k, _ in unet_ref.param_shapes(ref)] == [k for k, _ in unet_ref.param_shapes(unet_ref.UNetRef())]
flat = unet_ref.make_params(SEED, ref)
unet_ref.load_flat(ref, flat)
rng = np.random.default_rng(SEED + 1)
x = rng.uniform(0.0, 1.0, (2, 3, 16, 24)).astype(np.float32)
with torch.no_grad():
    y = ref(torch.from_numpy(x)).numpy()
np.savez_compressed(HERE / "unet_golden.npz", seed=SEED, x=x, y=y, n_params=len(flat),
                    param_sum=np.float64(flat.astype(np.float64).sum()))
print("wrote", HERE / "unet_golden.npz", "params", len(flat), "out mean", float(y.mean()))

# The 12-channel variant (train.py --gbuffer: colour + albedo + normal + position).
ref12 = UNet(base=32, in_ch=12).eval()
flat12 = unet_ref.make_params(SEED + 12, ref12)
unet_ref.load_flat(ref12, flat12)
x12 = np.random.default_rng(SEED + 13).uniform(0.0, 1.0, (2, 12, 16, 24)).astype(np.float32)
with torch.no_grad():
    y12 = ref12(torch.from_numpy(x12)).numpy()
np.savez_compressed(HERE / "unet12_golden.npz", seed=SEED + 12, x=x12, y=y12, n_params=len(flat12),
                    param_sum=np.float64(flat12.astype(np.float64).sum()))
print("wrote", HERE / "unet12_golden.npz", "params", len(flat12), "out mean", float(y12.mean()))

"""The C++ drop-in boundary: the reference's own CLI source (src/main.cpp,
unchanged) must compile against this repository's headers (include/) and
link against liblumina.so, resolving LoadSceneJSON, BuildBVH,
RenderSceneCUDA and RenderSceneCUDASorted from the library.

CPU-only: the link, the usage exit code (1) and the scene-load failure exit
code (2), which main.cpp reaches before any CUDA call.  The rendering of the
linked binary is checked on the GPU in test_dropin_render_gpu.py.  Skipped
where the reference checkout (REF, default /root/reference) is absent."""
import os
import pathlib
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
REF = pathlib.Path(os.environ.get("REF", "/root/reference"))
LIB = ROOT / "luminagi-cudaref_b200" / "lib"


@pytest.fixture(scope="module")
def linked(tmp_path_factory):
    main = REF / "src" / "main.cpp"
    if not main.exists():
        pytest.skip("reference checkout not present")
    if not (LIB / "liblumina.so").exists():
        pytest.skip("liblumina.so not built")
    out = tmp_path_factory.mktemp("dropin") / "cuda_ref_main"
    cmd = ["g++", "-O1", "-std=c++17", f"-I{ROOT / 'include'}", f"-I{REF / 'third_party'}", "-o", str(out),
           str(main), f"-L{LIB}", "-llumina", f"-Wl,-rpath,{LIB}"]
    p = subprocess.run(cmd, capture_output=True, text=True)
    assert p.returncode == 0, p.stderr[-3000:]
    return out


def test_reference_main_links_against_the_library(linked):
    syms = subprocess.run(["nm", "-DC", str(LIB / "liblumina.so")], capture_output=True, text=True).stdout
    for name in ("LoadSceneJSON(", "BuildBVH(", "RenderSceneCUDA(", "RenderSceneCUDASorted("):
        assert name in syms, name
    assert linked.exists()


def test_reference_main_usage_and_load_failure(linked, tmp_path):
    p = subprocess.run([str(linked)], capture_output=True, text=True)
    assert p.returncode == 1 and "usage:" in p.stderr
    p = subprocess.run([str(linked), str(tmp_path / "missing.json"), str(tmp_path / "out.png")],
                       capture_output=True, text=True)
    assert p.returncode == 2
    assert not (tmp_path / "out.png").exists()

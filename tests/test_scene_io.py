"""scene.json loader/writer, PNG/HDR writers and the C ABI surface, on the CPU.

The loader is checked float-bit for float-bit against what the reference's
own LoadSceneJSON produced for the committed fixtures
(tests/golden/*_ref.json, made by tests/golden/make_scene_golden.py), and
against the reference loader itself when oracle/_ref is built."""
import json
import pathlib
import re
import struct
import subprocess

import numpy as np
import pytest

import lumina
import oracle as O
from lumina import _ffi

GOLD = pathlib.Path(__file__).resolve().parent / "golden"
ROOT = pathlib.Path(__file__).resolve().parent.parent


def bits(a):
    return [struct.unpack("<I", struct.pack("<f", float(x)))[0] for x in np.asarray(a, np.float32).ravel()]


@pytest.mark.parametrize("name", ["mock_scene", "tricky_scene"])
def test_loader_matches_reference_fixture(name):
    ref = json.loads((GOLD / f"{name}_ref.json").read_text())
    s = lumina.Scene.load_json(GOLD / f"{name}.json")
    c = s.camera
    assert bits(c.pos) == ref["camera"]["pos"]
    assert bits(c.camera_to_world) == ref["camera"]["m"]
    assert bits([c.fov_y_deg]) == ref["camera"]["fov"] and bits([c.aspect]) == ref["camera"]["aspect"]
    assert bits([c.near_z]) == ref["camera"]["near"] and bits([c.far_z]) == ref["camera"]["far"]
    assert (c.width, c.height) == (ref["camera"]["w"], ref["camera"]["h"])
    assert bits(list(s.sun["dir"]) + list(s.sun["color"]) + [s.sun["intensity"]]) == ref["sun"]
    assert bits(s.tris.view(np.float32).reshape(len(s.tris), 25)[:, :24]) == ref["tris"]
    assert [int(m) for m in s.tris["material"]] == ref["mats"]
    assert bits(s.mat_albedo) == ref["albedo"] and bits(s.mat_emissive) == ref["emissive"]
    assert len(s.points) == ref["n_points"] and bits(s.points.view(np.float32)) == ref["points"]
    assert len(s.directionals) == ref["n_directionals"]
    assert bits(s.directionals.view(np.float32)) == ref["directionals"]


def test_mock_scene_bvh_pins():
    # The reference's test_bvh on scenes/mock_scene.json: 1 node, root bounds (-2,-2,0)..(2,2,5).
    ref = json.loads((GOLD / "mock_scene_ref.json").read_text())
    s = lumina.Scene.load_json(GOLD / "mock_scene.json")
    nodes, _, _, _ = O.oracle_build_bvh(s.tris)
    assert len(nodes) == ref["n_nodes"] == 1
    assert nodes.view(np.uint32).ravel().tolist() == ref["bvh_nodes"]
    assert list(nodes[0]["bbMin"]) == [-2, -2, 0] and list(nodes[0]["bbMax"]) == [2, 2, 5]


def test_texture_path_and_escapes():
    h = _ffi.C.c_void_p() if hasattr(_ffi, "C") else None
    import ctypes as C
    h = C.c_void_p()
    _ffi.check(_ffi.lib().lg_scene_load_json(str(GOLD / "tricky_scene.json").encode(), 0, 1, C.byref(h)))
    try:
        assert _ffi.lib().lg_scene_texture(h, 0) == b""
        assert _ffi.lib().lg_scene_texture(h, 1) == 'tex\\stone "a".png'.encode()
    finally:
        _ffi.lib().lg_scene_destroy(h)


def test_round_trip_and_reference_reads_our_json(tmp_path, box_scene):
    p = tmp_path / "box.json"
    box_scene.save_json(p)
    back = lumina.Scene.load_json(p, threads=4)
    assert back.tris.tobytes() == box_scene.tris.tobytes()
    assert back.mat_albedo.tobytes() == box_scene.mat_albedo.tobytes()
    assert back.points.tobytes() == box_scene.points.tobytes()
    assert np.array_equal(back.camera.camera_to_world, box_scene.camera.camera_to_world)
    if O.ref_available():
        r = O.ref_load_scene(str(p))
        assert r["tris"].tobytes() == box_scene.tris.tobytes()


def test_parallel_parse_equals_serial(tmp_path, small_engine_scene):
    p = tmp_path / "eng.json"
    small_engine_scene.save_json(p)
    a = lumina.Scene.load_json(p, threads=1)
    b = lumina.Scene.load_json(p, threads=8)
    assert a.tris.tobytes() == b.tris.tobytes() == small_engine_scene.tris.tobytes()


@pytest.mark.parametrize("text,code,needle", [
    (None, _ffi.LG_ERR_IO, "failed to open"),
    ('{"version": 1, "camera": {', _ffi.LG_ERR_PARSE, "JSON parse error"),
    ('{"version": 2}', _ffi.LG_ERR_PARSE, "unsupported version 2"),
    ('{"camera": {}}', _ffi.LG_ERR_PARSE, "unsupported version 0"),
    ('{"version": 1, "sun": {}}', _ffi.LG_ERR_PARSE, "missing key"),
    ('{"version": 1} trailing', _ffi.LG_ERR_PARSE, "JSON parse error"),
])
def test_loader_errors(tmp_path, text, code, needle):
    p = tmp_path / "bad.json"
    if text is not None:
        p.write_text(text)
    with pytest.raises(lumina.LuminaError) as e:
        lumina.Scene.load_json(p)
    assert e.value.code == code
    assert needle in str(e.value)


def test_png_and_hdr_writers(tmp_path):
    from PIL import Image
    rng = np.random.default_rng(0)
    img = rng.integers(0, 256, (37, 53, 3), dtype=np.uint8)
    p = tmp_path / "x.png"
    _ffi.check(_ffi.lib().lg_write_png(str(p).encode(), 53, 37, _ffi.ptr(img)))
    assert np.array_equal(np.asarray(Image.open(p).convert("RGB")), img)
    lin = rng.uniform(0, 4, (5, 7, 3)).astype(np.float32)
    q = tmp_path / "x.hdr"
    _ffi.check(_ffi.lib().lg_write_hdr(str(q).encode(), 7, 5, _ffi.ptr(lin)))
    data = q.read_bytes()
    hdr_end = data.index(b"-Y 5 +X 7\n") + len(b"-Y 5 +X 7\n")
    rgbe = np.frombuffer(data[hdr_end:], np.uint8).reshape(5, 7, 4).astype(np.float64)
    dec = rgbe[..., :3] * np.ldexp(1.0, (rgbe[..., 3:4] - 136).astype(int))
    # RGBE keeps 8 mantissa bits relative to the pixel's largest component.
    assert (np.abs(dec - lin) <= lin.max(axis=2, keepdims=True) / 128.0).all()


def test_look_at_matches_reference_formula():
    cam = lumina.look_at_camera([1.0, 2.0, 3.0], [4.0, -2.0, 3.5], 64, 32)
    f = np.array([3.0, -4.0, 0.5], np.float32)
    f /= np.float32(np.sqrt(np.float32(f @ f)))
    l = np.array([-f[1], f[0], 0.0], np.float32)
    l /= np.float32(np.sqrt(np.float32(l @ l)))
    m = cam.camera_to_world
    assert np.allclose(m[0:3], f, atol=1e-7) and np.allclose(m[4:7], l, atol=1e-7)
    assert np.allclose(m[8:11], np.cross(f, l), atol=1e-6) and np.allclose(m[12:15], [1, 2, 3])


def test_numpy_look_at_is_bit_identical_to_the_library():
    """The scene generators' float32 restatement of overwrite_camera equals
    lg_look_at bit for bit (so generated scenes need no CUDA library)."""
    from lumina.scene import look_at_f32
    rng = np.random.default_rng(3)
    poses = [([1.0, 2.0, 3.0], [4.0, -2.0, 3.5]), ([0, 0, 0], [0, 0, 5.0]), ([0, 0, 0], [0, 0, -1.0]),
             ([20.0, -6.0, 5.0], [0.3, 0.1, 1.7])]
    poses += [(rng.uniform(-30, 30, 3), rng.uniform(-30, 30, 3)) for _ in range(200)]
    base = lumina.Camera(np.zeros(3, np.float32), np.eye(4, dtype=np.float32).ravel(), 60.0, 2.0, 0.1, 1000.0,
                         64, 32)
    for pos, tgt in poses:
        lib_cam = base.look_at(pos, tgt)
        p, m = look_at_f32(pos, tgt, base.camera_to_world)
        assert lib_cam.camera_to_world.tobytes() == m.tobytes(), (pos, tgt)
        assert lib_cam.pos.tobytes() == p.tobytes()


def test_abi_exports_every_declared_symbol():
    header = (ROOT / "include" / "lumina.h").read_text()
    declared = set(re.findall(r"\b(lg_[a-z0-9_]+)\s*\(", header))
    assert len(declared) > 30
    exported = subprocess.run(["nm", "-D", "--defined-only", str(_ffi.LIB_PATH)], capture_output=True,
                              text=True).stdout
    names = set(re.findall(r" T (lg_[a-z0-9_]+)", exported))
    assert declared <= names, declared - names
    assert declared <= set(_ffi.SIGNATURES), declared - set(_ffi.SIGNATURES)
    lib = _ffi.lib()
    assert lib.lg_version() >= 100


def test_cli_usage_and_load_errors(tmp_path):
    cli = str(_ffi.CLI_PATH)
    r = subprocess.run([cli], capture_output=True, text=True)
    assert r.returncode == 1 and "usage:" in r.stderr
    r = subprocess.run([cli, str(tmp_path / "missing.json")], capture_output=True, text=True)
    assert r.returncode == 2 and "[scene] failed to open" in r.stderr
    bad = tmp_path / "v2.json"
    bad.write_text('{"version": 2}')
    r = subprocess.run([cli, str(bad)], capture_output=True, text=True)
    assert r.returncode == 2 and "unsupported version 2" in r.stderr


def _big_json(n, extra="", bad_at=-1, seed=0):
    """A scene.json with n triangles (a few MB, so the loader splits the array
    across threads); `extra` is spliced into every triangle object."""
    rng = np.random.default_rng(seed)
    vals = rng.uniform(-5, 5, (n, 24)).round(4)
    head = ('{"version": 1, "camera": {"pos": [0,0,1], "camera_to_world": [1,0,0,0,0,1,0,0,0,0,1,0,0,0,1,1],'
            ' "fov_y_deg": 60, "aspect": 2, "near": 0.1, "far": 100, "image_width": 64, "image_height": 32},'
            ' "sun": {"direction": [0,0,-1], "color": [1,1,1], "intensity": 1}, "lights": [],'
            ' "materials": [{"albedo": [0.5,0.5,0.5], "emissive": [0,0,0]}], "triangles": [\n')
    parts = []
    for i in range(n):
        v = vals[i]
        mat = "" if i == bad_at else ', "mat": 0'
        parts.append('{"v": [[%s,%s,%s],[%s,%s,%s],[%s,%s,%s]], "n": [[%s,%s,%s],[%s,%s,%s],[%s,%s,%s]], '
                     '"uv": [[%s,%s],[%s,%s],[%s,%s]]%s%s}' % (*v, extra, mat))
    return head + ",\n".join(parts) + "\n]}\n"


@pytest.mark.parametrize("extra", ["", ', "x": {"a": "{{{", "b": [1, {"c": "}"}]}', ', "s": "{\\"v\\": [1]}"'])
def test_split_parse_matches_serial_and_reference(tmp_path, extra):
    """The array is parsed in byte shares from guessed element starts; objects
    and braces inside elements make guesses fail, and the loader must then fall
    back to the serial scan with the same result."""
    p = tmp_path / "big.json"
    p.write_text(_big_json(24000, extra))
    assert p.stat().st_size > 4 << 20
    a = lumina.Scene.load_json(p, threads=1)
    for t in (2, 5, 8):
        b = lumina.Scene.load_json(p, threads=t)
        assert b.tris.tobytes() == a.tris.tobytes()
    assert a.n_tris == 24000
    if O.ref_available():
        assert O.ref_load_scene(str(p))["tris"].tobytes() == a.tris.tobytes()


def test_split_parse_error_message_matches_serial(tmp_path):
    p = tmp_path / "bad_big.json"
    p.write_text(_big_json(24000, bad_at=17000))
    msgs = []
    for t in (1, 8):
        with pytest.raises(lumina.LuminaError) as e:
            lumina.Scene.load_json(p, threads=t)
        msgs.append(str(e.value))
    assert msgs[0] == msgs[1] and 'missing key "mat"' in msgs[0]


def test_binary_scene_round_trip(tmp_path, small_engine_scene):
    sc = small_engine_scene
    sc2 = lumina.Scene(sc.camera, sc.sun, sc.tris, sc.mat_albedo, sc.mat_emissive, sc.points,
                       textures=["tex/a.png"] + [""] * (len(sc.mat_albedo) - 1))
    p = tmp_path / "eng.lgscene"
    sc2.save_bin(p)
    assert p.read_bytes()[:8] == b"LGSCENE1"
    back = lumina.Scene.load_json(p)
    assert back.tris.tobytes() == sc.tris.tobytes()
    assert back.mat_albedo.tobytes() == sc.mat_albedo.tobytes()
    assert back.mat_emissive.tobytes() == sc.mat_emissive.tobytes()
    assert back.points.tobytes() == sc.points.tobytes()
    assert back.sun.tobytes() == np.asarray(sc.sun).tobytes()
    assert np.array_equal(back.camera.camera_to_world, sc.camera.camera_to_world)
    assert back.camera.width == sc.camera.width and back.camera.height == sc.camera.height
    assert back.textures == sc2.textures
    # JSON and binary files of one scene load to the same arrays
    q = tmp_path / "eng.json"
    sc2.save_json(q)
    assert lumina.Scene.load_json(q).tris.tobytes() == back.tris.tobytes()
    # truncation is an error, not a short scene
    t = tmp_path / "trunc.lgscene"
    t.write_bytes(p.read_bytes()[:-100])
    with pytest.raises(lumina.LuminaError) as e:
        lumina.Scene.load_json(t)
    assert "truncated binary scene" in str(e.value)


def test_split_parse_fuzz_matches_serial(tmp_path):
    """Random byte edits inside the triangle array: the parallel split parse must
    agree with the serial parse on success, triangles and error message."""
    base = _big_json(12000).encode()
    assert len(base) > 2 << 20
    start = base.index(b'"triangles"')
    rng = np.random.default_rng(11)
    alphabet = b'{}[],:" 0123456789.-eE\\nx'
    p = tmp_path / "fuzz.json"
    outcomes = set()
    for trial in range(60):
        b = bytearray(base)
        for _ in range(int(rng.integers(1, 4))):
            pos = int(rng.integers(start, len(b)))
            op = int(rng.integers(0, 3))
            ch = alphabet[int(rng.integers(0, len(alphabet)))]
            if op == 0:
                b[pos] = ch
            elif op == 1:
                b.insert(pos, ch)
            else:
                del b[pos]
        p.write_bytes(bytes(b))
        res = []
        for t in (1, 6):
            try:
                res.append(("ok", lumina.Scene.load_json(p, threads=t).tris.tobytes()))
            except lumina.LuminaError as e:
                res.append(("err", str(e)))
        assert res[0] == res[1], (trial, res[0][0], res[1][0])
        outcomes.add(res[0][0])
    assert outcomes == {"ok", "err"}


def _number_tokens(n, seed):
    """JSON real tokens of many forms: %.9g coordinates (the writers' form),
    short and long digit strings, leading and trailing zeros, exponents inside
    and outside 1e+-22, more than 19 significant digits, signed zeros,
    subnormal and overflowing floats, and decimal halfway points between
    adjacent floats (where a second rounding would show)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        k = rng.integers(0, 10)
        x = float(rng.standard_normal() * 10.0 ** rng.integers(-8, 9))
        if k == 0:
            out.append("%.9g" % x)
        elif k == 1:
            out.append("%.17g" % x)
        elif k == 2:
            out.append("%.*f" % (int(rng.integers(1, 12)), x))
        elif k == 3:
            out.append("%.*e" % (int(rng.integers(0, 20)), x * 10.0 ** rng.integers(-40, 40)))
        elif k == 4:  # 20 to 30 significant digits
            d = str(rng.integers(1, 10)) + "".join(str(v) for v in rng.integers(0, 10, int(rng.integers(19, 30))))
            out.append(("-" if x < 0 else "") + d[:3] + "." + d[3:])
        elif k == 5:  # leading zeros in the fraction, trailing zeros after it
            out.append("%s0.%s%d%s" % ("-" if x < 0 else "", "0" * int(rng.integers(0, 25)),
                                       int(rng.integers(1, 10**6)), "0" * int(rng.integers(0, 15))))
        elif k == 6:
            out.append(rng.choice(["0.0", "-0.0", "-0.000e5", "0e-400", "1e-46", "1.4e-45", "7e-46",
                                   "3.4028235e38", "3.5e38", "1e39", "-1e300", "1.17549435e-38", "123456789012345678.5",
                                   "9007199254740993.0", "9007199254740992.0", "4.9406564584124654e-324"]))
        elif k == 7:  # halfway between two adjacent floats, printed exactly
            f = np.float32(x)
            g = np.nextafter(f, np.float32(np.inf))
            out.append("%.20e" % ((float(f) + float(g)) / 2))
        elif k == 8:
            out.append("%de%d" % (int(rng.integers(-999, 1000)), int(rng.integers(-30, 31))))
        else:
            out.append("%.*fE+%d" % (int(rng.integers(0, 6)), x, int(rng.integers(0, 25))))
    return out


def test_real_tokens_convert_as_strtod_then_float(tmp_path):
    """Every real token converts to the float nearest the correctly rounded
    double (nlohmann::json's strtod then get<float>): Python's float() is the
    correctly rounded double, numpy narrows it to float as a C cast does."""
    toks = _number_tokens(24 * 3000, 5)
    n = len(toks) // 24
    head = ('{"version": 1, "camera": {"pos": [0,0,1], "camera_to_world": [1,0,0,0,0,1,0,0,0,0,1,0,0,0,1,1],'
            ' "fov_y_deg": 60, "aspect": 2, "near": 0.1, "far": 100, "image_width": 64, "image_height": 32},'
            ' "sun": {"direction": [0,0,-1], "color": [1,1,1], "intensity": 1}, "lights": [],'
            ' "materials": [{"albedo": [0.5,0.5,0.5], "emissive": [0,0,0]}], "triangles": [\n')
    parts = []
    for i in range(n):
        t = toks[24 * i:24 * i + 24]
        parts.append('{"v": [[%s,%s,%s],[%s,%s,%s],[%s,%s,%s]], "n": [[%s,%s,%s],[%s,%s,%s],[%s,%s,%s]], '
                     '"uv": [[%s,%s],[%s,%s],[%s,%s]], "mat": 0}' % tuple(t))
    p = tmp_path / "numbers.json"
    p.write_text(head + ",\n".join(parts) + "\n]}\n")
    with np.errstate(over="ignore"):
        want = np.array([np.float32(float(s)) for s in toks[:24 * n]], np.float32)
    s = lumina.Scene.load_json(p, threads=1)
    got = s.tris.view(np.float32).reshape(n, 25)[:, :24].ravel()
    bad = np.flatnonzero(got.view(np.uint32) != want.view(np.uint32))
    assert bad.size == 0, [(toks[i], got[i], want[i]) for i in bad[:8]]
    if O.ref_available():
        ref = O.ref_load_scene(str(p))["tris"]
        assert ref.tobytes() == s.tris.tobytes()


@pytest.mark.parametrize("where,token", [("coordinate", "-1e400"), ("coordinate", "1" + "0" * 309),
                                         ("material index", "2e308"), ("skipped value", "1.5E+999")])
def test_number_overflow_rejected_as_reference(tmp_path, where, token):
    """A number whose double is not finite fails the load, with nlohmann's
    message, as the reference's LoadSceneJSON does (its parser rejects it
    wherever it stands); 3.5e38, finite as a double, loads as float inf."""
    tri = {"coordinate": '{"v": [[0,0,%s],[1,0,0],[0,1,0]], "n": [[0,0,1],[0,0,1],[0,0,1]], '
                         '"uv": [[0,0],[1,0],[0,1]], "mat": 0}' % token,
           "material index": '{"v": [[0,0,0],[1,0,0],[0,1,0]], "n": [[0,0,1],[0,0,1],[0,0,1]], '
                             '"uv": [[0,0],[1,0],[0,1]], "mat": %s}' % token,
           "skipped value": '{"v": [[0,0,0],[1,0,0],[0,1,0]], "n": [[0,0,1],[0,0,1],[0,0,1]], '
                            '"uv": [[0,0],[1,0],[0,1]], "mat": 0, "extra": %s}' % token}[where]
    head = ('{"version": 1, "camera": {"pos": [0,0,1], "camera_to_world": [1,0,0,0,0,1,0,0,0,0,1,0,0,0,1,1],'
            ' "fov_y_deg": 60, "aspect": 2, "near": 0.1, "far": 100, "image_width": 64, "image_height": 32},'
            ' "sun": {"direction": [0,0,-1], "color": [1,1,1], "intensity": 1}, "lights": [],'
            ' "materials": [{"albedo": [0.5,0.5,0.5], "emissive": [0,0,0]}], "triangles": [\n')
    p = tmp_path / "overflow.json"
    p.write_text(head + tri + "\n]}\n")
    r = subprocess.run([str(_ffi.CLI_PATH), str(p), "--spp", "1"],
                       capture_output=True, text=True)
    want = "[scene] JSON parse error: [json.exception.out_of_range.406] number overflow parsing '%s'" % token
    assert r.returncode == 2 and want in r.stderr, r.stderr
    if O.ref_available():
        assert O.ref_load_scene(str(p)) is None
    p.write_text(head + tri.replace(token, "3.5e38") + "\n]}\n")
    if where == "coordinate":
        s = lumina.Scene.load_json(p)
        assert np.isinf(s.tris["v"][0][0][2])


_UTF8_CASES = [  # (bytes inside a string, well-formed per RFC 3629)
    (b"caf\xc3\xa9", True), (b"\xe2\x82\xac", True), (b"\xf0\x9f\x98\x80", True), (b"\xef\xbf\xbf", True),
    (b"\xf4\x8f\xbf\xbf", True), (b"\xed\x9f\xbf", True), (b"\xee\x80\x80", True), (b"\xe0\xa0\x80", True),
    (b"\xc0\x80", False), (b"\xc1\xbf", False), (b"\xe0\x80\x80", False), (b"\xe0\x9f\xbf", False),
    (b"\xed\xa0\x80", False), (b"\xed\xbf\xbf", False), (b"\xf0\x8f\xbf\xbf", False), (b"\xf4\x90\x80\x80", False),
    (b"\xf5\x80\x80\x80", False), (b"\xf8\x88\x80\x80\x80", False), (b"\xff", False), (b"\x80", False),
    (b"\xbf", False), (b"\xe2\x82", False), (b"\xe2\x28\xa1", False), (b"\xc3", False), (b"\xf0\x9f\x98", False),
]


@pytest.mark.parametrize("where", ["texture path", "skipped member"])
@pytest.mark.parametrize("seq,ok", _UTF8_CASES)
def test_string_utf8_accepted_as_reference(tmp_path, where, seq, ok):
    """Strings accept exactly the well-formed UTF-8 sequences, as nlohmann's
    lexer does (the reference's loader fails on the others); an accepted
    sequence reaches the texture path byte for byte."""
    tex = b'"tex/a' + seq + b'b.png"'
    mat = b'{"albedo": [0.5,0.5,0.5], "emissive": [0,0,0]' + (b', "diffuse_tex": ' + tex if where ==
                                                              "texture path" else b"") + b"}"
    doc = (b'{"version": 1, "camera": {"pos": [0,0,1], "camera_to_world": [1,0,0,0,0,1,0,0,0,0,1,0,0,0,1,1],'
           b' "fov_y_deg": 60, "aspect": 2, "near": 0.1, "far": 100, "image_width": 64, "image_height": 32},'
           b' "sun": {"direction": [0,0,-1], "color": [1,1,1], "intensity": 1}, "lights": [],'
           + (b' "note": ' + tex + b"," if where == "skipped member" else b"")
           + b' "materials": [' + mat + b'], "triangles": [{"v": [[0,0,0],[1,0,0],[0,1,0]],'
           b' "n": [[0,0,1],[0,0,1],[0,0,1]], "uv": [[0,0],[1,0],[0,1]], "mat": 0}]}\n')
    p = tmp_path / "utf8.json"
    p.write_bytes(doc)
    import ctypes as C
    h = C.c_void_p()
    rc = _ffi.lib().lg_scene_load_json(str(p).encode(), 0, 1, C.byref(h))
    assert (rc == 0) == ok, _ffi.lib().lg_last_error()
    if ok:
        try:
            if where == "texture path":
                assert _ffi.lib().lg_scene_texture(h, 0) == b"tex/a" + seq + b"b.png"
        finally:
            _ffi.lib().lg_scene_destroy(h)
    else:
        assert b"ill-formed UTF-8" in _ffi.lib().lg_last_error() or b"unterminated" in _ffi.lib().lg_last_error()
    if O.ref_available():
        assert (O.ref_load_scene(str(p)) is not None) == ok


_CAM = ('"camera": {"pos": [0,0,1], "camera_to_world": [1,0,0,0,0,1,0,0,0,0,1,0,0,0,1,1], "fov_y_deg": 60,'
        ' "aspect": 2, "near": 0.1, "far": 100, "image_width": 64, "image_height": 32}')
_SUN = '"sun": {"direction": [0,0,-1], "color": [1,1,1], "intensity": 1}'
_MAT = '"materials": [{"albedo": [0.5,0.5,0.5], "emissive": [0,0,0]}]'
_TRI = '{"v": [[0,0,0],[1,0,0],[0,1,0]], "n": [[0,0,1],[0,0,1],[0,0,1]], "uv": [[0,0],[1,0],[0,1]], "mat": 0}'


def _doc(tris=_TRI, extra="", head=b"", tail=b""):
    body = '{"version": 1, %s, %s, "lights": [], %s%s, "triangles": [%s]}' % (_CAM, _SUN, _MAT, extra, tris)
    return head + body.encode() + tail


def _many(n, sep=", "):
    return sep.join([_TRI] * n)


# (name, document, the reference's LoadSceneJSON accepts it)
_DOCS = [
    ("plain", _doc(), True),
    ("byte-order mark", _doc(head=b"\xef\xbb\xbf"), True),
    ("text after the object (f >> j reads one value)", _doc(tail=b" x {"), True),
    ("second object after the first", _doc(tail=b" {}"), True),
    ("duplicate triangles key: last wins", _doc()[:-1] + b', "triangles": []}', True),
    ("lone low surrogate escape", _doc(extra=', "x": "\\udc00"'), False),
    ("lone high surrogate escape", _doc(extra=', "x": "\\ud800x"'), False),
    ("escaped NUL", _doc(extra=', "x": "\\u0000"'), True),
    ("form feed as whitespace", _doc(extra=',\f"x": 1'), False),
    ("skipped member: empty array element", _doc(extra=', "x": [1,,2]'), False),
    ("skipped member: missing colon", _doc(extra=', "x": {"a" 1}'), False),
    ("skipped member: trailing comma", _doc(extra=', "x": [1,2,]'), False),
    ("skipped member: bad literal", _doc(extra=', "x": [tru]'), False),
    ("skipped member: mismatched bracket", _doc(extra=', "x": {"a": [1}'), False),
    ("skipped member: 5,000 levels deep", _doc(extra=', "x": ' + "[" * 5000 + "]" * 5000), True),
    ("triangles: missing comma", _doc(_TRI + " " + _TRI), False),
    ("triangles: trailing comma", _doc(_TRI + ","), False),
    ("triangles: double comma", _doc(_TRI + ",," + _TRI), False),
    ("triangle with a malformed extra member", _doc(_TRI.replace('"mat": 0', '"mat": 0, "q": [1 2]')), False),
    ("triangle with a nested extra member", _doc(_TRI.replace('"mat": 0', '"mat": 0, "q": {"z": [1, "s", null]}')),
     True),
    ("lights: trailing comma", _doc().replace(b'"lights": []', b'"lights": [1,]'), False),
    ("30,000 triangles", _doc(_many(30000)), True),
    ("30,000 triangles, missing comma in the middle", _doc(_many(15000) + " " + _many(15000)), False),
    ("30,000 triangles, trailing comma", _doc(_many(30000) + ","), False),
    ("30,000 triangles, malformed extra member in the middle",
     _doc(_many(15000) + ", " + _TRI.replace('"mat": 0', '"mat": 0, "q": [1,,2]') + ", " + _many(15000)), False),
    ("30,000 triangles, element-like text inside a string",
     _doc(_many(15000) + ", " + _TRI.replace('"mat": 0', '"mat": 0, "q": "}, {\\"v\\": ["') + ", " + _many(15000)),
     True),
]


@pytest.mark.parametrize("name,doc,ok", _DOCS, ids=[d[0] for d in _DOCS])
def test_document_accepted_as_reference(tmp_path, name, doc, ok):
    """Which documents load: the reference's LoadSceneJSON (nlohmann's
    non-strict `f >> j`, scene_loader.cpp:38) decides, on the serial path and
    on the parallel triangle parse (30,000 triangles span several 1 MB
    shares)."""
    import ctypes as C
    p = tmp_path / "doc.json"
    p.write_bytes(doc)
    for threads in (1, 8):
        h = C.c_void_p()
        rc = _ffi.lib().lg_scene_load_json(str(p).encode(), 0, threads, C.byref(h))
        if rc == 0:
            _ffi.lib().lg_scene_destroy(h)
        assert (rc == 0) == ok, (threads, _ffi.lib().lg_last_error())
    if ok:
        s = lumina.Scene.load_json(p)
        assert s.n_tris == (0 if "duplicate" in name else doc.count(b'"mat": 0'))
    if O.ref_available():
        r = O.ref_load_scene(str(p))
        assert (r is not None) == ok
        if ok:
            assert r["tris"].tobytes() == s.tris.tobytes()


_PL = '{"type": "point", "pos": [0,0,3], "color": [1,1,1], "intensity": %d, "radius": 10}'
_T_AT = lambda z: _TRI.replace("[0,0,0],[1,0,0]", "[0,0,%d],[1,0,0]" % z)


def _doc_with(lights="[]", mats=None, tris=None):
    mats = mats if mats is not None else '[{"albedo": [0.5,0.5,0.5], "emissive": [0,0,0]}]'
    tris = tris if tris is not None else "[" + _TRI + "]"
    return ('{"version": 1, %s, %s, "lights": %s, "materials": %s, "triangles": %s}'
            % (_CAM, _SUN, lights, mats, tris)).encode()


# (name, document, point intensities, material albedo reds, first-vertex z per triangle), as the reference loads them
_VALUE_FORMS = [
    ("lights as an object: values in key order", _doc_with('{"b": %s, "a": %s}' % (_PL % 5, _PL % 7)),
     [7, 5], [0.5], [0]),
    ("lights object with duplicate keys: the last kept", _doc_with('{"b": %s, "b": %s, "B": %s}' % (_PL % 5, _PL % 7, _PL % 3)),
     [3, 7], [0.5], [0]),
    ("lights null", _doc_with("null"), [], [0.5], [0]),
    ("materials as an object, keys compared as bytes",
     _doc_with(mats='{"z": {"albedo": [0.5,0.5,0.5], "emissive": [0,0,0]}, "\\u00e9": {"albedo": [0.25,0.2,0.3],'
                    ' "emissive": [0,0,0]}, "a": {"albedo": [0.75,0.7,0.7], "emissive": [0,0,0]}}'),
     [], [0.75, 0.5, 0.25], [0]),
    ("materials null", _doc_with(mats="null"), [], [], [0]),
    ("triangles as an object", _doc_with(tris='{"t2": %s, "t10": %s, "t1": %s}' % (_T_AT(2), _T_AT(10), _T_AT(1))),
     [], [0.5], [1, 10, 2]),
    ("triangles null", _doc_with(tris="null"), [], [0.5], []),
]


@pytest.mark.parametrize("name,doc,points,reds,zs", _VALUE_FORMS, ids=[v[0] for v in _VALUE_FORMS])
def test_lights_materials_triangles_objects_and_null_as_reference(tmp_path, name, doc, points, reds, zs):
    """The reference's range-for over `j.at("lights")` (and materials,
    triangles) visits an object's values in its std::map's key order, keeping
    the last of duplicate keys, and nothing for null; this loader does the
    same."""
    p = tmp_path / "forms.json"
    p.write_bytes(doc)
    s = lumina.Scene.load_json(p)
    assert s.points["intensity"].tolist() == points
    assert s.mat_albedo[:, 0].tolist() == reds
    assert s.tris["v"][:, 0, 2].tolist() == zs
    if O.ref_available():
        r = O.ref_load_scene(str(p))
        assert r["tris"].tobytes() == s.tris.tobytes() and r["points"].tobytes() == s.points.tobytes()
        assert r["albedo"].tobytes() == s.mat_albedo.tobytes()

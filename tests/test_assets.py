"""Asset path: OBJ/MTL, PLY and EXR loaders and the reference's built-in scenes.

Pinned against the reference's own readers (src/parsers/*.cpp and its vendored tinyexr
LoadEXR, compiled for the host as oracle/_ref/libref_assets.so) on the reference's scene
files, where that tree is present. The synthetic cases below need neither and cover the
parser rules one by one: the accepted OBJ face forms, MTL order, PLY layouts, and every EXR
compression the reader handles except PIZ (pinned by the reference's own PIZ file)."""
import glob
import os
import struct
import zlib

import numpy as np
import pytest

import oracle as orc
import pathed

SCENES = os.path.join(orc.REF_TREE, "scenes")
HAVE_REF = os.path.isdir(SCENES) and os.path.exists(orc.REF_ASSETS_LIB)
needs_ref = pytest.mark.skipif(not HAVE_REF, reason="reference scene files or libref_assets.so absent")
CAM = [0, 1, 6.8, 0, 1, 0, 0, 1, 0, 0.34, 0]


def _load(files, mats=(0,), **kw):
    s = pathed.Session(8, 8)
    s.load_request(files, list(mats), CAM, **kw)
    e = s.export_scene()
    s.close()
    return e


@needs_ref
def test_mesh_files_match_reference_parsers():
    R = orc.RefAssets()
    files = sorted(glob.glob(os.path.join(SCENES, "*", "*.obj")) + glob.glob(os.path.join(SCENES, "*", "*.ply")))
    assert len(files) >= 10
    for f in files:
        ply = f.endswith(".ply")
        r = R.mesh(f, ply)
        e = _load([(f, pathed.MESH_PLY if ply else pathed.MESH_OBJ, 0)])
        assert np.array_equal(e["tri_vertices"].reshape(-1, 9), r["p"]), f
        assert np.array_equal(e["tri_normals"].reshape(-1, 9), np.where(np.isfinite(r["n"]), r["n"], 0)), f
        # MTL materials follow the request's one material, in the reference's order
        want = 1 + r["mtl"] if len(r["mtls"]) else np.zeros_like(r["mtl"])
        assert np.array_equal(e["tri_materials"], want), f
        assert np.array_equal(e["material_albedo"][1:], r["mtls"][:, :3]), f
        assert np.array_equal(e["material_emit"][1:], r["mtls"][:, 3:]), f


@needs_ref
@pytest.mark.parametrize("name", ["1_pixel_test.exr", "20060807_wells6_hd.exr"])  # PIZ and ZIP
def test_exr_matches_reference_loader(name):
    f = os.path.join(SCENES, "assets", name)
    ref = orc.RefAssets().exr(f)
    ours = pathed.read_exr(f)
    assert ours.shape == ref.shape and np.array_equal(ours, ref)


@pytest.mark.skipif(not os.path.exists(orc.REF_ASSETS_LIB), reason="libref_assets.so absent")
@pytest.mark.parametrize("w,h,half,smooth", [(37, 23, True, True), (203, 70, False, False), (64, 33, True, False),
                                              (5, 130, False, True)])
def test_piz_files_written_by_tinyexr(tmp_path, w, h, half, smooth):
    """PIZ blocks of every wavelet depth: odd and even sizes, HALF and FLOAT words, smooth
    data (few distinct words: the exact 14-bit pair rule) and noise (more than 2^14 distinct
    words in a block: the modulo rule), written by the reference's tinyexr and read back by
    both loaders"""
    rng = np.random.default_rng(w * 1000 + h)
    if smooth:
        y, x = np.mgrid[0:h, 0:w]
        planes = np.stack([np.sin(x / 7.0 + c) * np.cos(y / 5.0) + 1.5 for c in range(3)]).astype(np.float32)
    else:
        planes = rng.lognormal(0.0, 2.0, (3, h, w)).astype(np.float32)
    f = str(tmp_path / "piz.exr")
    R = orc.RefAssets()
    R.exr_save_piz(f, planes, b"BGR", half=half)
    ref = R.exr(f)
    ours = pathed.read_exr(f)
    assert ours.shape == ref.shape == (h, w, 4)
    assert np.array_equal(ours, ref)
    if not half:
        assert np.array_equal(ours[..., 2], planes[0]) and np.array_equal(ours[..., 0], planes[2])


@needs_ref
def test_reference_scenes_assemble_as_scene_cu():
    """SceneParameters::getSceneData / getCamera (src/scene.cu:14-218) over the reference's parsers"""
    R = orc.RefAssets()
    expect = {
        0: (["cornell-box/CornellBox-Original.obj"], [], 1, 0),
        1: (["cornell-glossy/CornellBox-Glossy.obj", "cornell-glossy/box.obj"], [], 3, 1),
        2: (["tests/plane.obj"], [], 1, 0),
        3: ([], ["mis/floor.ply", "mis/plate1.ply", "mis/plate2.ply", "mis/plate3.ply", "mis/plate4.ply"], 10, 5),
    }
    for idx, (objs, plys, nreq, nsph) in expect.items():
        s = pathed.Session(64, 48)
        s.load_reference_scene(idx, SCENES)
        e, c = s.export_scene(), s.counts()
        parts = [R.mesh(os.path.join(SCENES, f)) for f in objs] + [R.mesh(os.path.join(SCENES, f), True)
                                                                     for f in plys]
        assert np.array_equal(e["tri_vertices"].reshape(-1, 9), np.concatenate([p["p"] for p in parts]))
        assert c.num_spheres == nsph
        assert c.num_materials == nreq + sum(len(p["mtls"]) for p in parts)
        # emitters: triangles with an emitting material, then emitting spheres
        emit = np.abs(e["material_emit"]).sum(1) > 0
        want = [(0, i) for i, m in enumerate(e["tri_materials"]) if emit[m]] + \
               [(1, i) for i, m in enumerate(e["sphere_materials"]) if emit[m]]
        assert list(zip(e["light_types"], e["light_indices"])) == want
        assert (len(want) > 0) == (idx != 2)  # scene 2 is lit by its environment only
        assert (c.default_depth, c.default_nee) == (3, 1)  # Scene's defaults (include/scene.h:17-29)
        s.close()
    # cameras (getCamera): scenes 0-2 share one, scene 3 is flipped with its own vertical FOV
    s = pathed.Session(64, 48)
    s.load_reference_scene(3, SCENES)
    cam = s.export_scene()["camera"]
    fov = np.float32(np.float32(28.0000262073138) / np.float32(180.0))  # float division, then * M_PI
    assert cam[10] == 1 and cam[9] == np.float32(float(fov) * np.pi)
    assert s.counts().env_width == 1000 and s.counts().env_height == 500
    s.close()


def test_obj_face_forms_and_mtl_order(tmp_path):
    (tmp_path / "m.mtl").write_text("newmtl zeta\nKd 0.1 0.2 0.3\n\nnewmtl alpha\n  Kd 0.4 0.5 0.6\nKe 1 2 3\n"
                                    "Ns 10\nillum 2\n")
    (tmp_path / "a.obj").write_text(
        "# comment\nmtllib m.mtl\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv  0 1   0\nvn 0 0 1\nvt 0 0\n"
        "f 1 2 3\n"                  # a plain triangle: no reference pattern matches, skipped
        "usemtl zeta\nf 1 2 3 4\n"   # quad: two triangles with the geometric normal
        "usemtl nosuch\nf -4//1 -3//1 -2//1\n"  # unknown material name: index 0
        "usemtl alpha\nf 1/1/1 2/1/1 4/1/1 \n"
        "f 1/1/1  2/1/1 4/1/1\n")    # two spaces between groups: skipped
    e = _load([(str(tmp_path / "a.obj"), pathed.MESH_OBJ, 0)], mats=(0, 1))
    p = e["tri_vertices"].reshape(-1, 3, 3)
    assert p.shape[0] == 4
    assert np.array_equal(p[0], [[0, 0, 0], [1, 0, 0], [1, 1, 0]]) and np.array_equal(p[1], [[0, 0, 0], [1, 1, 0],
                                                                                            [0, 1, 0]])
    assert np.array_equal(p[3], [[0, 0, 0], [1, 0, 0], [0, 1, 0]])
    assert np.array_equal(e["tri_normals"].reshape(-1, 3, 3), np.tile([0, 0, 1], (4, 3, 1)).astype(np.float32))
    # MTL materials sorted by name after the request's two: alpha = 2, zeta = 3
    assert list(e["tri_materials"]) == [3, 3, 2, 2]
    assert np.allclose(e["material_albedo"][2:], [[0.4, 0.5, 0.6], [0.1, 0.2, 0.3]])
    assert np.allclose(e["material_emit"][2:], [[1, 2, 3], [0, 0, 0]])
    assert e["light_types"].size == 2  # the two triangles of the emitting alpha material


def test_obj_errors_and_missing_library(tmp_path):
    (tmp_path / "b.obj").write_text("mtllib none.mtl\nusemtl x\nv 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\nf 1 2 3 4\n")
    e = _load([(str(tmp_path / "b.obj"), pathed.MESH_OBJ, 1)], mats=(0, 0))
    assert list(e["tri_materials"]) == [1, 1]  # no MTL materials: the file's default material
    (tmp_path / "c.obj").write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3 9\n")
    with pytest.raises(pathed.PathedError, match="out of range"):
        _load([(str(tmp_path / "c.obj"), pathed.MESH_OBJ, 0)])
    (tmp_path / "d.obj").write_text("v 0 0\n")
    with pytest.raises(pathed.PathedError, match="d.obj:1"):
        _load([(str(tmp_path / "d.obj"), pathed.MESH_OBJ, 0)])
    with pytest.raises(pathed.PathedError, match="cannot read"):
        _load([(str(tmp_path / "missing.obj"), pathed.MESH_OBJ, 0)])
    with pytest.raises(pathed.PathedError, match="default material"):
        _load([(str(tmp_path / "b.obj"), pathed.MESH_OBJ, 5)])
    # coincident corners: the reference's 0/0 normal becomes zero, the face is kept
    (tmp_path / "e.obj").write_text("v 0 0 0\nv 1 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3 4\n")
    e = _load([(str(tmp_path / "e.obj"), pathed.MESH_OBJ, 0)])
    n = e["tri_normals"].reshape(-1, 9)
    assert n.shape[0] == 2 and np.all(n[0] == 0) and np.array_equal(n[1], [0, 0, 1] * 3)


def _ply(path, verts, faces, extra_vertex_prop=False, index_type="int", count_type="uchar", fmt="binary_little_endian"):
    props = "property float x\nproperty float y\nproperty float z\n" + ("property uchar red\n" if extra_vertex_prop else "")
    head = (f"ply\nformat {fmt} 1.0\ncomment synthetic\nelement vertex {len(verts)}\n{props}"
            f"element face {len(faces)}\nproperty list {count_type} {index_type} vertex_indices\nend_header\n")
    body = b""
    for v in verts:
        body += struct.pack("<3f", *v) + (b"\x07" if extra_vertex_prop else b"")
    ic = {"int": "i", "uint": "I", "short": "h"}[index_type]
    cc = {"uchar": "B", "ushort": "H"}[count_type]
    for f in faces:
        body += struct.pack("<" + cc, len(f)) + struct.pack("<%d%s" % (len(f), ic), *f)
    path.write_bytes(head.encode() + body)


def test_ply_layouts(tmp_path):
    verts = [(0, 0, 0), (2, 0, 0), (2, 1, 0), (0, 1, 0), (0, 0, 3)]
    _ply(tmp_path / "a.ply", verts, [(0, 1, 2), (0, 2, 3, 4)], extra_vertex_prop=True)
    e = _load([(str(tmp_path / "a.ply"), pathed.MESH_PLY, 0)])
    p = e["tri_vertices"].reshape(-1, 3, 3)
    assert p.shape[0] == 3  # the quad becomes a fan of two triangles
    assert np.array_equal(p[2], np.array([verts[0], verts[3], verts[4]], np.float32))
    assert np.array_equal(e["tri_normals"].reshape(-1, 9)[0], [0, 0, 1] * 3)
    _ply(tmp_path / "b.ply", verts, [(0, 1, 2)], index_type="uint", count_type="ushort")
    assert _load([(str(tmp_path / "b.ply"), pathed.MESH_PLY, 0)])["tri_vertices"].size == 9
    _ply(tmp_path / "c.ply", verts, [(0, 1, 7)])
    with pytest.raises(pathed.PathedError, match="out of range"):
        _load([(str(tmp_path / "c.ply"), pathed.MESH_PLY, 0)])
    _ply(tmp_path / "d.ply", verts, [(0, 1, 2)], fmt="ascii")
    with pytest.raises(pathed.PathedError, match="binary_little_endian"):
        _load([(str(tmp_path / "d.ply"), pathed.MESH_PLY, 0)])
    (tmp_path / "e.ply").write_bytes((tmp_path / "a.ply").read_bytes()[:-5])
    with pytest.raises(pathed.PathedError, match="truncated"):
        _load([(str(tmp_path / "e.ply"), pathed.MESH_PLY, 0)])


# ---- a small OpenEXR writer (scanline, NONE / RLE / ZIPS / ZIP) for the reader's tests --------
def _attr(name, typ, data):
    return name.encode() + b"\0" + typ.encode() + b"\0" + struct.pack("<i", len(data)) + data


def _rle(b):
    out, i = bytearray(), 0
    while i < len(b):
        j = i
        while j < len(b) and j - i < 128 and b[j] == b[i]:
            j += 1
        if j - i >= 3:
            out += struct.pack("<b", j - i - 1) + b[i:i + 1]
            i = j
        else:
            k = i
            while k < len(b) and k - i < 127 and not (k + 2 < len(b) and b[k] == b[k + 1] == b[k + 2]):
                k += 1
            out += struct.pack("<b", -(k - i)) + b[i:k]
            i = k
    return bytes(out)


def write_exr(path, chans, types, compression):
    names = sorted(chans)
    h, w = chans[names[0]].shape
    chl = b"".join(n.encode() + b"\0" + struct.pack("<iB3xii", types[n], 0, 1, 1) for n in names) + b"\0"
    box = struct.pack("<4i", 0, 0, w - 1, h - 1)
    head = (struct.pack("<II", 20000630, 2) + _attr("channels", "chlist", chl) +
            _attr("compression", "compression", bytes([compression])) + _attr("dataWindow", "box2i", box) +
            _attr("displayWindow", "box2i", box) + _attr("lineOrder", "lineOrder", b"\0") +
            _attr("pixelAspectRatio", "float", struct.pack("<f", 1)) +
            _attr("screenWindowCenter", "v2f", struct.pack("<2f", 0, 0)) +
            _attr("screenWindowWidth", "float", struct.pack("<f", 1)) + b"\0")
    lpc = {0: 1, 1: 1, 2: 1, 3: 16}[compression]
    chunks, raw_chunks = [], 0
    for y0 in range(0, h, lpc):
        raw = b"".join(chans[n][y].astype(np.float16 if types[n] == 1 else np.float32).tobytes()
                       for y in range(y0, min(h, y0 + lpc)) for n in names)
        data = raw
        if compression:
            t = np.frombuffer(raw[0::2] + raw[1::2], np.uint8).astype(np.int32)
            d = t.copy()
            d[1:] = (t[1:] - t[:-1] + 128) & 255
            d = d.astype(np.uint8).tobytes()
            data = _rle(d) if compression == 1 else zlib.compress(d)
            if len(data) >= len(raw):
                data, raw_chunks = raw, raw_chunks + 1  # stored uncompressed
        chunks.append(struct.pack("<ii", y0, len(data)) + data)
    off = len(head) + 8 * len(chunks)
    table = b""
    for c in chunks:
        table += struct.pack("<Q", off)
        off += len(c)
    path.write_bytes(head + table + b"".join(chunks))
    return raw_chunks


@pytest.mark.parametrize("compression", [0, 1, 2, 3], ids=["none", "rle", "zips", "zip"])
def test_exr_reader_compressions(tmp_path, compression):
    rng = np.random.default_rng(compression)
    h, w = 37, 23
    smooth = np.add.outer(np.linspace(0, 4, h), np.linspace(0, 2, w)).astype(np.float32)
    noisy = rng.lognormal(0, 2, (h, w)).astype(np.float32)
    flat = np.full((h, w), 0.25, np.float32)
    # FLOAT RGB + HALF A; noise makes some chunks store raw bytes
    chans = {"R": smooth, "G": noisy, "B": flat, "A": smooth * 0.5}
    types = {"R": 2, "G": 2, "B": 2, "A": 1}
    write_exr(tmp_path / "a.exr", chans, types, compression)
    img = pathed.read_exr(tmp_path / "a.exr")
    assert img.shape == (h, w, 4)
    for k, n in enumerate("RGB"):
        assert np.array_equal(img[..., k], chans[n])
    assert np.array_equal(img[..., 3], (smooth * 0.5).astype(np.float16).astype(np.float32))
    # RGB without alpha: A = 1; a single channel fills all four
    write_exr(tmp_path / "b.exr", {"R": flat, "G": flat, "B": noisy}, {"R": 1, "G": 1, "B": 2}, compression)
    assert np.all(pathed.read_exr(tmp_path / "b.exr")[..., 3] == 1)
    write_exr(tmp_path / "c.exr", {"Y": noisy}, {"Y": 2}, compression)
    assert np.array_equal(pathed.read_exr(tmp_path / "c.exr"), np.repeat(noisy[..., None], 4, -1))


def test_exr_reader_errors(tmp_path):
    f = np.ones((4, 4), np.float32)
    write_exr(tmp_path / "a.exr", {"R": f, "G": f}, {"R": 2, "G": 2}, 0)
    with pytest.raises(pathed.PathedError, match="B channel"):
        pathed.read_exr(tmp_path / "a.exr")
    write_exr(tmp_path / "b.exr", {"R": f, "G": f, "B": f}, {"R": 2, "G": 2, "B": 2}, 3)
    b = bytearray((tmp_path / "b.exr").read_bytes())
    (tmp_path / "c.exr").write_bytes(bytes(b[:-3]))
    with pytest.raises(pathed.PathedError):
        pathed.read_exr(tmp_path / "c.exr")
    b[4:8] = struct.pack("<I", 2 | 0x200)  # tiled flag
    (tmp_path / "d.exr").write_bytes(bytes(b))
    with pytest.raises(pathed.PathedError, match="tiled"):
        pathed.read_exr(tmp_path / "d.exr")
    with pytest.raises(pathed.PathedError, match="cannot read"):
        pathed.read_exr(tmp_path / "none.exr")


def _file_scene(tmp_path):
    """an OBJ room with an MTL emitter, a PLY mesh, a sphere and an EXR environment"""
    (tmp_path / "r.mtl").write_text("newmtl wall\nKd 0.7 0.6 0.5\nnewmtl lamp\nKd 0 0 0\nKe 8 8 6\n")
    (tmp_path / "r.obj").write_text(
        "mtllib r.mtl\nusemtl wall\n"
        "v -2 0 -2\nv 2 0 -2\nv 2 0 2\nv -2 0 2\nf -1 -2 -3 -4\n"
        "v -2 0 -2\nv -2 3 -2\nv 2 3 -2\nv 2 0 -2\nf -4 -3 -2 -1\n"
        "usemtl lamp\nv -0.5 2.9 -0.5\nv 0.5 2.9 -0.5\nv 0.5 2.9 0.5\nv -0.5 2.9 0.5\nf -1 -2 -3 -4\n")
    verts = [(-0.6, 0.2, 0.0), (0.0, 1.4, 0.3), (0.7, 0.2, -0.2), (0.0, 0.3, 0.9)]
    _ply(tmp_path / "m.ply", verts, [(0, 1, 2), (0, 3, 1), (2, 1, 3)])
    rng = np.random.default_rng(3)
    env = rng.lognormal(-1, 1, (16, 32)).astype(np.float32)
    write_exr(tmp_path / "e.exr", {"R": env, "G": env * 0.8, "B": env * 0.6}, {"R": 2, "G": 2, "B": 2}, 3)
    files = [(str(tmp_path / "r.obj"), pathed.MESH_OBJ, 0), (str(tmp_path / "m.ply"), pathed.MESH_PLY, 1)]
    kw = dict(material_albedo=[[0.5, 0.5, 0.5], [0, 0, 0], [0, 0, 0]], material_ior=[1, 1, 1.5],
              material_alpha=[0.1, 0.2, 0.1], spheres=[[1.2, 0.5, 0.8, 0.45]], sphere_materials=[2],
              env_exr=str(tmp_path / "e.exr"))
    return files, [0, 3, 2], kw


def test_request_scene_host_side(tmp_path):
    files, types, kw = _file_scene(tmp_path)
    e = _load(files, mats=types, **kw)
    assert e["tri_materials"].size == 6 + 3
    assert list(e["material_types"]) == [0, 3, 2, 0, 0]  # request materials, then MTL lamp, wall
    assert list(e["tri_materials"][:6]) == [4, 4, 4, 4, 3, 3] and list(e["tri_materials"][6:]) == [1, 1, 1]
    assert e["env_rgba"].shape == (16, 32, 4)


@pytest.mark.gpu
def test_request_scene_renders_as_its_arrays(tmp_path):
    """a scene loaded from files renders bit-identically to the same scene given as arrays"""
    files, types, kw = _file_scene(tmp_path)
    a = pathed.Session(96, 64)
    a.load_request(files, types, [0, 1.5, 6, 0, 1, 0, 0, 1, 0, 0.7, 0], **kw)
    a.set_max_depth(5)
    e = a.export_scene()
    b = pathed.Session(96, 64)
    b.load_arrays(tri_vertices=e["tri_vertices"], tri_normals=e["tri_normals"], tri_materials=e["tri_materials"],
                  spheres=e["spheres"], sphere_materials=e["sphere_materials"], material_types=e["material_types"],
                  material_albedo=e["material_albedo"], material_emit=e["material_emit"],
                  material_ior=e["material_ior"], material_alpha=e["material_alpha"], env_rgba=e["env_rgba"])
    b.set_camera(e["camera"][0:3], e["camera"][3:6], e["camera"][6:9], float(e["camera"][9]), bool(e["camera"][10]))
    b.set_max_depth(5)
    imgs = []
    for s in (a, b):
        s.set_seed(9)
        for _ in range(3):
            s.render(8)
        imgs.append(s.readback())
        s.close()
    assert np.isfinite(imgs[0]).all() and imgs[0].mean() > 0
    assert np.array_equal(imgs[0], imgs[1])


@needs_ref
def test_module_loads_reference_scene():
    """path_tracer.RenderSession.load_reference_scene: the reference GUI's scene 0 path"""
    import path_tracer as ptm

    s = ptm.RenderSession(64, 48)
    s.load_reference_scene(0, SCENES)
    m = s.getSceneModel()
    assert m.getMaxDepth() == 3 and m.getNextEventEstimation()
    o = m.getCameraOrigin()
    assert (o.x(), o.y(), o.z()) == (0.0, 1.0, np.float32(6.8))
    with pytest.raises(RuntimeError):
        s.load_reference_scene(4, SCENES)


def _exr_specials():
    # rounding ties (away from zero in the vendored writer), half subnormals, overflow, inf, NaN
    return np.array([0, -0.0, 1e-8, 6e-8, 3e-5, 65504, 65519, 65520, 1e6, -2.5, np.inf, np.nan,
                     1 + 2 ** -11, 1 + 3 * 2 ** -11, 2 ** -24 * 1.5, 2 ** -14 * (1 + 2 ** -11)], np.float32)


@needs_ref
@pytest.mark.parametrize("shape", [(7, 11), (64, 96), (1, 1), (300, 17)])
def test_exr_writer_matches_image_save(tmp_path, shape):
    """pt_write_exr writes the same bytes as the reference's Image::save (src/io/image.cpp)"""
    rng = np.random.default_rng(shape[0])
    rgb = rng.lognormal(0, 3, shape + (3,)).astype(np.float32)
    sp = _exr_specials()
    rgb.reshape(-1)[:min(sp.size, rgb.size)] = sp[:rgb.size]
    pathed.write_exr(tmp_path / "ours.exr", rgb)
    orc.RefAssets().image_save(tmp_path / "ref.exr", rgb)
    assert (tmp_path / "ours.exr").read_bytes() == (tmp_path / "ref.exr").read_bytes()


def test_exr_writer_round_trip(tmp_path):
    rng = np.random.default_rng(5)
    rgb = rng.lognormal(0, 2, (13, 9, 3)).astype(np.float32)
    # move exact half-way values off the tie (the writer rounds ties away from zero, numpy to
    # even; ties are pinned byte for byte against Image::save above)
    tie = (rgb.view(np.uint32) & 0x1FFF) == 0x1000
    rgb[tie] = np.nextafter(rgb[tie], np.float32(np.inf))
    pathed.write_exr(tmp_path / "a.exr", rgb)
    img = pathed.read_exr(tmp_path / "a.exr")
    assert img.shape == (13, 9, 4) and np.all(img[..., 3] == 1)
    # HALF channels, top row first: the buffer's row 0 (image bottom) is the file's last row
    assert np.array_equal(img[::-1, :, :3], rgb.astype(np.float16).astype(np.float32))
    with pytest.raises(pathed.PathedError):
        pathed.write_exr(tmp_path / "missing_dir" / "a.exr", rgb)


@pytest.mark.gpu
def test_snapshots_at_powers_of_two(tmp_path):
    """RenderSession's out.exr at every power-of-two spp (render_session.h:87-101)"""
    import path_tracer as ptm

    rs = ptm.RenderSession(48, 32)
    rs.init()
    path = str(tmp_path / "out.exr")
    rs.setSnapshotPath(path)
    spp, written = [], []
    for _ in range(6):
        rs.renderAsync()
        while rs.pollRender().isRendering:
            pass
        spp.append(rs.getSceneModel().getSpp())
        written.append(rs.snapshots)
    crossings = sum(any(s >= t > p for t in (2 ** k for k in range(1, 21))) for p, s in zip([0] + spp, spp))
    assert written[-1] == crossings and crossings >= 1
    # the last snapshot holds the radiance buffer of the frame that crossed a threshold
    last = max(i for i in range(len(spp)) if written[i] > (written[i - 1] if i else 0))
    if last == len(spp) - 1:
        img = pathed.read_exr(path)
        want = rs.getRadianceBuffer().astype(np.float16).astype(np.float32)
        assert np.allclose(img[::-1, :, :3], want, rtol=1e-3, atol=0)
    rs.setSnapshotPath("")
    s = pathed.Session(32, 24)
    s.load_config(0)
    s.render(4)
    s.save_exr(tmp_path / "s.exr")
    assert np.allclose(pathed.read_exr(tmp_path / "s.exr")[::-1, :, :3], s.readback(), rtol=1e-3)
    s.close()

"""Host-side I/O: FileImagePlane::Finalize and the headless image writers of
the C library, and the OBJ/MTL reader (no GPU needed)."""
import numpy as np
import pytest

from banshee_b200 import abi


def _accum(h=5, w=7, seed=0):
    rng = np.random.default_rng(seed)
    a = np.zeros((h, w, 4), np.float32)
    a[..., 3] = rng.integers(1, 9, size=(h, w))
    a[..., :3] = (rng.random((h, w, 3)) * 2.0).astype(np.float32) * a[..., 3:4]
    return a


def test_finalize_is_fileimageplane_finalize():
    from banshee_b200 import capi
    a = _accum()
    got = capi.image_finalize(a)
    want = np.power(a[..., :3] / a[..., 3:4], np.float32(1.0 / 2.2)).astype(np.float32)
    np.testing.assert_allclose(got, want, rtol=2e-6)


def test_pfm_and_ppm_writers(tmp_path):
    from banshee_b200 import capi
    a = _accum()
    h, w = a.shape[:2]
    fin = capi.image_finalize(a)
    p = tmp_path / "img.pfm"
    capi.image_write(p, a)
    raw = p.read_bytes()
    head = b"PF\n%d %d\n-1.0\n" % (w, h)
    assert raw.startswith(head)
    data = np.frombuffer(raw[len(head):], dtype="<f4").reshape(h, w, 3)
    assert (data == fin).all()                      # PFM scanlines bottom-up = buffer order
    q = tmp_path / "img.ppm"
    capi.image_write(q, a)
    raw = q.read_bytes()
    head = b"P6\n%d %d\n255\n" % (w, h)
    assert raw.startswith(head)
    px = np.frombuffer(raw[len(head):], dtype=np.uint8).reshape(h, w, 3)
    want = (np.clip(fin[::-1], 0, 1) * np.float32(255) + np.float32(0.5)).astype(np.uint8)
    assert (px == want).all()
    with pytest.raises(capi.BansheeError):
        capi.image_write(tmp_path / "img.png", a)


OBJ = """# two quads: a floor and a light above it
mtllib box.mtl
v 0 0 0
v 1 0 0
v 1 0 1
v 0 0 1
v 0.25 1 0.25
v 0.75 1 0.25
v 0.75 1 0.75
v 0.25 1 0.75
vn 0 1 0
vn 0 -1 0
usemtl floor
f 1//1 4//1 3//1 2//1
usemtl light
f 5//2 6//2 7//2 8//2
"""
MTL = """newmtl floor
Kd 0.7 0.6 0.5
newmtl light
Kd 0 0 0
Ke 1 1 1
"""


def test_obj_reader_builds_lambert_and_area_lights(tmp_path, oracle_built):
    from banshee_b200 import obj
    from banshee_b200.scene import camera
    (tmp_path / "box.obj").write_text(OBJ)
    (tmp_path / "box.mtl").write_text(MTL)
    sc = obj.load_obj(str(tmp_path / "box.obj"), width=16, height=16)
    assert [m.nfaces for m in sc.meshes] == [2, 2]
    assert sc.materials[0]["type"] == abi.BG_MAT_LAMBERT
    assert sc.materials[1]["type"] == abi.BG_MAT_EMISSIVE
    assert len(sc.lights) == 2
    assert np.allclose(sc.meshes[0].vertices[sc.meshes[0].vidx[0]], [[0, 0, 0], [0, 0, 1], [1, 0, 1]])
    sc.camera = camera((0.5, 0.5, 2.5), (0.5, 0.3, 0.5), (0, 1, 0), 0.01, 100.0, 50.0, 1.0)
    img = oracle_built.Oracle(sc).render(spp=4, seed=1, maxdepth=3, nthreads=1)
    m = img[..., :3] / img[..., 3:4]
    assert np.isfinite(m).all() and m.max() > 0

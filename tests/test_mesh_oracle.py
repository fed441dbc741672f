"""The marching-tetrahedra oracle on an analytic volume (CPU): a sphere's
truncated distance in a 32^3 volume gives a closed, consistently oriented,
outward-facing mesh whose vertices lie on the sphere; the OBJ writer."""
import dataclasses

import numpy as np


def sphere_words(n, size, radius, trunc):
    vs = size / n
    c = -0.5 * size + (np.arange(n) + 0.5) * vs
    x, y, z = np.meshgrid(c, c, c, indexing="ij")
    t = np.clip((np.sqrt(x * x + y * y + z * z) - radius) / trunc, -1.0, 1.0)
    q = np.round(t * 32767.0).astype(np.int16).view(np.uint16).astype(np.uint32)
    return (q | (1 << 16)).reshape(-1), vs


def test_sphere_mesh_is_closed_and_outward(of, ora):
    cfg = dataclasses.replace(of.CONFIGS["c1"], resolution=32, size_mm=1000.0, trunc_mm=100.0)
    words, vs = sphere_words(32, 1000.0, 300.0, 100.0)
    tris, ids = ora.mesh(cfg, words)
    assert len(tris) > 1000 and np.all(np.diff(ids.astype(np.int64)) > 0)
    r = np.linalg.norm(tris.reshape(-1, 3), axis=1)
    assert np.abs(r - 300.0).max() < 0.05 * vs  # linear interpolation of a smooth field
    # every directed edge once, its reverse once: closed and consistently oriented
    key = np.round(tris / 1e-3).astype(np.int64)
    edges = {}
    for t in key:
        for a, b in ((0, 1), (1, 2), (2, 0)):
            e = (tuple(t[a]), tuple(t[b]))
            edges[e] = edges.get(e, 0) + 1
    assert all(v == 1 for v in edges.values())
    assert all((b, a) in edges for (a, b) in edges)
    # normals point away from the centre
    n = np.cross(tris[:, 1] - tris[:, 0], tris[:, 2] - tris[:, 0])
    assert np.all(np.einsum("ij,ij->i", n, tris.mean(axis=1)) > 0)


def test_unobserved_cells_give_no_triangles(of, ora):
    cfg = dataclasses.replace(of.CONFIGS["c1"], resolution=32, size_mm=1000.0, trunc_mm=100.0)
    words, _ = sphere_words(32, 1000.0, 300.0, 100.0)
    w = words.reshape(32, 32, 32).copy()
    w[:16] &= 0xFFFF  # weight 0 in the lower half
    tris, _ = ora.mesh(cfg, w.reshape(-1))
    assert len(tris) > 0 and tris[:, :, 0].min() > -0.5 * 1000.0 + 15 * 1000.0 / 32


def test_obj_writer(of, tmp_path):
    t = np.arange(18, dtype=np.float32).reshape(2, 3, 3)
    of.write_obj(tmp_path / "m.obj", t)
    lines = (tmp_path / "m.obj").read_text().splitlines()
    v = [l for l in lines if l.startswith("v ")]
    f = [l for l in lines if l.startswith("f ")]
    assert len(v) == 6 and v[0] == "v 0 1 2" and v[5] == "v 15 16 17"
    assert f == ["f 1 2 3", "f 4 5 6"]

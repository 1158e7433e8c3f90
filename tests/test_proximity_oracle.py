"""The proximity restatement (signed vertex-face and edge-edge distances) on
cases with known answers."""
import numpy as np
import pytest


def test_vertex_over_face(oracle):
    # first triangle a small one 0.05 above the second's face
    verts = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0],
                      [0.2, 0.3, 0.05], [0.25, 0.3, 0.05], [0.2, 0.35, 0.05]], np.float32)
    faces = np.array([[3, 4, 5], [0, 1, 2]], np.int32)
    r = oracle.proximity([[0, 1]], faces, verts, h=0.1)
    vf = r[r["kind"] == 0]
    assert sorted(vf["fa"]) == [0, 1, 2] and (r["kind"] == 0).sum() == len(r)
    z = np.float64(np.float32(0.05))
    assert np.allclose(vf["dist"], z, rtol=0, atol=1e-15)
    assert np.allclose(vf["n"], [0, 0, 1], atol=1e-15)
    x, y = np.float64(np.float32(0.2)), np.float64(np.float32(0.3))
    v0 = vf[vf["fa"] == 0][0]
    assert np.allclose(v0["w"], [1, -(1 - x - y), -x, -y], atol=1e-12)
    assert len(oracle.proximity([[0, 1]], faces, verts, h=0.04)) == 0


def test_crossing_edges(oracle):
    verts = np.array([[0, 0, 0.1], [1, 0, 0.1], [0.5, -1, 0.1],
                      [0.5, -0.5, 0], [0.5, 0.5, 0], [1.5, 0, 0]], np.float32)
    faces = np.array([[0, 1, 2], [3, 4, 5]], np.int32)
    r = oracle.proximity([[0, 1]], faces, verts, h=0.2)
    e = r[(r["kind"] == 2) & (r["fa"] == 0) & (r["fb"] == 0)]
    assert len(e) == 1
    e = e[0]
    assert abs(e["dist"] - np.float64(np.float32(0.1))) < 1e-15
    assert np.allclose(e["n"], [0, 0, 1], atol=1e-15)
    assert np.allclose(e["w"], [0.5, 0.5, -0.5, -0.5], atol=1e-12)
    # the records come in the kernel's order: kinds ascending, features i-major
    key = r["kind"] * 16 + (r["fa"] + 1) * 4 + (r["fb"] + 1)
    assert np.all(np.diff(key) > 0)


def test_shared_vertices_are_skipped_in_one_mesh(oracle):
    # two triangles sharing the edge (0, 1), folded by a small angle
    verts = np.array([[0, 0, 0], [1, 0, 0], [0.5, 1, 0], [0.5, -1, 0.01]], np.float32)
    faces = np.array([[0, 1, 2], [1, 0, 3]], np.int32)
    r = oracle.proximity([[0, 1]], faces, verts, h=0.5)
    for rec in r:
        fa = faces[0][rec["fa"]] if rec["fa"] >= 0 else None
        fb = faces[1][rec["fb"]] if rec["fb"] >= 0 else None
        if rec["kind"] == 0:
            assert fa not in faces[1]
        if rec["kind"] == 1:
            assert fb not in faces[0]
    # as two meshes (ids unrelated), the shared corners count
    r2 = oracle.proximity([[0, 1]], faces, verts, faces, verts, h=0.5)
    assert len(r2) > len(r)


def test_degenerate_face_gives_nothing(oracle):
    verts = np.array([[0, 0, 0], [1, 0, 0], [2, 0, 0], [0.5, 0.1, 0.01], [0.6, 0.1, 0.01], [0.5, 0.2, 0.01]],
                     np.float32)
    faces = np.array([[3, 4, 5], [0, 1, 2]], np.int32)
    r = oracle.proximity([[0, 1]], faces, verts, h=1.0)
    assert not (r["kind"] == 0).any()

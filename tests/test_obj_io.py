"""Mesh files in (bvhcd_obj_read): host-side parsing, no GPU needed."""
import os

import numpy as np
import pytest


def _write(path, pos, faces, style=0):
    with open(path, "w") as f:
        f.write("# written by the test\nmtllib none.mtl\no cloth\n")
        for v in pos:
            f.write("v %.9g %.9g %.9g\n" % tuple(v))
        f.write("vt 0 0\nvn 0 0 1\ns off\n")
        n = len(pos)
        for k, t in enumerate(faces):
            if style == 0:
                f.write("f %d %d %d\n" % tuple(t + 1))
            elif style == 1:
                f.write("f %d/1/1 %d/1/1 %d/1/1\n" % tuple(t + 1))
            elif style == 2:
                f.write("f %d//1\t%d//1 %d//1\r\n" % tuple(t + 1))
            else:  # negative (relative) ids
                f.write("f %d %d %d\n" % tuple(t - n))


@pytest.mark.parametrize("style", [0, 1, 2, 3])
def test_obj_round_trip(lib_built, tmp_path, style):
    import scenes
    faces, frames = scenes.cloth_fold_frames(24, 1)
    pos = frames[0]
    p = tmp_path / "m.obj"
    _write(p, pos, faces, style)
    got_pos, got_faces = lib_built.load_obj(str(p))
    assert np.array_equal(got_pos, pos)
    assert np.array_equal(got_faces, faces)


def test_obj_polygons_are_fans(lib_built, tmp_path):
    p = tmp_path / "q.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nv 0.5 2 0\nf 1 2 3 4\nf 4 3 5\ng two\nf 1 2 3 4 5\n")
    pos, faces = lib_built.load_obj(str(p))
    assert pos.shape == (5, 3)
    assert faces.tolist() == [[0, 1, 2], [0, 2, 3], [3, 2, 4], [0, 1, 2], [0, 2, 3], [0, 3, 4]]


@pytest.mark.parametrize("text", ["v 0 0 0\nv 1 0 0\nf 1 2\n", "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n",
                                  "v 0 0\n", "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 x 3\n",
                                  "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 0 1 2\n"])
def test_obj_malformed_records_are_rejected(lib_built, tmp_path, text):
    p = tmp_path / "bad.obj"
    p.write_text(text)
    with pytest.raises(lib_built.BvhcdError):
        lib_built.load_obj(str(p))


def test_obj_missing_file_and_capacity(lib_built, tmp_path):
    import ctypes
    with pytest.raises(lib_built.BvhcdError):
        lib_built.load_obj(str(tmp_path / "none.obj"))
    p = tmp_path / "t.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0\nf 1 2 3\nf 2 4 3\n")
    V, T = ctypes.c_int32(), ctypes.c_int32()
    pos = np.zeros((4, 3), np.float32)
    faces = np.zeros((1, 3), np.int32)
    st = lib_built.lib().bvhcd_obj_read(os.fsencode(str(p)), pos.ctypes.data, 4, faces.ctypes.data, 1,
                                        ctypes.byref(V), ctypes.byref(T))
    assert st == 3 and (V.value, T.value) == (4, 2)  # CAPACITY_EXCEEDED with the full counts
    assert faces.tolist() == [[0, 1, 2]]


def test_obj_sequence(lib_built, tmp_path):
    import scenes
    faces, frames = scenes.cloth_fold_frames(16, 3)
    for f, pos in enumerate(frames):
        _write(tmp_path / ("seq_%03d.obj" % (f + 5)), pos, faces)
    got = list(lib_built.obj_frames(str(tmp_path / "seq_%03d.obj"), 5, 3))
    assert len(got) == 3
    for (p, fc), pos in zip(got, frames):
        assert np.array_equal(p, pos) and np.array_equal(fc, faces)


@pytest.mark.gpu
def test_obj_sequence_through_the_pipeline(cuda, lib_built, oracle, tmp_path):
    """A benchmark sequence read from OBJ files frame by frame (Scene::update)
    through the reference's schedule: pairs equal the oracle's on the same
    frames."""
    import scenes
    faces, frames = scenes.cloth_over_sphere_frames(40, frames=8, sphere_freq=6)
    for f, pos in enumerate(frames):
        _write(tmp_path / ("frame%d.obj" % f), pos, faces, style=f % 4)
    T, V = faces.shape[0], frames[0].shape[0]
    bvh = lib_built.LBvh(T, V, enable_restr=True)
    front = lib_built.BvttFront(bvh, int_front_capacity=2_000_000, ext_front_capacity=2_000_000,
                                pair_capacity=1_000_000, cull_adjacent=True, narrow_phase=True)
    p = oracle.Pipeline(True, True, True)
    for f, (pos, fc) in enumerate(lib_built.obj_frames(str(tmp_path / "frame%d.obj"), 0, len(frames))):
        b, fr = lib_built.schedule(f)
        lib_built.frame(bvh, front, f, 0, pos, fc)
        p.frame(fc, pos, b, fr)
        assert np.array_equal(oracle.canon_pairs(front.pairs()), oracle.canon_pairs(p.pairs())), f
        assert np.array_equal(oracle.canon_pairs(front.pairs(narrow=True)), oracle.canon_pairs(p.pairs(narrow=True))), f

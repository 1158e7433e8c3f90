"""Host-side tests of the C ABI that need no GPU: the shared library loads,
exports every entry point include/bvhcd.h declares, and its pure host
functions (status strings, the heuristic scheduler, argument checks) behave
like the reference's."""
import ctypes
import os
import re

import numpy as np

from conftest import ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "bvhcd.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bvhcd_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(lib_built):
    L = lib_built.lib()
    names = _declared()
    assert len(names) >= 18
    for n in names:
        assert hasattr(L, n), n
    assert sorted(lib_built.EXPORTED) == names


def test_status_strings(lib_built):
    L = lib_built.lib()
    assert L.bvhcd_status_string(0) == b"ok"
    assert L.bvhcd_status_string(3) == b"capacity exceeded"


def test_heuristic_schedule_matches_oracle(lib_built, oracle):
    for start in (0, 5):
        for f in range(start, start + 40):
            assert lib_built.schedule(f, start) == oracle.schedule(f, start)


def test_invalid_arguments_are_rejected(lib_built):
    L = lib_built.lib()
    assert L.bvhcd_bvh_create(None, None) == 1
    assert L.bvhcd_bvh_maintain(None, 0, None, None) == 1
    assert L.bvhcd_front_create(None, None, None) == 1
    assert L.bvhcd_front_maintain(None, 0, None) == 1
    b, f = ctypes.c_int32(), ctypes.c_int32()
    assert L.bvhcd_schedule_heuristic(3, 5, ctypes.byref(b), ctypes.byref(f)) == 1


def test_scene_generators_shapes():
    import scenes
    faces, frames = scenes.cloth_fold_frames(128, 2)
    assert faces.shape == (32258, 3) and frames[0].shape == (16384, 3)
    v, f = scenes.icosphere(45)
    assert f.shape == (40500, 3) and v.shape == (20252, 3)
    # shared vertices: every edge is used by exactly two triangles (closed surface)
    e = np.sort(np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]]), axis=1)
    _, cnt = np.unique(e, axis=0, return_counts=True)
    assert (cnt == 2).all()

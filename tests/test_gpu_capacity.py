"""Fronts near their capacity, without auto-grow, on the GPU.

Chunked emission reserves front slots eight at a time per lane; the slots a
lane does not fill are holes that still count against the capacity.  On a
small scene run by a full grid that waste used to reach seven slots per entry
and overflow a capacity several times the front, after which the update's
output (and every later keep) was corrupt.  Here a 5,669-triangle scene runs
the reference's schedule with front capacities of 1.5x the largest front the
oracle reports plus the traversals' bound of eight slots per triangle, and
room for the pair stream's holes: no frame may overflow, and every frame's
fronts and pair sets must equal the oracle's.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _multiset(x):
    x = np.asarray(x, dtype=np.int64).reshape(-1, 2)
    x = x[x[:, 0] >= 0]
    return x[np.lexsort((x[:, 1], x[:, 0]))]


def test_tight_capacity_schedule_matches_oracle(cuda, lib_built):
    import bvhcd
    import pyoracle
    import scenes
    faces, frames = scenes.cloth_over_sphere_frames(48, frames=14, sphere_freq=8)
    T, V = faces.shape[0], frames[0].shape[0]
    orc = pyoracle.Pipeline(True, True, True)
    ref = []
    for f, pos in enumerate(frames):
        b, fr = bvhcd.schedule(f)
        orc.frame(faces, pos, b, fr)
        ref.append((orc.front(0), orc.front(1), pyoracle.canon_pairs(orc.pairs()), orc.info()))
    fi = max(r[3]["F_int"] for r in ref)
    fe = max(r[3]["F_ext"] for r in ref)
    fp = max(r[3]["P"] for r in ref)
    bvh = bvhcd.LBvh(T, V, enable_restr=True)
    front = bvhcd.BvttFront(bvh, int_front_capacity=int(1.5 * fi) + 8 * T,
                            ext_front_capacity=int(1.5 * fe) + 8 * T,
                            pair_capacity=8 * fp + 4096, cull_adjacent=True, narrow_phase=True, auto_grow=False)
    for f, pos in enumerate(frames):
        bvhcd.frame(bvh, front, f, 0, pos, faces, faces_static=f > 0)
        st = front.stats()
        assert st["overflow"] == 0, (f, st)
        assert np.array_equal(_multiset(front.export(0)), _multiset(ref[f][0])), f
        assert np.array_equal(_multiset(front.export(1)), _multiset(ref[f][1])), f
        assert np.array_equal(pyoracle.canon_pairs(front.pairs(narrow=False)), ref[f][2]), f

"""Batched scenes (bvhcd_bvh_set_scenes) and graph-launched frames
(bvhcd_frame_graph) on the GPU.

A batch is one forest: each scene's subtree must be the tree the scene gets
on its own (shifted by the scene's slot and node offsets), and each scene's
pair sets must be those of the scene run alone -- the oracle's, per scene.
Graph-launched frames must give the same pairs as ordinary launches.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch(num_scenes=10, t_max=12_000, seed=7):
    import scenes
    return scenes.BatchedScenes(num_scenes=num_scenes, t_min=200, t_max=t_max, seed=seed)


def _split(pairs, tri_offsets):
    """Global-id pairs -> per-scene canonical local pairs; asserts no pair
    crosses scenes."""
    out = []
    p = np.sort(np.asarray(pairs, dtype=np.int64).reshape(-1, 2), axis=1)
    sa = np.searchsorted(tri_offsets, p[:, 0], side="right") - 1
    sb = np.searchsorted(tri_offsets, p[:, 1], side="right") - 1
    assert np.array_equal(sa, sb), "a pair crosses scenes"
    for s in range(len(tri_offsets) - 1):
        q = p[sa == s] - tri_offsets[s]
        out.append(q[np.lexsort((q[:, 1], q[:, 0]))] if q.size else np.zeros((0, 2), np.int64))
    return out


def _canon(oracle, p):
    c = oracle.canon_pairs(p).astype(np.int64)
    return c.reshape(-1, 2)


def test_forest_trees_equal_single_scene_trees(cuda, lib_built):
    b = _batch()
    off = b.tri_offsets
    pos = b.positions(0)
    bvh = lib_built.LBvh(b.num_faces, b.num_vertices, enable_restr=False)
    bvh.set_scenes(off)
    bvh.maintain(lib_built.BVH_BUILD, pos, b.faces)
    T, _, I = bvh.sizes()
    assert (T, I) == (b.num_faces, b.num_faces - b.num_scenes)
    fo = bvh.export()
    for s in range(b.num_scenes):
        faces_s, pos_s = b.scene(s, 0)
        one = lib_built.LBvh(faces_s.shape[0], pos_s.shape[0], enable_restr=False)
        one.maintain(lib_built.BVH_BUILD, pos_s, faces_s)
        t = one.export()
        a0, a1 = int(off[s]), int(off[s + 1])
        n0 = a0 - s
        Ts = a1 - a0
        assert np.array_equal(fo["codes"][a0:a1], t["codes"])
        assert np.array_equal(fo["leaf"][a0:a1, 0] - a0, t["leaf"][:, 0])          # triangle ids
        assert np.array_equal(fo["leaf"][a0:a1, 1] - n0, t["leaf"][:, 1])          # parents
        assert np.array_equal(fo["lbox"][a0:a1], t["lbox"])
        assert np.array_equal(fo["primmap"][a0:a1] - a0, t["primmap"])
        inode = fo["inode"][n0:n0 + Ts - 1].copy()
        ti = t["inode"]
        mark = ti[:, 3]
        exp = ti.copy()
        exp[:, 0] += np.where(mark & 1, a0, n0)
        exp[:, 1] += np.where(mark & 2, a0, n0)
        exp[:, 2] = np.where(ti[:, 2] >= 0, ti[:, 2] + n0, -1)
        exp[:, 4:6] += a0
        assert np.array_equal(inode, exp), s
        assert np.array_equal(fo["ibox"][n0:n0 + Ts - 1], t["ibox"])
        lca = t["lca"][:Ts]
        exp_lca = np.where(lca & 1, ((lca >> 1) + a0) * 2 + 1, ((lca >> 1) + n0) * 2)
        assert np.array_equal(fo["lca"][a0:a1], exp_lca), s
        one.close()


def test_batched_pairs_equal_per_scene_oracle(cuda, lib_built, oracle):
    b = _batch(num_scenes=8, t_max=8_000, seed=11)
    off = b.tri_offsets
    bvh = lib_built.LBvh(b.num_faces, b.num_vertices, enable_restr=False)
    bvh.set_scenes(off)
    front = lib_built.BvttFront(bvh, 6_000_000, 6_000_000, 3_000_000, cull_adjacent=True, narrow_phase=True)
    refs = [oracle.Pipeline(restructure=False, cull_adjacent=True, narrow=True) for _ in range(b.num_scenes)]
    for f in range(14):
        bop, fop = lib_built.schedule(f)
        bvh.maintain(bop, b.positions(f), b.faces)
        front.maintain(fop)
        st = front.stats()
        assert st["overflow"] == 0
        broad = _split(front.pairs(), off)
        hits = _split(front.pairs(narrow=True), off)
        for s, ref in enumerate(refs):
            faces_s, pos_s = b.scene(s, f)
            ref.frame(faces_s, pos_s, bop, fop)
            assert np.array_equal(broad[s], _canon(oracle, ref.pairs())), (f, s)
            assert np.array_equal(hits[s], _canon(oracle, ref.pairs(narrow=True))), (f, s)
        assert st["broad_pairs"] == sum(len(x) for x in broad)


def test_graph_frames_equal_plain_frames(cuda, lib_built):
    torch = cuda
    b = _batch(num_scenes=6, t_max=6_000, seed=3)
    off = b.tri_offsets
    stream = torch.cuda.Stream()
    faces_d = torch.from_numpy(b.faces).cuda()
    pos_d = torch.empty((b.num_vertices, 3), dtype=torch.float32, device="cuda")
    runs = []
    for graph in (False, True):
        bvh = lib_built.LBvh(b.num_faces, b.num_vertices, enable_restr=False)
        bvh.set_scenes(off)
        front = lib_built.BvttFront(bvh, 4_000_000, 4_000_000, 2_000_000, cull_adjacent=True,
                                    narrow_phase=True, auto_grow=False)
        out = []
        with torch.cuda.stream(stream):
            for f in range(16):
                bop, fop = lib_built.schedule(f)
                pos_d.copy_(torch.from_numpy(b.positions(f)))
                if graph:
                    lib_built.frame_graph(bvh, front, pos_d, faces_d, bop, fop, stream=stream)
                else:
                    bvh.maintain(bop, pos_d, faces_d, stream=stream)
                    front.maintain(fop, stream=stream)
                st = front.stats(stream=stream)
                out.append((st["int_front"], st["ext_front"], st["broad_pairs"], st["narrow_hits"],
                            _split(front.pairs(stream=stream), off),
                            _split(front.pairs(narrow=True, stream=stream), off)))
        runs.append(out)
        front.close()
        bvh.close()
    for f, (a, g) in enumerate(zip(*runs)):
        assert a[:4] == g[:4], f
        for x, y in zip(a[4] + a[5], g[4] + g[5]):
            assert np.array_equal(x, y), f


def test_batched_argument_checks(cuda, lib_built):
    b = _batch(num_scenes=3, t_max=3_000, seed=5)
    bvh = lib_built.LBvh(b.num_faces, b.num_vertices, enable_restr=True)
    with pytest.raises(lib_built.BvhcdError):
        bvh.set_scenes(b.tri_offsets)          # restructuring is on
    bvh2 = lib_built.LBvh(b.num_faces, b.num_vertices, enable_restr=False)
    bad = b.tri_offsets.copy()
    bad[1] = bad[0] + 1                        # a one-triangle scene
    with pytest.raises(lib_built.BvhcdError):
        bvh2.set_scenes(bad)
    with pytest.raises(lib_built.BvhcdError):
        bvh2.set_scenes(b.tri_offsets + 1)     # does not start at 0
    bvh2.set_scenes(b.tri_offsets)
    with pytest.raises(lib_built.BvhcdError):  # triangle count differs from the layout
        bvh2.maintain(lib_built.BVH_BUILD, b.positions(0), b.faces[:-2])
    front = lib_built.BvttFront(bvh2, 1_000_000, 1_000_000, 500_000)
    stream = cuda.cuda.Stream()
    with pytest.raises(lib_built.BvhcdError):  # host input cannot be graph-launched
        lib_built.frame_graph(bvh2, front, b.positions(0), b.faces, 0, 1, stream=stream)


def test_autotune_and_shapes_leave_results_unchanged(cuda, lib_built, oracle, cloth_c1):
    """Launch shapes change only how the work is spread: every shape the
    autotuner picks or the caller forces gives the oracle's pair sets."""
    faces, frames = cloth_c1
    T, V = faces.shape[0], frames[0].shape[0]
    bvh = lib_built.LBvh(T, V, enable_restr=False)
    front = lib_built.BvttFront(bvh, 4_000_000, 4_000_000, 2_000_000, cull_adjacent=True, narrow_phase=True)
    ref = oracle.Pipeline(restructure=False, cull_adjacent=True, narrow=True)
    forced = [{k: (1, 128) for k in lib_built.SHAPE_STAGES}, {k: (4, 512) for k in lib_built.SHAPE_STAGES}]
    for f in range(14):
        b, fr = lib_built.schedule(f)
        bvh.maintain(b, frames[f], faces)
        front.maintain(fr)
        ref.frame(faces, frames[f], b, fr)
        if f == 1:
            shapes, best = front.autotune(2)
            assert front.shapes() == shapes
            for k, (u, blk) in shapes.items():
                assert u in (1, 2, 4) and blk in (128, 256, 512), k
                assert best[k] > 0.0, k
            assert front.stats()["front_op_run"] == lib_built.FRONT_GENERATE
        if f in (5, 9):
            front.set_shapes(forced[(f // 5) - 1])
        assert np.array_equal(_canon(oracle, front.pairs()), _canon(oracle, ref.pairs())), f
        assert np.array_equal(_canon(oracle, front.pairs(narrow=True)), _canon(oracle, ref.pairs(narrow=True))), f
    with pytest.raises(lib_built.BvhcdError):
        front.set_shapes({"keep": (3, 256)})
    with pytest.raises(lib_built.BvhcdError):
        front.set_shapes({"narrow": (1, 64)})

"""Parity with the reference's own pipeline.

tests/golden/ref_<workload>.json were produced by running the reference's
unmodified LBvhFixedDeformable + BvttFrontLooseIntra (its sources compiled as
host C++ with every kernel run one thread at a time, oracle/ref/
Makefile.refemu) under its own schedule (tests/golden/make_golden.py).  Each
holds, per frame, the reference's own report (front sizes, broad-phase pair
count, narrow-phase hit count, BVH operation tag, restructure decision) and
digests of its broad-phase pair set and of its tree arrays, plus the subtree
roots marked for restructuring before the frame.  The reference's standalone
build has no adjacency culling, so both sides run with culling off.

The CPU tests pin the oracle to those fixtures; when oracle/_ref/
ref_emu_driver has been built they also run the reference live on a small
case.  The GPU test holds the CUDA path to the same fixtures through the
C ABI.
"""
import glob
import hashlib
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden")
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "ref_*.json")))
EMU_DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_emu_driver")


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _load(path):
    with open(path) as f:
        return json.load(f)


def _inputs(fx):
    sys.path.insert(0, os.path.join(ROOT, "bvh-based-collision-detection-scheme_b200"))
    import scenes
    faces, frames = eval("scenes." + fx["workload"], {"scenes": scenes})
    assert fx["input_sha256"] == digest(np.stack(frames)) + ":" + digest(faces), \
        "the seeded frames differ from the ones the fixture was made from"
    return faces, frames


def _tree_digests(tree):
    inode = tree["inode"]
    leaf = tree["leaf"]
    return {
        "leaf_lca": digest(tree["lca"].astype(np.int32)),
        "leaf_par": digest(leaf[:, 1].astype(np.int32)),
        "prim_idx": digest(leaf[:, 0].astype(np.int32)),
        "prim_map": digest(tree["primmap"].astype(np.int32)),
        "codes": digest(tree["codes"].astype(np.uint32)),
        "int_par": digest(inode[:, 2].astype(np.int32)),
        "int_lbd": digest(inode[:, 4].astype(np.int32)),
        "int_rbd": digest(inode[:, 5].astype(np.int32)),
        "int_mark": digest(inode[:, 3].astype(np.uint32)),
    }


def test_fixtures_present():
    names = {os.path.basename(p) for p in FIXTURES}
    assert {"ref_cloth_fold_128.json", "ref_cloth_fold_128_restructure.json",
            "ref_stacked_layers_64.json"} <= names


def test_fixtures_cover_every_restructure_branch():
    tags, branches = set(), set()
    for path in FIXTURES:
        for e in _load(path)["frames"]:
            tags.add(e["opt_tag"])
            if e["restructure_decision"]:
                branches.add(e["restructure_decision"]["branch"])
    assert tags == {0, 1, 2}
    assert branches == {"refit", "restr", "build"}


def comparable(frames, full_on_restructure):
    """Per fixture frame, which checks hold against the reference.

    The reference's restructure moves primitives with a racy, inverted
    permutation (updatePrimMap, Mine/collision/lbvh/LBvhRestructureKernels.cu:
    68-77) that leaves its slot->triangle map inconsistent until the next
    full build, while the product moves them by the sort permutation.  So a
    frame whose BVH was restructured (opt tag 1) from a consistent tree is
    held to the restructure decision -- or to everything, when
    `full_on_restructure` (the oracle in reference-permutation mode) -- and
    the frames after it, until a clean rebuild, to nothing: their fronts, and
    the quality checks that read them, start from the reference's
    inconsistent map.  A rebuild chosen by a restructure decision taken on
    such a frame is held to everything but that decision ("rebuilt").
    Yields (entry, "full" | "rebuilt" | "decision" | "none")."""
    dirty = False
    for e in frames:
        rebuilt = e["opt_tag"] == 2 or (e["bvh_op"] == 0 and e["restructure_decision"] is None)
        if rebuilt and dirty:
            dirty = False
            yield e, "rebuilt"
        elif dirty:
            yield e, "none"
        elif e["opt_tag"] == 1:
            yield e, ("full" if full_on_restructure else "decision")
            dirty = True
        else:
            yield e, "full"


def _check_frame(e, kind, opt_tag, decision, counts, pairs, tree):
    f = e["frame"]
    if kind == "none":
        return
    assert opt_tag == e["opt_tag"], f
    if e["restructure_decision"] and kind != "rebuilt":
        d = e["restructure_decision"]
        assert decision == (d["subtrees"], d["int_nodes"]), f
    if kind != "full":
        return
    F_int, F_ext, P, H = counts
    assert (F_int, F_ext) == (e["int_front"], e["ext_front"]), f
    assert P == e["broad_pairs"], f
    # the reference skips its narrow phase on a restructured frame and
    # reports the previous frame's count (BvttFrontLooseIntra.cu:84-109)
    if e["opt_tag"] != 1:
        assert H == e["narrow_hits"], f
    assert digest(pairs) == e["pairs_sha256"], f
    assert _tree_digests(tree) == e["tree_sha256"], f


def _run_oracle(oracle, fx, reference_permutation):
    faces, frames = _inputs(fx)
    p = oracle.Pipeline(restructure=True, cull_adjacent=False, narrow=True,
                        reference_permutation=reference_permutation)
    kinds = []
    for e, kind in comparable(fx["frames"], reference_permutation):
        f = e["frame"]
        assert (e["bvh_op"], e["front_op"]) == oracle.schedule(f)
        if e["restructure_roots"]:
            p.mark_restructure(np.asarray(e["restructure_roots"], dtype=np.int32))
        p.frame(faces, frames[f], e["bvh_op"], e["front_op"])
        i = p.info()
        _check_frame(e, kind, i["opt_tag"], (i["num_rt_subtree"], i["num_rt_int"]),
                     (i["F_int"], i["F_ext"], i["P"], i["H"]), oracle.canon_pairs(p.pairs()),
                     p.tree())
        kinds.append(kind)
    return kinds


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_oracle_matches_reference_pipeline(oracle, path):
    """The oracle as the product computes (sort permutation on restructure)."""
    kinds = _run_oracle(oracle, _load(path), reference_permutation=False)
    assert kinds.count("full") + kinds.count("rebuilt") >= len(kinds) // 2


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_oracle_reference_permutation_matches_restructure_frames(oracle, path):
    """With the reference's own permutation update the oracle reproduces the
    reference's restructured tree, fronts and pairs bit for bit, which pins
    the rest of the restructure (decision, keys, confined rebuild, DFS
    renumbering, front regeneration) against the reference's code."""
    fx = _load(path)
    kinds = _run_oracle(oracle, fx, reference_permutation=True)
    restructured = [k for e, k in zip(fx["frames"], kinds) if e["opt_tag"] == 1]
    assert all(k == "full" for k in restructured)


@pytest.mark.skipif(not os.path.exists(EMU_DRIVER), reason="oracle/_ref/ref_emu_driver not built")
def test_oracle_matches_reference_live(oracle, tmp_path):
    """Runs the reference itself (host build) on a fresh seeded case that no
    fixture holds, with a forced restructure, and compares every frame."""
    sys.path.insert(0, GOLDEN)
    import make_golden
    import scenes
    faces, frames = scenes.cloth_fold_frames(48, 14, seed=99)
    T, V = faces.shape[0], frames[0].shape[0]
    p = oracle.Pipeline(restructure=True, cull_adjacent=False, narrow=True,
                        reference_permutation=True)
    marks = [[] for _ in frames]
    ours = []
    for f, pos in enumerate(frames):
        if f == 4:
            marks[f] = make_golden.choose_roots(p.tree()["inode"], 0.3, 5)
            p.mark_restructure(np.asarray(marks[f], dtype=np.int32))
        b, fr = oracle.schedule(f)
        p.frame(faces, pos, b, fr)
        i = p.info()
        ours.append((i["opt_tag"], (i["num_rt_subtree"], i["num_rt_int"]),
                     (i["F_int"], i["F_ext"], i["P"], i["H"]), oracle.canon_pairs(p.pairs()),
                     p.tree()))
    fin, fmk, fout = (str(tmp_path / n) for n in ("frames.bin", "marks.bin", "out.bin"))
    with open(fin, "wb") as f:
        np.array([0x49485642, T, V, len(frames)], np.int32).tofile(f)
        faces.astype(np.int32).tofile(f)
        np.stack(frames).astype(np.float32).tofile(f)
    with open(fmk, "wb") as f:
        for m in marks:
            np.array([len(m)] + list(m), np.int32).tofile(f)
    run = subprocess.run([EMU_DRIVER, fin, fout, fmk], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr[-2000:]
    recs = make_golden.read_output(fout)
    rep = make_golden.frame_reports(run.stdout)
    assert len(recs) == len(rep) == len(frames)
    entries = []
    for r, (counts, restr) in zip(recs, rep):
        entries.append(dict(frame=r["frame"], bvh_op=r["bvh_op"], opt_tag=r["opt_tag"],
                            restructure_decision=restr, int_front=counts[0], ext_front=counts[1],
                            broad_pairs=counts[2], narrow_hits=counts[3],
                            pairs_sha256=digest(make_golden.canon(r["pairs"])),
                            tree_sha256={k: digest(r[k]) for k in make_golden.TREE_FIELDS}))
    assert [e["opt_tag"] for e in entries].count(1) == 1
    for (e, kind), o in zip(comparable(entries, True), ours):
        _check_frame(e, kind, *o)


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_cuda_path_matches_reference_pipeline(cuda, lib_built, oracle, path):
    fx = _load(path)
    faces, frames = _inputs(fx)
    T, V = faces.shape[0], frames[0].shape[0]
    bvh = lib_built.LBvh(T, V, enable_restr=True)
    front = lib_built.BvttFront(bvh, 4_000_000, 4_000_000, 2_000_000, cull_adjacent=False,
                                narrow_phase=True)
    for e, kind in comparable(fx["frames"], False):
        f = e["frame"]
        if e["restructure_roots"]:
            bvh.request_restructure(np.asarray(e["restructure_roots"], dtype=np.int32))
        bvh.maintain(e["bvh_op"], frames[f], faces)
        front.maintain(e["front_op"])
        st = front.stats()
        _check_frame(e, kind, st["bvh_opt_tag"], (st["num_rt_subtrees"], st["num_rt_int_nodes"]),
                     (st["int_front"], st["ext_front"], st["broad_pairs"], st["narrow_hits"]),
                     oracle.canon_pairs(front.pairs()), bvh.export())

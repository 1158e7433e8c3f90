"""Generates the golden fixtures tests/golden/ref_<workload>.json by running
the reference's own pipeline (LBvhFixedDeformable + BvttFrontLooseIntra,
compiled unmodified from the reference sources) through
oracle/ref/ref_pipeline_driver.cpp on seeded synthetic frames.

    python tests/golden/make_golden.py [--driver PATH] [--only NAME] [--out DIR]

The driver is oracle/_ref/ref_emu_driver (oracle/ref/Makefile.refemu): the
reference's sources built as host C++, every kernel run one thread at a time.
(Built for the GPU, the reference faults on a B200 inside its own front
generation, after a tree build whose bottom-up merge has no memory fence, so
it is not run there.)

Each fixture records, per frame of the reference schedule, what the reference
itself reports (front sizes, broad-phase pair count, narrow-phase hit count,
BVH operation tag, and the subtree / internal-node counts of its restructure
decision when it prints one) and SHA-256 digests of its broad-phase pair set
(as sorted (min, max) original-id pairs) and of its tree arrays.  Workloads
with forced restructuring also record, per frame, the subtree roots that were
marked just before the frame's BVH maintenance; they are chosen from the
tree the oracle holds at that point (the oracle and the reference agree on it
frame by frame, which is what the fixture then checks).  The reference is
compiled without adjacency culling (its standalone build), so the oracle and
the CUDA path are compared with culling off.
"""
import argparse
import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "bvh-based-collision-detection-scheme_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_emu_driver")
TREE_FIELDS = ["leaf_lca", "leaf_par", "prim_idx", "prim_map", "codes", "int_par", "int_lbd", "int_rbd",
               "int_mark"]

# name -> (scene call as text, {frame: (fraction of internal nodes to mark, seed)})
WORKLOADS = {
    "cloth_fold_128": ("cloth_fold_frames(128, 20)", {}),
    # fractions chosen to land in each branch of the restructure decision
    # (Mine/collision/lbvh/LBvhFixedDeformable.cu:243-270): > 1/2 of the
    # internal nodes rebuilds, < 1/8 refits, in between restructures.
    "cloth_fold_128_restructure": ("cloth_fold_frames(128, 20)",
                                   {3: (0.25, 11), 9: (0.60, 13), 15: (0.05, 14), 17: (0.20, 15)}),
    "stacked_layers_64": ("stacked_layers_frames(64, 4, 14)", {5: (0.22, 21)}),
}


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def canon(p):
    p = np.asarray(p, dtype=np.int64).reshape(-1, 2)
    if p.size == 0:
        return np.zeros((0, 2), np.int64)
    q = np.sort(p, axis=1)
    return q[np.lexsort((q[:, 1], q[:, 0]))]


def workload(call):
    import scenes
    return eval("scenes." + call, {"scenes": scenes})


def choose_roots(inode, frac, seed):
    """Disjoint subtree roots of the current tree covering about `frac` of
    its internal nodes, drawn in a seeded order among subtrees of 16 to 1024
    leaves.  inode[:, 4:6] hold each internal node's leaf range; in DFS
    order the subtree of node i is the id range [i, i + size - 1)."""
    I = inode.shape[0]
    size = inode[:, 5] - inode[:, 4] + 1
    cand = np.flatnonzero((size >= 16) & (size <= 1024))
    rng = np.random.default_rng(seed)
    rng.shuffle(cand)
    taken = np.zeros(I, dtype=bool)
    roots, covered = [], 0
    for i in cand:
        s = int(size[i])
        if taken[i:i + s - 1].any():
            continue
        anc = i
        clash = False
        while anc != -1:
            if taken[anc]:
                clash = True
                break
            anc = int(inode[anc, 2])
        if clash:
            continue
        taken[i:i + s - 1] = True
        roots.append(int(i))
        covered += s - 1
        if covered >= frac * I:
            break
    return sorted(roots)


def read_output(path):
    frames = []
    buf = open(path, "rb").read()
    off = 0
    while off < len(buf):
        magic, f, b, fr, tag, n, T = np.frombuffer(buf, np.int32, 7, off)
        off += 28
        assert magic == 0x4D415246
        rec = dict(frame=int(f), bvh_op=int(b), front_op=int(fr), opt_tag=int(tag), n=int(n))
        rec["pairs"] = np.frombuffer(buf, np.int32, 2 * n, off).reshape(-1, 2)
        off += 8 * n
        for name, cnt, dt in [("leaf_lca", T + 1, np.int32), ("leaf_par", T, np.int32),
                              ("prim_idx", T, np.int32), ("prim_map", T, np.int32),
                              ("codes", T, np.uint32), ("int_par", T - 1, np.int32),
                              ("int_lbd", T - 1, np.int32), ("int_rbd", T - 1, np.int32),
                              ("int_mark", T - 1, np.uint32)]:
            rec[name] = np.frombuffer(buf, dt, cnt, off)
            off += 4 * cnt
        frames.append(rec)
    return frames


def frame_reports(log):
    """Splits the reference's stdout at its per-frame report line
    (BvttFrontLooseIntra::inspectResults) and reads, per frame, that report
    and the restructure decision LBvhFixedDeformable::restructure printed."""
    out = []
    restr = None
    for line in log.splitlines():
        m = re.search(r"(\d+) subtrees and (\d+) \((\d+)\) internal nodes need restructuring\. (\w+)", line)
        if m:
            restr = {"subtrees": int(m.group(1)), "int_nodes": int(m.group(2)), "branch": m.group(4)}
            continue
        m = re.search(r"front \((\d+), (\d+)\) cpNum (\d+) actualCpNum (\d+)", line)
        if m:
            out.append((tuple(int(g) for g in m.groups()), restr))
            restr = None
    return out


def marks_for(name, faces, frames):
    """Per-frame restructure roots, chosen from the oracle's tree just before
    each marked frame's BVH maintenance."""
    import pyoracle
    plan = WORKLOADS[name][1]
    marks = [[] for _ in frames]
    if not plan:
        return marks
    p = pyoracle.Pipeline(restructure=True, cull_adjacent=False, narrow=False)
    for f, pos in enumerate(frames):
        if f in plan:
            frac, seed = plan[f]
            marks[f] = choose_roots(p.tree()["inode"], frac, seed)
            p.mark_restructure(np.asarray(marks[f], dtype=np.int32))
        b, fr = pyoracle.schedule(f)
        p.frame(faces, pos, b, fr)
    return marks


def make(name, driver, outdir):
    call = WORKLOADS[name][0]
    faces, frames = workload(call)
    T, V = faces.shape[0], frames[0].shape[0]
    marks = marks_for(name, faces, frames)
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "frames.bin")
        fmk = os.path.join(td, "marks.bin")
        fout = os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            np.array([0x49485642, T, V, len(frames)], np.int32).tofile(f)
            faces.astype(np.int32).tofile(f)
            np.stack(frames).astype(np.float32).tofile(f)
        with open(fmk, "wb") as f:
            for m in marks:
                np.array([len(m)] + list(m), np.int32).tofile(f)
        run = subprocess.run([driver, fin, fout, fmk], capture_output=True, text=True)
        if run.returncode != 0:
            raise SystemExit(f"reference driver failed with status {run.returncode}: "
                             f"{run.stdout[-2000:]}\n{run.stderr[-2000:]}")
        recs = read_output(fout)
    rep = frame_reports(run.stdout)
    assert len(rep) == len(recs), (len(rep), len(recs))
    out = {"workload": call, "triangles": int(T), "vertices": int(V),
           "input_sha256": digest(np.stack(frames)) + ":" + digest(faces),
           "adjacency_culling": False, "frames": []}
    for r, m, ((fi, fe, cp, hits), restr) in zip(recs, marks, rep):
        e = {k: r[k] for k in ("frame", "bvh_op", "front_op", "opt_tag")}
        e.update(int_front=fi, ext_front=fe, broad_pairs=cp, narrow_hits=hits,
                 restructure_roots=m, restructure_decision=restr,
                 pairs_sha256=digest(canon(r["pairs"])))
        e["tree_sha256"] = {k: digest(r[k]) for k in TREE_FIELDS}
        out["frames"].append(e)
    path = os.path.join(outdir, f"ref_{name}.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {path}: {len(recs)} frames, opt tags {[e['opt_tag'] for e in out['frames']]}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--driver", default=DRIVER)
    ap.add_argument("--only", default=None)
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    for name in WORKLOADS:
        if a.only is None or a.only == name:
            make(name, a.driver, a.out)


if __name__ == "__main__":
    main()

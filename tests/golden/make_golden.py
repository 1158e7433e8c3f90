"""Generates tests/golden/ref_gpu_cloth128.json by running the reference's own
CUDA pipeline (oracle/_ref/ref_gpu_driver, built from the reference sources by
oracle/ref/Makefile.refgpu) on the 128x128 folding-cloth frames.

Run on a machine with a GPU:  python tests/golden/make_golden.py [out.json [driver.log]]

The fixture records, per frame of the reference schedule, what the reference
itself reports (front sizes, broad-phase pair count, narrow-phase hit count,
BVH operation tag) and SHA-256 digests of its broad-phase pair set (as
sorted (min, max) original-id pairs) and of its tree arrays.  The reference
is compiled without adjacency culling (its standalone build), so the oracle
and the CUDA path are compared with culling off.
"""
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

FIXTURE = os.path.join(HERE, "ref_gpu_cloth128.json")
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_driver")
TREE_FIELDS = ["leaf_lca", "leaf_par", "prim_idx", "prim_map", "codes", "int_par", "int_lbd", "int_rbd",
               "int_mark"]


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def canon(p):
    p = np.asarray(p, dtype=np.int64).reshape(-1, 2)
    if p.size == 0:
        return np.zeros((0, 2), np.int64)
    q = np.sort(p, axis=1)
    return q[np.lexsort((q[:, 1], q[:, 0]))]


def workload():
    import scenes
    return scenes.cloth_fold_frames(128, 20)


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


def main():
    faces, frames = workload()
    T, V = faces.shape[0], frames[0].shape[0]
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "frames.bin")
        fout = os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            np.array([0x49485642, T, V, len(frames)], np.int32).tofile(f)
            faces.astype(np.int32).tofile(f)
            np.stack(frames).astype(np.float32).tofile(f)
        log = subprocess.run([DRIVER, fin, fout], check=True, capture_output=True, text=True).stdout
        recs = read_output(fout)
    # the reference's own per-frame report (BvttFrontLooseIntra::inspectResults)
    rep = [tuple(map(int, m)) for m in
           re.findall(r"front \((\d+), (\d+)\) cpNum (\d+) actualCpNum (\d+)", log)]
    assert len(rep) == len(recs), (len(rep), len(recs))
    out = {"workload": "cloth_fold_frames(128, 20)", "triangles": int(T), "vertices": int(V),
           "input_sha256": digest(np.stack(frames)) + ":" + digest(faces),
           "adjacency_culling": False, "frames": []}
    for r, (fi, fe, cp, hits) in zip(recs, rep):
        e = {k: r[k] for k in ("frame", "bvh_op", "front_op", "opt_tag")}
        e.update(int_front=fi, ext_front=fe, broad_pairs=cp, narrow_hits=hits,
                 pairs_sha256=digest(canon(r["pairs"])))
        e["tree_sha256"] = {k: digest(r[k]) for k in TREE_FIELDS}
        out["frames"].append(e)
    path = sys.argv[1] if len(sys.argv) > 1 else FIXTURE
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    if len(sys.argv) > 2:
        with open(sys.argv[2], "w") as f:
            f.write(log)
    print(f"wrote {path}: {len(recs)} frames")


if __name__ == "__main__":
    main()

"""Trace recording, counterfactual labelling, GPU training and evaluation of
the learned scheduler (bvhcd_learner_*, bvhcd_mlp_*).

    python learn.py train --out learned_scheduler.npz     (on a GPU)
    python learn.py eval  --weights learned_scheduler.npz (on a GPU)

Traces.  Seeded variants of the cloth-over-sphere workload (wave amplitude
0.05-0.4, wave frequency 1-6) run under the learned mode's base policy (BVH
refit every frame, the front kept, no mandatory rebuild) with random
exploratory restructures and front regenerations.  At every decision frame
the learner's features of the cut's subtrees are recorded, and the run is
forked (bvhcd_bvh_copy_state / bvhcd_front_copy_state) into six branches that
run the next H frames (24 by default: an operation has that long to pay
back): refit only; four branches that each restructure one quarter of the
cut (a quarter stays between 1/8 and 1/2 of the internal nodes, so it is a
restructure, not a rebuild); a front regeneration.

Labels.  A branch's cost for a subtree is the branch's measured frame time
(CUDA events) shared out by the subtree's share of the front entries
(bvhcd_learner_work) plus, for the branch's one-off operation (restructure and
the regeneration that follows it, or the regeneration alone), that
operation's measured stage time shared out by leaves.  A subtree's label is
the cheapest of refit, the restructure branch that holds it, and the
regeneration; an operation has to beat refit by `margin` to win.

Training.  The project's own kernels (bvhcd_mlp_train: forward, backward and
Adam on the GPU) with inverse-frequency class weights; validation on held-out
sequences.

Evaluation.  Held-out seeds of a 708x708 cloth over the sphere (about 1 M
triangles) for 200 frames under the heuristic (the reference's schedule:
build every 12 frames, front cycle 6, quality-triggered restructuring), under
the learned scheduler, and under two schedules without the network: the
reference's front cycle with the BVH refit every frame ("cycle"), and the
learned mode's base policy alone, refit and keep ("keep"); frame by frame:
device time per frame and the broad and narrow pair sets, which must be
equal.  The host's garbage collector is off while a sequence is timed (a
collection between a frame's launches would stall the GPU inside the frame's
events).
"""
from __future__ import annotations

import argparse
import gc
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import bvhcd  # noqa: E402
import scenes  # noqa: E402

WEIGHTS = os.path.join(HERE, "learned_scheduler.npz")
N_BRANCH_QUARTERS = 4


def base_front_op(f: int) -> int:
    """The learned mode's front operation between decisions: keep."""
    return bvhcd.FRONT_KEEP


def cycle_front_op(f: int) -> int:
    """The reference's front cycle (BenchmarkLogic.hpp:102-117) without its
    mandatory rebuilds: UPDATE every 6th frame, REORDER before it, KEEP."""
    k = f % 6
    if k == 0:
        return bvhcd.FRONT_UPDATE
    if k == 5:
        return bvhcd.FRONT_REORDER
    return bvhcd.FRONT_KEEP


class Pipe:
    """A BVH (restructuring on) and its front.  A Learner bound to it turns
    the front's own quality check off, so it restructures only when told."""

    def __init__(self, T, V, caps, smax, profile=False):
        self.bvh = bvhcd.LBvh(T, V, enable_restr=True)
        self.front = bvhcd.BvttFront(self.bvh, *caps, cull_adjacent=True, narrow_phase=True)
        self.learner = bvhcd.Learner(self.bvh, self.front, smax)
        if profile:
            self.bvh.profile(True)

    def close(self):
        self.learner.close()
        self.front.close()
        self.bvh.close()


def _caps(T):
    return (40 * T + 100_000, 30 * T + 100_000, 8 * T + 100_000)


def record_sequence(torch, seed, n, frames, amplitude, freq, H, stride, smax, explore, rng):
    """Features and per-subtree branch costs of one sequence."""
    faces, pos = scenes.cloth_over_sphere_frames(n, frames + H + 1, seed=seed, sphere_freq=max(2, n // 12),
                                                 amplitude=amplitude, wave_freq=freq)
    T, V = faces.shape[0], pos[0].shape[0]
    caps = _caps(T)
    main = Pipe(T, V, caps, smax)
    lrn = main.learner                 # records features; the run below is driven, not voted
    branches = [Pipe(T, V, caps, smax, profile=True) for _ in range(2 + N_BRANCH_QUARTERS)]
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    rows, labels, meta = [], [], []
    for f in range(frames):
        if f == 0:
            main.bvh.maintain(bvhcd.BVH_BUILD, pos[0], faces)
            main.front.maintain(bvhcd.FRONT_GENERATE)
            lrn.observe(True, True)
            continue
        # exploration: random restructure of one quarter, or a regeneration
        roots = lrn.cut()
        act = rng.random()
        if act < explore and len(roots) >= 8:
            q = rng.permutation(len(roots))[: len(roots) // 4]
            main.bvh.request_restructure(roots[np.sort(q)])
        main.bvh.maintain(bvhcd.BVH_REFIT, pos[f], faces)
        tag = main.bvh.opt_tag()
        regen = tag in (1, 2) or explore <= act < 2 * explore
        fop = bvhcd.FRONT_GENERATE if regen else base_front_op(f)
        main.front.maintain(fop)
        lrn.observe(tag in (1, 2), fop == bvhcd.FRONT_GENERATE)
        if f % stride:
            continue
        X = lrn.features()
        roots = lrn.cut()
        C = len(roots)
        if C < 8:
            continue
        size = np.zeros(C, np.int64)
        inode = main.bvh.export()["inode"]
        size[:] = inode[roots, 5] - inode[roots, 4] + 1
        perm = rng.permutation(C)
        quarter = np.empty(C, np.int64)
        for k in range(N_BRANCH_QUARTERS):
            quarter[perm[k::N_BRANCH_QUARTERS]] = k
        cost = np.full((C, 2 + N_BRANCH_QUARTERS), np.nan)
        for b, pipe in enumerate(branches):
            bvhcd.copy_state(pipe.bvh, main.bvh, pipe.front, main.front)
            if 1 <= b <= N_BRANCH_QUARTERS:
                pipe.bvh.request_restructure(roots[np.sort(np.flatnonzero(quarter == b - 1))])
            pipe.bvh.stage_times(reset=True)
            c = np.zeros(C)
            op_ms = 0.0
            for h in range(1, H + 1):
                g = f + h
                fop_b = bvhcd.FRONT_GENERATE if (b == 1 + N_BRANCH_QUARTERS and h == 1) else base_front_op(g)
                ev[0].record()
                pipe.bvh.maintain(bvhcd.BVH_REFIT, pos[g], faces)
                pipe.front.maintain(fop_b)
                ev[1].record()
                torch.cuda.synchronize()
                ms = ev[0].elapsed_time(ev[1])
                st = pipe.bvh.stage_times(reset=True)
                one_off = 0.0
                if h == 1 and b >= 1:
                    one_off = st["bvh_restructure"][0] + st["front_generate"][0] + st["front_reorder"][0]
                    op_ms = one_off
                w = lrn.work(pipe.front, C).astype(np.float64)
                tot = w.sum()
                if tot > 0:
                    c += (ms - one_off) * w / tot
            if 1 <= b <= N_BRANCH_QUARTERS:
                mine = quarter == b - 1
                leaves = size[mine].sum()
                c[mine] += op_ms * size[mine] / max(leaves, 1)
                cost[mine, 1] = c[mine]
            elif b == 0:
                cost[:, 0] = c
            else:
                cost[:, 2] = c + op_ms * size / max(size.sum(), 1)
        rows.append(X)
        labels.append(cost[:, :3])
        meta.append(np.stack([np.full(C, seed), np.full(C, f), size], 1))
    for pipe in branches + [main]:
        pipe.close()
    return rows, labels, meta


def make_labels(cost, margin):
    """argmin of (refit, restructure, regenerate) costs; an operation must
    beat refit by `margin` (relative)."""
    y = np.zeros(cost.shape[0], np.int32)
    ref = cost[:, 0]
    best_op = np.where(cost[:, 1] <= cost[:, 2], 1, 2)
    best_cost = np.minimum(cost[:, 1], cost[:, 2])
    y[best_cost < ref * (1.0 - margin)] = best_op[best_cost < ref * (1.0 - margin)]
    return y


def cmd_train(args):
    import torch
    torch.cuda.set_device(0)
    rng = np.random.default_rng(args.seed)
    X, Cst, M = [], [], []
    t0 = time.time()
    seq = 0
    while (sum(x.shape[0] for x in X) < args.rows and time.time() - t0 < args.budget_s) or seq < 2:
        amp = float(rng.uniform(0.05, 0.4))
        freq = float(rng.uniform(1.0, 6.0))
        r, c, m = record_sequence(torch, 1000 + seq, args.n, args.frames, amp, freq, args.horizon, args.stride,
                                  args.smax, args.explore, rng)
        X += r
        Cst += c
        M += m
        seq += 1
        print(f"sequence {seq}: amp {amp:.3f} freq {freq:.2f} rows {sum(x.shape[0] for x in X)} "
              f"({time.time() - t0:.0f} s)", flush=True)
    X = np.concatenate(X).astype(np.float32)
    cost = np.concatenate(Cst)
    meta = np.concatenate(M)
    y = make_labels(cost, args.margin)
    counts = np.bincount(y, minlength=3)
    cw = (counts.sum() / np.maximum(counts, 1) / 3.0).astype(np.float32)
    cw = np.minimum(cw, 20.0)
    # validation: the last sequence
    val = meta[:, 0] == meta[:, 0].max()
    bvh = bvhcd.LBvh(64, 64, enable_restr=True)
    front = bvhcd.BvttFront(bvh, 10_000, 10_000, 10_000)
    lrn = bvhcd.Learner(bvh, front, 256)
    Xt, yt = torch.from_numpy(X[~val]).cuda(), torch.from_numpy(y[~val]).cuda()
    Xv = torch.from_numpy(X[val]).cuda()
    losses = []
    for stage, (ep, lr) in enumerate([(args.epochs, args.lr), (args.epochs // 2, args.lr / 4)]):
        losses.append(lrn.train(Xt, yt, class_weight=cw, epochs=ep, batch=args.batch, lr=lr, seed=stage))
    _, vt = lrn.predict(Xt)
    _, vv = lrn.predict(Xv)
    acc_t = float(np.mean(vt == y[~val]))
    acc_v = float(np.mean(vv == y[val]))
    # what the votes would have cost on the validation rows, against refit everywhere
    cv = cost[val]
    pick = np.take_along_axis(cv, vv[:, None].astype(np.int64), 1)[:, 0]
    oracle_pick = np.take_along_axis(cv, y[val][:, None].astype(np.int64), 1)[:, 0]
    report = {"rows": int(X.shape[0]), "sequences": seq, "label_counts": counts.tolist(),
              "class_weight": cw.tolist(), "train_loss": losses, "train_acc": acc_t, "val_acc": acc_v,
              "val_cost_ratio_vs_refit": float(pick.sum() / cv[:, 0].sum()),
              "val_label_cost_ratio_vs_refit": float(oracle_pick.sum() / cv[:, 0].sum()),
              "n": args.n, "frames": args.frames, "horizon": args.horizon, "stride": args.stride,
              "smax": args.smax, "margin": args.margin, "seconds": round(time.time() - t0, 1)}
    params = lrn.params()
    np.savez(args.out, params=params, smax=np.int32(args.smax), report=json.dumps(report))
    if args.dataset:
        np.savez_compressed(args.dataset, X=X, cost=cost, meta=meta)
    print(json.dumps(report), flush=True)


def _digest(p):
    p = np.sort(np.asarray(p, np.int64).reshape(-1, 2), axis=1)
    p = p[np.lexsort((p[:, 1], p[:, 0]))]
    return hashlib.sha256(p.tobytes()).hexdigest()


def evaluate(torch, weights, n, frames, seed, check_every=1, decide_every=3):
    """Heuristic vs learned on one held-out sequence: device ms per frame and
    equal pair sets.  A third run, "cycle", is the learned mode's cycle with
    no network (refit every frame, the front cycle, never a rebuild): what
    the network adds beyond dropping the mandatory rebuilds."""
    w = np.load(weights)
    smax = int(w["smax"])
    faces, pos = scenes.cloth_over_sphere_frames(n, frames, seed=seed, amplitude=0.2)
    T, V = faces.shape[0], pos[0].shape[0]
    caps = _caps(T)
    dpos = torch.from_numpy(np.stack(pos)).cuda()
    dfaces = torch.from_numpy(faces).cuda()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * frames)]
    out = {}
    digests = {}
    for mode in ("heuristic", "learned", "cycle", "keep"):
        bvh = bvhcd.LBvh(T, V, enable_restr=mode in ("heuristic", "learned"))
        front = bvhcd.BvttFront(bvh, *caps, cull_adjacent=True, narrow_phase=True)
        lrn = None
        if mode == "learned":
            lrn = bvhcd.Learner(bvh, front, smax)
            lrn.set_params(w["params"])
            lrn.set_decide_every(decide_every)
        tags, ops, dig = [], [], []
        torch.cuda.synchronize()
        gc.collect()
        gc.disable()
        for f in range(frames):
            ev[2 * f].record()
            if mode == "heuristic":
                bvhcd.frame(bvh, front, f, 0, dpos[f], dfaces, faces_static=f > 0)
            elif mode in ("cycle", "keep"):
                bvh.maintain(bvhcd.BVH_BUILD if f == 0 else bvhcd.BVH_REFIT, dpos[f], dfaces, faces_static=f > 0)
                front.maintain(bvhcd.FRONT_GENERATE if f == 0 else
                               (cycle_front_op(f) if mode == "cycle" else base_front_op(f)))
            else:
                tag, op = lrn.frame(dpos[f], dfaces, f)
            ev[2 * f + 1].record()
            if lrn is None:      # read after the frame's end event: no sync inside the timed region
                tag = bvh.opt_tag() if f else 2
                op = front.stats()["front_op_run"]
            tags.append(tag)
            ops.append(op)
            if f % check_every == 0:
                dig.append((_digest(front.pairs()), _digest(front.pairs(narrow=True))))
        torch.cuda.synchronize()
        gc.enable()
        ms = [ev[2 * f].elapsed_time(ev[2 * f + 1]) for f in range(frames)]
        st = front.stats()
        assert st["overflow_any"] == 0, st
        out[mode] = {"total_ms": round(float(sum(ms)), 3), "mean_ms": round(float(np.mean(ms)), 4),
                     "slowest_frames": [[int(f), round(float(ms[f]), 3)] for f in np.argsort(ms)[::-1][:3]],
                     "p50_ms": round(float(np.median(ms)), 4), "p99_ms": round(float(np.percentile(ms, 99)), 4),
                     "builds": int(sum(1 for f, t in enumerate(tags)
                                       if t == 2 or (mode == "heuristic" and f % 12 == 0))),
                     "restructures": int(sum(1 for t in tags if t == 1)),
                     "generates": int(sum(1 for o in ops if o == bvhcd.FRONT_GENERATE))}
        digests[mode] = dig
        if lrn is not None:
            lrn.close()
        front.close()
        bvh.close()
    out["pairs_equal"] = digests["heuristic"] == digests["learned"] == digests["cycle"] == digests["keep"]
    out["frames_checked"] = len(digests["heuristic"])
    out["speedup"] = round(out["heuristic"]["total_ms"] / out["learned"]["total_ms"], 4)
    out["speedup_cycle"] = round(out["heuristic"]["total_ms"] / out["cycle"]["total_ms"], 4)
    out["speedup_keep"] = round(out["heuristic"]["total_ms"] / out["keep"]["total_ms"], 4)
    out["learned_vs_cycle"] = round(out["cycle"]["total_ms"] / out["learned"]["total_ms"], 4)
    out["decide_every"] = decide_every
    out["workload"] = f"cloth {n}x{n} over icosphere, {T} triangles, {frames} frames, seed {seed}"
    return out


def cmd_eval(args):
    import torch
    torch.cuda.set_device(0)
    res = [evaluate(torch, args.weights, args.n, args.frames, s, args.check_every, args.decide_every)
           for s in args.seeds]
    print(json.dumps(res), flush=True)


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--out", default=WEIGHTS)
    t.add_argument("--dataset", default=None)
    t.add_argument("--rows", type=int, default=1_000_000)
    t.add_argument("--budget-s", type=float, default=900.0)
    t.add_argument("--n", type=int, default=256)
    t.add_argument("--frames", type=int, default=72)
    t.add_argument("--horizon", type=int, default=24)
    t.add_argument("--stride", type=int, default=2)
    t.add_argument("--smax", type=int, default=256)
    t.add_argument("--explore", type=float, default=0.08)
    t.add_argument("--margin", type=float, default=0.02)
    t.add_argument("--epochs", type=int, default=30)
    t.add_argument("--batch", type=int, default=4096)
    t.add_argument("--lr", type=float, default=2e-3)
    t.add_argument("--seed", type=int, default=7)
    e = sub.add_parser("eval")
    e.add_argument("--weights", default=WEIGHTS)
    e.add_argument("--n", type=int, default=708)
    e.add_argument("--frames", type=int, default=200)
    e.add_argument("--seeds", type=int, nargs="+", default=[90001, 90002])
    e.add_argument("--check-every", type=int, default=1)
    e.add_argument("--decide-every", type=int, default=3)
    a = ap.parse_args()
    cmd_train(a) if a.cmd == "train" else cmd_eval(a)


if __name__ == "__main__":
    main()

"""Seeded synthetic frame generators for the collision workloads.

The reference reads mesh sequences from disk through assimp
(Mine/world/Scene.cpp:14-42) and hands the pipeline a ``SceneData{pos, fids}``
(Mine/world/Scene.h:16-20): float3 positions and int3 faces, meshes
concatenated with vertex offsets (Scene.cpp:31-40).  The benchmark datasets it
was evaluated on are not available, so every workload here is generated from
a fixed seed with the shapes, sizes and motion the workload names:

* ``cloth_fold``      128x128 (or n x n) square cloth, analytic fold
                      z = 0.3 sin(2 pi x t) cos(2 pi y t) + N(0, 1e-3),
                      t = (f + 1) / frames.
* ``cloth_over_sphere`` 512x512 cloth with a seeded damped-wave fold of
                      amplitude 0.2 over a geodesic icosphere (frequency 45,
                      40,500 triangles, radius 0.25); per-frame vertex motion
                      at most 2% of an edge length.
* ``stacked_layers``  four cloth layers 1e-3 apart with seeded in-plane shear.
* ``batched_cloth_sphere`` 256 independent cloth-over-sphere scenes whose
                      triangle counts are drawn log-uniform in [1k, 200k]
                      (about 90% cloth, 10% icosphere), each with its own
                      seeded damped wave; concatenated with triangle offsets.

All arrays are float32 positions (V, 3) and int32 faces (T, 3).
"""
from __future__ import annotations

import math

import numpy as np


def cloth_grid(n: int, size: float = 1.0):
    """n x n vertex grid on [0, size]^2, two triangles per quad with a fixed
    diagonal: T = 2 (n - 1)^2."""
    xs = np.linspace(0.0, size, n, dtype=np.float64)
    X, Y = np.meshgrid(xs, xs, indexing="xy")
    idx = np.arange(n * n, dtype=np.int32).reshape(n, n)
    a = idx[:-1, :-1].ravel()
    b = idx[:-1, 1:].ravel()
    c = idx[1:, :-1].ravel()
    d = idx[1:, 1:].ravel()
    f1 = np.stack([a, b, d], axis=1)
    f2 = np.stack([a, d, c], axis=1)
    faces = np.empty((2 * a.size, 3), dtype=np.int32)
    faces[0::2] = f1
    faces[1::2] = f2
    return X.ravel(), Y.ravel(), faces


def cloth_fold_frames(n: int = 128, frames: int = 20, seed: int = 1234,
                      noise: float = 1e-3):
    """Square cloth under the analytic fold; yields (frame, pos) with the
    shared faces returned first.  Frame f uses t = (f + 1) / frames."""
    x, y, faces = cloth_grid(n)
    rng = np.random.default_rng(seed)
    out = []
    for f in range(frames):
        t = (f + 1) / frames
        z = 0.3 * np.sin(2 * np.pi * x * t) * np.cos(2 * np.pi * y * t)
        z = z + rng.normal(0.0, noise, size=z.shape)
        out.append(np.stack([x, y, z], axis=1).astype(np.float32))
    return faces, out


def icosphere(freq: int, radius: float = 1.0, center=(0.0, 0.0, 0.0)):
    """Geodesic icosahedron of the given frequency: 20 freq^2 triangles,
    10 freq^2 + 2 shared vertices, projected on a sphere."""
    p = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([[-1, p, 0], [1, p, 0], [-1, -p, 0], [1, -p, 0],
                  [0, -1, p], [0, 1, p], [0, -1, -p], [0, 1, -p],
                  [p, 0, -1], [p, 0, 1], [-p, 0, -1], [-p, 0, 1]], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    ico = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
           (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
           (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
           (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    keys = {}
    verts = []

    def vid(face, i, j):
        # canonical key of the lattice point i*(B-A)/freq + j*(C-A)/freq + A on
        # the face (A, B, C): weights on the sorted corner ids
        a, b, c = face
        w = {a: freq - i - j, b: i, c: j}
        key = tuple(sorted((k, wt) for k, wt in w.items() if wt > 0))
        if key not in keys:
            pt = sum(v[k] * wt for k, wt in w.items()) / freq
            keys[key] = len(verts)
            verts.append(pt / np.linalg.norm(pt))
        return keys[key]

    faces = []
    for face in ico:
        grid = {}
        for i in range(freq + 1):
            for j in range(freq + 1 - i):
                grid[(i, j)] = vid(face, i, j)
        for i in range(freq):
            for j in range(freq - i):
                faces.append((grid[(i, j)], grid[(i + 1, j)], grid[(i, j + 1)]))
                if i + j < freq - 1:
                    faces.append((grid[(i + 1, j)], grid[(i + 1, j + 1)], grid[(i, j + 1)]))
    verts = np.asarray(verts) * radius + np.asarray(center, dtype=np.float64)
    return verts.astype(np.float64), np.asarray(faces, dtype=np.int32)


def cloth_over_sphere_frames(n: int = 512, frames: int = 100, seed: int = 2024,
                             sphere_freq: int = 45, amplitude: float = 0.2,
                             height: float = 0.2, radius: float = 0.25,
                             first_frame: int = 0, wave_freq: float | None = None):
    """Cloth (n x n on [0,1]^2) folded by a seeded damped radial wave,
    z = height + A e^{-lambda t} sin(k r - omega t + phi), over a static
    icosphere centred under the cloth.  The step in t is chosen so that no
    vertex moves more than 2% of an edge length (1/(n-1)) per frame.
    wave_freq, when given, fixes the wave number k = 2 pi wave_freq (else k is
    drawn from the seed in 2 pi [2, 4]).
    Returns (faces, [pos per frame]) with the sphere appended after the cloth
    (vertex ids offset by the cloth's vertex count)."""
    x, y, cfaces = cloth_grid(n)
    rng = np.random.default_rng(seed)
    cx, cy = rng.uniform(0.3, 0.7, size=2)
    phi = rng.uniform(0.0, 2 * np.pi)
    k = 2 * np.pi * rng.uniform(2.0, 4.0)
    if wave_freq is not None:      # the learned scheduler's training variants set it
        k = 2 * np.pi * float(wave_freq)
    lam, omega = 0.5, 2 * np.pi
    edge = 1.0 / (n - 1)
    dt = 0.02 * edge / (amplitude * (omega + lam)) * 0.999
    r = np.hypot(x - cx, y - cy)
    sv, sf = icosphere(sphere_freq, radius, (0.5, 0.5, 0.0))
    faces = np.concatenate([cfaces, sf + x.size]).astype(np.int32)
    out = []
    prev = None
    for f in range(first_frame, first_frame + frames):
        t = f * dt
        z = height + amplitude * math.exp(-lam * t) * np.sin(k * r - omega * t + phi)
        cloth = np.stack([x, y, z], axis=1)
        if prev is not None:
            assert np.abs(cloth - prev).max() <= 0.02 * edge + 1e-12
        prev = cloth
        out.append(np.concatenate([cloth, sv]).astype(np.float32))
    return faces, out


def stacked_layers_frames(n: int = 512, layers: int = 4, frames: int = 50, seed: int = 77,
                          gap: float = 1e-3, max_shear: float = 0.5, z_noise: float = 0.0):
    """`layers` cloths at z = 0, gap, 2 gap, ... with a seeded in-plane shear
    of up to +-max_shear edge lengths per frame per layer.  z_noise > 0 adds a
    seeded, frame-constant vertical jitter of up to +-z_noise gaps, so that
    neighbouring layers cut through each other at grazing angles."""
    x, y, cf = cloth_grid(n)
    rng = np.random.default_rng(seed)
    edge = 1.0 / (n - 1)
    V = x.size
    faces = np.concatenate([cf + l * V for l in range(layers)]).astype(np.int32)
    shear = np.zeros((layers, 2))
    jit = (rng.uniform(-z_noise, z_noise, size=(layers, x.size)) * gap if z_noise > 0
           else np.zeros((layers, x.size)))
    out = []
    for f in range(frames):
        shear += rng.uniform(-max_shear, max_shear, size=(layers, 2)) * edge
        pts = []
        for l in range(layers):
            sx = x + shear[l, 0] * y
            sy = y + shear[l, 1] * x
            pts.append(np.stack([sx, sy, l * gap + jit[l]], axis=1))
        out.append(np.concatenate(pts).astype(np.float32))
    return faces, out


_ICO_CACHE: dict = {}


def _unit_icosphere(freq: int):
    if freq not in _ICO_CACHE:
        _ICO_CACHE[freq] = icosphere(freq)
    return _ICO_CACHE[freq]


class BatchedScenes:
    """Independent cloth-over-sphere scenes concatenated into one triangle
    and vertex list.  Scene s owns triangles [tri_offsets[s],
    tri_offsets[s+1]) and vertices [vert_offsets[s], vert_offsets[s+1]);
    its faces hold global vertex ids.  positions(f) gives frame f of every
    scene at once.  Every scene lives in its own unit frame (cloth on
    [0,1]^2 at height 0.2 over a sphere of radius 0.25 centred at (0.5, 0.5,
    0)), so the scenes overlap in space: only the batching keeps them apart."""

    def __init__(self, num_scenes: int = 256, t_min: int = 1000, t_max: int = 200_000, seed: int = 4242,
                 amplitude: float = 0.2, height: float = 0.2, radius: float = 0.25):
        rng = np.random.default_rng(seed)
        target = np.exp(rng.uniform(math.log(t_min), math.log(t_max), size=num_scenes))
        faces, tri_off, vert_off = [], [0], [0]
        xs, ys, rs, par = [], [], [], []
        static = []
        lam, omega = 0.5, 2 * np.pi
        self.cloth_verts = []
        for sc in range(num_scenes):
            n = max(3, int(round(math.sqrt(0.45 * target[sc]))) + 1)
            nu = max(1, int(round(math.sqrt(0.005 * target[sc]))))
            x, y, cf = cloth_grid(n)
            sv, sf = _unit_icosphere(nu)
            sv = sv * radius + np.array([0.5, 0.5, 0.0])
            v0 = vert_off[-1]
            faces.append(cf + v0)
            faces.append(sf + v0 + x.size)
            tri_off.append(tri_off[-1] + cf.shape[0] + sf.shape[0])
            vert_off.append(v0 + x.size + sv.shape[0])
            cx, cy = rng.uniform(0.3, 0.7, size=2)
            phi = rng.uniform(0.0, 2 * np.pi)
            k = 2 * np.pi * rng.uniform(2.0, 4.0)
            edge = 1.0 / (n - 1)
            dt = 0.02 * edge / (amplitude * (omega + lam)) * 0.999
            xs.append(x)
            ys.append(y)
            rs.append(np.hypot(x - cx, y - cy))
            par.append(np.repeat(np.array([[k, phi, dt]]), x.size, axis=0))
            static.append((v0 + x.size, sv))
            self.cloth_verts.append((v0, x.size))
        self.num_scenes = num_scenes
        self.faces = np.concatenate(faces).astype(np.int32)
        self.tri_offsets = np.asarray(tri_off, dtype=np.int32)
        self.vert_offsets = np.asarray(vert_off, dtype=np.int64)
        self.num_faces = int(self.tri_offsets[-1])
        self.num_vertices = int(self.vert_offsets[-1])
        self._cloth_idx = np.concatenate([np.arange(v0, v0 + nv) for v0, nv in self.cloth_verts])
        self._x = np.concatenate(xs)
        self._y = np.concatenate(ys)
        self._r = np.concatenate(rs)
        p = np.concatenate(par)
        self._k, self._phi, self._dt = p[:, 0], p[:, 1], p[:, 2]
        self._amp, self._h, self._lam, self._omega = amplitude, height, lam, omega
        self._base = np.zeros((self.num_vertices, 3), dtype=np.float32)
        for v0, sv in static:
            self._base[v0:v0 + sv.shape[0]] = sv
        self._base[self._cloth_idx, 0] = self._x
        self._base[self._cloth_idx, 1] = self._y

    def positions(self, f: int) -> np.ndarray:
        t = f * self._dt
        z = self._h + self._amp * np.exp(-self._lam * t) * np.sin(self._k * self._r - self._omega * t + self._phi)
        out = self._base.copy()
        out[self._cloth_idx, 2] = z
        return out

    def scene(self, s: int, f: int):
        """(faces, positions) of scene s alone at frame f, local vertex ids."""
        v0, v1 = int(self.vert_offsets[s]), int(self.vert_offsets[s + 1])
        t0, t1 = int(self.tri_offsets[s]), int(self.tri_offsets[s + 1])
        return self.faces[t0:t1] - v0, self.positions(f)[v0:v1]

    def subset(self, ids):
        """The scenes `ids` (sorted) as their own batch: (faces with batch-local
        vertex ids, triangle offsets, global vertex index of every batch
        vertex)."""
        ids = np.asarray(sorted(ids), dtype=np.int64)
        vidx = np.concatenate([np.arange(self.vert_offsets[s], self.vert_offsets[s + 1]) for s in ids])
        remap = np.full(self.num_vertices, -1, dtype=np.int64)
        remap[vidx] = np.arange(vidx.size)
        faces = np.concatenate([self.faces[self.tri_offsets[s]:self.tri_offsets[s + 1]] for s in ids])
        off = np.concatenate([[0], np.cumsum([self.tri_offsets[s + 1] - self.tri_offsets[s] for s in ids])])
        return remap[faces].astype(np.int32), off.astype(np.int32), vidx


def shard_scenes(sizes, world: int, rank: int):
    """Scenes of rank `rank` when `world` ranks share a batch: scenes dealt
    largest first to the rank with the fewest triangles so far (ties to the
    lowest rank).  Returns the sorted scene ids."""
    sizes = np.asarray(sizes)
    load = np.zeros(world)
    owner = np.empty(sizes.size, dtype=np.int64)
    for sc in np.argsort(-sizes, kind="stable"):
        r = int(np.argmin(load))
        owner[sc] = r
        load[r] += sizes[sc]
    return np.flatnonzero(owner == rank)

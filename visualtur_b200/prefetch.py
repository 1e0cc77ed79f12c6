"""Learned brick prefetch (no reference counterpart).

A small MLP maps a camera pose to the probability that a frame rendered
from it marches each coarse octree node (level 4: 16^3 nodes).  It is
trained on brick-access traces that the plain renderer logs
(record_trace) during random fly-throughs, by libvt's own forward and
backward kernels (vt_mlp_*).  Before each frame the predicted nodes' bricks
are handed to the renderer as a prefetch hint; demand paging stays the
fallback, so a wrong prediction costs time and never changes a pixel.
"""
import math

import numpy as np

from . import MLP, Camera, vt_camera

TRACE_LEVEL = 4
FEATURES = 12


def pose_features(cam, n, fov_deg):
    """12 normalised features: position (3), forward (3), up (3), FOV (1),
    near/far distance to the volume's bounding sphere (2)."""
    c = (n - 1) / 2.0
    pos = np.array(cam.position[:], np.float64)
    d = np.linalg.norm(pos - c)
    rad = math.sqrt(3.0) * n / 2.0
    f = np.empty(FEATURES, np.float32)
    f[0:3] = (pos - c) / n
    f[3:6] = cam.look[:]
    f[6:9] = cam.up[:]
    f[9] = fov_deg / 90.0
    f[10] = max(d - rad, 0.0) / n
    f[11] = (d + rad) / n
    return f


def look_at(W, H, dist, fov, pos, target, up=(0.0, 1.0, 0.0)):
    """vt_camera at `pos` looking at `target` (right = cross(look, up), the
    reference's basis convention)."""
    cam = Camera(H, W, dist, fov, fov).c
    pos = np.asarray(pos, np.float32)
    look = np.asarray(target, np.float32) - pos
    look = (look / np.sqrt(np.float32((look * look).sum()))).astype(np.float32)
    upv = np.asarray(up, np.float32)
    right = np.cross(look, upv).astype(np.float32)
    rn = np.linalg.norm(right)
    if rn < 1e-6:
        upv = np.array([1, 0, 0], np.float32)
        right = np.cross(look, upv).astype(np.float32)
    upv = np.cross(right, look).astype(np.float32)
    upv /= np.float32(np.linalg.norm(upv))
    right = np.cross(look, upv).astype(np.float32)
    for i in range(3):
        cam.look[i], cam.up[i], cam.right[i], cam.position[i] = look[i], upv[i], right[i], pos[i]
    return cam


def catmull_rom(points, frames):
    """Uniform Catmull-Rom spline through `points` (closed), `frames` samples."""
    P = np.asarray(points, np.float64)
    k = len(P)
    out = []
    for f in range(frames):
        u = f * k / frames
        i = int(u)
        t = u - i
        p0, p1, p2, p3 = P[(i - 1) % k], P[i % k], P[(i + 1) % k], P[(i + 2) % k]
        out.append(0.5 * ((2 * p1) + (-p0 + p2) * t + (2 * p0 - 5 * p1 + 4 * p2 - p3) * t * t +
                          (-p0 + 3 * p1 - 3 * p2 + p3) * t * t * t))
    return np.array(out)


def random_flythrough(rng, n, frames, r_lo, r_hi, ctrl=6):
    """Camera positions on a spline through `ctrl` random points at radius
    [r_lo, r_hi] around the volume centre, each looking at a point of a
    spline through random targets in the volume's inner half."""
    c = (n - 1) / 2.0

    def sphere_pts(m):
        v = rng.standard_normal((m, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        return c + v * rng.uniform(r_lo, r_hi, (m, 1))

    pos = catmull_rom(sphere_pts(ctrl), frames)
    tgt = catmull_rom(c + rng.uniform(-n / 4, n / 4, (ctrl, 3)), frames)
    return pos, tgt


def node_bricks(brick_list, levelC, level=TRACE_LEVEL):
    """coarse node offset (0..8^level-1) -> sorted brick codes inside it"""
    b = np.asarray(brick_list, np.uint64)
    anc = (b >> np.uint64(3 * (levelC - level))) - np.uint64(8 ** level)
    out = {}
    order = np.argsort(anc, kind="stable")
    anc_s, b_s = anc[order], b[order]
    cuts = np.flatnonzero(np.diff(anc_s)) + 1
    for grp_a, grp_b in zip(np.split(anc_s, cuts), np.split(b_s, cuts)):
        if grp_a.size:
            out[int(grp_a[0])] = grp_b
    return out


def trace_to_targets(bits, level=TRACE_LEVEL):
    """bitmask words -> float {0,1} vector over the level's nodes"""
    w = np.asarray(bits, np.uint32)
    return np.unpackbits(w.view(np.uint8), bitorder="little")[:8 ** level].astype(np.float32)


class Prefetcher:
    """Trains the pose -> node network and turns predictions into brick hints."""

    def __init__(self, n, fov, levelC, brick_list, seed=0, hidden=512, level=TRACE_LEVEL):
        self.n, self.fov, self.levelC, self.level = n, fov, levelC, level
        self.mlp = MLP((FEATURES, hidden, hidden, 8 ** level), seed=seed)
        self.set_bricks(brick_list, levelC)

    def set_bricks(self, brick_list, levelC):
        """Brick codes (at levelC) that hints are drawn from: a renderer with
        another brick size takes its own list; the network is unchanged."""
        self.levelC = levelC
        self.groups = node_bricks(brick_list, levelC, self.level)
        # bricks with the coarse node each lies in, for vectorised selection
        self.bricks = np.sort(np.asarray(brick_list, np.uint64))
        self.brick_node = ((self.bricks >> np.uint64(3 * (levelC - self.level))) -
                           np.uint64(8 ** self.level)).astype(np.int64)

    def train(self, torch, X, Y, epochs=30, batch=256, lr=1e-3, seed=0):
        """X: N x 12 features, Y: N x 8^level targets; returns per-epoch loss"""
        dx = torch.from_numpy(np.ascontiguousarray(X, np.float32)).cuda()
        dy = torch.from_numpy(np.ascontiguousarray(Y, np.float32)).cuda()
        rng = np.random.default_rng(seed)
        n = X.shape[0]
        hist = []
        for ep in range(epochs):
            perm = torch.from_numpy(rng.permutation(n)).cuda()
            xs, ys = dx[perm].contiguous(), dy[perm].contiguous()
            tot, cnt = 0.0, 0
            for i in range(0, n - batch + 1, batch):
                tot += self.mlp.train_step(xs[i:i + batch], ys[i:i + batch], batch, lr, want_loss=(i == 0))
                cnt += 1 if i == 0 else 0
            hist.append(tot / max(cnt, 1))
        return hist

    def predict(self, torch, feats):
        f = torch.from_numpy(np.ascontiguousarray(np.atleast_2d(feats), np.float32)).cuda()
        p = torch.empty(f.shape[0] * 8 ** self.level, dtype=torch.float32, device="cuda")
        self.mlp.forward(f, f.shape[0], p)
        torch.cuda.synchronize()
        return p.cpu().numpy().reshape(f.shape[0], -1)

    def bricks_for(self, probs, threshold):
        """sorted brick codes of every node whose probability exceeds threshold"""
        return self.bricks[np.asarray(probs)[self.brick_node] > threshold]

    def reset_hints(self):
        """Forget what was hinted (after the renderer's cache was dropped)."""
        self._last_hint = None

    def new_bricks_for(self, probs, threshold, refresh=32):
        """bricks_for, less those already hinted in the last `refresh` calls:
        once a brick has been hinted it is loaded (or was resident), so
        repeating it only costs the renderer a lookup.  Bricks come back
        after `refresh` calls, in case the cache has evicted them since."""
        if getattr(self, "_last_hint", None) is None or len(self._last_hint) != len(self.bricks):
            self._last_hint = np.full(len(self.bricks), -(1 << 30), np.int64)
            self._calls = 0
        self._calls += 1
        sel = np.asarray(probs)[self.brick_node] > threshold
        sel &= self._last_hint <= self._calls - refresh
        self._last_hint[sel] = self._calls
        return self.bricks[sel]


def collect_traces(renderer, n, W, H, fov, rng, paths, frames, r_lo, r_hi, level=TRACE_LEVEL, dist=50.0):
    """(pose features, marched-node targets) pairs from `paths` random
    fly-throughs of `frames` poses, rendered by `renderer` (record_trace on
    at `level`).  Returns X (N x 12) and Y (N x 8^level)."""
    X, Y = [], []
    for _ in range(paths):
        pos, tgt = random_flythrough(rng, n, frames, r_lo, r_hi)
        for p_, t_ in zip(pos, tgt):
            cam = look_at(W, H, dist, fov, p_, t_)
            renderer.set_camera(cam)
            renderer.updateVisibleCubes(None)
            X.append(pose_features(cam, n, fov))
            Y.append(trace_to_targets(renderer.trace(level), level))
    return np.array(X, np.float32), np.array(Y, np.float32)

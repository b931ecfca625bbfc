"""Seeded synthetic scenes and ray sets for the benchmark configurations.

Every random number comes from Philox4x32-10 (Salmon et al., SC'11) with a
counter made of (element id, draw id, stream tag, 0) and a key of
(seed, config tag), so a scene is a pure function of its parameters and does
not depend on the order or device it is generated on.  Floats in [0, 1) are
``(word >> 8) * 2**-24``.

The scenes restate the benchmark inputs:

* ``uniform_soup``      -- triangles with centres U[0,1]^3 and three vertex
                           offsets U[-s,s]^3 (the 65,536-triangle plain
                           uniform-grid case uses s = 0.01);
* ``cluster_in_field``  -- 90% of the triangles centred in a sphere of radius
                           0.05 about the origin with offsets +-0.002, 10%
                           centred U[-50,50]^3 with offsets +-0.5;
* ``heightfield_boxes`` -- a W x H quad heightfield over [0,1]^2 with Perlin
                           height (amplitude 0.1) plus closed boxes of
                           lognormal(mu=-4, sigma=0.5) side;
* ``random_rays``       -- origins U[-1,2]^3 and uniform unit directions.

Vertices are float32 xyz triples and triangles uint32 index triples
(three unique vertices per triangle unless stated otherwise).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

M0 = np.uint64(0xD2511F53)
M1 = np.uint64(0xCD9E8D57)
W0 = 0x9E3779B9
W1 = 0xBB67AE85
_MASK = np.uint64(0xFFFFFFFF)

TAG_SOUP = 0x534F5550      # "SOUP"
TAG_CLUSTER = 0x434C5553   # "CLUS"
TAG_HEIGHT = 0x48474854    # "HGHT"
TAG_RAYS = 0x52415953      # "RAYS"
TAG_BATCH = 0x42415443     # "BATC"


def philox4x32(c0, c1, c2, c3, k0: int, k1: int):
    """Philox4x32-10 on uint32 counter arrays; returns four uint32 arrays."""
    c0 = np.asarray(c0, dtype=np.uint64) & _MASK
    c1 = np.asarray(c1, dtype=np.uint64) & _MASK
    c2 = np.asarray(c2, dtype=np.uint64) & _MASK
    c3 = np.asarray(c3, dtype=np.uint64) & _MASK
    c0, c1, c2, c3 = np.broadcast_arrays(c0, c1, c2, c3)
    k0 = int(k0) & 0xFFFFFFFF
    k1 = int(k1) & 0xFFFFFFFF
    for _ in range(10):
        p0 = M0 * c0
        p1 = M1 * c2
        h0 = p0 >> np.uint64(32)
        l0 = p0 & _MASK
        h1 = p1 >> np.uint64(32)
        l1 = p1 & _MASK
        n0 = h1 ^ c1 ^ np.uint64(k0)
        n2 = h0 ^ c3 ^ np.uint64(k1)
        c0, c1, c2, c3 = n0, l1, n2, l0
        k0 = (k0 + W0) & 0xFFFFFFFF
        k1 = (k1 + W1) & 0xFFFFFFFF
    return (c0.astype(np.uint32), c1.astype(np.uint32), c2.astype(np.uint32),
            c3.astype(np.uint32))


def u01(words) -> np.ndarray:
    """uint32 -> float32 in [0, 1) with 24 random bits (exact)."""
    return ((np.asarray(words, dtype=np.uint32) >> np.uint32(8)).astype(np.float32)
            * np.float32(1.0 / 16777216.0))


def uniform_draws(n: int, ndraw: int, seed: int, tag: int, stream: int = 0) -> np.ndarray:
    """(n, ndraw) float32 uniforms; draw j of element i uses counter (i, j//4, stream, 0)."""
    nblk = (ndraw + 3) // 4
    ids = np.arange(n, dtype=np.uint64)
    out = np.empty((n, nblk * 4), dtype=np.float32)
    for b in range(nblk):
        w = philox4x32(ids, b, stream, 0, seed, tag)
        for j in range(4):
            out[:, 4 * b + j] = u01(w[j])
    return out[:, :ndraw]


@dataclass
class Scene:
    vertices: np.ndarray   # (nv, 3) float32
    indices: np.ndarray    # (nt, 3) uint32
    name: str = ""

    @property
    def num_triangles(self) -> int:
        return int(self.indices.shape[0])

    @property
    def num_vertices(self) -> int:
        return int(self.vertices.shape[0])


def _soup_from(centers: np.ndarray, offsets: np.ndarray) -> Scene:
    """centers (n,3), offsets (n,3,3) float32 -> one scene with 3 unique vertices per tri."""
    n = centers.shape[0]
    v = (centers[:, None, :] + offsets).astype(np.float32).reshape(n * 3, 3)
    idx = np.arange(n * 3, dtype=np.uint32).reshape(n, 3)
    return Scene(np.ascontiguousarray(v), idx)


def uniform_soup(n: int, seed: int = 0, offset_scale: float = 0.01) -> Scene:
    """Centres U[0,1]^3, vertex offsets U[-s,s]^3, all in float32 arithmetic."""
    u = uniform_draws(n, 12, seed, TAG_SOUP)
    c = u[:, 0:3]
    s = np.float32(offset_scale)
    off = (u[:, 3:12].reshape(n, 3, 3) * np.float32(2.0) - np.float32(1.0)) * s
    sc = _soup_from(c, off)
    sc.name = f"uniform_soup(n={n},seed={seed},s={offset_scale})"
    return sc


def cluster_in_field(n: int, seed: int = 0, cluster_frac: float = 0.9, radius: float = 0.05,
                     cluster_offset: float = 0.002, field_half: float = 50.0,
                     field_offset: float = 0.5) -> Scene:
    """Dense cluster in a sparse field (two-level grid workload)."""
    nc = int(round(cluster_frac * n))
    u = uniform_draws(n, 12, seed, TAG_CLUSTER)
    # cluster centres: uniform in the ball (radius * cbrt(u), isotropic direction)
    uc = u[:nc].astype(np.float64)
    r = radius * np.cbrt(uc[:, 0])
    z = 2.0 * uc[:, 1] - 1.0
    phi = 2.0 * math.pi * uc[:, 2]
    rho = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    cc = np.stack([r * rho * np.cos(phi), r * rho * np.sin(phi), r * z], axis=1).astype(np.float32)
    offc = ((u[:nc, 3:12].reshape(nc, 3, 3) * np.float32(2.0) - np.float32(1.0))
            * np.float32(cluster_offset))
    nf = n - nc
    fc = ((u[nc:, 0:3] * np.float32(2.0) - np.float32(1.0)) * np.float32(field_half))
    offf = ((u[nc:, 3:12].reshape(nf, 3, 3) * np.float32(2.0) - np.float32(1.0))
            * np.float32(field_offset))
    centers = np.concatenate([cc, fc], axis=0)
    offs = np.concatenate([offc, offf], axis=0)
    sc = _soup_from(centers, offs)
    sc.name = f"cluster_in_field(n={n},seed={seed})"
    return sc


def _perlin_grad_table(seed: int) -> np.ndarray:
    w = philox4x32(np.arange(256, dtype=np.uint64), 0, 7, 0, seed, TAG_HEIGHT)
    perm = np.argsort(w[0].astype(np.uint64) * np.uint64(256) + np.arange(256, dtype=np.uint64),
                      kind="stable")
    return np.concatenate([perm, perm]).astype(np.int64)


def perlin2(x: np.ndarray, y: np.ndarray, seed: int) -> np.ndarray:
    """2D gradient (Perlin, SIGGRAPH 2002 'improved noise') in float64, range about [-1, 1]."""
    p = _perlin_grad_table(seed)
    xi = np.floor(x).astype(np.int64)
    yi = np.floor(y).astype(np.int64)
    xf = x - xi
    yf = y - yi
    xi &= 255
    yi &= 255

    def fade(t):
        return t * t * t * (t * (t * 6 - 15) + 10)

    def grad(h, dx, dy):
        h = h & 7
        gx = np.where(h < 4, 1.0, -1.0) * np.where((h & 1) == 0, 1.0, 0.5)
        gy = np.where((h & 2) == 0, 1.0, -1.0) * np.where((h & 1) == 0, 0.5, 1.0)
        return gx * dx + gy * dy

    aa = p[p[xi] + yi]
    ab = p[p[xi] + yi + 1]
    ba = p[p[xi + 1] + yi]
    bb = p[p[xi + 1] + yi + 1]
    u = fade(xf)
    v = fade(yf)
    x1 = grad(aa, xf, yf) * (1 - u) + grad(ba, xf - 1, yf) * u
    x2 = grad(ab, xf, yf - 1) * (1 - u) + grad(bb, xf - 1, yf - 1) * u
    return x1 * (1 - v) + x2 * v


_BOX_TRIS = np.array([
    [0, 2, 1], [1, 2, 3],   # -z
    [4, 5, 6], [5, 7, 6],   # +z
    [0, 1, 4], [1, 5, 4],   # -y
    [2, 6, 3], [3, 6, 7],   # +y
    [0, 4, 2], [2, 4, 6],   # -x
    [1, 3, 5], [3, 7, 5],   # +x
], dtype=np.uint32)


def heightfield_boxes(w: int = 2048, h: int = 1024, seed: int = 2, amplitude: float = 0.1,
                      nboxes: int = 1000, mu: float = -4.0, sigma: float = 0.5,
                      octaves: int = 4) -> Scene:
    """W x H quads (2 triangles each) over [0,1]^2, Perlin height, plus closed boxes."""
    xs = np.linspace(0.0, 1.0, w + 1)
    ys = np.linspace(0.0, 1.0, h + 1)
    gx, gy = np.meshgrid(xs, ys)  # (h+1, w+1)
    z = np.zeros_like(gx)
    freq, amp = 4.0, 1.0
    for _ in range(octaves):
        z += amp * perlin2(gx * freq, gy * freq, seed)
        freq *= 2.0
        amp *= 0.5
    z *= amplitude
    hv = np.stack([gx, gy, z], axis=-1).reshape(-1, 3).astype(np.float32)
    ii, jj = np.meshgrid(np.arange(w), np.arange(h))
    v00 = (jj * (w + 1) + ii).ravel()
    v10 = v00 + 1
    v01 = v00 + (w + 1)
    v11 = v01 + 1
    t0 = np.stack([v00, v10, v11], axis=1)
    t1 = np.stack([v00, v11, v01], axis=1)
    hidx = np.stack([t0, t1], axis=1).reshape(-1, 3).astype(np.uint32)
    # boxes: centre uniform over the field, resting on the local height
    ub = uniform_draws(nboxes, 4, seed, TAG_HEIGHT, stream=1).astype(np.float64)
    # Box-Muller for the lognormal side
    g = np.sqrt(-2.0 * np.log(np.maximum(ub[:, 2], 1e-12))) * np.cos(2.0 * math.pi * ub[:, 3])
    side = np.exp(mu + sigma * g)
    cx, cy = ub[:, 0], ub[:, 1]
    cz = np.zeros_like(cx)
    freq, amp = 4.0, 1.0
    for _ in range(octaves):
        cz += amp * perlin2(cx * freq, cy * freq, seed)
        freq *= 2.0
        amp *= 0.5
    cz *= amplitude
    corners = np.array([[(i >> 0) & 1, (i >> 1) & 1, (i >> 2) & 1] for i in range(8)], dtype=np.float64)
    lo = np.stack([cx - side / 2, cy - side / 2, cz - side / 4], axis=1)
    bv = (lo[:, None, :] + corners[None, :, :] * side[:, None, None]).reshape(-1, 3).astype(np.float32)
    base = hv.shape[0] + (np.arange(nboxes, dtype=np.uint32) * 8)
    bidx = (base[:, None, None] + _BOX_TRIS[None, :, :]).reshape(-1, 3).astype(np.uint32)
    sc = Scene(np.ascontiguousarray(np.concatenate([hv, bv], axis=0)),
               np.ascontiguousarray(np.concatenate([hidx, bidx], axis=0)))
    sc.name = f"heightfield_boxes({w}x{h},seed={seed},boxes={nboxes})"
    return sc


def random_rays(n: int, seed: int, lo: float = -1.0, hi: float = 2.0, stream: int = 0):
    """Origins U[lo,hi]^3 and uniform unit directions; returns (org (n,3), dir (n,3)) float32."""
    u = uniform_draws(n, 5, seed, TAG_RAYS, stream=stream)
    span = np.float32(hi - lo)
    org = (u[:, 0:3] * span + np.float32(lo)).astype(np.float32)
    ud = u[:, 3:5].astype(np.float64)
    z = 2.0 * ud[:, 0] - 1.0
    phi = 2.0 * math.pi * ud[:, 1]
    rho = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    d = np.stack([rho * np.cos(phi), rho * np.sin(phi), z], axis=1).astype(np.float32)
    return np.ascontiguousarray(org), np.ascontiguousarray(d)


def log_uniform_ints(n: int, lo: float, hi: float, seed: int, tag: int, stream: int) -> np.ndarray:
    u = uniform_draws(n, 1, seed, tag, stream=stream)[:, 0].astype(np.float64)
    return np.floor(np.exp(math.log(lo) + u * (math.log(hi) - math.log(lo)))).astype(np.int64)


@dataclass
class Camera:
    eye: tuple
    forward: tuple
    up: tuple
    fov_deg: float
    res_x: int
    res_y: int


# Camera of the plain uniform-grid case (pinhole at (0.5,0.5,-1.5) looking +z, 45 deg).
CAMERA_SOUP = Camera((0.5, 0.5, -1.5), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 45.0, 512, 512)
# Camera of the cluster-in-field case: inside the field, 0.25 in front of the
# cluster, looking at it (+z), 45 deg vertical opening, 1920 x 1080.
CAMERA_CLUSTER = Camera((0.0, 0.0, -0.25), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 45.0, 1920, 1080)
# Camera of the heightfield path-tracing case: above the field looking down at 45 deg.
CAMERA_HEIGHTFIELD = Camera((0.5, -0.35, 0.65), (0.0, 0.70710678, -0.70710678),
                            (0.0, 0.0, 1.0), 45.0, 1920, 1080)


# ---------------------------------------------------------------------------
# Device-side generation (torch on CUDA) for the large batched workloads: the
# same Philox counters and float32 arithmetic as the numpy functions above,
# so the outputs are identical, only produced on the GPU.
def _philox_torch(c0, c1, c2, c3, k0: int, k1: int):
    import torch
    m = 0xFFFFFFFF
    M0t, M1t = 0xD2511F53, 0xCD9E8D57
    k0 &= m
    k1 &= m
    for _ in range(10):
        p0 = c0 * M0t
        p1 = c2 * M1t
        h0 = (p0 >> 32) & m
        l0 = p0 & m
        h1 = (p1 >> 32) & m
        l1 = p1 & m
        n0 = h1 ^ c1 ^ k0
        n2 = h0 ^ c3 ^ k1
        c0, c1, c2, c3 = n0, l1, n2, l0
        k0 = (k0 + W0) & m
        k1 = (k1 + W1) & m
    return c0, c1, c2, c3


def _u01_torch(w):
    import torch
    return (w >> 8).to(torch.float32) * torch.tensor(1.0 / 16777216.0, dtype=torch.float32, device=w.device)


def uniform_soup_device(n: int, seed: int = 0, offset_scale: float = 0.01, device="cuda", chunk=1 << 22):
    """uniform_soup generated on the GPU: returns (vertices (3n,3) float32, indices (n,3) int32)."""
    import torch
    verts = torch.empty(3 * n, 3, dtype=torch.float32, device=device)
    s = torch.tensor(offset_scale, dtype=torch.float32, device=device)
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        ids = torch.arange(a, b, dtype=torch.int64, device=device)
        zero = torch.zeros_like(ids)
        u = []
        for blk in range(3):
            w = _philox_torch(ids, zero + blk, zero, zero, seed, TAG_SOUP)
            u.extend(_u01_torch(x) for x in w)
        c = torch.stack(u[0:3], dim=1)
        off = (torch.stack(u[3:12], dim=1).reshape(-1, 3, 3) * 2.0 - 1.0) * s
        verts[3 * a:3 * b] = (c[:, None, :] + off).reshape(-1, 3)
    idx = torch.arange(3 * n, dtype=torch.int32, device=device).reshape(n, 3)
    return verts, idx


def random_rays_device(n: int, seed: int, lo: float = -1.0, hi: float = 2.0, stream: int = 0,
                       device="cuda"):
    """random_rays generated on the GPU (float64 trigonometry, then float32)."""
    import torch
    ids = torch.arange(n, dtype=torch.int64, device=device)
    zero = torch.zeros_like(ids)
    w = _philox_torch(ids, zero, zero + stream, zero, seed, TAG_RAYS)
    w2 = _philox_torch(ids, zero + 1, zero + stream, zero, seed, TAG_RAYS)
    u = [_u01_torch(x) for x in w] + [_u01_torch(w2[0])]
    span = torch.tensor(hi - lo, dtype=torch.float32, device=device)
    org = torch.stack(u[0:3], dim=1) * span + torch.tensor(lo, dtype=torch.float32, device=device)
    z = 2.0 * u[3].double() - 1.0
    phi = 2.0 * math.pi * u[4].double()
    rho = torch.sqrt(torch.clamp(1.0 - z * z, min=0.0))
    d = torch.stack([rho * torch.cos(phi), rho * torch.sin(phi), z], dim=1).float()
    return org.contiguous(), d.contiguous()


def batch_workload_sizes(num_scenes: int = 256, seed: int = 3):
    """Per-scene triangle counts log-U[1K, 2M], offset scales log-U[0.001, 0.05], ray counts log-U[64K, 1M]."""
    tris = log_uniform_ints(num_scenes, 1e3, 2e6, seed, TAG_BATCH, 0)
    u = uniform_draws(num_scenes, 1, seed, TAG_BATCH, stream=1)[:, 0].astype(np.float64)
    scales = np.exp(math.log(0.001) + u * (math.log(0.05) - math.log(0.001))).astype(np.float32)
    rays = log_uniform_ints(num_scenes, 65536, 1 << 20, seed, TAG_BATCH, 2)
    return tris, scales, rays

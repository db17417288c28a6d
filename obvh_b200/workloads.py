"""Seeded synthetic inputs with the shapes of the reference's benchmark scenes.

The reference's bundled glTF scenes ship without their geometry blobs, so
these generators stand in for them (shapes, sizes and value distributions as
specified for each workload; all float32):

* ``ellipsoid_points``   - points uniform on an ellipsoid surface, rotated,
  noised and offset (the plain DiTO fit).
* ``triangle_soup``      - thin randomly oriented triangles around uniform
  centroids, a hairball-like soup (the LBVH + OBB-tree build).
* ``torus_knot_mesh``    - a closed (2,3) torus-knot tube with a bumpy surface
  (the ATRBVH + OBB-tree build).
* ``gaussian_sets``      - many anisotropic Gaussian clouds of log-uniform
  sizes in one CSR buffer (batched DiTO fits).
"""
from __future__ import annotations

import math

import numpy as np


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    """Uniform (Haar) random rotation from a normalised Gaussian quaternion."""
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def unit_vectors(rng: np.random.Generator, n: int) -> np.ndarray:
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v


def ellipsoid_points(n: int, seed: int = 0, axes=(4.0, 1.0, 0.25), noise: float = 0.01,
                     offset_range: float = 10.0, chunk: int = 1 << 22) -> np.ndarray:
    """n points uniform (by area) on the ellipsoid surface with semi-axes `axes`,
    rotated by a Haar rotation, with N(0, noise^2) per coordinate and a uniform
    [-offset_range, offset_range]^3 offset.  Area-uniformity by rejection: a
    sphere direction u maps to axes*u and is kept with probability
    |area element| / max."""
    rng = np.random.default_rng(seed)
    a = np.asarray(axes, np.float64)
    rot = random_rotation(rng)
    off = rng.uniform(-offset_range, offset_range, size=3)
    gmax = max(a[1] * a[2], a[0] * a[2], a[0] * a[1])
    out = np.empty((n, 3), np.float32)
    filled = 0
    while filled < n:
        m = min(chunk, 2 * (n - filled) + 1024)
        u = unit_vectors(rng, m)
        g = np.sqrt((a[1] * a[2] * u[:, 0]) ** 2 + (a[0] * a[2] * u[:, 1]) ** 2 + (a[0] * a[1] * u[:, 2]) ** 2)
        keep = rng.uniform(size=m) * gmax < g
        p = u[keep] * a
        take = min(len(p), n - filled)
        p = p[:take] @ rot.T + rng.normal(scale=noise, size=(take, 3)) + off
        out[filled:filled + take] = p
        filled += take
    return out


def ellipsoid_points_torch(n: int, seed: int = 0, device="cuda", axes=(4.0, 1.0, 0.25), noise: float = 0.01,
                           offset_range: float = 10.0):
    """Same distribution as ellipsoid_points, generated with torch on `device`
    (fast enough for the 100M-point roofline runs; a different random stream)."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    rng = np.random.default_rng(seed)
    rot = torch.tensor(random_rotation(rng), dtype=torch.float32, device=device)
    off = torch.tensor(rng.uniform(-offset_range, offset_range, size=3), dtype=torch.float32, device=device)
    a = torch.tensor(axes, dtype=torch.float32, device=device)
    gmax = max(axes[1] * axes[2], axes[0] * axes[2], axes[0] * axes[1])
    out = torch.empty((n, 3), dtype=torch.float32, device=device)
    filled = 0
    while filled < n:
        m = min(1 << 25, 2 * (n - filled) + 1024)
        u = torch.randn((m, 3), generator=g, device=device)
        u /= u.norm(dim=1, keepdim=True)
        el = torch.sqrt((a[1] * a[2] * u[:, 0]) ** 2 + (a[0] * a[2] * u[:, 1]) ** 2 + (a[0] * a[1] * u[:, 2]) ** 2)
        keep = torch.rand(m, generator=g, device=device) * gmax < el
        p = u[keep] * a
        take = min(p.shape[0], n - filled)
        p = p[:take] @ rot.T + noise * torch.randn((take, 3), generator=g, device=device) + off
        out[filled:filled + take] = p
        filled += take
    return out


def triangle_soup(n_tris: int, seed: int = 1, rmin: float = 0.002, rmax: float = 0.02):
    """(vertices [3n x 3] float32, faces [n x 4] uint32): face i = (3i, 3i+1, 3i+2, 0);
    centroid uniform in [0,1]^3, each vertex at centroid + r*u with u uniform on the
    sphere and r log-uniform in [rmin, rmax]."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.0, 1.0, size=(n_tris, 1, 3))
    u = unit_vectors(rng, 3 * n_tris).reshape(n_tris, 3, 3)
    r = np.exp(rng.uniform(math.log(rmin), math.log(rmax), size=(n_tris, 3, 1)))
    v = (c + r * u).reshape(-1, 3).astype(np.float32)
    f = np.zeros((n_tris, 4), np.uint32)
    f[:, 0] = np.arange(0, 3 * n_tris, 3, dtype=np.uint32)
    f[:, 1] = f[:, 0] + 1
    f[:, 2] = f[:, 0] + 2
    return v, f


def torus_knot_mesh(segments: int = 1024, around: int = 448, seed: int = 2, p: int = 2, q: int = 3,
                    tube: float = 0.15, bump: float = 0.02, noise: float = 0.005):
    """Closed (p,q) torus-knot tube: (vertices [segments*around x 3] float32,
    faces [2*segments*around x 4] uint32).

    Centre curve (theta in [0, 2pi)):
        r(theta) = 2 + cos(q theta)
        c(theta) = (r cos(p theta), r sin(p theta), -sin(q theta))
    The tube cross-section uses a parallel-transport-free Frenet-like frame from
    the curve tangent and the z axis; the surface radius at (theta, phi) is
    tube + bump*sin(13 theta)*cos(7 phi) + U[0, noise]."""
    rng = np.random.default_rng(seed)
    th = np.arange(segments) * (2 * math.pi / segments)
    ph = np.arange(around) * (2 * math.pi / around)
    r = 2.0 + np.cos(q * th)
    c = np.stack([r * np.cos(p * th), r * np.sin(p * th), -np.sin(q * th)], axis=1)
    dr = -q * np.sin(q * th)
    t = np.stack([dr * np.cos(p * th) - r * p * np.sin(p * th),
                  dr * np.sin(p * th) + r * p * np.cos(p * th),
                  -q * np.cos(q * th)], axis=1)
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    zaxis = np.array([0.0, 0.0, 1.0])
    nrm = np.cross(t, zaxis)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    bin_ = np.cross(t, nrm)
    rad = tube + bump * np.sin(13 * th)[:, None] * np.cos(7 * ph)[None, :] + rng.uniform(0, noise, size=(segments, around))
    cp, sp = np.cos(ph)[None, :, None], np.sin(ph)[None, :, None]
    v = c[:, None, :] + rad[:, :, None] * (cp * nrm[:, None, :] + sp * bin_[:, None, :])
    v = v.reshape(-1, 3).astype(np.float32)
    i = np.arange(segments)[:, None]
    j = np.arange(around)[None, :]
    a = i * around + j
    b = ((i + 1) % segments) * around + j
    a1 = i * around + (j + 1) % around
    b1 = ((i + 1) % segments) * around + (j + 1) % around
    f = np.zeros((segments, around, 2, 4), np.uint32)
    f[:, :, 0, 0], f[:, :, 0, 1], f[:, :, 0, 2] = a, b, b1
    f[:, :, 1, 0], f[:, :, 1, 1], f[:, :, 1, 2] = a, b1, a1
    return v, f.reshape(-1, 4)


def gaussian_sets(n_sets: int = 4096, seed: int = 3, size_min: int = 64, size_max: int = 262144,
                  sigma_min: float = 0.01, sigma_max: float = 5.0, offset_range: float = 100.0):
    """(points [total x 3] float32, offsets [n_sets+1] int64): set s is
    points[offsets[s]:offsets[s+1]], an anisotropic Gaussian cloud (per-axis
    sigma log-uniform), rotated and offset; sizes log-uniform."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(size_min), math.log(size_max), size=n_sets)).astype(np.int64)
    offsets = np.zeros(n_sets + 1, np.int64)
    np.cumsum(sizes, out=offsets[1:])
    pts = np.empty((offsets[-1], 3), np.float32)
    for s in range(n_sets):
        sig = np.exp(rng.uniform(math.log(sigma_min), math.log(sigma_max), size=3))
        rot = random_rotation(rng)
        off = rng.uniform(-offset_range, offset_range, size=3)
        x = rng.normal(size=(sizes[s], 3)) * sig
        pts[offsets[s]:offsets[s + 1]] = x @ rot.T + off
    return pts, offsets


def gaussian_sets_torch(n_sets: int = 4096, seed: int = 3, size_min: int = 64, size_max: int = 262144,
                        sigma_min: float = 0.01, sigma_max: float = 5.0, offset_range: float = 100.0,
                        device="cuda"):
    """Same distribution as gaussian_sets, generated with torch on `device`
    (fast enough for the 4,096-set runs; a different random stream for the
    points).  Returns (points [total x 3] float32 tensor, offsets int64 numpy)."""
    import torch
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(size_min), math.log(size_max), size=n_sets)).astype(np.int64)
    offsets = np.zeros(n_sets + 1, np.int64)
    np.cumsum(sizes, out=offsets[1:])
    sig = np.exp(rng.uniform(math.log(sigma_min), math.log(sigma_max), size=(n_sets, 3)))
    rot = np.stack([random_rotation(rng) for _ in range(n_sets)])
    off = rng.uniform(-offset_range, offset_range, size=(n_sets, 3))
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    out = torch.empty((int(offsets[-1]), 3), dtype=torch.float32, device=device)
    # a few thousand sets per slab keeps the temporaries small
    step = 256
    for s0 in range(0, n_sets, step):
        s1 = min(n_sets, s0 + step)
        a, b = int(offsets[s0]), int(offsets[s1])
        ids = torch.repeat_interleave(torch.arange(s1 - s0, device=device),
                                      torch.tensor(sizes[s0:s1], device=device))
        x = torch.randn((b - a, 3), generator=g, device=device, dtype=torch.float64)
        x = x * torch.tensor(sig[s0:s1], device=device)[ids]
        r = torch.tensor(rot[s0:s1], device=device)[ids]
        y = torch.einsum("nij,nj->ni", r, x) + torch.tensor(off[s0:s1], device=device)[ids]
        out[a:b] = y.to(torch.float32)
    return out, offsets


def triangle_soup_torch(n_tris: int, seed: int = 1, rmin: float = 0.002, rmax: float = 0.02, device="cuda"):
    """Same distribution as triangle_soup, generated with torch on `device` (a
    different random stream): (vertices [3n x 3] float32, faces [n x 4] int32
    with face i = (3i, 3i+1, 3i+2, 0))."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    c = torch.rand((n_tris, 1, 3), generator=g, device=device, dtype=torch.float64)
    u = torch.randn((n_tris, 3, 3), generator=g, device=device, dtype=torch.float64)
    u = u / u.norm(dim=2, keepdim=True)
    r = torch.exp(torch.rand((n_tris, 3, 1), generator=g, device=device, dtype=torch.float64)
                  * (math.log(rmax) - math.log(rmin)) + math.log(rmin))
    v = (c + r * u).reshape(-1, 3).to(torch.float32)
    f = torch.zeros((n_tris, 4), dtype=torch.int32, device=device)
    base = torch.arange(0, 3 * n_tris, 3, dtype=torch.int32, device=device)
    f[:, 0] = base
    f[:, 1] = base + 1
    f[:, 2] = base + 2
    return v, f


def gaussian_cloud_torch(n: int, rng: np.random.Generator, device="cuda", sigma_min: float = 0.01,
                         sigma_max: float = 5.0, offset_range: float = 100.0):
    """One anisotropic Gaussian cloud (the gaussian_sets generator for a single
    set): per-axis sigma log-uniform, Haar rotation, uniform offset."""
    import torch
    sig = np.exp(rng.uniform(math.log(sigma_min), math.log(sigma_max), size=3))
    rot = random_rotation(rng)
    off = rng.uniform(-offset_range, offset_range, size=3)
    g = torch.Generator(device=device)
    g.manual_seed(int(rng.integers(0, 2 ** 62)))
    x = torch.randn((n, 3), generator=g, device=device, dtype=torch.float64) * torch.tensor(sig, device=device)
    y = x @ torch.tensor(rot.T, device=device) + torch.tensor(off, device=device)
    return y.to(torch.float32).contiguous()


RAY = np.dtype([("origin", "<f4", (3,)), ("tmin", "<f4"), ("direction", "<f4", (3,)), ("tmax", "<f4")])
ISECT = np.dtype([("normal", "<f4", (3,)), ("barys", "<f4", (2,)), ("primitive", "<u4"), ("instance", "<u4")])


def probe_rays(n: int, lo, hi, seed: int = 5, tmax: float = 1e30) -> np.ndarray:
    """n rays (kr_ray records) into the box [lo, hi]: origins uniform on the
    sphere of twice the box's half-diagonal around its centre, directions
    (unnormalised) towards uniform points inside the box, tmin 0."""
    rng = np.random.default_rng(seed)
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    c = 0.5 * (lo + hi)
    radius = float(np.linalg.norm(hi - lo))
    o = c + radius * unit_vectors(rng, n)
    target = lo + rng.uniform(0.0, 1.0, size=(n, 3)) * (hi - lo)
    r = np.zeros(n, RAY)
    r["origin"] = o.astype(np.float32)
    r["direction"] = (target - o).astype(np.float32)
    r["tmax"] = np.float32(tmax)
    return r

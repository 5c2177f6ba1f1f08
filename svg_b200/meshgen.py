"""Seeded synthetic triangle meshes standing in for the reference's benchmark
meshes (Fertility 30K, Stanford Bunny 72K, Dragon 750K, README.md:8-10), which
are not available here.  All geometry is float64.

Layout conventions (fixed, so every consumer sees identical arrays):
  torus:        vertex (i, j), i over the major angle u (nu steps), j over the
                minor angle v (nv steps), index i*nv + j.
  height field: vertex (ix, iy) on an n x n grid over [0,1]^2, index iy*n + ix.
  Each grid quad a=(i,j) b=(i+1,j) c=(i+1,j+1) d=(i,j+1) is split along a-c on
  even rows (row = i for the torus, iy for the height field) and along b-d on
  odd rows, triangles oriented consistently (a,b,c)/(a,c,d) or (a,b,d)/(b,c,d).

Random draws use numpy.random.default_rng(seed) in the order documented in
each function.
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "torus", "torus_value_noise", "height_field", "config_mesh", "pool_meshes",
    "write_obj", "grid_faces",
]


def grid_faces(nu: int, nv: int, wrap_u: bool, wrap_v: bool, index) -> np.ndarray:
    """Triangles of an (nu x nv) vertex grid; index(i, j) -> vertex id arrays."""
    iu = np.arange(nu if wrap_u else nu - 1)
    jv = np.arange(nv if wrap_v else nv - 1)
    I, J = np.meshgrid(iu, jv, indexing="ij")
    I1 = (I + 1) % nu
    J1 = (J + 1) % nv
    a, b, c, d = index(I, J), index(I1, J), index(I1, J1), index(I, J1)
    even = (I % 2) == 0
    t0 = np.where(even[..., None], np.stack([a, b, c], -1), np.stack([a, b, d], -1))
    t1 = np.where(even[..., None], np.stack([a, c, d], -1), np.stack([b, c, d], -1))
    # per quad: t0 then t1, quads in (i, j) row-major order
    faces = np.stack([t0, t1], axis=2).reshape(-1, 3)
    return faces.astype(np.int32)


def _torus_points(R: float, rr: np.ndarray, nu: int, nv: int) -> np.ndarray:
    u = 2.0 * np.pi * np.arange(nu) / nu
    v = 2.0 * np.pi * np.arange(nv) / nv
    U, Vv = np.meshgrid(u, v, indexing="ij")
    rr = rr.reshape(nu, nv)
    ring = R + rr * np.cos(Vv)
    pos = np.stack([ring * np.cos(U), ring * np.sin(U), rr * np.sin(Vv)], -1)
    return pos.reshape(-1, 3).astype(np.float64)


def torus(R: float = 1.0, r: float = 0.35, nu: int = 200, nv: int = 150,
          noise: float = 0.02, seed: int = 0):
    """Closed torus; tube radius displaced by noise*r*N(0,1) per vertex
    (one standard_normal draw per vertex, in vertex-index order)."""
    rng = np.random.default_rng(seed)
    V = nu * nv
    rr = r + noise * r * rng.standard_normal(V)
    pos = _torus_points(R, rr, nu, nv)
    faces = grid_faces(nu, nv, True, True, lambda i, j: i * nv + j)
    return pos, faces


def _value_noise(rng, f: int, uf: np.ndarray, vf: np.ndarray) -> np.ndarray:
    """Periodic value noise: an f x f lattice of U[-1,1] values over the unit
    torus, smoothstep-bilinear interpolation at (uf, vf) in [0,1)^2."""
    lat = rng.uniform(-1.0, 1.0, size=(f, f))
    x = uf * f
    y = vf * f
    x0 = np.floor(x).astype(np.int64)
    y0 = np.floor(y).astype(np.int64)
    tx = x - x0
    ty = y - y0
    sx = tx * tx * (3.0 - 2.0 * tx)
    sy = ty * ty * (3.0 - 2.0 * ty)
    i0, i1 = x0 % f, (x0 + 1) % f
    j0, j1 = y0 % f, (y0 + 1) % f
    a = lat[i0, j0] * (1 - sx) + lat[i1, j0] * sx
    b = lat[i0, j1] * (1 - sx) + lat[i1, j1] * sx
    return a * (1 - sy) + b * sy


def torus_value_noise(R: float = 1.0, r: float = 0.4, nu: int = 1000, nv: int = 750,
                      octaves: int = 5, amp: float = 0.03, base_freq: int = 8, seed: int = 2):
    """Closed torus whose tube radius is displaced by the sum over octaves o of
    amp*r*0.5^o * value_noise(frequency base_freq*2^o); one lattice draw per
    octave, octave 0 first."""
    rng = np.random.default_rng(seed)
    uf = (np.arange(nu) / nu)[:, None] * np.ones((1, nv))
    vf = np.ones((nu, 1)) * (np.arange(nv) / nv)[None, :]
    disp = np.zeros((nu, nv))
    for o in range(octaves):
        disp += amp * r * 0.5 ** o * _value_noise(rng, base_freq * 2 ** o, uf, vf)
    pos = _torus_points(R, r + disp.reshape(-1), nu, nv)
    faces = grid_faces(nu, nv, True, True, lambda i, j: i * nv + j)
    return pos, faces


def height_field(n: int = 270, bumps: int = 64, jitter: float = 0.2, seed: int = 1,
                 sigma_range=(0.02, 0.15), amp_std: float = 0.08):
    """Open height field on [0,1]^2.  Draw order: jitter U[-j,j]*h for every
    vertex (x then y; boundary vertices then reset to 0), bump centres
    U[0,1]^2 (bumps x 2), sigmas U[sigma_range] (bumps), amplitudes
    N(0, amp_std) (bumps)."""
    rng = np.random.default_rng(seed)
    h = 1.0 / (n - 1)
    ix, iy = np.meshgrid(np.arange(n), np.arange(n), indexing="xy")
    ix = ix.reshape(-1)
    iy = iy.reshape(-1)
    jit = rng.uniform(-jitter, jitter, size=(n * n, 2)) * h
    boundary = (ix == 0) | (iy == 0) | (ix == n - 1) | (iy == n - 1)
    jit[boundary] = 0.0
    x = ix * h + jit[:, 0]
    y = iy * h + jit[:, 1]
    centres = rng.uniform(0.0, 1.0, size=(bumps, 2))
    sig = rng.uniform(sigma_range[0], sigma_range[1], size=bumps)
    amp = rng.normal(0.0, amp_std, size=bumps)
    z = np.zeros_like(x)
    for k in range(bumps):
        d2 = (x - centres[k, 0]) ** 2 + (y - centres[k, 1]) ** 2
        z += amp[k] * np.exp(-d2 / (2.0 * sig[k] ** 2))
    pos = np.stack([x, y, z], -1).astype(np.float64)
    # row index for the diagonal rule is iy: pass (iy, ix) as (i, j)
    faces = grid_faces(n, n, False, False, lambda i, j: i * n + j)
    return pos, faces


def config_mesh(idx: int, scale: float = 1.0):
    """Meshes of the benchmark configurations; scale < 1 shrinks the grid
    (same generator and seed) for quick tests."""
    def s(k):
        return max(4, int(round(k * scale)))
    if idx == 0:
        return torus(1.0, 0.35, s(200), s(150), 0.02, seed=0)
    if idx == 1:
        return height_field(s(270), seed=1)
    if idx == 2:
        return torus_value_noise(1.0, 0.4, s(1000), s(750), seed=2)
    raise ValueError(f"no mesh for configuration {idx}")


def pool_meshes(scale: float = 1.0):
    """The mixed build+query pool: 8 meshes of 5K..300K vertices (seeds 10-17),
    tori (even slots) and height fields (odd slots)."""
    sizes = [5000, 12000, 30000, 50000, 80000, 120000, 200000, 300000]
    out = []
    for k, nverts in enumerate(sizes):
        seed = 10 + k
        nverts = max(64, int(nverts * scale))
        if k % 2 == 0:
            nv = max(4, int(round(np.sqrt(nverts * 3.0 / 4.0))))
            nu = max(4, int(round(nverts / nv)))
            out.append(torus(1.0, 0.35, nu, nv, 0.02, seed=seed))
        else:
            n = max(4, int(round(np.sqrt(nverts))))
            out.append(height_field(n, seed=seed))
    return out


def write_obj(path: str, pos: np.ndarray, faces: np.ndarray) -> None:
    """OBJ with %.17g coordinates: parsing them back with strtod (or a C++
    stream, as the reference loader does) reproduces every double exactly."""
    with open(path, "w") as f:
        f.write("".join("v %.17g %.17g %.17g\n" % tuple(p) for p in pos))
        f.write("".join("f %d %d %d\n" % (a + 1, b + 1, c + 1) for a, b, c in faces))

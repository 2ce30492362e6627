"""Synthetic Delaunay scenes with the shapes of the rmeshvk benchmark configs.

Tet meshes come from ``scipy.spatial.Delaunay`` of seeded point clouds.  Per-tet
parameters follow the distributions named by the benchmark configurations:
densities ``exp(N(0,1))``, color gradients ``N(0, 0.1)``, degree-0 SH
coefficients ``N(0, 0.5)``.  In base-color mode (the reference training path,
which copies ``base_colors`` straight into the per-tet colour,
project_compute.wgsl:319-324) the base colour is the degree-0 SH value
``0.5 + C0 * sh0``.

``circumspheres`` follows crates/rmesh-util/src/test_util.rs:133-163
(and the Python twin in crates/rmesh-python/tests/test_autograd.py:14-31):
``denom = 2 a.(b x c)``, replaced by 1 when ``|denom| < 1e-12``.
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "circumspheres", "delaunay_tets", "uniform_cloud", "gmm_cloud", "shell_cloud",
    "make_scene", "CONFIGS", "scene_for_config", "SH_C0",
]

SH_C0 = 0.28209479177387814


def circumspheres(vertices: np.ndarray, indices: np.ndarray) -> np.ndarray:
    """(cx, cy, cz, r^2) per tet, float32 [4M]; computed in float64."""
    v = np.asarray(vertices, dtype=np.float64).reshape(-1, 3)
    t = np.asarray(indices, dtype=np.int64).reshape(-1, 4)
    v0, v1, v2, v3 = v[t[:, 0]], v[t[:, 1]], v[t[:, 2]], v[t[:, 3]]
    a, b, c = v1 - v0, v2 - v0, v3 - v0
    aa = np.einsum("ij,ij->i", a, a)[:, None]
    bb = np.einsum("ij,ij->i", b, b)[:, None]
    cc = np.einsum("ij,ij->i", c, c)[:, None]
    cbc, cca, cab = np.cross(b, c), np.cross(c, a), np.cross(a, b)
    denom = 2.0 * np.einsum("ij,ij->i", a, cbc)
    denom = np.where(np.abs(denom) < 1e-12, 1.0, denom)[:, None]
    r = (aa * cbc + bb * cca + cc * cab) / denom
    center = v0 + r
    out = np.concatenate([center, np.einsum("ij,ij->i", r, r)[:, None]], axis=1)
    return np.ascontiguousarray(out.astype(np.float32).ravel())


def delaunay_tets(points: np.ndarray) -> np.ndarray:
    """uint32 [4M] tet indices of the Delaunay tetrahedralisation."""
    from scipy.spatial import Delaunay

    tri = Delaunay(np.asarray(points, dtype=np.float64))
    return np.ascontiguousarray(tri.simplices.astype(np.uint32).ravel())


def uniform_cloud(n: int, rng: np.random.Generator, lo=-1.0, hi=1.0) -> np.ndarray:
    return rng.uniform(lo, hi, size=(n, 3))


def gmm_cloud(n: int, rng: np.random.Generator, k: int = 8, sigma=(0.15, 0.4)) -> np.ndarray:
    """``k``-component Gaussian mixture: means U[-1,1]^3, isotropic sigma U[sigma]."""
    means = rng.uniform(-1.0, 1.0, size=(k, 3))
    sig = rng.uniform(sigma[0], sigma[1], size=k)
    comp = rng.integers(0, k, size=n)
    return means[comp] + rng.normal(size=(n, 3)) * sig[comp, None]


def shell_cloud(n: int, rng: np.random.Generator, radius_range=(0.3, 0.9), jitter=0.01) -> np.ndarray:
    """Points jittered near a random sphere shell inside [-1,1]^3."""
    r = rng.uniform(*radius_range)
    c = rng.uniform(-(1.0 - r), 1.0 - r, size=3)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return c + d * r + rng.normal(size=(n, 3)) * jitter


def make_scene(points: np.ndarray, rng: np.random.Generator, sh_degree: int = 0) -> dict:
    """Delaunay mesh + parameters.  Returns a dict of flat contiguous arrays."""
    pts = np.asarray(points, dtype=np.float64)
    indices = delaunay_tets(pts)
    m = indices.size // 4
    nc = (sh_degree + 1) ** 2
    sh = rng.normal(0.0, 0.5, size=(m, 3, nc)).astype(np.float32)
    densities = np.exp(rng.normal(0.0, 1.0, size=m)).astype(np.float32)
    color_grads = rng.normal(0.0, 0.1, size=(m, 3)).astype(np.float32)
    vertices = np.ascontiguousarray(pts.astype(np.float32).ravel())
    base_colors = (0.5 + SH_C0 * sh[:, :, 0]).astype(np.float32)
    return {
        "vertices": vertices,
        "indices": indices,
        "base_colors": np.ascontiguousarray(base_colors.ravel()),
        "densities": densities,
        "color_grads": np.ascontiguousarray(color_grads.ravel()),
        "circumdata": circumspheres(vertices, indices),
        "sh_coeffs": np.ascontiguousarray(sh.ravel()),  # [M, 3, nc], coefficient c*nc + i
        "sh_degree": int(sh_degree),
    }


def grid_scene(grid_size: int, rng: np.random.Generator, jitter: float = 0.1) -> dict:
    """Regular-grid tet mesh (the structure of the reference's grid_tet_scene,
    crates/rmesh-util/src/test_util.rs:231-324): grid_size^3 vertices on the
    unit cube, each jittered by U(-0.5, 0.5) x jitter x the cell step, and every
    cube cell cut into the reference's five tets (A B D F, A D C G, A E F G,
    D F G H and the central A F D G, with A..H the corners 000, 100, 010, 110,
    001, 101, 011, 111; the renderer orients faces by the opposite vertex, so
    vertex order does not matter); densities U(0.5, 3.5), colour gradients
    U(-0.1, 0.1), base colours U(0.2, 0.8).  The random numbers come from
    ``rng`` (the reference draws them from a ChaCha8 stream), so the layout
    is the reference's and the values are seeded here.  jitter = 0 leaves
    the faces exactly axis-aligned and coplanar across cells."""
    n = int(grid_size)
    step = 1.0 / (n - 1)
    iz, iy, ix = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    base = np.stack([ix, iy, iz], axis=-1).reshape(-1, 3).astype(np.float64) * step
    pts = base + (rng.random(base.shape) - 0.5) * (jitter * step)
    vid = lambda x, y, z: x + y * n + z * n * n
    cells = []
    for z in range(n - 1):
        for y in range(n - 1):
            for x in range(n - 1):
                A, B, C, D = vid(x, y, z), vid(x + 1, y, z), vid(x, y + 1, z), vid(x + 1, y + 1, z)
                E, F, G, H = vid(x, y, z + 1), vid(x + 1, y, z + 1), vid(x, y + 1, z + 1), vid(x + 1, y + 1, z + 1)
                cells += [A, B, D, F, A, D, C, G, A, E, F, G, D, F, G, H, A, F, D, G]
    indices = np.asarray(cells, dtype=np.uint32)
    m = indices.size // 4
    vertices = np.ascontiguousarray(pts.astype(np.float32).ravel())
    return {
        "vertices": vertices,
        "indices": indices,
        "base_colors": rng.uniform(0.2, 0.8, 3 * m).astype(np.float32),
        "densities": (rng.random(m) * 3.0 + 0.5).astype(np.float32),
        "color_grads": ((rng.random(3 * m) - 0.5) * 0.2).astype(np.float32),
        "circumdata": circumspheres(vertices, indices),
        "sh_coeffs": np.zeros(3 * m, np.float32),
        "sh_degree": 0,
    }


# The five benchmark configurations (point counts, cloud recipe, views).
CONFIGS = {
    "c1": dict(points=2_000, cloud="uniform", sh_degree=0, views=1, res=((512, 512),), seed=0),
    "c2": dict(points=10_000, cloud="gmm", sh_degree=3, views=1, res=((512, 512),), seed=0),
    "c3": dict(points=100_000, cloud="gmm", sh_degree=3, views=16,
               res=((256, 256), (512, 512), (800, 600), (1024, 1024)), seed=0),
    "c4": dict(points=1_000_000, cloud="uniform+shell", sh_degree=3, views=8, res=((1920, 1080),), seed=0),
    "c5": dict(points=250_000, cloud="gmm", sh_degree=3, views=32, res=((800, 800),), seed=0),
}


def scene_for_config(name: str, points: int | None = None, seed: int | None = None) -> dict:
    """Build the mesh of a benchmark configuration (optionally with fewer points)."""
    cfg = CONFIGS[name]
    n = int(points if points is not None else cfg["points"])
    rng = np.random.default_rng(cfg["seed"] if seed is None else seed)
    if cfg["cloud"] == "uniform":
        pts = uniform_cloud(n, rng)
    elif cfg["cloud"] == "gmm":
        pts = gmm_cloud(n, rng)
    else:
        pts = np.concatenate([uniform_cloud(n, rng), shell_cloud(n // 10, rng)], axis=0)
    return make_scene(pts, rng, sh_degree=cfg["sh_degree"])

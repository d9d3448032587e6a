"""Seeded synthetic tetrahedral meshes, transfer functions and cameras.

The reference ships no datasets (its README points at ``../tet_offs/spx.off``
and friends, which are not part of the project), so every workload here is
generated from a seed with numpy's PCG64:

* ``freudenthal_mesh``: the unit cube split into N^3 cells, each cell cut into
  6 tetrahedra along its main diagonal (Freudenthal / Kuhn split, conforming
  across cells).  Interior vertices are jittered uniformly by +/-0.2 of a cell
  width; boundary vertices stay on the cube so the hull remains convex.
* ``gaussian_field``: a sum of isotropic Gaussians used as the per-vertex
  scalar (normalised to [0,1]) and, with another seed, as the carving field.
* ``carve``: removes tets whose centroid value of a second field exceeds a
  percentile, drops unreferenced vertices and re-indexes, so the mesh has
  cavities and rays re-enter it.  Unreferenced vertices must go: the
  reference's incidence builder gives up on them (vfRayPreComp.cc:260-262).
* ``transfer_function``: 256 RGBA entries, piecewise linear between 4 seeded
  control points, alpha 0 below scalar 0.1 (the reference fetches entry
  ``(uint)(255*s)``, vfRayKernelCPU.cc:279).
* ``random_rotation`` / ``orbit_views``: row-major 4x4 model-view matrices in
  the layout ``rotateVolume`` consumes (vfRayPreComp.cc:886-906).

The same functions build every workload: the plain single view of a 24^3
convex mesh, the 64-view orbit of a carved 64^3 mesh, the uneven job mix over
carved meshes of 16..128 cells per side, and the served request stream.
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "freudenthal_mesh", "gaussian_field", "carve", "transfer_function",
    "random_rotation", "orbit_views", "rotate_points", "make_mesh",
    "write_off", "write_tf", "permute_tet_vertices",
]

# The 6 Freudenthal tets of a unit cell: a monotone lattice path from corner
# (0,0,0) to (1,1,1), one per permutation of the axes.
_PERMS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))


def freudenthal_mesh(n: int, jitter: float = 0.2, seed: int = 0):
    """Return ``(xyz float64 (nV,3), tets uint32 (nT,4))`` for an n^3 grid."""
    m = n + 1
    g = np.arange(m, dtype=np.float64) / n
    zz, yy, xx = np.meshgrid(g, g, g, indexing="ij")
    xyz = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1)
    if jitter:
        rng = np.random.default_rng(seed)
        d = rng.uniform(-jitter / n, jitter / n, size=xyz.shape)
        ii = np.arange(m)
        inner = (ii > 0) & (ii < n)
        mask = (inner[:, None, None] & inner[None, :, None] & inner[None, None, :]).ravel()
        xyz[mask] += d[mask]
    # cell origins, x fastest
    cz, cy, cx = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    cx, cy, cz = cx.ravel(), cy.ravel(), cz.ravel()

    def vid(dx, dy, dz):
        return (cx + dx) + m * ((cy + dy) + m * (cz + dz))

    tets = np.empty((cx.size, 6, 4), dtype=np.uint32)
    for k, p in enumerate(_PERMS):
        off = [0, 0, 0]
        tets[:, k, 0] = vid(*off)
        for j in range(3):
            off[p[j]] = 1
            tets[:, k, j + 1] = vid(*off)
    return xyz, tets.reshape(-1, 4)


def gaussian_field(points: np.ndarray, count: int, seed: int) -> np.ndarray:
    """Sum of ``count`` isotropic Gaussians with centres U[0.1,0.9]^3,
    sigma U[0.05,0.2] and amplitude U[0.5,1], evaluated at ``points``."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.1, 0.9, size=(count, 3))
    sig = rng.uniform(0.05, 0.2, size=count)
    amp = rng.uniform(0.5, 1.0, size=count)
    out = np.zeros(points.shape[0], dtype=np.float64)
    for k in range(count):
        d2 = ((points - c[k]) ** 2).sum(axis=1)
        out += amp[k] * np.exp(-d2 / (2.0 * sig[k] ** 2))
    return out


def carve(xyz: np.ndarray, tets: np.ndarray, seed: int, count: int = 16,
          percentile: float = 85.0):
    """Drop tets whose centroid value of a seeded Gaussian field exceeds the
    given percentile; drop and re-index unreferenced vertices (vertex and tet
    order are otherwise preserved)."""
    # centroid field in chunks on a thread pool (numpy's array operations
    # release the interpreter lock; each chunk does the same operations on
    # its elements, so the values do not depend on the chunking or the
    # threads), with bounded temporaries for meshes of 10^8 tets
    from concurrent.futures import ThreadPoolExecutor
    import os

    val = np.empty(tets.shape[0], dtype=np.float64)
    step = 1 << 20

    def chunk(lo):
        cen = xyz[tets[lo:lo + step]].mean(axis=1)
        val[lo:lo + step] = gaussian_field(cen, count, seed)

    with ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1)) as ex:
        list(ex.map(chunk, range(0, tets.shape[0], step)))
    keep = val <= np.percentile(val, percentile)
    tets = tets[keep]
    used = np.zeros(xyz.shape[0], dtype=bool)
    used[tets.ravel()] = True
    remap = np.full(xyz.shape[0], -1, dtype=np.int64)
    remap[used] = np.arange(int(used.sum()))
    return xyz[used], remap[tets].astype(np.uint32), used


def transfer_function(seed: int = 2, cutoff: float = 0.1) -> np.ndarray:
    """256x4 float32 RGBA: piecewise linear between 4 seeded control points
    spanning [cutoff, 1]; alpha is 0 below ``cutoff``."""
    rng = np.random.default_rng(seed)
    knots = np.concatenate([[cutoff], np.sort(rng.uniform(cutoff, 1.0, size=2)), [1.0]])
    rgb = rng.uniform(0.0, 1.0, size=(4, 3))
    alpha = rng.uniform(0.1, 0.9, size=4)
    s = np.arange(256, dtype=np.float64) / 255.0
    tf = np.zeros((256, 4), dtype=np.float64)
    for ch in range(3):
        tf[:, ch] = np.interp(s, knots, rgb[:, ch])
    tf[:, 3] = np.interp(s, knots, alpha)
    tf[s < cutoff, 3] = 0.0
    return tf.astype(np.float32)


def random_rotation(seed: int) -> np.ndarray:
    """Uniform random rotation (QR of a Gaussian matrix) as a 3x3 float64."""
    rng = np.random.default_rng(seed)
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))[None, :]
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def _mv(rot3: np.ndarray) -> np.ndarray:
    mv = np.eye(4, dtype=np.float32)
    mv[:3, :3] = rot3.astype(np.float32)
    return mv


def orbit_views(count: int, seed: int) -> np.ndarray:
    """``count`` row-major 4x4 model-view matrices on a seeded orbit: a fixed
    random tilt followed by ``count`` equal steps about the vertical axis."""
    tilt = random_rotation(seed)
    out = np.empty((count, 4, 4), dtype=np.float32)
    for k in range(count):
        a = 2.0 * np.pi * k / count
        ry = np.array([[np.cos(a), 0.0, np.sin(a)], [0.0, 1.0, 0.0],
                       [-np.sin(a), 0.0, np.cos(a)]])
        out[k] = _mv(ry @ tilt)
    return out


def rotate_points(xyz: np.ndarray, rot3: np.ndarray, centre=(0.5, 0.5, 0.5)) -> np.ndarray:
    c = np.asarray(centre, dtype=np.float64)
    return (xyz - c) @ rot3.T + c


def make_mesh(n: int, carved: bool = False, view_seed: int | None = 3,
              jitter_seed: int = 0, scalar_seed: int = 1, carve_seed: int = 4,
              scalar_count: int = 8, carve_count: int = 16, percentile: float = 85.0):
    """Build a mesh as float32 ``vert4 (nV,4)`` [x y z s] and ``tets (nT,4)``.

    With ``view_seed`` set, a seeded rotation is baked into the coordinates
    (the reference CLI renders a mesh as stored, so a camera for the plain
    path is a rotation of the file's coordinates)."""
    xyz, tets = freudenthal_mesh(n, seed=jitter_seed)
    s = gaussian_field(xyz, scalar_count, scalar_seed)
    if carved:
        xyz, tets, used = carve(xyz, tets, carve_seed, carve_count, percentile)
        s = s[used]
    s = (s - s.min()) / (s.max() - s.min())
    if view_seed is not None:
        xyz = rotate_points(xyz, random_rotation(view_seed))
    vert4 = np.empty((xyz.shape[0], 4), dtype=np.float32)
    vert4[:, :3] = xyz
    vert4[:, 3] = s
    return vert4, np.ascontiguousarray(tets, dtype=np.uint32)


def permute_tet_vertices(tets: np.ndarray, seed: int) -> np.ndarray:
    """The same tets, each listing its 4 vertices in a seeded random order.
    Lattice-built tets list theirs in increasing id order, so a face shared
    by two tets appears in both in the same order; real meshes need not.
    Face order drives the exact arithmetic of the render, so tests use this
    to cover every vertex permutation between neighbouring tets."""
    rng = np.random.default_rng(seed)
    order = np.argsort(rng.random(tets.shape), axis=1)
    return np.ascontiguousarray(np.take_along_axis(tets, order, axis=1), dtype=np.uint32)


def write_off(path: str, vert4: np.ndarray, tets: np.ndarray) -> None:
    """Write the reference's .off layout (vfRayPreComp.cc:29-63): a header
    ``nV nT`` with no magic, nV lines ``x y z s``, nT lines of 4 ids.  Floats
    are written with 9 significant digits so they read back exactly."""
    with open(path, "w") as f:
        f.write(f"{vert4.shape[0]} {tets.shape[0]}\n")
        np.savetxt(f, vert4.astype(np.float32), fmt="%.9g")
        np.savetxt(f, tets, fmt="%d")


def write_tf(path: str, tf: np.ndarray) -> None:
    """Write the reference's .tf layout (vfRayPreComp.cc:628-649)."""
    with open(path, "w") as f:
        f.write("256\n")
        np.savetxt(f, tf.astype(np.float32), fmt="%.9g")

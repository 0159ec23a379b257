"""Seeded synthetic meshes for the benchmark workloads, and the reference's OBJ -> triangle
tuple conversion on the host.

* icosphere(R, subdiv): icosahedron subdivided `subdiv` times, projected to radius R
  (subdiv = 3 -> 642 vertices, 1280 faces).
* star_mesh(...): a closed UV sphere of n_lon x n_bands faces whose radius is perturbed by
  real spherical harmonics up to degree lmax (n_lon = 250, n_bands = 101 -> 25,002 vertices,
  50,000 faces).
* shape_def_from_mesh: ObjectShapeReader::get_triangle_params / convert_to_shape
  (src/file/objectshape_reader.cpp:248-300) vectorised, with the 7 -> 8 padding of
  NumericFormFactor::read_shapes_file (src/ff/ff_num.cpp:1016-1030).  Degenerate triangles
  are dropped as the reference drops them.
"""
from __future__ import annotations

import numpy as np

DEFAULT_SEED = 20240601


def icosphere(radius: float = 10.0, subdiv: int = 3, jitter: float = 0.0,
              seed: int = DEFAULT_SEED):
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t),
         (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
         (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
         (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    faces = list(f)
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    V = np.array(verts) * radius
    F = np.array(faces, dtype=np.int32)
    if jitter > 0:
        rng = np.random.default_rng(seed)
        V = V + rng.normal(scale=jitter, size=V.shape)
    return V, _orient_outward(V, F)


def _orient_outward(V, F):
    """Flips faces whose normal points toward the centroid (star-shaped meshes)."""
    a, b, c = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    n = np.cross(b - a, c - a)
    ctr = (a + b + c) / 3.0 - V.mean(axis=0)
    flip = np.einsum("ij,ij->i", n, ctr) < 0
    F = F.copy()
    F[flip] = F[flip][:, [0, 2, 1]]
    return F


def _real_sph_harm(l, m, theta, phi):
    """Real orthonormal spherical harmonic Y_lm(theta = polar, phi = azimuth)."""
    from scipy.special import lpmv, factorial

    am = abs(m)
    norm = np.sqrt((2 * l + 1) / (4 * np.pi) * factorial(l - am) / factorial(l + am))
    # lpmv includes the Condon-Shortley phase; undo it so the basis is the usual real one
    P = lpmv(am, l, np.cos(theta)) * ((-1) ** am)
    if m > 0:
        return np.sqrt(2) * norm * P * np.cos(am * phi)
    if m < 0:
        return np.sqrt(2) * norm * P * np.sin(am * phi)
    return norm * P


def star_mesh(mean_radius: float = 15.0, n_lon: int = 250, n_bands: int = 101, lmax: int = 8,
              amp: float = 0.05, seed: int = DEFAULT_SEED):
    """Closed UV-sphere mesh with radius 15*(1 + sum_{l<=lmax,m} a_lm Y_lm), a_lm ~ N(0,(amp/l)^2).

    Vertices: 2 poles + n_lon*(n_bands-1) ring vertices; faces: 2*n_lon*(n_bands-1)."""
    rng = np.random.default_rng(seed)
    coef = {(l, m): rng.normal(scale=amp / l) for l in range(1, lmax + 1)
            for m in range(-l, l + 1)}
    rings = n_bands - 1
    th = np.pi * (np.arange(1, rings + 1) / n_bands)       # polar angles of the rings
    ph = 2 * np.pi * (np.arange(n_lon) / n_lon)
    TH, PH = np.meshgrid(th, ph, indexing="ij")
    theta = np.concatenate([[0.0], TH.ravel(), [np.pi]])
    phi = np.concatenate([[0.0], PH.ravel(), [0.0]])
    pert = np.zeros_like(theta)
    for (l, m), a in coef.items():
        pert += a * _real_sph_harm(l, m, theta, phi)
    r = mean_radius * np.maximum(1.0 + pert, 0.1)
    V = np.stack([r * np.sin(theta) * np.cos(phi), r * np.sin(theta) * np.sin(phi),
                  r * np.cos(theta)], axis=1)
    top, bot = 0, len(V) - 1

    def vid(i, j):  # ring i (0..rings-1), longitude j
        return 1 + i * n_lon + (j % n_lon)

    F = []
    for j in range(n_lon):
        F.append((top, vid(0, j), vid(0, j + 1)))
    for i in range(rings - 1):
        for j in range(n_lon):
            a, b, c, d = vid(i, j), vid(i, j + 1), vid(i + 1, j), vid(i + 1, j + 1)
            F.append((a, c, b))
            F.append((b, c, d))
    for j in range(n_lon):
        F.append((bot, vid(rings - 1, j + 1), vid(rings - 1, j)))
    F = np.array(F, dtype=np.int32)
    return V, _orient_outward(V, F)


def shape_def_from_mesh(V, F, keep_degenerate: bool = False):
    """(T, 8) float64 rows (s, nx, ny, nz, cx, cy, cz, 0) per the reference's
    get_triangle_params; degenerate triangles are dropped unless keep_degenerate."""
    V = np.asarray(V, dtype=np.float64)
    F = np.asarray(F, dtype=np.int64)
    v1, v2, v3 = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    c = (v1 + v2 + v3) / 3.0
    a = v2 - v1
    b = v3 - v1
    na = np.sqrt((a * a).sum(1))
    nb = np.sqrt((b * b).sum(1))
    dot = (a * b).sum(1)
    cr = np.cross(a, b)
    nc = np.sqrt((cr * cr).sum(1))
    ok = (nc != 0) & (na != 0) & (nb != 0)
    with np.errstate(invalid="ignore", divide="ignore"):
        n = cr / nc[:, None]
        cosv = dot / (na * nb)
        s = na * nb * np.sqrt(1 - cosv * cosv) / 2
    out = np.zeros((len(F), 8))
    out[:, 0] = s
    out[:, 1:4] = n
    out[:, 4:7] = c
    if not keep_degenerate:
        out = out[ok]
    return np.ascontiguousarray(out)


def write_obj(path, verts, faces):
    """Writes a mesh as Wavefront OBJ (1-based faces)."""
    v = np.asarray(verts, dtype=np.float64).reshape(-1, 3)
    f = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
    with open(path, "w") as fh:
        for x in v:
            fh.write(f"v {x[0]:.17g} {x[1]:.17g} {x[2]:.17g}\n")
        for t in f:
            fh.write(f"f {t[0] + 1} {t[1] + 1} {t[2] + 1}\n")


def load_obj(path):
    """hgx_obj_load: (vertices[nv, 3], faces[nf, 3] 0-based, info) of an OBJ file; info has
    the counts of 4-vertex faces left out (nquads) and larger faces skipped (nskipped)."""
    import ctypes as C

    from ._capi import check, lib
    h = C.c_void_p()
    check(lib().hgx_obj_load(str(path).encode(), C.byref(h)))
    try:
        nv, nf, nq, ns = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(lib().hgx_mesh_info(h, C.byref(nv), C.byref(nf), C.byref(nq), C.byref(ns)))
        v = np.zeros((nv.value, 3))
        f = np.zeros((nf.value, 3), dtype=np.int32)
        check(lib().hgx_mesh_read(h, v.ctypes.data, f.ctypes.data))
    finally:
        lib().hgx_mesh_destroy(h)
    return v, f, {"nquads": nq.value, "nskipped": ns.value}


def read_shapes_file(ctx, path):
    """hgx_read_shapes_file: the (T, 8) shape_def of an .obj or raw .dat shape file (ctx may be
    None for .dat files)."""
    import ctypes as C

    from ._capi import check, lib
    h = None if ctx is None else ctx.handle
    n = C.c_int()
    check(lib().hgx_read_shapes_file(h, str(path).encode(), None, 0, C.byref(n)))
    out = np.zeros((n.value, 8))
    check(lib().hgx_read_shapes_file(h, str(path).encode(), out.ctypes.data, n.value, C.byref(n)))
    return out

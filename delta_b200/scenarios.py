"""Synthetic inputs (seeded) for the contact pipeline.

No dataset is involved: the reference's benchmarks are re-created with the shapes,
sizes and value distributions of each workload.

``narrowphase_pairs`` builds the independent triangle-pair workload: triangle A has
vertices U[0,1]^3; triangle B is a rotated triangle with edge lengths U(0.05,1), placed
so that the true separation is lognormal(ln 1e-3, 2).  10% of pairs are near-parallel
(planes within 1e-3 rad) and 5% intersect.  The separation is exact by construction:
a unit direction n is chosen in the normal cone of a feature of A (vertex, edge or
face) and B is oriented so that a feature of it (vertex, edge or face) is extreme in -n;
the two features are placed at distance d along n, so the plane orthogonal to n
separates A from B and d = dist(A, B).
"""
from __future__ import annotations

import numpy as np

GENERAL, NEAR_PARALLEL, INTERSECTING = 0, 1, 2
CLASS_NAMES = ("general", "near_parallel", "intersecting")


def _unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def _random_unit(rng, n):
    return _unit(rng.normal(size=(n, 3)))


def _perp_unit(rng, n_vec):
    """A random unit vector orthogonal to each row of n_vec."""
    r = rng.normal(size=n_vec.shape)
    r -= np.sum(r * n_vec, axis=1, keepdims=True) * n_vec
    return _unit(r)


def _random_rotations(rng, n):
    q = _unit(rng.normal(size=(n, 4)))
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], 1)


def _random_barycentric(rng, n):
    u = rng.random((n, 2))
    flip = u.sum(1) > 1
    u[flip] = 1 - u[flip]
    return np.stack([1 - u[:, 0] - u[:, 1], u[:, 0], u[:, 1]], 1)


def _triangle_2d(rng, n):
    """Planar triangles (n,3,2) with edge lengths U(0.05,1): edge v0->v1 on +x, v2 above."""
    out = np.empty((n, 3, 2))
    todo = np.arange(n)
    while todo.size:
        l = rng.uniform(0.05, 1.0, size=(todo.size, 3))  # |v0v1|, |v1v2|, |v2v0|
        ok = (l[:, 0] + l[:, 1] > l[:, 2]) & (l[:, 1] + l[:, 2] > l[:, 0]) & (l[:, 2] + l[:, 0] > l[:, 1])
        l, idx = l[ok], todo[ok]
        px = (l[:, 0] ** 2 + l[:, 2] ** 2 - l[:, 1] ** 2) / (2 * l[:, 0])
        py = np.sqrt(np.maximum(l[:, 2] ** 2 - px ** 2, 0.0))
        out[idx, 0] = 0.0
        out[idx, 1, 0], out[idx, 1, 1] = l[:, 0], 0.0
        out[idx, 2, 0], out[idx, 2, 1] = px, py
        todo = todo[~ok]
    return out


def narrowphase_pairs(n: int, seed: int = 0, near_parallel: float = 0.10, intersecting: float = 0.05):
    """Returns a (9,n), b (9,n) float64 planes (3*vertex+coord), true separation (n,)
    and class (n,) uint8 (GENERAL, NEAR_PARALLEL, INTERSECTING)."""
    rng = np.random.default_rng(seed)
    A = rng.random((n, 3, 3))
    NA = _unit(np.cross(A[:, 1] - A[:, 0], A[:, 2] - A[:, 0]))
    u = rng.random(n)
    cls = np.full(n, GENERAL, np.uint8)
    cls[u < near_parallel + intersecting] = NEAR_PARALLEL
    cls[u < intersecting] = INTERSECTING
    d = np.exp(rng.normal(np.log(1e-3), 2.0, size=n))
    d[cls == INTERSECTING] = 0.0

    # ---- feature of A and direction n -------------------------------------------------
    a_type = rng.integers(0, 3, n)  # 0 vertex, 1 edge, 2 face
    b_type = rng.integers(0, 3, n)
    b_type[(a_type == 2) & (b_type == 2)] = 1
    a_type[cls == NEAR_PARALLEL] = 2
    b_type[cls == NEAR_PARALLEL] = 2
    sign = np.where(rng.random(n) < 0.5, -1.0, 1.0)[:, None]
    nvec = np.empty((n, 3))
    p = np.empty((n, 3))
    # vertex: random direction, extreme vertex of A
    m = a_type == 0
    nv = _random_unit(rng, m.sum())
    iv = np.argmax(np.einsum("nvk,nk->nv", A[m], nv), axis=1)
    nvec[m] = nv
    p[m] = A[m][np.arange(m.sum()), iv]
    # edge: n in the half circle orthogonal to the edge, outward in the plane
    m = a_type == 1
    e = rng.integers(0, 3, m.sum())
    Am = A[m]
    i0 = Am[np.arange(m.sum()), e]
    i1 = Am[np.arange(m.sum()), (e + 1) % 3]
    i2 = Am[np.arange(m.sum()), (e + 2) % 3]
    te = _unit(i1 - i0)
    mo = np.cross(te, NA[m])
    mo *= np.where(np.sum(mo * (i2 - i0), 1) > 0, -1.0, 1.0)[:, None]
    phi = rng.uniform(-0.45 * np.pi, 0.45 * np.pi, m.sum())[:, None]
    nvec[m] = _unit(np.cos(phi) * mo + np.sin(phi) * NA[m])
    p[m] = i0 + rng.random((m.sum(), 1)) * (i1 - i0)
    # face: n = +-normal of A, any point of A
    m = a_type == 2
    nvec[m] = sign[m] * NA[m]
    p[m] = np.einsum("nv,nvk->nk", _random_barycentric(rng, m.sum()), A[m])

    # ---- B oriented with a feature extreme in -n -----------------------------------------
    T2 = _triangle_2d(rng, n)
    B = np.empty((n, 3, 3))
    q = np.empty((n, 3))
    t = _perp_unit(rng, nvec)
    t2 = np.cross(nvec, t)
    # vertex: random rotation, vertex minimal along n
    m = (b_type == 0) & (cls != INTERSECTING)
    R = _random_rotations(rng, m.sum())
    Bm = np.einsum("nij,nvj->nvi", R, np.concatenate([T2[m], np.zeros((m.sum(), 3, 1))], 2))
    iv = np.argmin(np.einsum("nvk,nk->nv", Bm, nvec[m]), axis=1)
    B[m] = Bm
    q[m] = Bm[np.arange(m.sum()), iv]
    # edge: edge v0v1 along t, the triangle leaning into +n at angle psi
    m = (b_type == 1) & (cls != INTERSECTING)
    psi = rng.uniform(-0.45 * np.pi, 0.45 * np.pi, m.sum())[:, None]
    inward = np.cos(psi) * nvec[m] + np.sin(psi) * t2[m]
    B[m] = T2[m][:, :, :1] * t[m][:, None, :] + T2[m][:, :, 1:] * inward[:, None, :]
    q[m] = B[m][:, 0] + rng.random((m.sum(), 1)) * (B[m][:, 1] - B[m][:, 0])
    # face: the triangle in a plane orthogonal to n, any point of it
    m = (b_type == 2) & (cls == GENERAL)
    B[m] = T2[m][:, :, :1] * t[m][:, None, :] + T2[m][:, :, 1:] * t2[m][:, None, :]
    q[m] = np.einsum("nv,nvk->nk", _random_barycentric(rng, m.sum()), B[m])
    # near-parallel: face orthogonal to n tilted by alpha < 1e-3 rad about t, lowest vertex
    m = cls == NEAR_PARALLEL
    alpha = rng.uniform(0.0, 1e-3, m.sum())[:, None]
    tt2 = np.cos(alpha) * t2[m] + np.sin(alpha) * nvec[m]
    Bm = T2[m][:, :, :1] * t[m][:, None, :] + T2[m][:, :, 1:] * tt2[:, None, :]
    iv = np.argmin(np.einsum("nvk,nk->nv", Bm, nvec[m]), axis=1)
    B[m] = Bm
    q[m] = Bm[np.arange(m.sum()), iv]
    # intersecting: random rotation, an interior point of B put on an interior point of A
    m = cls == INTERSECTING
    R = _random_rotations(rng, m.sum())
    Bm = np.einsum("nij,nvj->nvi", R, np.concatenate([T2[m], np.zeros((m.sum(), 3, 1))], 2))
    B[m] = Bm
    q[m] = np.einsum("nv,nvk->nk", _random_barycentric(rng, m.sum()), Bm)

    B += (p + d[:, None] * nvec - q)[:, None, :]
    a = np.ascontiguousarray(A.reshape(n, 9).T)
    b = np.ascontiguousarray(B.reshape(n, 9).T)
    return a, b, d, cls


# ---------------------------------------------------------------------------------------
# particle meshes
# ---------------------------------------------------------------------------------------
def icosphere(subdiv: int):
    """Unit icosphere: 20 * 4**subdiv triangles, outward winding.  Returns (V, F)."""
    g = (1.0 + 5 ** 0.5) / 2
    V = [(-1, g, 0), (1, g, 0), (-1, -g, 0), (1, -g, 0), (0, -1, g), (0, 1, g), (0, -1, -g), (0, 1, -g),
         (g, 0, -1), (g, 0, 1), (-g, 0, -1), (-g, 0, 1)]
    V = [tuple(np.array(v) / np.linalg.norm(v)) for v in V]
    F = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache = {}
        Vl = list(V)

        def mid(i, j):
            key = (min(i, j), max(i, j))
            if key not in cache:
                m = (np.array(Vl[i]) + np.array(Vl[j])) / 2
                Vl.append(tuple(m / np.linalg.norm(m)))
                cache[key] = len(Vl) - 1
            return cache[key]

        NF = []
        for a, b, c in F:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            NF += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        V, F = Vl, NF
    return np.array(V, float), np.array(F, np.int64)


def _hull_sphere(n_tri: int):
    """Convex hull of (n_tri+4)/2 Fibonacci points on the unit sphere: n_tri triangles."""
    from scipy.spatial import ConvexHull

    npts = (n_tri + 4) // 2
    i = np.arange(npts) + 0.5
    phi = np.arccos(1 - 2 * i / npts)
    th = np.pi * (1 + 5 ** 0.5) * i
    V = np.stack([np.cos(th) * np.sin(phi), np.sin(th) * np.sin(phi), np.cos(phi)], 1)
    F = ConvexHull(V).simplices.astype(np.int64)
    if F.shape[0] != n_tri:
        raise ValueError(f"hull gave {F.shape[0]} triangles, wanted {n_tri}")
    return V, _outward(V, F)


def _outward(V, F):
    n = np.cross(V[F[:, 1]] - V[F[:, 0]], V[F[:, 2]] - V[F[:, 0]])
    c = V[F].mean(1) - V.mean(0)
    flip = np.sum(n * c, 1) < 0
    F = F.copy()
    F[flip] = F[flip][:, [0, 2, 1]]
    return F


def sphere_mesh(n_tri: int, rng=None, radius: float = 1.0, perturb=None):
    """A closed sphere-like triangle mesh with exactly n_tri triangles (an icosphere when
    n_tri is 20*4**k, otherwise the convex hull of Fibonacci points, the hull-of-points
    particle type of the reference's granulate generator).  `perturb=(lo, hi)` scales
    each vertex radius by U(lo, hi).  Returns (V, F) with outward winding."""
    k = {20: 0, 80: 1, 320: 2, 1280: 3}.get(n_tri)
    V, F = icosphere(k) if k is not None else _hull_sphere(n_tri)
    if perturb is not None:
        rng = rng if rng is not None else np.random.default_rng()
        V = V * rng.uniform(perturb[0], perturb[1], size=(V.shape[0], 1))
    return V * radius, F


def _pairs_chunk(args):
    n, seed = args
    a, b, d, cls = narrowphase_pairs(n, seed)
    return a, b, d, cls


def narrowphase_pairs_chunked(n: int, seed: int = 0, chunk: int = 1 << 20, workers: int = 0):
    """narrowphase_pairs over chunks of `chunk` pairs (chunk k seeded with (seed, k)),
    generated in a spawn-started process pool.  Same distribution, deterministic in
    (n, seed, chunk)."""
    import os
    from concurrent.futures import ProcessPoolExecutor
    import multiprocessing as mp

    sizes = [min(chunk, n - s) for s in range(0, n, chunk)]
    seeds = [int(np.random.SeedSequence([seed, k]).generate_state(1)[0]) for k in range(len(sizes))]
    workers = workers or min(len(sizes), os.cpu_count() or 1, 32)
    if workers <= 1 or len(sizes) == 1:
        parts = [_pairs_chunk(x) for x in zip(sizes, seeds)]
    else:
        with ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
            parts = list(ex.map(_pairs_chunk, zip(sizes, seeds)))
    a = np.concatenate([p[0] for p in parts], 1)
    b = np.concatenate([p[1] for p in parts], 1)
    d = np.concatenate([p[2] for p in parts])
    cls = np.concatenate([p[3] for p in parts])
    return a, b, d, cls


# ---------------------------------------------------------------------------------------
# rigid-body scenes
# ---------------------------------------------------------------------------------------
def mass_properties(V, F, density):
    """Mass, centre of mass and inertia tensor (about the centre) of the solid bounded by
    the closed, outward-wound mesh (V, F): sum of the signed tetrahedra (origin, a, b, c),
    each with covariance det * A C0 A^T, C0 = [[2,1,1],[1,2,1],[1,1,2]]/120."""
    o = V.mean(0)
    T = V[F] - o  # (nT, 3 vertices, 3)
    det = np.einsum("ij,ij->i", T[:, 0], np.cross(T[:, 1], T[:, 2]))
    vol = det.sum() / 6.0
    mass = density * vol
    com = o + (det[:, None] * T.sum(1)).sum(0) / (24.0 * vol)
    C0 = (np.ones((3, 3)) + np.eye(3)) / 120.0
    Acol = np.transpose(T, (0, 2, 1))  # columns are the vertices
    cov = density * np.einsum("n,nij,jk,nlk->il", det, Acol, C0, Acol)
    d = (com - o)[:, None]
    cov_c = cov - mass * (d @ d.T)
    inertia = np.trace(cov_c) * np.eye(3) - cov_c
    return mass, com, inertia


def lattice_scene(seed: int = 0, nx: int = 8, ny: int = 4, nz: int = 8, spacing: float = 0.025,
                  jitter: float = 0.002, radius: float = 0.01, perturb=(0.8, 1.2), n_tri: int = 80,
                  density: float = 2500.0, eps: float = 1e-4, floor_half: float = 0.5, friction: bool = False):
    """The small plain-method workload: perturbed sphere meshes on an nx*ny*nz lattice
    (y vertical) above a floor of two triangles at y = 0 spanning (2*floor_half)^2."""
    rng = np.random.default_rng(seed)
    bodies = []
    base = np.array([-(nx - 1) / 2 * spacing, 1.5 * radius * perturb[1], -(nz - 1) / 2 * spacing])
    for ix in range(nx):
        for iy in range(ny):
            for iz in range(nz):
                V, F = sphere_mesh(n_tri, rng, radius, perturb)
                c = base + np.array([ix, iy, iz]) * spacing + rng.uniform(-jitter, jitter, 3)
                bodies.append((V + c, F))
    h = floor_half
    floor_V = np.array([[-h, 0, -h], [h, 0, -h], [h, 0, h], [-h, 0, h]], float)
    floor_F = np.array([[0, 2, 1], [0, 3, 2]])
    return build_scene(bodies, obstacles=[(floor_V, floor_F)], density=density, eps=eps, friction=friction)


def build_scene(bodies, obstacles=(), density=2500.0, eps=1e-4, friction=False):
    """Scene dict (AoS per body: pos[3n], rot[9n], ...; SoA-tri vertices) from lists of
    (V, F) meshes in world coordinates.  Moving bodies first, then obstacles."""
    all_meshes = [(V, F, False) for V, F in bodies] + [(V, F, True) for V, F in obstacles]
    n = len(all_meshes)
    counts = [F.shape[0] for _, F, _ in all_meshes]
    tri_offset = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    xyz = np.concatenate([V[F].reshape(-1, 3) for V, F, _ in all_meshes])
    pos = np.zeros((n, 3)); inertia = np.zeros((n, 3, 3)); inverse = np.zeros((n, 3, 3))
    mass = np.zeros(n); radius = np.zeros(n); obst = np.zeros(n, np.uint8)
    for i, (V, F, is_obst) in enumerate(all_meshes):
        if is_obst:
            c = V.mean(0)
            pos[i] = c
            mass[i] = np.inf
            obst[i] = 1
        else:
            m, c, J = mass_properties(V, F, density)
            pos[i], mass[i], inertia[i] = c, m, J
            inverse[i] = np.linalg.inv(J)
        radius[i] = np.linalg.norm(V - pos[i], axis=1).max()
    tri_body = np.repeat(np.arange(n, dtype=np.int32), counts)
    rot = np.tile(np.eye(3).reshape(9), n)
    # 3x3 matrices are stored column-major (dynamics.cpp); J and its inverse are symmetric
    return {
        "n_bodies": n, "tri_offset": tri_offset, "tri_body": tri_body,
        "x": xyz[:, 0].copy(), "y": xyz[:, 1].copy(), "z": xyz[:, 2].copy(),
        "rx": xyz[:, 0].copy(), "ry": xyz[:, 1].copy(), "rz": xyz[:, 2].copy(),
        "pos": pos.reshape(-1).copy(), "ref_pos": pos.reshape(-1).copy(),
        "vel": np.zeros(3 * n), "ang": np.zeros(3 * n), "ref_ang": np.zeros(3 * n), "rot": rot,
        "inertia": inertia.transpose(0, 2, 1).reshape(-1).copy(), "inverse": inverse.transpose(0, 2, 1).reshape(-1).copy(),
        "mass": mass, "eps": np.full(n, eps), "radius": radius,
        "friction": np.full(n, 1 if friction else 0, np.uint8), "obstacle": obst,
    }


def _batched_mass_properties(V, F, density):
    """mass_properties for a batch of meshes sharing connectivity F: V (B, nV, 3)."""
    o = V.mean(1, keepdims=True)
    T = V[:, F] - o[:, None]  # (B, nT, 3, 3)
    det = np.einsum("btj,btj->bt", T[:, :, 0], np.cross(T[:, :, 1], T[:, :, 2]))
    vol = det.sum(1) / 6.0
    mass = density * vol
    com = o[:, 0] + np.einsum("bt,btj->bj", det, T.sum(2)) / (24.0 * vol[:, None])
    # sum over tetrahedra of det * A C0 A^T with C0 = (I + 1 1^T)/120, i.e.
    # det/120 * (sum_v v v^T + s s^T), s = sum of the three vertices
    ssum = T.sum(2)
    cov = density / 120.0 * (np.einsum("bt,btvi,btvj->bij", det, T, T, optimize=True) +
                             np.einsum("bt,bti,btj->bij", det, ssum, ssum, optimize=True))
    d = com - o[:, 0]
    cov_c = cov - mass[:, None, None] * np.einsum("bi,bj->bij", d, d)
    tr = np.trace(cov_c, axis1=1, axis2=2)
    inertia = tr[:, None, None] * np.eye(3) - cov_c
    return mass, com, inertia


def particle_cloud_scene(centres, radii, n_tri, obstacles, seed=0, perturb=(0.8, 1.2), density=2500.0,
                         eps=1e-4, friction=False):
    """Scene dict for many particles (perturbed sphere meshes of n_tri[i] triangles, radius
    radii[i], centred at centres[i]) plus static obstacle meshes, built per mesh size."""
    rng = np.random.default_rng(seed)
    n = len(centres)
    n_tri = np.asarray(n_tri)
    counts = np.concatenate([n_tri, [F.shape[0] for _, F in obstacles]]).astype(np.int64)
    nb = n + len(obstacles)
    tri_offset = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    xyz = np.empty((tri_offset[-1] * 3, 3))
    mass = np.zeros(n); com = np.zeros((n, 3)); inertia = np.zeros((n, 3, 3)); rad = np.zeros(n)
    for nt in np.unique(n_tri):
        idx = np.flatnonzero(n_tri == nt)
        V0, F = sphere_mesh(int(nt), None, 1.0)
        for lo in range(0, idx.size, 20000):  # bounded temporaries
            sub = idx[lo:lo + 20000]
            scale = rng.uniform(perturb[0], perturb[1], size=(sub.size, V0.shape[0], 1)) * radii[sub][:, None, None]
            V = V0[None] * scale + centres[sub][:, None, :]
            m, c, J = _batched_mass_properties(V, F, density)
            mass[sub], com[sub], inertia[sub] = m, c, J
            rad[sub] = np.linalg.norm(V - c[:, None], axis=2).max(1)
            vidx = (3 * tri_offset[sub])[:, None] + np.arange(3 * int(nt))[None]
            xyz[vidx.reshape(-1)] = V[:, F].reshape(-1, 3)
    pos = np.zeros((nb, 3)); pos[:n] = com
    inv = np.zeros((nb, 3, 3)); inv[:n] = np.linalg.inv(inertia)
    J = np.zeros((nb, 3, 3)); J[:n] = inertia
    m = np.full(nb, np.inf); m[:n] = mass
    r = np.zeros(nb); r[:n] = rad
    obst = np.zeros(nb, np.uint8); obst[n:] = 1
    for k, (V, F) in enumerate(obstacles):
        i = n + k
        xyz[3 * tri_offset[i]:3 * tri_offset[i + 1]] = V[F].reshape(-1, 3)
        pos[i] = V.mean(0)
        r[i] = np.linalg.norm(V - pos[i], axis=1).max()
    return {
        "n_bodies": nb, "tri_offset": tri_offset, "tri_body": np.repeat(np.arange(nb, dtype=np.int32), counts),
        "x": xyz[:, 0].copy(), "y": xyz[:, 1].copy(), "z": xyz[:, 2].copy(),
        "rx": xyz[:, 0].copy(), "ry": xyz[:, 1].copy(), "rz": xyz[:, 2].copy(),
        "pos": pos.reshape(-1).copy(), "ref_pos": pos.reshape(-1).copy(),
        "vel": np.zeros(3 * nb), "ang": np.zeros(3 * nb), "ref_ang": np.zeros(3 * nb),
        "rot": np.tile(np.eye(3).reshape(9), nb),
        "inertia": J.transpose(0, 2, 1).reshape(-1).copy(), "inverse": inv.transpose(0, 2, 1).reshape(-1).copy(),
        "mass": m, "eps": np.full(nb, eps), "radius": r,
        "friction": np.full(nb, 1 if friction else 0, np.uint8), "obstacle": obst,
    }


def _jittered_lattice(n, spacing, origin, jitter, rng, shape_xz):
    nx, nz = shape_xz
    ny = -(-n // (nx * nz))
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1).reshape(-1, 3)
    g = g[np.lexsort((g[:, 2], g[:, 0], g[:, 1]))][:n]  # fill layer by layer from the bottom
    return origin + g * spacing + rng.uniform(-jitter, jitter, (n, 3))


def hopper_obstacles(n_around=64, n_along=16, half_angle_deg=30.0, outlet=0.08, height=0.8, patch=(4, 2)):
    """Conical hopper wall (axis y, outlet at y = 0) with 2*n_around*n_along triangles,
    split into patches of patch[0] x patch[1] quads (one obstacle body each)."""
    r0 = outlet / 2
    r1 = r0 + height * np.tan(np.radians(half_angle_deg))
    th = np.linspace(0, 2 * np.pi, n_around + 1)
    ys = np.linspace(0, height, n_along + 1)
    out = []
    for a0 in range(0, n_around, patch[0]):
        for h0 in range(0, n_along, patch[1]):
            V, F = [], []
            for a in range(a0, min(a0 + patch[0], n_around)):
                for h in range(h0, min(h0 + patch[1], n_along)):
                    q = []
                    for (ai, hi) in ((a, h), (a + 1, h), (a + 1, h + 1), (a, h + 1)):
                        rr = r0 + (r1 - r0) * ys[hi] / height
                        q.append((rr * np.cos(th[ai]), ys[hi], rr * np.sin(th[ai])))
                    b = len(V)
                    V += q
                    F += [(b, b + 1, b + 2), (b, b + 2, b + 3)]
            out.append((np.array(V), np.array(F)))
    return out


def hopper_scene(n_particles=10000, seed=0, sizes=(40, 80, 160, 320), radius=(0.005, 0.015), eps=1e-4):
    """The batched uneven hopper workload: particles of mixed mesh sizes above a conical hopper."""
    rng = np.random.default_rng(seed)
    radii = rng.uniform(radius[0], radius[1], n_particles)
    n_tri = rng.choice(np.asarray(sizes), n_particles)
    sp = 2.0 * radius[1] * 1.2 * 1.05
    side = int(np.ceil(np.sqrt(n_particles / 30)))
    cen = _jittered_lattice(n_particles, sp, np.array([-(side - 1) * sp / 2, 0.3, -(side - 1) * sp / 2]),
                            0.1 * sp, rng, (side, side))
    return particle_cloud_scene(cen, radii, n_tri, hopper_obstacles(), seed=seed + 1, eps=eps)


def box_scene(n_particles=200000, seed=0, sizes=(80, 160, 320, 500), radius=(0.004, 0.012), eps=1e-4,
              box=(0.6, 1.2, 0.6)):
    """The large box workload: particles poured from a jittered lattice into a box of 12
    wall triangles (6 faces, x and z sides 0.6 m, height 1.2 m; y vertical)."""
    rng = np.random.default_rng(seed)
    radii = rng.uniform(radius[0], radius[1], n_particles)
    n_tri = rng.choice(np.asarray(sizes), n_particles)
    sp = 2.0 * radius[1] * 1.2 * 1.02
    nx = int(box[0] / sp) - 1
    cen = _jittered_lattice(n_particles, sp, np.array([-(nx - 1) * sp / 2, sp, -(nx - 1) * sp / 2]), 0.05 * sp, rng,
                            (nx, nx))
    hx, hy, hz = box[0] / 2, box[1], box[2] / 2
    C = np.array([[-hx, 0, -hz], [hx, 0, -hz], [hx, 0, hz], [-hx, 0, hz],
                  [-hx, hy, -hz], [hx, hy, -hz], [hx, hy, hz], [-hx, hy, hz]], float)
    quads = [(0, 1, 2, 3), (4, 7, 6, 5), (0, 4, 5, 1), (1, 5, 6, 2), (2, 6, 7, 3), (3, 7, 4, 0)]
    walls = [(C[list(q)], np.array([[0, 1, 2], [0, 2, 3]])) for q in quads]
    return particle_cloud_scene(cen, radii, n_tri, walls, seed=seed + 1, eps=eps)

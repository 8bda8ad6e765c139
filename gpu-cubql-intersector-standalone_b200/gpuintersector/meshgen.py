"""Seeded synthetic workloads (numpy), standing in for the reference's trimesh
data (pythonDataGeneration/PythonDataGenerationScript.py:5-54, which needs
trimesh) at the shapes and sizes of the five configurations:

  1. two UV spheres 128 x 80 (20,224 triangles), B translated (0.5, 0, 0) and
     rotated by a seeded uniform rotation;
  2. two level-8 displaced icospheres (1,310,720 triangles each),
     r = 1 + 0.05 * sum_{k=1..8} sin(f_k <dir, a_k> + phi_k) / k with seeded unit
     axes a_k, phases phi_k ~ U[0, 2 pi) and f_k = 2 pi k (1 + 0.25 U[-1, 1]);
     B = A offset (0.3, 0.1, 0) plus a seeded rotation;
  3. two 512 x 512-quad integer grids (524,288 triangles) with cell 2048 on a 2^20
     grid; B coplanar, shifted half a cell in x, each vertex lifted by the
     z in {-1, 0, +1} of its 8 x 8-quad tile;
  4. batched pairs of displaced geodesic icospheres with T = 20 n^2 triangles,
     n chosen so T is log-uniform in [t_min, t_max];
  5. serving: resident displaced geodesic spheres and a Poisson pose stream.

Poses are returned as (R, center, trans) triples for gpuintersector.pose_raw.
"""
import numpy as np


def uv_sphere(segments=128, rings=80, radius=1.0):
    """UV sphere: 2 poles + (rings-1) rings of `segments` vertices; 2*segments*(rings-1) triangles."""
    phi = np.pi * np.arange(1, rings) / rings
    th = 2.0 * np.pi * np.arange(segments) / segments
    sp, cp = np.sin(phi)[:, None], np.cos(phi)[:, None]
    ring = np.stack([radius * sp * np.cos(th)[None, :], radius * sp * np.sin(th)[None, :],
                     radius * np.broadcast_to(cp, (rings - 1, segments))], axis=-1).reshape(-1, 3)
    verts = np.concatenate([[[0.0, 0.0, radius]], ring, [[0.0, 0.0, -radius]]]).astype(np.float64)
    north, south = 0, verts.shape[0] - 1
    idx = lambda i, j: 1 + i * segments + (j % segments)
    tris = []
    j = np.arange(segments)
    tris.append(np.stack([np.full(segments, north), idx(0, j), idx(0, j + 1)], axis=1))
    for i in range(rings - 2):
        a, b, c, d = idx(i, j), idx(i, j + 1), idx(i + 1, j), idx(i + 1, j + 1)
        tris.append(np.stack([a, c, b], axis=1))
        tris.append(np.stack([b, c, d], axis=1))
    tris.append(np.stack([np.full(segments, south), idx(rings - 2, j + 1), idx(rings - 2, j)], axis=1))
    return verts, np.concatenate(tris).astype(np.uint32)


def _icosahedron():
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    return v, f


def icosphere(level):
    """Unit icosphere by `level` midpoint subdivisions: 20*4^L triangles, 10*4^L+2 vertices."""
    v, f = _icosahedron()
    for _ in range(level):
        nv = v.shape[0]
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        key = e[:, 0] * (nv + 1) + e[:, 1]
        uk, inv = np.unique(key, return_inverse=True)
        a, b = uk // (nv + 1), uk % (nv + 1)
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = inv.reshape(3, -1).T + nv  # midpoints of edges (01, 12, 20)
        v = np.concatenate([v, mid])
        f0, f1, f2 = f[:, 0], f[:, 1], f[:, 2]
        m01, m12, m20 = m[:, 0], m[:, 1], m[:, 2]
        f = np.concatenate([np.stack([f0, m01, m20], 1), np.stack([f1, m12, m01], 1), np.stack([f2, m20, m12], 1),
                            np.stack([m01, m12, m20], 1)])
    return v, f.astype(np.uint32)


def geodesic_sphere(n):
    """Class-I geodesic sphere of frequency n: each icosahedron face split into
    n^2 triangles, points projected to the unit sphere; 20 n^2 triangles,
    10 n^2 + 2 vertices.  Vectorised: a grid point is sum(w_k * corner_k) / n
    with the corners taken in increasing index order, so a point shared by two
    faces is computed bit-identically from both and exact duplicates merge."""
    n = int(n)
    v0, f0 = _icosahedron()
    i, j = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    keep = (i + j) <= n
    i, j = i[keep], j[keep]
    npf = i.size
    local = -np.ones((n + 1, n + 1), dtype=np.int64)
    local[i, j] = np.arange(npf)
    ids = np.repeat(f0[:, None, :], npf, axis=1)                         # (20, npf, 3) corner ids
    w = np.stack([n - i - j, i, j], axis=-1)[None].repeat(20, axis=0)   # (20, npf, 3) weights
    order = np.argsort(ids, axis=-1, kind="stable")
    ids = np.take_along_axis(ids, order, -1)
    w = np.take_along_axis(w, order, -1).astype(np.float64)
    p = (w[..., 0:1] * v0[ids[..., 0]] + w[..., 1:2] * v0[ids[..., 1]]) + w[..., 2:3] * v0[ids[..., 2]]
    p = p.reshape(-1, 3) / n
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    verts, inv = np.unique(p, axis=0, return_inverse=True)
    inv = inv.reshape(20, npf)
    a_i, a_j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    up = (a_i + a_j) <= n - 1
    ui, uj = a_i[up], a_j[up]
    dn = (a_i + a_j) <= n - 2
    di, dj = a_i[dn], a_j[dn]
    t_up = np.stack([local[ui, uj], local[ui + 1, uj], local[ui, uj + 1]], axis=1)
    t_dn = np.stack([local[di + 1, dj], local[di + 1, dj + 1], local[di, dj + 1]], axis=1)
    tl = np.concatenate([t_up, t_dn])                                      # per-face local triangles
    tris = (inv[:, tl]).reshape(-1, 3)
    return verts.astype(np.float64), tris.astype(np.uint32)


def displacement_params(rng, k=8):
    ax = rng.standard_normal((k, 3))
    ax /= np.linalg.norm(ax, axis=1, keepdims=True)
    ph = rng.uniform(0.0, 2.0 * np.pi, k)
    fr = 2.0 * np.pi * np.arange(1, k + 1) * (1.0 + 0.25 * rng.uniform(-1.0, 1.0, k))
    return ax, ph, fr


def displace(unit_verts, params, amp=0.05, radius=1.0):
    ax, ph, fr = params
    d = unit_verts
    r = np.ones(d.shape[0])
    for k in range(ax.shape[0]):
        r += amp * np.sin(fr[k] * (d @ ax[k]) + ph[k]) / (k + 1)
    return (d * (radius * r)[:, None]).astype(np.float64)


def random_rotation(rng):
    """Uniform rotation from a normalised 4-D Gaussian quaternion."""
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]], dtype=np.float64)


def grid_mesh(n=512, cell=2048.0, shift_x=0.0, z=None):
    """(n+1)^2 vertices on integer coordinates, 2 n^2 triangles; z: per-vertex z or None."""
    i, j = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    x = i * cell + shift_x
    y = j * cell
    zz = np.zeros_like(x, dtype=np.float64) if z is None else z
    verts = np.stack([x.ravel(), y.ravel(), np.asarray(zz, dtype=np.float64).ravel()], axis=1).astype(np.float64)
    vid = lambda a, b: a * (n + 1) + b
    a, b = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    a, b = a.ravel(), b.ravel()
    v00, v10, v01, v11 = vid(a, b), vid(a + 1, b), vid(a, b + 1), vid(a + 1, b + 1)
    tris = np.concatenate([np.stack([v00, v10, v11], 1), np.stack([v00, v11, v01], 1)]).astype(np.uint32)
    return verts, tris


# ------------------------------------------------------------------ configurations
def config1(seed=1):
    rng = np.random.default_rng(seed)
    v, t = uv_sphere(128, 80, 1.0)
    R = random_rotation(rng)
    return dict(name="uv_sphere_128x80", vA=v, tA=t, vB=v.copy(), tB=t.copy(),
                poseA=None, poseB=(R, np.zeros(3), np.array([0.5, 0.0, 0.0])))


def config2(seed=2, level=8):
    rng = np.random.default_rng(seed)
    u, t = icosphere(level)
    v = displace(u, displacement_params(rng))
    R = random_rotation(rng)
    return dict(name="icosphere_L%d_displaced" % level, vA=v, tA=t, vB=v.copy(), tB=t.copy(),
                poseA=None, poseB=(R, np.zeros(3), np.array([0.3, 0.1, 0.0])))


def config3(seed=3, n=512, cell=2048.0, tile=8):
    rng = np.random.default_rng(seed)
    vA, tA = grid_mesh(n, cell)
    ntile = n // tile + 1
    tz = rng.integers(-1, 2, size=(ntile, ntile)).astype(np.float64)
    i, j = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    z = tz[i // tile, j // tile]
    vB, tB = grid_mesh(n, cell, shift_x=cell / 2.0, z=z)
    return dict(name="coplanar_grid_%dx%d" % (n, n), vA=vA, tA=tA, vB=vB, tB=tB, poseA=None, poseB=None)


_geo_cache = {}


def geodesic_cached(n):
    if n not in _geo_cache:
        _geo_cache[n] = geodesic_sphere(n)
    return _geo_cache[n]


def freq_for_tris(T):
    return max(2, int(round((T / 20.0) ** 0.5)))


def _freq_grid(t_min, t_max, steps=24):
    """Geodesic frequencies on a geometric grid covering [t_min, t_max] triangles
    (20 n^2 each): drawing T log-uniformly and taking the nearest grid frequency
    keeps the distribution while only `steps` distinct spheres are built."""
    f = np.unique(np.round(np.geomspace(freq_for_tris(t_min), freq_for_tris(t_max), steps)).astype(int))
    return f


def _draw_tris(rng, t_min, t_max):
    return float(np.exp(rng.uniform(np.log(t_min), np.log(t_max))))


def _sphere_of_size(rng, grid, T):
    n = int(grid[np.argmin(np.abs(np.log(20.0 * grid.astype(float) ** 2) - np.log(T)))])
    u, t = geodesic_cached(n)
    return displace(u, displacement_params(rng)), t


def config4_sizes(seed=4, pairs=4096, t_min=1000, t_max=200000):
    """Triangle counts (drawn, before the frequency grid) of every pair's meshes,
    without building them: the first two draws of each pair's own generator."""
    out = []
    for p in range(pairs):
        rng = np.random.default_rng([seed, p])
        out.append((_draw_tris(rng, t_min, t_max), _draw_tris(rng, t_min, t_max)))
    return out


def config4_iter(seed=4, pairs=4096, t_min=1000, t_max=200000, which=None):
    """Batched pairs, one at a time (pair p from its own seeded generator, so any
    subset can be built alone): each mesh a displaced geodesic sphere with T
    log-uniform in [t_min, t_max]; B posed with an offset of [0.2, 1.5] *
    radius in a random direction and a random rotation."""
    grid = _freq_grid(t_min, t_max)
    for p in (range(pairs) if which is None else which):
        rng = np.random.default_rng([seed, p])
        TA, TB = _draw_tris(rng, t_min, t_max), _draw_tris(rng, t_min, t_max)
        vA, tA = _sphere_of_size(rng, grid, TA)
        vB, tB = _sphere_of_size(rng, grid, TB)
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        off = rng.uniform(0.2, 1.5) * d
        R = random_rotation(rng)
        yield dict(vA=vA, tA=tA, vB=vB, tB=tB, poseA=None, poseB=(R, np.zeros(3), off))


def config4(seed=4, pairs=4096, t_min=1000, t_max=200000):
    return list(config4_iter(seed, pairs, t_min, t_max))


def config5(seed=5, pairs=64, t_min=10000, t_max=2000000):
    """Serving set: mesh pairs of displaced geodesic spheres with T log-uniform
    in [t_min, t_max]; B's base pose an offset of 0.3 along a random direction
    plus a random rotation."""
    rng = np.random.default_rng(seed)
    grid = _freq_grid(t_min, t_max)
    out = []
    for p in range(pairs):
        vA, tA = _sphere_of_size(rng, grid, _draw_tris(rng, t_min, t_max))
        vB, tB = _sphere_of_size(rng, grid, _draw_tris(rng, t_min, t_max))
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        out.append(dict(vA=vA, tA=tA, vB=vB, tB=tB, poseB=(random_rotation(rng), np.zeros(3), 0.3 * d)))
    return out


def pose_stream(rng, n, max_rot_deg=5.0, max_trans=0.05):
    """Small random rigid updates: rotation <= max_rot_deg about a uniform axis."""
    out = []
    for _ in range(n):
        ax = rng.standard_normal(3)
        ax /= np.linalg.norm(ax)
        ang = np.deg2rad(rng.uniform(0.0, max_rot_deg))
        K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
        R = np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * (K @ K)
        tr = rng.standard_normal(3)
        tr *= rng.uniform(0.0, max_trans) / np.linalg.norm(tr)
        out.append((R, tr))
    return out

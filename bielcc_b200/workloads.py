"""Seeded synthetic workloads for the field / assembly paths.

No public dataset is involved: meshes, currents and observation points are
generated here with the shapes, sizes and distributions of the five workload
configurations (UV sphere PEC scatterer, refined sphere with near-field
points, perturbed icosphere assembly, 256-mesh batch, serving stream).

Physical-optics currents follow the plane-wave formulas of
electrodynamics/incident_field.h:20-59 in normalised units (|E0| = 1, H_inc =
k_hat x E0 e^{ik.x}, i.e. impedance 1): J = 2 n x H_inc on lit cells
(n . k_hat < 0) and 0 on shadow cells.
"""
import numpy as np


# ---------------------------------------------------------------- meshes
def uv_sphere(n_lat, n_lon, radius=1.0):
    """UV-parameterised quad mesh: n_lat x n_lon cells, vertex order
    (theta_i, phi_j), (theta_i+1, phi_j), (theta_i+1, phi_j+1), (theta_i, phi_j+1),
    which gives outward normals under norm_func; pole rows are degenerate quads
    (two equal vertices), as in examples/data/surface_mesh/sphere_quad.dat."""
    th = np.linspace(0.0, np.pi, n_lat + 1)
    ph = np.linspace(0.0, 2.0 * np.pi, n_lon + 1)

    def P(t, p):
        st = np.sin(t)
        return np.stack([radius * st * np.cos(p), radius * st * np.sin(p), radius * np.cos(t) * np.ones_like(p)], -1)

    cells = np.zeros((n_lat, n_lon, 4, 3))
    T, Pp = np.meshgrid(th[:-1], ph[:-1], indexing="ij")
    T1, Pp1 = np.meshgrid(th[1:], ph[1:], indexing="ij")
    cells[:, :, 0] = P(T, Pp)
    cells[:, :, 1] = P(T1, Pp)
    cells[:, :, 2] = P(T1, Pp1)
    cells[:, :, 3] = P(T, Pp1)
    # exact pole coordinates (sin(0) = 0, sin(pi) ~ 1e-16): make the degenerate
    # vertices bit-identical
    cells[0, :, 0] = cells[0, :, 3] = np.array([0.0, 0.0, radius])
    cells[-1, :, 1] = cells[-1, :, 2] = np.array([0.0, 0.0, -radius])
    return cells.reshape(-1, 4, 3)


def _icosahedron():
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]])
    return v / np.linalg.norm(v, axis=1, keepdims=True), f


def icosphere(level):
    """Unit icosphere, 20 * 4**level triangles, outward (counter-clockwise) order.
    Returns (vertices [V,3], faces [F,3])."""
    v, f = _icosahedron()
    verts = list(v)
    for _ in range(level):
        cache = {}

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        f = np.array(nf)
    return np.array(verts), f


def perturbed_icosphere(level=5, amp=0.05, seed=2, smooth_iters=8, radius=1.0):
    """Icosphere with radius * (1 + amp * s(v)), s = N(0,1) noise per vertex
    averaged `smooth_iters` times over the vertex 1-ring and rescaled to unit
    standard deviation. Returns triangle cells [F][3][3]."""
    v, f = icosphere(level)
    rng = np.random.default_rng(seed)
    s = rng.standard_normal(len(v))
    nb = [set() for _ in range(len(v))]
    for a, b, c in f:
        nb[a].update((b, c))
        nb[b].update((a, c))
        nb[c].update((a, b))
    idx = [np.fromiter(n, dtype=np.int64) for n in nb]
    for _ in range(smooth_iters):
        s = np.array([(s[i] + s[idx[i]].sum()) / (1 + len(idx[i])) for i in range(len(v))])
    s = (s - s.mean()) / s.std()
    vv = v * (radius * (1.0 + amp * s))[:, None]
    return vv[f]


def spheroid(n_lat, n_lon, a=1.0, c=2.0):
    """Prolate spheroid (semi-axes a, a, c) as a UV quad mesh."""
    cells = uv_sphere(n_lat, n_lon, 1.0)
    return cells * np.array([a, a, c])


def torus(n_u, n_v, R=1.5, r=0.5):
    """Torus quad mesh (major radius R, minor r), outward normals."""
    u = np.linspace(0, 2 * np.pi, n_u + 1)
    v = np.linspace(0, 2 * np.pi, n_v + 1)

    def P(uu, vv):
        return np.stack([(R + r * np.cos(vv)) * np.cos(uu), (R + r * np.cos(vv)) * np.sin(uu), r * np.sin(vv)], -1)

    U0, V0 = np.meshgrid(u[:-1], v[:-1], indexing="ij")
    U1, V1 = np.meshgrid(u[1:], v[1:], indexing="ij")
    cells = np.stack([P(U0, V0), P(U1, V0), P(U1, V1), P(U0, V1)], 2)
    return cells.reshape(-1, 4, 3)


def rounded_cube(n, edge_radius=0.1, half=1.0):
    """Cube [-half, half]^3 with rounded edges/corners: a UV sphere pushed onto
    the super-ellipsoid-like rounded box (point = core clamp + edge_radius *
    direction). Quad cells, n x 2n."""
    cells = uv_sphere(n, 2 * n, 1.0)
    core = half - edge_radius
    flat = cells.reshape(-1, 3)
    # map each sphere direction d to the rounded box surface along d
    d = flat / np.maximum(np.linalg.norm(flat, axis=1, keepdims=True), 1e-300)
    # support-function style projection: scale so that max-norm hits `half`
    m = np.max(np.abs(d), axis=1, keepdims=True)
    box = d / m * core
    out = box + edge_radius * d
    return out.reshape(cells.shape)


# ---------------------------------------------------------------- cell geometry (numpy)
def triangulate(cells):
    """Each quad split into triangles (v0, v1, v2) and (v2, v3, v0); triangles
    of (near) zero area, the collapsed halves of pole quads, are dropped."""
    cells = np.asarray(cells, np.float64)
    tri = np.concatenate([cells[:, [0, 1, 2]], cells[:, [2, 3, 0]]], axis=0)
    order = np.stack([np.arange(len(cells)), np.arange(len(cells)) + len(cells)], 1).ravel()
    tri = tri[order]  # the two halves of a quad next to each other
    area = 0.5 * np.linalg.norm(np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]), axis=1)
    return np.ascontiguousarray(tri[area > 1e-9 * area.max()])


def _mixed_shape(kind, target, triangles, rng):
    """One mesh of the batched / serving distributions: a spheroid (axis ratio
    1-4), a rounded cube (edge radius 0.1) or a torus (R/r = 3) of about
    `target` cells, as quads or (triangles=True) as their triangulation."""
    t = target / 2 if triangles else target
    if kind == 0:
        n_lat = max(4, int(round((t / 2) ** 0.5)))
        cells = spheroid(n_lat, 2 * n_lat, 1.0, rng.uniform(1.0, 4.0))
    elif kind == 1:
        cells = rounded_cube(max(4, int(round((t / 2) ** 0.5))), 0.1, 1.0)
    else:
        nv = max(4, int(round((t / 3) ** 0.5)))
        cells = torus(3 * nv, nv, 1.5, 0.5)
    return triangulate(cells) if triangles else cells


def centres(cells):
    if cells.shape[1] == 4:
        return (cells[:, 0] + cells[:, 1] + cells[:, 2] + cells[:, 3]) * 0.25
    return (cells[:, 0] + cells[:, 1] + cells[:, 2]) / 3.0


def normals(cells):
    if cells.shape[1] == 4:
        n = np.cross(cells[:, 2] - cells[:, 0], cells[:, 3] - cells[:, 1])
    else:
        n = np.cross(cells[:, 1] - cells[:, 0], cells[:, 2] - cells[:, 0])
    return n / np.linalg.norm(n, axis=1, keepdims=True)


def diameters(cells):
    if cells.shape[1] == 4:
        segs = [cells[:, 2] - cells[:, 0], cells[:, 3] - cells[:, 1]] + [cells[:, (s + 1) % 4] - cells[:, s] for s in range(4)]
    else:
        segs = [cells[:, (s + 1) % 3] - cells[:, s] for s in range(3)]
    return np.max(np.stack([np.linalg.norm(s, axis=1) for s in segs], 1), axis=1)


# ---------------------------------------------------------------- currents and incident field
def planewave(k, direction=(0.0, 0.0, 1.0), e0=(1.0, 0.0, 0.0)):
    """(k_vec, e0, h_scale) of a plane wave; h_scale = 1/k so H = k_hat x e0."""
    d = np.asarray(direction, float)
    d = d / np.linalg.norm(d)
    return k * d, np.asarray(e0, float), 1.0 / k


def po_currents(cells, k, directions=None, seed=None):
    """Physical-optics currents J = 2 n x H_inc (lit), 0 (shadow), evaluated at
    cell centres; one RHS per incidence direction. directions None -> +z with x
    polarisation; an int -> that many seeded uniform directions on S^2 with a
    random polarisation orthogonal to each. Returns J [S][N][3] complex128."""
    c = centres(cells)
    n = normals(cells)
    if directions is None:
        dirs = np.array([[0.0, 0.0, 1.0]])
        pols = np.array([[1.0, 0.0, 0.0]])
    else:
        rng = np.random.default_rng(seed)
        dirs = rng.standard_normal((int(directions), 3))
        dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
        tmp = rng.standard_normal((int(directions), 3))
        pols = tmp - (tmp * dirs).sum(1, keepdims=True) * dirs
        pols /= np.linalg.norm(pols, axis=1, keepdims=True)
    J = np.zeros((len(dirs), len(cells), 3), np.complex128)
    for s, (d, e0) in enumerate(zip(dirs, pols)):
        ph = np.exp(1j * k * (c @ d))
        h = np.cross(d, e0)[None, :] * ph[:, None]
        lit = (n @ d) < 0
        J[s] = np.where(lit[:, None], 2.0 * np.cross(n, h), 0.0)
    return J


# ---------------------------------------------------------------- observation points
def sphere_points(m, radius, seed):
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((m, 3))
    return radius * d / np.linalg.norm(d, axis=1, keepdims=True)


def shell_points(m, r_min, r_max, rng):
    d = rng.standard_normal((m, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return d * rng.uniform(r_min, r_max, size=(m, 1))


def near_points(cells, m, d_min, d_max, rng):
    idx = rng.integers(0, len(cells), size=m)
    return centres(cells)[idx] + normals(cells)[idx] * rng.uniform(d_min, d_max, size=(m, 1))


# ---------------------------------------------------------------- the workload configurations
def config1():
    """512-quad UV sphere (16 x 32), k = 2 pi, 1000 points on r = 3 (seed 0)."""
    cells = uv_sphere(16, 32)
    k = 2.0 * np.pi
    return dict(name="sphere512_k2pi_pts1000", cells=cells, k=k, J=po_currents(cells, k),
                pts=sphere_points(1000, 3.0, 0), inc=planewave(k))


def config2(n_far=18000, n_near=2000, n_lat=64):
    """8192-quad UV sphere (64 x 128), k = 2 pi, 18000 points on 2-5 m shells +
    2000 near-field points 0.02-0.1 m along normals of random cells (seed 1).
    n_lat (and the point counts) give the same construction at another size,
    for reduced profiling runs."""
    cells = uv_sphere(n_lat, 2 * n_lat)
    k = 2.0 * np.pi
    rng = np.random.default_rng(1)
    pts = np.concatenate([shell_points(n_far, 2.0, 5.0, rng), near_points(cells, n_near, 0.02, 0.1, rng)])
    return dict(name=f"sphere{len(cells)}_k2pi_pts{n_far + n_near}", cells=cells, k=k, J=po_currents(cells, k),
                pts=pts, inc=planewave(k))


def config3(level=5):
    """Perturbed icosphere (20 * 4**level triangles, seed 2), k = 4 pi."""
    cells = perturbed_icosphere(level=level, seed=2)
    return dict(name=f"icosphere{len(cells)}_k4pi_assembly", cells=cells, k=4.0 * np.pi)


def batch_meshes(n_meshes=256, seed=3, n_min=200, n_max=20000, pts_per_mesh=2000, rhs_max=64):
    """The 256-mesh batch: spheroids (axis ratio 1-4), rounded cubes (edge
    radius 0.1), tori (R/r = 3), every other triple of meshes as triangles
    (the quads split in two); 200-20000 cells log-uniform; k log-uniform in
    [0.5, 20]; 1-rhs_max PO right-hand sides from uniform S^2 directions;
    pts_per_mesh far points (on a shell at 2-4 x the mesh extent)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_meshes):
        kind = i % 3
        target = float(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
        cells = _mixed_shape(kind, target, (i // 3) % 2 == 1, rng)
        k = float(np.exp(rng.uniform(np.log(0.5), np.log(20.0))))
        S = int(rng.integers(1, rhs_max + 1))
        J = po_currents(cells, k, directions=S, seed=int(rng.integers(1 << 31)))
        extent = float(np.max(np.linalg.norm(cells.reshape(-1, 3), axis=1)))
        pts = shell_points(pts_per_mesh, 2.0 * extent, 4.0 * extent, rng)
        out.append(dict(cells=cells, k=k, J=J, pts=pts))
    return out


def serving_stream(n_requests=400, seed=4, n_meshes=24, n_min=200, n_max=20000, p_min=100, p_max=50000,
                   rhs_max=16, assembly_frac=0.1, max_assembly_cells=2000, near_frac=0.1):
    """Request stream of the serving workload. Meshes are drawn like
    batch_meshes (spheroids, rounded cubes, tori, quads or triangles; 200-20000
    cells log-uniform;
    k log-uniform in [0.5, 20]) and stay resident; each carries rhs_max PO
    current sets and a pool of p_max observation points (near_frac of them
    0.02-0.1 x the mesh extent above random cells, the rest on a 1.5-4 x
    extent shell). Requests arrive as a Poisson process of unit rate (arrival
    times are scaled by the caller's rate); a field request takes 100-50000
    points (log-uniform, the first P of its mesh's pool) and 1-16 current
    sets (the first S); assembly requests (assembly_frac of them) go to meshes
    of at most max_assembly_cells cells."""
    rng = np.random.default_rng(seed)
    meshes = []
    for i in range(n_meshes):
        kind = i % 3
        target = float(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
        cells = _mixed_shape(kind, target, (i // 3) % 2 == 1, rng)
        k = float(np.exp(rng.uniform(np.log(0.5), np.log(20.0))))
        extent = float(np.max(np.linalg.norm(cells.reshape(-1, 3), axis=1)))
        n_near = int(near_frac * p_max)
        pool = np.concatenate([shell_points(p_max - n_near, 1.5 * extent, 4.0 * extent, rng),
                               near_points(cells, n_near, 0.02 * extent, 0.1 * extent, rng)])
        pool = pool[rng.permutation(len(pool))]
        J = po_currents(cells, k, directions=rhs_max, seed=int(rng.integers(1 << 31)))
        meshes.append(dict(cells=cells, k=k, J=J, pts=np.ascontiguousarray(pool)))
    small = [i for i, m in enumerate(meshes) if len(m["cells"]) <= max_assembly_cells]
    t = 0.0
    reqs = []
    for _ in range(n_requests):
        t += float(rng.exponential(1.0))
        if small and rng.uniform() < assembly_frac:
            reqs.append(dict(t=t, type="assemble", mesh=int(rng.choice(small))))
        else:
            P = int(round(np.exp(rng.uniform(np.log(p_min), np.log(p_max)))))
            reqs.append(dict(t=t, type="field", mesh=int(rng.integers(n_meshes)), P=P,
                             S=int(rng.integers(1, rhs_max + 1))))
    return meshes, reqs

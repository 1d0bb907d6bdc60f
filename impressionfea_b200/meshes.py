"""Synthetic inputs of the forging path: tetrahedral billets and height-field dies.

The reference meshes its billet internally by isosurface stuffing (ThreeD/IsosurfaceStuffing.cs) and builds dies
from presets (ThreeD/DiePresets3D.cs). The per-iteration path only consumes the resulting arrays, so the cases here
are generated directly: a seeded 2D Delaunay fill of the quarter disk, extruded in layers, each prism split into
three tetrahedra by the global-index rule (conforming across shared faces), with node jitter uniform in
+-jitter*h along every direction a node is free to move. The same arrays feed the CUDA path and the oracle.
"""
from dataclasses import dataclass

import numpy as np


@dataclass
class TetCase:
    x: np.ndarray          # (nn, 3) float64
    tets: np.ndarray       # (ne, 4) int32, positively oriented
    on_x0: np.ndarray      # (nn,) uint8
    on_y0: np.ndarray      # (nn,) uint8
    gap0: float            # initial die gap
    bounds_for_velocity: tuple  # (min_x, min_y, min_z, max_x, max_y) of the seated billet

    @property
    def nn(self):
        return len(self.x)

    @property
    def ne(self):
        return len(self.tets)


@dataclass
class HeightField:
    """Rigid die z = h(x, y) on a regular grid (HeightFieldDie): samples (ny+1) x (nx+1), row-major in y."""
    x0: float
    y0: float
    dx: float
    nx: int
    ny: int
    h: np.ndarray

    def height_at(self, x, y):
        """Bilinear height (HeightFieldDie.HeightAt, ThreeD/HeightFieldDie.cs:100-107), clamped to the grid."""
        fx = min(max((x - self.x0) / self.dx, 0.0), float(self.nx))
        fy = min(max((y - self.y0) / self.dx, 0.0), float(self.ny))
        i, j = min(int(fx), self.nx - 1), min(int(fy), self.ny - 1)
        u, v, w = fx - i, fy - j, self.nx + 1
        h = self.h
        return ((1 - u) * (1 - v) * h[j * w + i] + u * (1 - v) * h[j * w + i + 1] + (1 - u) * v * h[(j + 1) * w + i]
                + u * v * h[(j + 1) * w + i + 1])

    @staticmethod
    def flat(z, half_extent=100.0):
        """Flat die as one grid cell (two triangles)."""
        return HeightField(-half_extent, -half_extent, 2 * half_extent, 1, 1, np.full(4, float(z)))

    @staticmethod
    def sample(fn, x0, x1, y0, y1, dx):
        nx = int(np.ceil((x1 - x0) / dx))
        ny = int(np.ceil((y1 - y0) / dx))
        xs = x0 + np.arange(nx + 1) * dx
        ys = y0 + np.arange(ny + 1) * dx
        X, Y = np.meshgrid(xs, ys)
        return HeightField(x0, y0, dx, nx, ny, np.ascontiguousarray(fn(X, Y), np.float64).ravel())


@dataclass
class TriMeshDie:
    """Rigid die as a closed triangulated solid (TriMeshDie over TriMeshSolid, ThreeD/TriMeshSolid.cs:248-297):
    vertices (nv, 3), triangles (nt, 3) wound with outward normals; the top die given in its closed position."""
    vertices: np.ndarray
    triangles: np.ndarray

    @staticmethod
    def box(lo, hi):
        """An axis-aligned box (12 triangles, outward winding)."""
        (x0, y0, z0), (x1, y1, z1) = lo, hi
        v = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                      [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]], np.float64)
        t = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4],
                      [1, 2, 6], [1, 6, 5], [2, 3, 7], [2, 7, 6], [3, 0, 4], [3, 4, 7]], np.int32)
        return TriMeshDie(v, t)

    @staticmethod
    def grid_block(fn, x0, x1, y0, y1, n, z_far, top):
        """A solid bounded by the surface z = fn(x, y) sampled on an (n+1) x (n+1) grid and the plane z = z_far
        (below the surface for a bottom die, above it for a top die), closed by four side walls."""
        xs, ys = np.linspace(x0, x1, n + 1), np.linspace(y0, y1, n + 1)
        X, Y = np.meshgrid(xs, ys)
        Z = np.asarray(fn(X, Y), np.float64)
        m = (n + 1) * (n + 1)
        top_v = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
        far_v = np.stack([X.ravel(), Y.ravel(), np.full(m, float(z_far))], 1)
        v = np.concatenate([top_v, far_v])
        idx = lambda i, j: j * (n + 1) + i
        tris = []
        for j in range(n):
            for i in range(n):
                a, b, c, d = idx(i, j), idx(i + 1, j), idx(i + 1, j + 1), idx(i, j + 1)
                tris += [[a, b, c], [a, c, d]]                      # working surface, normal +z
                tris += [[m + a, m + c, m + b], [m + a, m + d, m + c]]  # far plane, normal -z
        ring = [idx(i, 0) for i in range(n)] + [idx(n, j) for j in range(n)] + \
               [idx(i, n) for i in range(n, 0, -1)] + [idx(0, j) for j in range(n, 0, -1)]
        for k in range(len(ring)):
            p, q = ring[k], ring[(k + 1) % len(ring)]
            tris += [[p, m + p, m + q], [p, m + q, q]]              # side walls, outward
        t = np.array(tris, np.int32)
        if top:  # the solid lies above its working surface: flip every triangle
            t = t[:, [0, 2, 1]]
        return TriMeshDie(v, t)


def _quarter_disk_points(R, h):
    """Boundary nodes (on x=0, y=0 and the arc) and hexagonal-lattice interior nodes of the quarter disk."""
    n_edge = max(2, int(round(R / h)))
    n_arc = max(2, int(round(0.5 * np.pi * R / h)))
    pts, kind = [], []  # kind: 0 interior, 1 on y=0 edge, 2 on x=0 edge, 3 on arc, 4 corner
    pts.append((0.0, 0.0)); kind.append(4)
    for i in range(1, n_edge):
        pts.append((R * i / n_edge, 0.0)); kind.append(1)
    pts.append((R, 0.0)); kind.append(4)
    for k in range(1, n_arc):
        th = 0.5 * np.pi * k / n_arc
        pts.append((R * np.cos(th), R * np.sin(th))); kind.append(3)
    pts.append((0.0, R)); kind.append(4)
    for i in range(n_edge - 1, 0, -1):
        pts.append((0.0, R * i / n_edge)); kind.append(2)
    dy = h * np.sqrt(3) / 2
    j = 0
    y = 0.5 * dy
    while y < R:
        xoff = 0.5 * h if j % 2 else 0.0
        x = 0.5 * h + xoff
        while x < R:
            if np.hypot(x, y) < R - 0.45 * h and x > 0.4 * h and y > 0.4 * h:
                pts.append((x, y)); kind.append(0)
            x += h
        y += dy
        j += 1
    return np.array(pts), np.array(kind)


def quarter_cylinder(R, H, h, z0=0.0, seed=0, jitter=0.1, shut=None):
    """Quarter-model vertical cylinder (x >= 0, y >= 0), radius R, height H, base at z0, edge length about h.

    Returns a TetCase. With ``shut`` (closed top-die height), gap0 = z0 + H - shut (DieSet3D.Place for flat dies).
    """
    from scipy.spatial import Delaunay

    p2, kind = _quarter_disk_points(R, h)
    tri = Delaunay(p2).simplices.astype(np.int64)
    a, b, c = p2[tri[:, 0]], p2[tri[:, 1]], p2[tri[:, 2]]
    area2 = (b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (b[:, 1] - a[:, 1]) * (c[:, 0] - a[:, 0])
    tri = tri[np.abs(area2) > 1e-12 * h * h]
    tri.sort(axis=1)
    nz = max(2, int(round(H / h)))
    n2 = len(p2)
    zs = z0 + H * np.arange(nz + 1) / nz
    nn = n2 * (nz + 1)
    x = np.zeros((nn, 3))
    for k in range(nz + 1):
        x[k * n2:(k + 1) * n2, :2] = p2
        x[k * n2:(k + 1) * n2, 2] = zs[k]
    tets = []
    for k in range(nz):
        base, top = k * n2, (k + 1) * n2
        v0, v1, v2 = base + tri[:, 0], base + tri[:, 1], base + tri[:, 2]
        v3, v4, v5 = top + tri[:, 0], top + tri[:, 1], top + tri[:, 2]
        tets.append(np.stack([v0, v1, v2, v3], 1))
        tets.append(np.stack([v1, v2, v3, v4], 1))
        tets.append(np.stack([v2, v3, v4, v5], 1))
    tets = np.concatenate(tets).astype(np.int64)
    # interleave prisms so consecutive tets are spatial neighbours (layer-major order already is)
    rng = np.random.default_rng(seed)
    kind3 = np.tile(kind, nz + 1)
    layer = np.repeat(np.arange(nz + 1), n2)
    amp = jitter * h
    d = rng.uniform(-amp, amp, size=(nn, 3))
    free_z = (layer > 0) & (layer < nz)
    disp = np.zeros((nn, 3))
    disp[:, 2] = np.where(free_z, d[:, 2], 0.0)
    inter = kind3 == 0
    disp[inter, 0] = d[inter, 0]
    disp[inter, 1] = d[inter, 1]
    on_y_edge = kind3 == 1
    disp[on_y_edge, 0] = d[on_y_edge, 0]
    on_x_edge = kind3 == 2
    disp[on_x_edge, 1] = d[on_x_edge, 1]
    on_arc = kind3 == 3

    def apply(scale):
        xx = x.copy()
        xx[:, 2] += disp[:, 2] * scale
        xx[inter | on_y_edge | on_x_edge, :2] += disp[inter | on_y_edge | on_x_edge, :2] * scale[inter | on_y_edge | on_x_edge, None]
        th = np.arctan2(x[on_arc, 1], x[on_arc, 0]) + d[on_arc, 0] / R * scale[on_arc]
        xx[on_arc, 0] = R * np.cos(th)
        xx[on_arc, 1] = R * np.sin(th)
        return xx

    scale = np.ones(nn)
    if jitter > 0:
        for _ in range(8):
            xx = apply(scale)
            det = _tet_det(xx, tets)
            bad = np.abs(det) < 0.05 * _tet_det(x, tets).__abs__()
            if not bad.any():
                break
            scale[np.unique(tets[bad])] *= 0.5
        x = apply(scale)
    det = _tet_det(x, tets)
    flip = det < 0
    tets[flip] = tets[flip][:, [0, 2, 1, 3]]
    det = _tet_det(x, tets)
    assert (det > 0).all(), "generated mesh has inverted tetrahedra"
    on_x0 = (x[:, 0] == 0.0).astype(np.uint8)
    on_y0 = (x[:, 1] == 0.0).astype(np.uint8)
    gap0 = (z0 + H - shut) if shut is not None else 0.0
    return TetCase(x=np.ascontiguousarray(x), tets=np.ascontiguousarray(tets.astype(np.int32)), on_x0=on_x0,
                   on_y0=on_y0, gap0=float(gap0), bounds_for_velocity=(-R, -R, z0, R, R))


def _tet_det(x, t):
    p0 = x[t[:, 0]]
    a, b, c = x[t[:, 1]] - p0, x[t[:, 2]] - p0, x[t[:, 3]] - p0
    return np.einsum("ij,ij->i", a, np.cross(b, c))


def h_for_tets(R, H, target_tets):
    """Edge length giving about ``target_tets`` tetrahedra in the quarter cylinder."""
    area = 0.25 * np.pi * R * R
    # triangles ~ area / (sqrt(3)/4 h^2), layers ~ H / h, 3 tets per prism
    return float((3 * area * H / (np.sqrt(3) / 4) / target_tets) ** (1.0 / 3.0))


def upset_case_3d(R, H, h, shut, seed=0, jitter=0.1):
    """Quarter cylinder between flat dies: bottom die z = 0, top die closed at z = shut."""
    mesh = quarter_cylinder(R, H, h, z0=0.0, seed=seed, jitter=jitter, shut=shut)
    dies = (HeightField.flat(0.0, 4 * R + 20), HeightField.flat(shut, 4 * R + 20))
    return mesh, dies


def gear_blank_thickness(r, hub_r=15.0, hub_t=22.0, web_t=6.0, rim_in=36.0, rim_r=45.0, rim_t=10.0, flash_t=3.0,
                         land_ratio=3.0, ramp=1.5):
    """Part thickness at closure of an axisymmetric gear blank, as a function of the radius: hub (r < hub_r), web
    of thickness web_t, rim (rim_in < r < rim_r), flash land of gap flash_t and width land_ratio * flash_t, then
    the gutter (open). Neighbouring levels are joined by linear ramps of width `ramp` (drafts of the impression).
    The published case gives the hub radius, web thickness, rim radius, flash gap and land ratio; the hub and rim
    thicknesses and the rim's inner radius are this generator's, chosen so that the cavity up to the land holds
    about the billet's volume (d40 x h50: 62.8 cm^3) and the excess goes to flash."""
    r = np.asarray(r, np.float64)
    land_out = rim_r + land_ratio * flash_t
    edges = [(hub_r, hub_t, web_t), (rim_in, web_t, rim_t), (rim_r, rim_t, flash_t), (land_out, flash_t, 4 * hub_t)]
    t = np.full(r.shape, hub_t)
    for e, a, b in edges:
        s = np.clip((r - (e - 0.5 * ramp)) / ramp, 0.0, 1.0)
        t = np.where(r >= e - 0.5 * ramp, a + (b - a) * s, t)
    return t


def stuffed_cylinder(R, H, h, z0=0.0):
    """Quarter-model vertical cylinder (x >= 0, y >= 0) of radius R and height H on z = z0, meshed the way the
    reference meshes its billets: isosurface stuffing of the solid at lattice spacing h
    (IsosurfaceStuffing.Stuff, ThreeD/IsosurfaceStuffing.cs:19-84, by the library's host mesher)."""
    from .remesh import stuff

    x, t = stuff(lambda px, py, pz: px * px + py * py < R * R and z0 < pz < z0 + H, (-R, -R, z0), (R, R, z0 + H), h,
                 True, True)
    on_x0 = (x[:, 0] == 0.0).astype(np.uint8)
    on_y0 = (x[:, 1] == 0.0).astype(np.uint8)
    return TetCase(x=np.ascontiguousarray(x), tets=np.ascontiguousarray(t, np.int32), on_x0=on_x0, on_y0=on_y0,
                   gap0=0.0, bounds_for_velocity=(-R, -R, z0, R, R))


def gear_blank_case_3d(h, R=20.0, H=50.0, dx=0.5, seed=0, jitter=0.1, stuffed=False, **profile):
    """Closed-die forging of a gear blank (quarter model): billet d = 2R, height H on the bottom die; both dies are
    height fields sampled at dx from gear_blank_thickness, mirrored about the part's mid-plane, the top die given at
    its closed position. The billet seats on the highest point of the bottom die under it (z0 = 0) and the top die
    starts touching it: gap0 = max over billet nodes of (z - top surface). stuffed: the billet is meshed by
    isosurface stuffing at h (as the reference does, and as every remesh does), else by the seeded Delaunay fill."""
    zm = 0.5 * float(np.min(gear_blank_thickness(np.linspace(0.0, R, 401), **profile)))  # seat: z0 = 0
    bottom = HeightField.sample(lambda X, Y: zm - 0.5 * gear_blank_thickness(np.hypot(X, Y), **profile),
                                -2.0, 70.0, -2.0, 70.0, dx)
    top = HeightField.sample(lambda X, Y: zm + 0.5 * gear_blank_thickness(np.hypot(X, Y), **profile),
                             -2.0, 70.0, -2.0, 70.0, dx)
    mesh = stuffed_cylinder(R, H, h) if stuffed else quarter_cylinder(R, H, h, z0=0.0, seed=seed, jitter=jitter)
    r = np.hypot(mesh.x[:, 0], mesh.x[:, 1])
    mesh.gap0 = float(np.max(mesh.x[:, 2] - (zm + 0.5 * gear_blank_thickness(r, **profile))))
    return mesh, (bottom, top)


def cavity_samples(dies, outline, x_max, y_max, sym_x=True, sym_y=True, x_min=None):
    """The closed cavity's sample points for FillPercent (BuildCavitySamples, ThreeD/Forging3DSolver.cs:2157-2172):
    a plan-view grid of spacing sqrt(area / 2500) over the part's extent, and at every grid point inside the outline
    (outline(x, y) < 0) where the closed dies leave a gap, points spread evenly through that gap. (n, 3) array."""
    x0 = 0.0 if sym_x else (-x_max if x_min is None else x_min)
    y0 = 0.0 if sym_y else -y_max
    d = np.sqrt((x_max - x0) * (y_max - y0) / 2500.0)
    out = []
    x = x0 + d / 2
    while x < x_max:
        y = y0 + d / 2
        while y < y_max:
            if outline(x, y) < 0:
                zb, zt = dies[0].height_at(x, y), dies[1].height_at(x, y)
                if zt > zb:
                    nz = max(1, int(round((zt - zb) / d)))
                    for k in range(nz):
                        out.append((x, y, zb + (k + 0.5) * (zt - zb) / nz))
            y += d
        x += d
    return np.array(out, np.float64).reshape(-1, 3)


def gear_blank_outline(x, y, rim_r=45.0, flash_t=3.0, land_ratio=3.0, ramp=4.0):
    """Plan-view outline of the gear blank's impression (negative inside): the flash land up to where the ramp to
    the open gutter starts."""
    return float(np.hypot(x, y)) - (rim_r + land_ratio * flash_t - 0.5 * ramp)

"""The forging cases the library is measured and checked on (synthetic inputs of the published configurations).

- ``upsetting_drop_in()``: 3D upsetting, quarter model of a d30 x h45 billet, ~30k linear tets from a seeded
  Delaunay fill (node jitter +-10 % of h), flat dies as two-triangle height fields, C = 150 MPa, eps0 = 0.01,
  n = 0.1, m = 0.12, friction m_f = 0.4, 40 % reduction in 80 increments, ram 50 mm/s, tolerance 1e-3.
- ``closed_die_gear_blank()``: closed-die forging of an axisymmetric gear blank (hub r15, web 6 mm, rim r45,
  flash gap 3 mm, land 3:1) as two height fields at dx = 0.5 mm, billet d40 x h50 meshed by isosurface stuffing
  at 1.0 mm (~202k tets), C = 140 MPa, n = 0.08, m = 0.15, friction 0.3, 200 increments to closure.
- ``upsetting_2d()``: 2D axisymmetric upsetting, r10 x h30 billet, 20 x 60 quads, flat dies, C = 120 MPa,
  eps0 = 0.01, n = 0.05, m = 0.15, friction 0.3, ram 10 mm/s, 50 % in 100 increments, tolerance 1e-6.

The reference builds its 3D billets by isosurface stuffing (ThreeD/IsosurfaceStuffing.cs); the closed-die billet
is stuffed the same way (by the library's host mesher), the upsetting billet is a seeded Delaunay fill. The same
arrays feed the CUDA path and the oracle, which is all the per-iteration path consumes.
"""
import numpy as np

from .config import Forging2DConfig, Forging3DConfig
from .meshes import gear_blank_case_3d, h_for_tets, upset_case_3d

UPSET_R, UPSET_H, UPSET_REDUCTION, UPSET_STEPS, UPSET_TETS = 15.0, 45.0, 0.40, 80, 30000


def upsetting_drop_in(target_tets=UPSET_TETS, seed=2024):
    h = round(h_for_tets(UPSET_R, UPSET_H, target_tets), 3)
    stroke = UPSET_REDUCTION * UPSET_H
    mesh, dies = upset_case_3d(UPSET_R, UPSET_H, h, shut=UPSET_H - stroke, seed=seed)
    cfg = Forging3DConfig(C=150, N=0.1, M=0.12, eps0=0.01, friction=0.4, ram=50.0, h=h, ds=stroke / UPSET_STEPS,
                          size=UPSET_H, tol=1e-3)
    return cfg, mesh, dies


def closed_die_gear_blank(target_tets=200000, seed=None):
    """The closed-die case; the billet is meshed by isosurface stuffing, like every remesh after it, at the lattice
    spacing that gives about target_tets tets (1.0 mm for 200k). seed=None: the published geometry (billet
    d40 x h50); a seed draws a geometry variant, billet radius and height each within +-5 % (training trajectories
    for the learned warm start)."""
    R, H = 20.0, 50.0
    if seed is not None:
        rng = np.random.default_rng(seed)
        R *= rng.uniform(0.95, 1.05)
        H *= rng.uniform(0.95, 1.05)
    h = round(1.0 * (200000.0 / target_tets) ** (1.0 / 3.0), 3)
    mesh, dies = gear_blank_case_3d(h, R=R, H=H, ramp=4.0, stuffed=True)
    cfg = Forging3DConfig(C=140, N=0.08, M=0.15, eps0=0.01, friction=0.3, ram=50.0, h=h, ds=mesh.gap0 / 200,
                          size=H, tol=1e-3)
    return cfg, mesh, dies


def upsetting_2d():
    return Forging2DConfig()


def batched_sweep(n_cases=64, seed=4096):
    """Independent upsetting cases of uneven size: half 2D axisymmetric (2k-20k quads), half 3D quarter models
    (5k-80k tets), each with its own seeded draw of aspect h/d ~ U[0.8, 2.0], friction m_f ~ U[0.1, 0.6],
    C ~ U[80, 200] MPa, n ~ U[0, 0.2], m ~ U[0.05, 0.25]. Returns [("2d", cfg) | ("3d", cfg, mesh, dies)]."""
    rng = np.random.default_rng(seed)
    cases = []
    for c in range(n_cases):
        aspect = rng.uniform(0.8, 2.0)
        friction, Cc, n, m = rng.uniform(0.1, 0.6), rng.uniform(80, 200), rng.uniform(0, 0.2), rng.uniform(0.05, 0.25)
        R = 10.0
        H = aspect * 2 * R
        if c % 2 == 0:
            ne = int(rng.uniform(2000, 20000))
            nx = max(4, int(round(np.sqrt(ne * R / H))))
            nz = max(4, int(round(ne / nx)))
            cfg = Forging2DConfig(C=Cc, N=n, M=m, eps0=0.01, friction=friction, ram=10.0, ds=0.5 * H / 100, tol=1e-6,
                                  radius=R, height=H, nx=nx, nz=nz,
                                  top_profile=np.array([[0.0, 0.5 * H], [200.0, 0.5 * H]]))
            cases.append(("2d", cfg))
        else:
            tets = int(rng.uniform(5000, 80000))
            h = round(h_for_tets(R, H, tets), 3)
            shut = 0.6 * H
            mesh, dies = upset_case_3d(R, H, h, shut, seed=c)
            cfg = Forging3DConfig(C=Cc, N=n, M=m, eps0=0.01, friction=friction, ram=50.0, h=h, ds=(H - shut) / 80,
                                  size=H, tol=1e-3)
            cases.append(("3d", cfg, mesh, dies))
    return cases

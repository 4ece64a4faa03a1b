"""Seeded test problems shared by the parity tests (small versions of the
benchmark workloads: 2D perturbed triangles with lognormal diffusivity, and
3D Kuhn tetrahedra with upwind convection)."""
import numpy as np


def diffusion_2d(fv, n=16, seed=3, sigma=1.0, jitter=0.2):
    m = fv.Mesh.square(n, jitter, seed)
    kf, _, sc = m.fields(seed, 1.0, sigma, source_const=1.0)
    nb = m.n_boundary_faces
    return dict(mesh=m, c_lap=-1.0, c_conv=0.0, c_src=-1.0, kappa=kf, flux=None, source=sc,
                bndi=np.zeros(nb), bnde=np.zeros(nb))


def convdiff_3d(fv, n=6, seed=5, sigma=0.5, jitter=0.15, velocity=(1.0, 0.5, 0.25)):
    m = fv.Mesh.cube(n, jitter, seed)
    h = 1.0 / n
    kappa0 = float(np.linalg.norm(velocity)) * h / 3.0
    kf, fl, sc = m.fields(seed, kappa0, sigma, velocity=velocity, source_uniform=True)
    nb = m.n_boundary_faces
    return dict(mesh=m, c_lap=-1.0, c_conv=1.0, c_src=-1.0, kappa=kf, flux=fl, source=sc,
                bndi=np.zeros(nb), bnde=np.zeros(nb))


def equation(fv, case):
    lap = fv.laplacian(fv.Orthogonal(), case["kappa"])
    src = fv.source(case["source"])
    if case["c_conv"] != 0.0:
        return fv.convection(fv.Upwind(case["flux"]), case["flux"]) - lap - src
    return -lap - src


def oracle_system(orc, case):
    return orc.assemble(case["mesh"], case["c_lap"], case["c_conv"], case["c_src"], kappa=case["kappa"],
                        flux=case["flux"], source=case["source"], bndi=case["bndi"], bnde=case["bnde"])

"""Shared test helpers: golden fixtures, synthetic cases, and the same problem built for the
GPU library (mhdarcy) and for the CPU oracle."""
import os

import numpy as np

import mhdarcy
from mhdarcy.mesh import Mesh

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_fixture(name):
    z = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    mesh = Mesh(z["nodes"], z["el_dim"], z["el_nodes"], z["bc_dim"], z["bc_nodes"])
    return z, mesh


def fixture_coeffs(z):
    n = len(z["el_dim"])
    aniso = np.zeros((n, 9))
    aniso[:, 0] = aniso[:, 4] = aniso[:, 8] = z["anisotropy"]
    return dict(conductivity=z["conductivity"], anisotropy=aniso, cross_section=z["cross_section"],
                sigma=z["sigma"], water_source_density=z["water_source_density"], storativity=z["storativity"])


def fixture_bc(z, topo):
    """Per boundary object: explicit boundary elements carry the case's data, implicit ones
    (created for outer sides without a boundary element) are homogeneous Neumann."""
    bb = topo["bdr_bc_element"]
    per = lambda a: np.array([a[b] if b >= 0 else 0.0 for b in bb])
    return dict(bc_type=np.array([z["bc_type"][b] if b >= 0 else 0 for b in bb], np.int32),
                pressure=per(z["bc_pressure"]), flux=per(z["bc_flux"]), robin_sigma=per(z["bc_robin_sigma"]))


def oracle_problem(mesh, topo, n_edges, coeffs, bc, **kw):
    import oracle as O
    return O.Problem(mesh, topo, n_edges, conductivity=coeffs.get("conductivity", 1.0),
                     anisotropy=coeffs.get("anisotropy"), cross_section=coeffs.get("cross_section", 1.0),
                     sigma=coeffs.get("sigma", 1.0), water_source_density=coeffs.get("water_source_density", 0.0),
                     storativity=coeffs.get("storativity", 1.0), bc_type=bc["bc_type"],
                     bc_pressure=bc.get("pressure", 0.0), bc_flux=bc.get("flux", 0.0),
                     bc_robin_sigma=bc.get("robin_sigma", 0.0), **kw)


def cube_case(n, planes=(), lines=(), seed=1234, log_mean=-6.0, log_std=1.0, frac_K=1e-3, frac_delta=1e-3,
              line_K=1e-2, line_delta=1e-4):
    """A Kuhn-cube case in the style of the benchmark configurations: log-normal 3D
    conductivity, fracture and channel coefficients, Dirichlet p=1 at x=0 and p=0 at x=1 on
    every dimension's outer sides, homogeneous Neumann elsewhere."""
    mesh = mhdarcy.cube_mesh(n, planes, lines)
    rng = np.random.default_rng(seed)
    ne = mesh.n_elements
    K = np.empty(ne)
    d = np.ones(ne)
    d3 = mesh.el_dim == 3
    K[d3] = 10.0 ** rng.normal(log_mean, log_std, d3.sum())
    K[mesh.el_dim == 2] = frac_K
    d[mesh.el_dim == 2] = frac_delta
    K[mesh.el_dim == 1] = line_K
    d[mesh.el_dim == 1] = line_delta
    coeffs = dict(conductivity=K, cross_section=d)
    return mesh, coeffs


def cube_bc(system_or_topo, mesh):
    """Dirichlet p = 1 on x = 0 and p = 0 on x = 1 (boundary sides of every dimension)."""
    from mhdarcy.cases import dirichlet_x_bc
    topo = system_or_topo.topology() if hasattr(system_or_topo, "topology") else system_or_topo
    return dirichlet_x_bc(topo, mesh)[0]

"""Synthetic fractured-cube cases with the shapes and value distributions of the benchmark
configurations (there is no public dataset for this path; everything is seeded):

  cfg1  n=16 Kuhn cube (24,576 tets) + z=0.5 fracture (512 triangles, delta=1e-3, K=1e-3)
        + 1D x-line at y=z=0.5 (16 segments, delta=1e-4, K=1e-2); log10 K3 ~ N(-6, 1) iid.
  cfg2  n=64 (1,572,864 tets), same fracture/line; log10 K3 ~ N(-6, 1.5) Gaussian-correlated,
        correlation length 0.1 (FFT-filtered white noise on a 128^3 grid, sampled at centroids).
  cfg3  instances: n in {8,12,16,24,32}, one z=0.5 fracture, N(-6,1), correlation 0.05..0.2.
  cfg4  n=48 + z=0.5 fracture, S3=1e-4, S2=1e-6, N(-6,1); p(x=0,t) = 1 + 0.5 sin(2 pi t).
  cfg5  n=96, 6 axis-aligned fractures at seeded interior grid planes (log10 K ~ U(-4,-2),
        delta=1e-3), 4 channels along grid lines inside fracture planes, log10 K3 ~ N(-7, 2)
        with correlation length 0.05 clipped to [1e-9, 1e-2].
Boundary conditions: Dirichlet p=1 on x=0 and p=0 on x=1 on the outer sides of every dimension,
homogeneous Neumann elsewhere.  Seeds: 1234 + config index (+ instance for cfg3).
"""
import numpy as np

_SIDE = {1: np.array([[0, -1, -1], [1, -1, -1]]), 2: np.array([[0, 1, -1], [1, 2, -1], [0, 2, -1]]),
         3: np.array([[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]])}


def correlated_normal(grid, corr_len, rng):
    """Zero-mean unit-variance Gaussian field on a periodic grid^3 with covariance
    exp(-r^2 / corr_len^2) (white noise filtered in Fourier space)."""
    w = rng.standard_normal((grid, grid, grid))
    k = 2.0 * np.pi * np.fft.fftfreq(grid, d=1.0 / grid)
    kx, ky, kz = np.meshgrid(k, k, np.fft.rfftfreq(grid, d=1.0 / grid) * 2.0 * np.pi, indexing="ij")
    filt = np.exp(-(kx ** 2 + ky ** 2 + kz ** 2) * corr_len ** 2 / 8.0)
    f = np.fft.irfftn(np.fft.rfftn(w) * filt, s=w.shape, axes=(0, 1, 2))
    f -= f.mean()
    return f / f.std()


def sample_at(field, pts):
    g = field.shape[0]
    idx = np.clip((pts * g).astype(np.int64), 0, g - 1)
    return field[idx[:, 0], idx[:, 1], idx[:, 2]]


def dirichlet_x_bc(topo, mesh, p_left=1.0, p_right=0.0):
    """Boundary arrays: Dirichlet p_left on x=0, p_right on x=1, homogeneous Neumann elsewhere."""
    ss, sb = topo["el_side_start"], topo["side_bdr"]
    nb = len(topo["bdr_edge"])
    typ = np.zeros(nb, np.int32)
    p = np.zeros(nb)
    bs = np.nonzero(sb >= 0)[0]
    side_el = np.searchsorted(ss, bs, side="right") - 1
    loc = bs - ss[side_el]
    dims = mesh.el_dim[side_el]
    xmin = np.full(len(bs), np.inf)
    xmax = np.full(len(bs), -np.inf)
    for d in (1, 2, 3):
        sel = np.nonzero(dims == d)[0]
        if len(sel) == 0:
            continue
        tab = _SIDE[d][loc[sel]]
        for k in range(d):
            x = mesh.nodes[mesh.el_nodes[side_el[sel], tab[:, k]], 0]
            xmin[sel] = np.minimum(xmin[sel], x)
            xmax[sel] = np.maximum(xmax[sel], x)
    left = xmax < 1e-12
    right = xmin > 1.0 - 1e-12
    typ[sb[bs[left]]] = 1
    p[sb[bs[left]]] = p_left
    typ[sb[bs[right]]] = 1
    p[sb[bs[right]]] = p_right
    return dict(bc_type=typ, pressure=p), sb[bs[left]]


def make_case(cfg, seed=None, n=None, corr_len=None, mesh_builder=None):
    """Mesh and coefficients of a benchmark configuration (1..5).  mesh_builder(n, planes,
    lines) makes the Kuhn cube mesh (default: the library's mhdarcy.cube_mesh); this module
    needs nothing else from the package, so a CPU-only caller can load it by file path and
    pass its own builder of the same mesh."""
    if mesh_builder is None:
        from .mesh import cube_mesh as mesh_builder
    cube_mesh = mesh_builder
    seed = 1234 + cfg if seed is None else seed
    rng = np.random.default_rng(seed)
    if cfg == 1:
        n = n or 16
        mesh = cube_mesh(n, [(2, n // 2)], [(0, n // 2, n // 2)])
        logk = rng.normal(-6.0, 1.0, mesh.n_elements)
    elif cfg == 2:
        n = n or 64
        mesh = cube_mesh(n, [(2, n // 2)], [(0, n // 2, n // 2)])
        f = correlated_normal(2 * n, 0.1, rng)
        logk = -6.0 + 1.5 * sample_at(f, mesh.centres())
    elif cfg == 3:
        n = n or int(rng.choice([8, 12, 16, 24, 32]))
        cl = corr_len or float(rng.uniform(0.05, 0.2))
        mesh = cube_mesh(n, [(2, n // 2)])
        f = correlated_normal(max(32, 2 * n), cl, rng)
        logk = -6.0 + 1.0 * sample_at(f, mesh.centres())
    elif cfg == 4:
        n = n or 48
        mesh = cube_mesh(n, [(2, n // 2)])
        logk = rng.normal(-6.0, 1.0, mesh.n_elements)
    elif cfg == 5:
        n = n or 96
        planes = []
        for ax in (0, 1, 2):
            pos = rng.choice(np.arange(n // 8, n - n // 8), size=2, replace=False)
            planes += [(ax, int(p)) for p in sorted(pos)]
        # channels along intersections of an x-plane and a z-plane (grid lines in both planes)
        xs = [p for a, p in planes if a == 0]
        ys = [p for a, p in planes if a == 1]
        zs = [p for a, p in planes if a == 2]
        lines = [(1, xs[0], zs[0]), (1, xs[1], zs[1]), (0, ys[0], zs[1]), (2, xs[1], ys[0])]
        mesh = cube_mesh(n, planes, lines)
        f = correlated_normal(2 * n, 0.05, rng)
        logk = np.clip(-7.0 + 2.0 * sample_at(f, mesh.centres()), -9.0, -2.0)
    else:
        raise ValueError(cfg)
    ne = mesh.n_elements
    K = 10.0 ** logk
    delta = np.ones(ne)
    sto = np.ones(ne)
    d2, d1 = mesh.el_dim == 2, mesh.el_dim == 1
    if cfg == 5:
        tri = np.nonzero(d2)[0]
        per_plane = 2 * n * n
        fk = 10.0 ** rng.uniform(-4.0, -2.0, len(tri) // per_plane)
        K[tri] = np.repeat(fk, per_plane)
    else:
        K[d2] = 1e-3
    delta[d2] = 1e-3
    K[d1] = 1e-2
    delta[d1] = 1e-4
    if cfg == 4:
        sto[mesh.el_dim == 3] = 1e-4
        sto[d2] = 1e-6
    coeffs = dict(conductivity=K, cross_section=delta, storativity=sto)
    return mesh, coeffs

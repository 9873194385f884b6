"""Intersections of 1D elements with 2D elements that do not share their nodes, in the form the
mortar coupling takes (mh_create_mortar): the reference reads them from the neighbouring file
of an external tool (Mesh::read_intersections, src/mesh/mesh.cc:703-755); this computes them
for segments that lie in the plane of the triangles.

Each intersection is the part of a segment (master) inside a triangle (slave): its two end
points X, Y with their local coordinates on the master (t in [0, 1] from node 0 to node 1) and
on the slave (t0, t1 with nodes 0, 1, 2 at (0, 0), (1, 0), (0, 1)), X before Y along the
segment.
"""
import ctypes as C

import numpy as np

from . import _lib


def plane_intersections(mesh, lines=None, triangles=None, tol=1e-12):
    """(master, slave, master_t [n, 2], slave_xy [n, 2, 2]) for the segments `lines` and the
    triangles `triangles` (element indices; default all of each dimension) that are coplanar:
    each segment is clipped against each triangle's three sides in the triangle's plane."""
    dim = np.asarray(mesh.el_dim)
    lines = np.nonzero(dim == 1)[0] if lines is None else np.asarray(lines)
    triangles = np.nonzero(dim == 2)[0] if triangles is None else np.asarray(triangles)
    X = mesh.nodes
    out_m, out_s, out_t, out_xy = [], [], [], []
    for ln in lines:
        P0, P1 = X[mesh.el_nodes[ln, 0]], X[mesh.el_nodes[ln, 1]]
        dvec = P1 - P0
        L = np.linalg.norm(dvec)
        for tr in triangles:
            A, B, Cc = (X[mesh.el_nodes[tr, k]] for k in range(3))
            nrm = np.cross(B - A, Cc - A)
            area2 = np.linalg.norm(nrm)
            if area2 == 0.0:
                continue
            nu = nrm / area2
            if abs(np.dot(P0 - A, nu)) > tol * max(1.0, L) or abs(np.dot(P1 - A, nu)) > tol * max(1.0, L):
                continue  # not in the triangle's plane
            lo, hi = 0.0, 1.0
            for Q0, Q1, Qo in ((A, B, Cc), (B, Cc, A), (Cc, A, B)):
                e = Q1 - Q0
                inward = np.cross(nu, e)
                if np.dot(inward, Qo - Q0) < 0:
                    inward = -inward
                f0 = np.dot(P0 - Q0, inward)
                f1 = np.dot(dvec, inward)
                if abs(f1) <= tol * np.linalg.norm(inward) * max(L, 1e-300):
                    if f0 < -tol * np.linalg.norm(inward):
                        lo, hi = 1.0, 0.0
                    continue
                t = -f0 / f1
                if f1 > 0:
                    lo = max(lo, t)
                else:
                    hi = min(hi, t)
            if hi - lo <= tol:
                continue
            G = np.array([[np.dot(B - A, B - A), np.dot(B - A, Cc - A)], [np.dot(B - A, Cc - A), np.dot(Cc - A, Cc - A)]])
            xy = []
            for t in (lo, hi):
                p = P0 + t * dvec - A
                xy.append(np.linalg.solve(G, [np.dot(p, B - A), np.dot(p, Cc - A)]))
            out_m.append(ln)
            out_s.append(tr)
            out_t.append([lo, hi])
            out_xy.append(xy)
    return (np.array(out_m, np.int32), np.array(out_s, np.int32), np.array(out_t, np.float64).reshape(-1, 2),
            np.array(out_xy, np.float64).reshape(-1, 2, 2))


def mortar_desc(method, sigma, master, slave, master_t, slave_xy):
    """mh_mortar_desc over numpy arrays (keep the returned arrays alive while it is used)."""
    keep = (np.ascontiguousarray(master, np.int32), np.ascontiguousarray(slave, np.int32),
            np.ascontiguousarray(master_t, np.float64).reshape(-1), np.ascontiguousarray(slave_xy, np.float64).reshape(-1))
    d = _lib.MortarDesc()
    d.method = int(method)
    d.sigma = float(sigma)
    d.n = len(keep[0])
    d.master = _lib.ptr(keep[0], C.c_int32)
    d.slave = _lib.ptr(keep[1], C.c_int32)
    d.master_t = _lib.ptr(keep[2], C.c_double)
    d.slave_xy = _lib.ptr(keep[3], C.c_double)
    return d, keep

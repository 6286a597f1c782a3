"""Locally refined hexahedral meshes in the ingestion form of
`MappedMesh` (mpdg_mesh_create_mapped).

`refine_box` refines a set of cells of a structured hexahedral mesh once,
isotropically (8 children through the parent's trilinear map), and returns
the cells' corners, their cell->DoF maps and the hanging-node constraints
that deal.II's DoFTools::make_hanging_node_constraints would produce on such
a mesh (utilities/constraints.hpp:117-135, after refinement by
utilities/amr.hpp:55).  One refinement level keeps the mesh 2:1 balanced.

DoFs are identified by position: a node shared by cells is one DoF.  A node of
a refined cell that lies on a face or an edge of an unrefined neighbour, and is
not one of that neighbour's own nodes, hangs: its value is the neighbour's
FE_Q(p) interpolant at that point, a combination of the neighbour's face or
edge DoFs with the weights of its Gauss-Lobatto Lagrange basis.
"""
from __future__ import annotations

import itertools

import numpy as np


def gauss_lobatto(n):
    """Gauss-Lobatto nodes on [0,1] (the roots of P'_{n-1} and the end points)."""
    if n == 2:
        return np.array([0.0, 1.0])
    m = n - 1
    c = np.zeros(m + 1)
    c[m] = 1.0
    roots = np.polynomial.legendre.legroots(np.polynomial.legendre.legder(c))
    return np.concatenate([[0.0], 0.5 * (np.sort(roots) + 1.0), [1.0]])


def lagrange(z, x):
    """Values of the Lagrange basis on nodes z at the point x."""
    v = np.ones(len(z))
    for i in range(len(z)):
        for k in range(len(z)):
            if k != i:
                v[i] *= (x - z[k]) / (z[i] - z[k])
    return v


def _trilinear(corners, xi):
    x = np.zeros(3)
    for v in range(8):
        b = [(v >> d) & 1 for d in range(3)]
        w = np.prod([xi[d] if b[d] else 1.0 - xi[d] for d in range(3)])
        x += w * corners[v]
    return x


def refine_box(nc, degree, refine, vertices=None, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    """Refines the cells `refine` (lexicographic indices ix + nc0 (iy + nc1 iz))
    of an nc[0] x nc[1] x nc[2] mesh once.  `vertices` ((nc+1)^3 x 3, x fastest)
    default to the box [lo, hi].  Returns a dict with cell_vertices (E x 8 x 3),
    cell_dofs (E x n^3), n_dofs, constraints {dof: [(master, weight)]},
    coordinates (n_dofs x 3) and boundary (uint8 mask of the box faces)."""
    nc = tuple(int(v) for v in nc)
    p, n = int(degree), int(degree) + 1
    if vertices is None:
        ax = [np.linspace(lo[d], hi[d], nc[d] + 1) for d in range(3)]
        Z, Y, X = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
        vertices = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    V = np.asarray(vertices, np.float64).reshape(nc[2] + 1, nc[1] + 1, nc[0] + 1, 3)
    refine = set(int(c) for c in refine)
    z = gauss_lobatto(n)
    scale = np.max(np.abs(V)) + 1.0

    def cid(ix, iy, iz):
        return ix + nc[0] * (iy + nc[1] * iz)

    def corners_of(ix, iy, iz):
        return np.array([V[iz + (v >> 2 & 1), iy + (v >> 1 & 1), ix + (v & 1)] for v in range(8)])

    keys = {}
    coords = []

    def dof_at(x):
        k = tuple(np.round(x / scale * 1e9).astype(np.int64))
        if k not in keys:
            keys[k] = len(coords)
            coords.append(x)
        return keys[k]

    cells, cverts, cref = [], [], []   # cref: (parent ix, iy, iz, child offset or None)
    local = [(i, j, k) for k in range(n) for j in range(n) for i in range(n)]
    for iz, iy, ix in itertools.product(range(nc[2]), range(nc[1]), range(nc[0])):
        C = corners_of(ix, iy, iz)
        if cid(ix, iy, iz) not in refine:
            cverts.append(C)
            cells.append([dof_at(_trilinear(C, (z[i], z[j], z[k]))) for i, j, k in local])
            cref.append((ix, iy, iz, None))
            continue
        for off in itertools.product((0, 1), repeat=3):  # (ox, oy, oz)
            ref_c = [0.5 * (np.array(off) + np.array([(v >> d) & 1 for d in range(3)])) for v in range(8)]
            cc = np.array([_trilinear(C, r) for r in ref_c])
            cverts.append(cc)
            cells.append([dof_at(_trilinear(C, 0.5 * (np.array(off) + np.array([z[i], z[j], z[k]]))))
                          for i, j, k in local])
            cref.append((ix, iy, iz, off))
    coords = np.array(coords)
    # hanging nodes: nodes of children on the boundary of an unrefined neighbour
    unref_nodes = {}
    for e, (ix, iy, iz, off) in enumerate(cref):
        if off is None:
            unref_nodes[(ix, iy, iz)] = set(cells[e])
    unref_cell = {(ix, iy, iz): e for e, (ix, iy, iz, off) in enumerate(cref) if off is None}
    constraints = {}
    for e, (ix, iy, iz, off) in enumerate(cref):
        if off is None:
            continue
        for t, (i, j, k) in enumerate(local):
            g = cells[e][t]
            if g in constraints:
                continue
            xi = 0.5 * (np.array(off) + np.array([z[i], z[j], z[k]]))  # in the parent's reference cube
            for d in itertools.product((-1, 0, 1), repeat=3):
                if d == (0, 0, 0):
                    continue
                nb = (ix + d[0], iy + d[1], iz + d[2])
                if nb not in unref_cell:
                    continue
                xu = xi - np.array(d, dtype=float)
                if np.any(xu < -1e-12) or np.any(xu > 1 + 1e-12):
                    continue
                if g in unref_nodes[nb]:
                    break  # a node of the neighbour itself: not hanging
                xu = np.clip(xu, 0.0, 1.0)
                lx, ly, lz = lagrange(z, xu[0]), lagrange(z, xu[1]), lagrange(z, xu[2])
                eu = unref_cell[nb]
                ent = []
                for tu, (a, b, c) in enumerate(local):
                    w = lx[a] * ly[b] * lz[c]
                    if abs(w) > 1e-13:
                        ent.append((cells[eu][tu], float(w)))
                constraints[g] = ent
                break
    gmin, gmax = V.reshape(-1, 3).min(axis=0), V.reshape(-1, 3).max(axis=0)
    tol = 1e-9 * scale
    boundary = np.any((np.abs(coords - gmin) < tol) | (np.abs(coords - gmax) < tol), axis=1).astype(np.uint8)
    return dict(cell_vertices=np.array(cverts), cell_dofs=np.array(cells, np.int64), n_dofs=len(coords),
                constraints=constraints, coordinates=coords, boundary=boundary)

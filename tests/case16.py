"""Restatement of the reference's case-16 system builder (test helper).

verification/case16_preconditioner.py:23-97 (_build_convdiff_system): 2D
convection-diffusion u dT/dx - gamma lap T = 0 on a channel mesh, harmonic-free
constant gamma, upwind convection with F = u A n_x, Dirichlet inlet (T=1) and walls
(T=0), zero-gradient outlet. Entries are appended in the reference's order so
scipy's coo->csr gives the same CSR.
"""
import numpy as np
from scipy import sparse

from kcfd import meshgen
from oracle import mesh as om


def channel_mesh(nx, ny, L=1.0, H=1.0):
    nodes, cells, bd = meshgen.quad_box_arrays(0.0, 0.0, L, H, nx, ny, meshgen.CHANNEL_2D_NAMES)
    return om.build_2d(nodes, cells, bd)


def convdiff_system(m, gamma_val=0.01, u_conv=1.0):
    n = m.n_cells
    dval = {}
    for bname, phi_b in (("inlet", 1.0), ("wall_bottom", 0.0), ("wall_top", 0.0)):
        for fid in m.boundary_patches.get(bname, []):
            dval[int(fid)] = phi_b
    rows, cols, vals = [], [], []
    rhs = np.zeros(n)
    for fid in range(m.n_faces):
        o = int(m.owner[fid])
        nx_dir = m.normal[fid, 0]
        nb = int(m.neighbour[fid])
        if nb >= 0:
            d = float(np.linalg.norm(m.ccenter[nb] - m.ccenter[o]))
            if d < 1e-30:
                continue
            dc = gamma_val * m.area[fid] / d
            F = u_conv * m.area[fid] * nx_dir
            rows += [o, nb, o, nb, o, o, nb, nb]
            cols += [o, nb, nb, o, o, nb, nb, o]
            vals += [dc, dc, -dc, -dc, max(F, 0.0), min(F, 0.0), max(-F, 0.0), min(-F, 0.0)]
        elif fid in dval:
            d = float(np.linalg.norm(m.fcenter[fid] - m.ccenter[o]))
            if d < 1e-30:
                continue
            dc = gamma_val * m.area[fid] / d
            rows.append(o); cols.append(o); vals.append(dc)
            rhs[o] += dc * dval[fid]
            F = u_conv * m.area[fid] * nx_dir
            if F >= 0:
                rows.append(o); cols.append(o); vals.append(F)
            else:
                rhs[o] += -F * dval[fid]
        else:
            F = u_conv * m.area[fid] * nx_dir
            if F >= 0:
                rows.append(o); cols.append(o); vals.append(F)
    A = sparse.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsr()
    return A, rhs

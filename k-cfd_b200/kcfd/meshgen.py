"""Mesh generators: node / cell / face-node arrays fed to the face-connectivity builder.

The structured generators produce exactly the arrays of the reference generators
(node numbering, cell order, per-cell face node order, boundary dict order):
  * quad_box_arrays      -- mesh/mesh_generator.py:13-93 (_make_structured_quad_mesh)
  * tri_channel_arrays   -- mesh/mesh_generator.py:266-325
  * hex_box_arrays       -- mesh/mesh_generator_3d.py:12-159 (generate_3d_channel_mesh)
Synthetic generators for the workloads the reference has no generator for:
  * jitter_interior      -- interior nodes displaced by U(-a, a) x spacing (seeded)
  * delaunay_tri_arrays  -- Delaunay triangulation of uniform random points
  * delaunay_tet_arrays  -- Delaunay tetrahedralisation of a jittered lattice
Everything here is vectorised numpy; the meshes are built from these arrays by
kcfd.mesh.build_mesh (native face discovery).

The reference's named generators return a kcfd Mesh built from the same arrays:
generate_channel_mesh, generate_cavity_mesh, generate_bubble_column_mesh,
generate_triangle_channel_mesh (mesh/mesh_generator.py:96-128,232-325),
generate_3d_channel_mesh, generate_3d_duct_mesh, generate_3d_cavity_mesh
(mesh/mesh_generator_3d.py:12-206).
"""
from __future__ import annotations

import numpy as np

CAVITY_2D_NAMES = {"bottom": "wall_bottom", "top": "lid", "left": "wall_left", "right": "wall_right"}
CHANNEL_2D_NAMES = {"bottom": "wall_bottom", "top": "wall_top", "left": "inlet", "right": "outlet"}
CAVITY_3D_NAMES = {"x_min": "wall_left", "x_max": "wall_right", "y_min": "wall_bottom",
                   "y_max": "lid", "z_min": "wall_front", "z_max": "wall_back"}
CHANNEL_3D_NAMES = {"x_min": "inlet", "x_max": "outlet", "y_min": "wall_bottom",
                    "y_max": "wall_top", "z_min": "wall_front", "z_max": "wall_back"}


def quad_box_arrays(x0, y0, x1, y1, nx, ny, names=None):
    """Structured quads; cells [n0,n1,n2,n3] counter-clockwise, j-major."""
    names = names or {"bottom": "bottom", "top": "top", "left": "left", "right": "right"}
    dx = (x1 - x0) / nx
    dy = (y1 - y0) / ny
    j, i = np.meshgrid(np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    nodes = np.stack([x0 + i.reshape(-1) * dx, y0 + j.reshape(-1) * dy], axis=1)
    jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    n0 = (jj * (nx + 1) + ii).reshape(-1)
    cells = np.stack([n0, n0 + 1, n0 + 1 + (nx + 1), n0 + (nx + 1)], axis=1)
    ar = np.arange(nx)
    bd = {}
    bd[names.get("bottom", "bottom")] = list(np.stack([ar, ar + 1], 1))
    top0 = ny * (nx + 1) + ar
    bd[names.get("top", "top")] = list(np.stack([top0, top0 + 1], 1))
    aj = np.arange(ny)
    bd[names.get("left", "left")] = list(np.stack([aj * (nx + 1), (aj + 1) * (nx + 1)], 1))
    bd[names.get("right", "right")] = list(np.stack([aj * (nx + 1) + nx, (aj + 1) * (nx + 1) + nx], 1))
    return nodes, cells, bd


def tri_channel_arrays(Lx, Ly, nx, ny):
    """Quads split along n0-n2 into (n0,n1,n2) and (n0,n2,n3)."""
    def nid(i, j):
        return j * (nx + 1) + i
    dx, dy = Lx / nx, Ly / ny
    j, i = np.meshgrid(np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    nodes = np.stack([i.reshape(-1) * dx, j.reshape(-1) * dy], axis=1)
    jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    jj, ii = jj.reshape(-1), ii.reshape(-1)
    n0, n1, n2, n3 = nid(ii, jj), nid(ii + 1, jj), nid(ii + 1, jj + 1), nid(ii, jj + 1)
    cells = np.stack([np.stack([n0, n1, n2], 1), np.stack([n0, n2, n3], 1)], axis=1).reshape(-1, 3)
    aj, ai = np.arange(ny), np.arange(nx)
    bd = {"inlet": list(np.stack([nid(0, aj), nid(0, aj + 1)], 1)),
          "outlet": list(np.stack([nid(nx, aj), nid(nx, aj + 1)], 1)),
          "wall_bottom": list(np.stack([nid(ai, 0), nid(ai + 1, 0)], 1)),
          "wall_top": list(np.stack([nid(ai, ny), nid(ai + 1, ny)], 1))}
    return nodes, cells, bd


# corners of each hex face, in the reference's face order and node order
HEX_FACE_CORNERS = np.array([[0, 3, 2, 1], [4, 5, 6, 7], [0, 1, 5, 4], [2, 3, 7, 6], [0, 4, 7, 3], [1, 2, 6, 5]])


def hex_box_arrays(Lx, Ly, Lz, nx, ny, nz, names=None):
    """Structured hexes (k, j, i order), six faces per cell in the reference order."""
    names = names or CHANNEL_3D_NAMES
    dx, dy, dz = Lx / nx, Ly / ny, Lz / nz

    def nid(i, j, k):
        return k * (ny + 1) * (nx + 1) + j * (nx + 1) + i

    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    nodes = np.stack([i.reshape(-1) * dx, j.reshape(-1) * dy, k.reshape(-1) * dz], axis=1)
    # cell (i, j, k) -> its corner n0 = nid(i, j, k); corners n0..n7 are fixed offsets from it
    base = nid(*np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")).transpose(2, 1, 0).reshape(-1)
    row, plane = nx + 1, (nx + 1) * (ny + 1)
    corner = np.array([0, 1, 1 + row, row, plane, plane + 1, plane + 1 + row, plane + row], dtype=np.int64)
    cells = base[:, None] + corner[None, :]
    # faces in the reference's order: z-, z+, y-, y+, x-, x+ (node lists as above)
    cfaces = base[:, None, None] + corner[HEX_FACE_CORNERS][None, :, :]
    bd = {}
    K, J = (a.reshape(-1) for a in np.meshgrid(np.arange(nz), np.arange(ny), indexing="ij"))
    bd[names.get("x_min", "inlet")] = np.stack([nid(0, J, K), nid(0, J, K + 1), nid(0, J + 1, K + 1), nid(0, J + 1, K)], 1)
    bd[names.get("x_max", "outlet")] = np.stack([nid(nx, J, K), nid(nx, J + 1, K), nid(nx, J + 1, K + 1), nid(nx, J, K + 1)], 1)
    K, I = (a.reshape(-1) for a in np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij"))
    bd[names.get("y_min", "wall_bottom")] = np.stack([nid(I, 0, K), nid(I + 1, 0, K), nid(I + 1, 0, K + 1), nid(I, 0, K + 1)], 1)
    bd[names.get("y_max", "wall_top")] = np.stack([nid(I + 1, ny, K), nid(I, ny, K), nid(I, ny, K + 1), nid(I + 1, ny, K + 1)], 1)
    J, I = (a.reshape(-1) for a in np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij"))
    bd[names.get("z_min", "wall_front")] = np.stack([nid(I, J, 0), nid(I, J + 1, 0), nid(I + 1, J + 1, 0), nid(I + 1, J, 0)], 1)
    bd[names.get("z_max", "wall_back")] = np.stack([nid(I, J, nz), nid(I + 1, J, nz), nid(I + 1, J + 1, nz), nid(I, J + 1, nz)], 1)
    return nodes, cells, cfaces, bd


def jitter_interior(nodes, shape, spacing, amp=0.2, seed=0):
    """Displace nodes not on any boundary plane by U(-amp, amp) x spacing per axis.

    shape = (nx, ny[, nz]) cell counts; nodes are numbered i fastest. The draw covers
    every node (rng.uniform(-amp, amp, (n_nodes, ndim))) so the field is a function of
    the seed and the lattice only.
    """
    ndim = len(shape)
    rng = np.random.default_rng(seed)
    disp = rng.uniform(-amp, amp, (len(nodes), ndim)) * np.asarray(spacing)[None, :]
    grids = np.meshgrid(*[np.arange(s + 1) for s in reversed(shape)], indexing="ij")
    idx = [g.reshape(-1) for g in reversed(grids)]  # i, j, k per node
    interior = np.ones(len(nodes), dtype=bool)
    for a, s in zip(idx, shape):
        interior &= (a > 0) & (a < s)
    out = nodes.copy()
    out[interior] += disp[interior]
    return out


def _morton_order(pts):
    """Cell order along a Morton curve of the centroids (locality for gathers)."""
    lo, hi = pts.min(0), pts.max(0)
    q = ((pts - lo) / np.maximum(hi - lo, 1e-300) * 1023.0).astype(np.int64)
    code = np.zeros(len(pts), dtype=np.int64)
    for bit in range(10):
        for d in range(pts.shape[1]):
            code |= ((q[:, d] >> bit) & 1) << (bit * pts.shape[1] + d)
    return np.argsort(code, kind="stable")


def delaunay_tri_arrays(n_points, rng, dirichlet_name="dirichlet", wall_name="wall", side_points=0):
    """Delaunay triangles of n_points uniform points in the unit square plus its corners.

    Cells are ordered along a Morton curve of their centroids. Boundary edges are
    the convex hull; hull edges whose midpoint has x < 1e-9 form the Dirichlet
    segment, the rest the wall patch. With corners alone the hull is the square's
    four sides, each one long edge under a sliver triangle; side_points > 0 puts that
    many equally spaced points inside each side, so every side is a chain of
    side_points + 1 edges.
    """
    from scipy.spatial import Delaunay
    extra = np.zeros((0, 2))
    if side_points > 0:
        t = np.arange(1, side_points + 1) / (side_points + 1.0)
        z, o = np.zeros_like(t), np.ones_like(t)
        extra = np.vstack([np.stack([t, z], 1), np.stack([o, t], 1), np.stack([t, o], 1), np.stack([z, t], 1)])
    pts = np.vstack([rng.uniform(0.0, 1.0, (n_points, 2)), [[0, 0], [1, 0], [1, 1], [0, 1]], extra])
    tri = Delaunay(pts)
    cells = tri.simplices.astype(np.int64)
    order = _morton_order(pts[cells].mean(axis=1))
    cells = cells[order]
    hull = tri.convex_hull.astype(np.int64)
    mid_x = pts[hull].mean(axis=1)[:, 0]
    left = mid_x < 1e-9
    bd = {dirichlet_name: list(hull[left]), wall_name: list(hull[~left])}
    return pts, cells, bd


def delaunay_tet_arrays(box, n_target, rng, jitter=0.25):
    """Delaunay tetrahedra of a jittered lattice in box = (Lx, Ly, Lz).

    The lattice is chosen so that the tetrahedralisation has about n_target cells: a
    Delaunay mesh of this jittered lattice has 6.35 tets per point (measured: 1,219,253
    tets on 34 x 34 x 166 points), and the lattice counts follow the box's aspect, the
    x count being the one whose predicted total is nearest n_target.
    Face node lists follow the reference's tet face order (_tet_faces in
    mesh/hybrid_mesh_generator.py:64-72); cells are ordered along a Morton curve.
    Boundary faces are the convex hull, tagged by face-centroid position: bottom
    (z = 0) 'inlet_gas', top (z = Lz) 'outlet', the rest 'wall'.
    """
    from scipy.spatial import Delaunay
    Lx, Ly, Lz = box
    best = None
    for nx in range(2, 4096):
        ny, nz = max(2, round(nx * Ly / Lx)), max(2, round(nx * Lz / Lx))
        pred = 6.35 * (nx + 1) * (ny + 1) * (nz + 1)
        if best is None or abs(pred - n_target) < best[0]:
            best = (abs(pred - n_target), nx, ny, nz)
        if pred > 2 * n_target:
            break
    _, nx, ny, nz = best
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    sp = np.array([Lx / nx, Ly / ny, Lz / nz])
    pts = np.stack([i.reshape(-1) * sp[0], j.reshape(-1) * sp[1], k.reshape(-1) * sp[2]], axis=1)
    pts = jitter_interior(pts, (nx, ny, nz), sp, amp=jitter, seed=int(rng.integers(0, 2**31)))
    tet = Delaunay(pts, qhull_options="Qbb Qc Qz Q12")
    cells = tet.simplices.astype(np.int64)
    # drop slivers of (near) zero volume that Qhull can leave on a lattice
    p = pts[cells]
    v6 = np.abs(np.einsum("ij,ij->i", p[:, 1] - p[:, 0], np.cross(p[:, 2] - p[:, 0], p[:, 3] - p[:, 0])))
    cells = cells[v6 > 1e-12 * sp.prod()]
    order = _morton_order(pts[cells].mean(axis=1))
    cells = cells[order]
    n0, n1, n2, n3 = cells[:, 0], cells[:, 1], cells[:, 2], cells[:, 3]
    cfaces = np.stack([np.stack([n0, n2, n1], 1), np.stack([n0, n1, n3], 1),
                       np.stack([n1, n2, n3], 1), np.stack([n0, n3, n2], 1)], axis=1)
    # boundary = faces used once
    allf = np.sort(cfaces.reshape(-1, 3), axis=1)
    key = (allf[:, 0] * (len(pts) + 1) + allf[:, 1]) * (len(pts) + 1) + allf[:, 2]
    uk, inv, cnt = np.unique(key, return_inverse=True, return_counts=True)
    once = cnt[inv] == 1
    bf = cfaces.reshape(-1, 3)[once]
    zc = pts[bf][:, :, 2].mean(axis=1)
    bd = {"inlet_gas": list(bf[zc < 1e-9 * Lz + 1e-12]), "outlet": list(bf[zc > Lz * (1 - 1e-9) - 1e-12])}
    rest = ~((zc < 1e-9 * Lz + 1e-12) | (zc > Lz * (1 - 1e-9) - 1e-12))
    bd["wall"] = list(bf[rest])
    return pts, cells, cfaces, bd


# ------------------------------------------------- the reference's named generators --
def _build(nodes, cells, bd, cf=None):
    from .mesh import build_mesh
    return build_mesh(nodes, cells, bd, ndim=3 if cf is not None else 2, cell_face_node_list=cf)


def generate_channel_mesh(length=1.0, height=0.1, nx=50, ny=20):
    """mesh/mesh_generator.py:96-110: inlet (left), outlet (right), wall_bottom, wall_top."""
    return _build(*quad_box_arrays(0.0, 0.0, length, height, nx, ny, CHANNEL_2D_NAMES))


def generate_cavity_mesh(size=1.0, n=64):
    """mesh/mesh_generator.py:113-126: lid (top), wall_bottom, wall_left, wall_right."""
    return _build(*quad_box_arrays(0.0, 0.0, size, size, n, n, CAVITY_2D_NAMES))


def generate_bubble_column_mesh(width=0.15, height=0.45, nx=30, ny=90):
    """mesh/mesh_generator.py:232-263: the bottom split into inlet_gas (faces whose
    centre x lies in [width/3, 2 width/3]) and wall_bottom, after outlet (top),
    wall_left and wall_right."""
    return _build(*bubble_column_arrays(width, height, nx, ny))


def bubble_column_arrays(width=0.15, height=0.45, nx=30, ny=90):
    """Nodes, cells and boundary dict of generate_bubble_column_mesh."""
    nodes, cells, bd = quad_box_arrays(0.0, 0.0, width, height, nx, ny,
                                       {"bottom": "_bottom", "top": "outlet", "left": "wall_left",
                                        "right": "wall_right"})
    bottom = np.asarray(bd.pop("_bottom"))
    xc = 0.5 * (nodes[bottom[:, 0], 0] + nodes[bottom[:, 1], 0])
    inlet = (width / 3.0 <= xc) & (xc <= 2.0 * width / 3.0)
    bd["inlet_gas"] = list(bottom[inlet])
    bd["wall_bottom"] = list(bottom[~inlet])
    return nodes, cells, bd


def generate_triangle_channel_mesh(Lx=1.0, Ly=0.1, nx=20, ny=5):
    """mesh/mesh_generator.py:266-325."""
    return _build(*tri_channel_arrays(Lx, Ly, nx, ny))


def generate_3d_channel_mesh(Lx=1.0, Ly=0.1, Lz=0.1, nx=20, ny=10, nz=10, boundary_names=None):
    """mesh/mesh_generator_3d.py:12-159 (default names: inlet, outlet, wall_bottom,
    wall_top, wall_front, wall_back)."""
    nodes, cells, cf, bd = hex_box_arrays(Lx, Ly, Lz, nx, ny, nz, boundary_names or CHANNEL_3D_NAMES)
    return _build(nodes, cells, bd, cf)


def generate_3d_duct_mesh(Lx=2.0, Ly=0.1, Lz=0.1, nx=20, ny=10, nz=10):
    """mesh/mesh_generator_3d.py:162-178."""
    return generate_3d_channel_mesh(Lx, Ly, Lz, nx, ny, nz, CHANNEL_3D_NAMES)


def generate_3d_cavity_mesh(Lx=1.0, Ly=1.0, Lz=1.0, nx=16, ny=16, nz=16):
    """mesh/mesh_generator_3d.py:181-206: lid (y = Ly), walls elsewhere."""
    return generate_3d_channel_mesh(Lx, Ly, Lz, nx, ny, nz, CAVITY_3D_NAMES)


def _split_quad(q):
    """Two triangles of a quad (a, b, c, d), cut on the diagonal through its smallest
    node id, so that the two cells sharing the quad cut it the same way."""
    a, b, c, d = (int(v) for v in q)
    if min(a, b, c, d) in (a, c):
        return [(a, b, c), (a, c, d)]
    return [(a, b, d), (b, c, d)]


def _hex_quads(h):
    """The six faces of a hex (n0..n7), outward, in the order z-, z+, y-, y+, x-, x+."""
    n0, n1, n2, n3, n4, n5, n6, n7 = (int(v) for v in h)
    return [(n0, n3, n2, n1), (n4, n5, n6, n7), (n0, n1, n5, n4), (n2, n3, n7, n6), (n0, n4, n7, n3),
            (n1, n2, n6, n5)]


def _tet_tris(t):
    n0, n1, n2, n3 = (int(v) for v in t)
    return [(n0, n2, n1), (n0, n1, n3), (n1, n2, n3), (n0, n3, n2)]


def hybrid_hex_tet_arrays(Lx=2.0, Ly=0.1, Lz=0.1, nx=20, ny=8, nz=8, tet_fraction=0.5, boundary_names=None):
    """mesh/hybrid_mesh_generator.py:93-260: hexes on the low-x side, and on the
    high-x side every hex replaced by 12 tets around an added centre node (each hex
    face cut by _split_quad, each triangle joined to the centre); the last hex column
    carries its x+ face as the two triangles its tet neighbours see. Boundary faces
    are the faces of one cell only (none through a centre node), each given to the
    first box plane (x_min, x_max, y_min, y_max, z_min, z_max) holding all its
    nodes, in the order the cells list them."""
    names = boundary_names or CHANNEL_3D_NAMES
    dx, dy, dz = Lx / nx, Ly / ny, Lz / nz
    nx_hex = max(1, int(nx * (1.0 - tet_fraction)))
    nx_tet = nx - nx_hex
    base = (nx + 1) * (ny + 1) * (nz + 1)

    def nid(i, j, k):
        return k * (ny + 1) * (nx + 1) + j * (nx + 1) + i

    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    lattice = np.stack([i.reshape(-1) * dx, j.reshape(-1) * dy, k.reshape(-1) * dz], axis=1)
    kc, jc, ic = (a.reshape(-1) for a in np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx_hex, nx),
                                                      indexing="ij"))
    centres = np.stack([(ic + 0.5) * dx, (jc + 0.5) * dy, (kc + 0.5) * dz], axis=1)
    nodes = np.concatenate([lattice, centres]) if len(centres) else lattice
    centre_of = {(int(a), int(b), int(c)): base + q for q, (a, b, c) in enumerate(zip(ic, jc, kc))}
    tol = 1e-10
    x, y, z = lattice[:, 0], lattice[:, 1], lattice[:, 2]
    planes = [("x_min", np.abs(x) < tol), ("x_max", np.abs(x - Lx) < tol), ("y_min", np.abs(y) < tol),
              ("y_max", np.abs(y - Ly) < tol), ("z_min", np.abs(z) < tol), ("z_max", np.abs(z - Lz) < tol)]
    cells, cfaces = [], []
    for kk in range(nz):
        for jj in range(ny):
            for ii in range(nx):
                h = [nid(ii, jj, kk), nid(ii + 1, jj, kk), nid(ii + 1, jj + 1, kk), nid(ii, jj + 1, kk),
                     nid(ii, jj, kk + 1), nid(ii + 1, jj, kk + 1), nid(ii + 1, jj + 1, kk + 1), nid(ii, jj + 1, kk + 1)]
                quads = _hex_quads(h)
                if ii < nx_hex:
                    faces = quads[:5] + _split_quad(quads[5]) if (ii == nx_hex - 1 and nx_tet > 0) else quads
                    cells.append(np.array(h))
                    cfaces.append([np.array(f) for f in faces])
                else:
                    c = centre_of[(ii, jj, kk)]
                    for q in quads:
                        for tri in _split_quad(q):
                            t = (*tri, c)
                            cells.append(np.array(t))
                            cfaces.append([np.array(f) for f in _tet_tris(t)])
    count = {}
    for fl in cfaces:
        for f in fl:
            key = tuple(sorted(int(v) for v in f))
            count[key] = count.get(key, 0) + 1
    bd = {names.get(p, p): [] for p, _ in planes}
    seen = set()
    for fl in cfaces:
        for f in fl:
            key = tuple(sorted(int(v) for v in f))
            if key in seen or count[key] != 1 or max(key) >= base:
                continue
            seen.add(key)
            for p, on in planes:
                if on[list(key)].all():
                    bd.setdefault(names.get(p, p), []).append(f)
                    break
    return nodes, cells, cfaces, bd


def generate_hybrid_hex_tet_mesh(Lx=2.0, Ly=0.1, Lz=0.1, nx=20, ny=8, nz=8, tet_fraction=0.5, boundary_names=None):
    """mesh/hybrid_mesh_generator.py:93-260 (the cell zone map is not kept)."""
    nodes, cells, cf, bd = hybrid_hex_tet_arrays(Lx, Ly, Lz, nx, ny, nz, tet_fraction, boundary_names)
    return _build(nodes, cells, bd, cf)

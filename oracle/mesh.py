"""Oracle: vectorised restatement of the reference mesh builder (test infrastructure).

Follows mesh/mesh_reader.py of the reference:
  * 2D path of build_fvmesh_from_arrays (mesh_reader.py:166-242): faces are the cell
    edges (n_k, n_{k+1}) discovered cell by cell; a face id is the rank of its first
    discovery; owner = first cell, neighbour = later cell; normal (dy,-dx)/len flipped
    to point away from the owner centre (:202-206); boundary faces tagged by an edge
    lookup into the patch dict (last assignment wins, :217-222); patches are created
    in the order their first face appears in face-id order (:224-231).
  * 3D path _build_fvmesh_3d (mesh_reader.py:245-323): cell centre = node mean
    (:263), face key = sorted node tuple (:254-255), Newell normal and area
    (_compute_face_geometry_3d :81-99), divergence-theorem volume with an
    owner-outward sign test (_compute_cell_geometry_3d :116-138).
  * 2D cell geometry: node mean and shoelace area (:102-113).

Every per-element expression keeps the reference's operation order so that the
results agree bit-for-bit where numpy's elementwise arithmetic allows it; the
golden fixtures in tests/golden pin that.
"""
from __future__ import annotations

import numpy as np


class Mesh:
    """Structure-of-arrays unstructured FV mesh (same content as the reference FVMesh)."""

    def __init__(self):
        self.ndim = 2
        self.nodes = None
        self.n_cells = 0
        self.n_faces = 0
        self.n_internal_faces = 0
        self.n_boundary_faces = 0
        self.owner = None        # (F,) int64
        self.neighbour = None    # (F,) int64, -1 on boundary
        self.area = None         # (F,)
        self.normal = None       # (F, ndim) unit, owner-outward
        self.fcenter = None      # (F, ndim)
        self.face_nodes = None   # (F, kmax) padded with -1
        self.ccenter = None      # (n, ndim)
        self.volume = None       # (n,)
        self.cell_faces = None   # (n, kmax) face ids per cell in discovery order, -1 pad
        self.boundary_patches = {}  # name -> int64 array of face ids


def _ragged(cells):
    """Return (ptr, flat) for a list/array of per-cell index arrays."""
    if isinstance(cells, np.ndarray) and cells.ndim == 2:
        n, k = cells.shape
        return np.arange(0, n * k + 1, k, dtype=np.int64), cells.reshape(-1).astype(np.int64)
    lens = np.fromiter((len(c) for c in cells), dtype=np.int64, count=len(cells))
    ptr = np.zeros(len(cells) + 1, dtype=np.int64)
    np.cumsum(lens, out=ptr[1:])
    flat = np.concatenate([np.asarray(c, dtype=np.int64) for c in cells]) if len(cells) else np.zeros(0, np.int64)
    return ptr, flat


def _group_first(keys_hi, keys_lo=None):
    """Group equal keys; return (gid per item, first item per group, last item per group).

    Group ids are NOT in discovery order; callers re-rank by the first index.
    A stable sort keeps the earliest occurrence first inside each group.
    """
    if keys_lo is None:
        order = np.argsort(keys_hi, kind="stable")
        hs = keys_hi[order]
        newg = np.empty(len(order), dtype=bool)
        if len(order):
            newg[0] = True
            newg[1:] = hs[1:] != hs[:-1]
    else:
        order = np.lexsort((keys_lo, keys_hi))
        hs, ls = keys_hi[order], keys_lo[order]
        newg = np.empty(len(order), dtype=bool)
        if len(order):
            newg[0] = True
            newg[1:] = (hs[1:] != hs[:-1]) | (ls[1:] != ls[:-1])
    gsorted = np.cumsum(newg) - 1
    gid = np.empty(len(order), dtype=np.int64)
    gid[order] = gsorted
    first = order[newg]
    lastmask = np.empty_like(newg)
    if len(order):
        lastmask[:-1] = newg[1:]
        lastmask[-1] = True
    last = order[lastmask]
    return gid, first, last


def _seq_mean(pts):
    """np.mean over axis 1 of (m, k, d) with the reference's sequential order."""
    k = pts.shape[1]
    s = pts[:, 0].copy()
    for i in range(1, k):
        s = s + pts[:, i]
    return s / k


def _finish_faces(mesh, ce, gid, first, last, cells_ptr, face_node_rows, face_sizes):
    """Face ids by first discovery; owner/neighbour; per-cell face lists."""
    E = len(ce)
    order = np.argsort(first, kind="stable")
    fid_of_group = np.empty(len(first), dtype=np.int64)
    fid_of_group[order] = np.arange(len(first), dtype=np.int64)
    fid_of_item = fid_of_group[gid]
    F = len(first)
    first_sorted = first[order]
    owner = ce[first_sorted]
    neighbour = -np.ones(F, dtype=np.int64)
    notfirst = np.ones(E, dtype=bool)
    notfirst[first] = False
    # the reference overwrites neighbour at every later discovery: the last one wins
    idx = np.nonzero(notfirst)[0]
    neighbour[fid_of_item[idx]] = ce[idx]
    mesh.owner = owner
    mesh.neighbour = neighbour
    mesh.face_nodes = face_node_rows[first_sorted]
    mesh.face_sizes = face_sizes[first_sorted]
    mesh.n_faces = F
    mesh.n_internal_faces = int(np.count_nonzero(neighbour >= 0))
    mesh.n_boundary_faces = F - mesh.n_internal_faces
    # per-cell face lists in discovery order (cell.faces in the reference)
    lens = np.diff(cells_ptr)
    kmax = int(lens.max()) if len(lens) else 0
    cf = -np.ones((len(lens), kmax), dtype=np.int64)
    cell_of_item = ce
    pos = np.arange(E, dtype=np.int64) - cells_ptr[cell_of_item]
    cf[cell_of_item, pos] = fid_of_item
    mesh.cell_faces = cf
    return fid_of_item


def _tag_boundary(mesh, keyfun_faces, bkeys, bnames_per_key):
    """Patch tagging: boundary face -> patch name by key lookup, 'default' otherwise.

    The lookup table is filled in patch-dict order, so a key listed twice keeps the
    last patch name, as the reference's dict assignment does (mesh_reader.py:217-222).
    """
    bfaces = np.nonzero(mesh.neighbour < 0)[0]
    bh, bl = bkeys
    table = {}
    if bl is None:
        for k, nm in zip(bh.tolist(), bnames_per_key.tolist()):
            table[k] = nm
    else:
        for k1, k2, nm in zip(bh.tolist(), bl.tolist(), bnames_per_key.tolist()):
            table[(k1, k2)] = nm
    patches = {}
    if len(bfaces):
        fh, fl = keyfun_faces(bfaces)
        keys = fh.tolist() if fl is None else list(zip(fh.tolist(), fl.tolist()))
        for fid, k in zip(bfaces.tolist(), keys):
            patches.setdefault(table.get(k, "default"), []).append(fid)
    mesh.boundary_patches = {k: np.asarray(v, dtype=np.int64) for k, v in patches.items()}


def _flatten_bdict(boundary_faces_dict, nnodes, ndim):
    names, rows = [], []
    for bname, lst in boundary_faces_dict.items():
        for bf in lst:
            rows.append(np.asarray(bf, dtype=np.int64))
            names.append(bname)
    return names, rows


def build_2d(node_coords, cell_node_list, boundary_faces_dict):
    """Restates build_fvmesh_from_arrays, 2D path (mesh/mesh_reader.py:166-242)."""
    mesh = Mesh()
    mesh.ndim = 2
    nodes = np.array(node_coords, dtype=np.float64)
    mesh.nodes = nodes
    ptr, flat = _ragged(cell_node_list)
    n = len(ptr) - 1
    lens = np.diff(ptr)
    mesh.n_cells = n
    # 1) cell geometry (_compute_cell_geometry_2d :102-113)
    cc = np.zeros((n, 2))
    vol = np.zeros(n)
    for k in np.unique(lens):
        sel = np.nonzero(lens == k)[0]
        idx = flat[ptr[sel][:, None] + np.arange(k)[None, :]]
        pts = nodes[idx]
        cc[sel] = _seq_mean(pts)
        area = np.zeros(len(sel))
        for i in range(k):
            j = (i + 1) % k
            area = area + (pts[:, i, 0] * pts[:, j, 1] - pts[:, j, 0] * pts[:, i, 1])
        vol[sel] = np.abs(area) / 2.0
    mesh.ccenter = cc
    mesh.volume = vol
    # 2) edges in discovery order (:189-214)
    ce = np.repeat(np.arange(n, dtype=np.int64), lens)
    pos = np.arange(len(flat), dtype=np.int64) - ptr[ce]
    nxt = ptr[ce] + (pos + 1) % lens[ce]
    e0, e1 = flat, flat[nxt]
    NN = len(nodes) + 1
    keys = np.minimum(e0, e1) * NN + np.maximum(e0, e1)
    gid, first, last = _group_first(keys)
    rows = np.stack([e0, e1], axis=1)
    _finish_faces(mesh, ce, gid, first, last, ptr, rows, np.full(len(e0), 2, dtype=np.int64))
    # face geometry (_compute_face_geometry_2d :66-78), normal flip (:203-206)
    fn = mesh.face_nodes
    p0, p1 = nodes[fn[:, 0]], nodes[fn[:, 1]]
    center = 0.5 * (p0 + p1)
    dx = p1[:, 0] - p0[:, 0]
    dy = p1[:, 1] - p0[:, 1]
    length = np.sqrt(dx ** 2 + dy ** 2)
    normal = np.stack([dy, -dx], axis=1)
    ok = length > 1e-15
    normal[ok] = normal[ok] / length[ok][:, None]
    to_face = center - cc[mesh.owner]
    flip = (normal[:, 0] * to_face[:, 0] + normal[:, 1] * to_face[:, 1]) < 0
    normal[flip] = -normal[flip]
    mesh.fcenter = center
    mesh.normal = normal
    mesh.area = length
    # 3) boundary tagging (:216-231)
    names, brows = _flatten_bdict(boundary_faces_dict, len(nodes), 2)
    if brows:
        B = np.stack([r[:2] for r in brows])
        bkeys = np.minimum(B[:, 0], B[:, 1]) * NN + np.maximum(B[:, 0], B[:, 1])
    else:
        bkeys = np.zeros(0, dtype=np.int64)

    def keyfun(bf):
        a, b = fn[bf, 0], fn[bf, 1]
        return np.minimum(a, b) * NN + np.maximum(a, b), None

    _tag_boundary(mesh, keyfun, (bkeys, None), np.array(names, dtype=object))
    return mesh


def _sorted_face_keys(rows, sizes, NN):
    """Two int64 keys of the sorted node tuple of each face (padding -1 -> NN-1)."""
    r = rows.copy()
    r[r < 0] = NN - 1
    r.sort(axis=1)
    k = r.shape[1]
    if k <= 3:
        hi = r[:, 0] * NN + r[:, 1] if k >= 2 else r[:, 0]
        lo = r[:, 2] if k == 3 else np.zeros(len(r), dtype=np.int64)
    else:
        hi = r[:, 0] * NN + r[:, 1]
        lo = r[:, 2] * NN + r[:, 3]
        for j in range(4, k):  # faces with more than four nodes fold into lo
            lo = lo * NN + r[:, j]
    return hi, lo


def build_3d(node_coords, cell_node_list, cell_face_node_list, boundary_faces_dict):
    """Restates _build_fvmesh_3d (mesh/mesh_reader.py:245-323)."""
    mesh = Mesh()
    mesh.ndim = 3
    nodes = np.array(node_coords, dtype=np.float64)
    mesh.nodes = nodes
    NN = len(nodes) + 1
    cptr, cflat = _ragged(cell_node_list)
    n = len(cptr) - 1
    clens = np.diff(cptr)
    mesh.n_cells = n
    cc = np.zeros((n, 3))
    for k in np.unique(clens):
        sel = np.nonzero(clens == k)[0]
        idx = cflat[cptr[sel][:, None] + np.arange(k)[None, :]]
        cc[sel] = _seq_mean(nodes[idx])
    mesh.ccenter = cc
    # flatten the per-cell face node lists into padded rows in discovery order
    if isinstance(cell_face_node_list, np.ndarray) and cell_face_node_list.ndim == 3:
        nc, kf, kn = cell_face_node_list.shape
        rows = cell_face_node_list.reshape(nc * kf, kn).astype(np.int64)
        sizes = np.full(nc * kf, kn, dtype=np.int64)
        fptr = np.arange(0, nc * kf + 1, kf, dtype=np.int64)
    else:
        flist, fsz, fcnt = [], [], []
        for fl in cell_face_node_list:
            fcnt.append(len(fl))
            for f in fl:
                flist.append(np.asarray(f, dtype=np.int64))
                fsz.append(len(f))
        kn = max(fsz)
        rows = -np.ones((len(flist), kn), dtype=np.int64)
        for i, f in enumerate(flist):
            rows[i, :len(f)] = f
        sizes = np.asarray(fsz, dtype=np.int64)
        fptr = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(fcnt, out=fptr[1:])
    ce = np.repeat(np.arange(n, dtype=np.int64), np.diff(fptr))
    hi, lo = _sorted_face_keys(rows, sizes, NN)
    gid, first, last = _group_first(hi, lo)
    _finish_faces(mesh, ce, gid, first, last, fptr, rows, sizes)
    F = mesh.n_faces
    fn, fs = mesh.face_nodes, mesh.face_sizes
    center = np.zeros((F, 3))
    normal = np.zeros((F, 3))
    for k in np.unique(fs):
        sel = np.nonzero(fs == k)[0]
        pts = nodes[fn[sel, :k]]
        center[sel] = _seq_mean(pts)
        nx = np.zeros(len(sel)); ny = np.zeros(len(sel)); nz = np.zeros(len(sel))
        for i in range(k):
            j = (i + 1) % k
            nx = nx + (pts[:, i, 1] - pts[:, j, 1]) * (pts[:, i, 2] + pts[:, j, 2])
            ny = ny + (pts[:, i, 2] - pts[:, j, 2]) * (pts[:, i, 0] + pts[:, j, 0])
            nz = nz + (pts[:, i, 0] - pts[:, j, 0]) * (pts[:, i, 1] + pts[:, j, 1])
        normal[sel] = np.stack([nx, ny, nz], axis=1)
    area = np.sqrt(normal[:, 0] * normal[:, 0] + normal[:, 1] * normal[:, 1] + normal[:, 2] * normal[:, 2])
    ok = area > 1e-15
    normal[ok] = normal[ok] / area[ok][:, None]
    area = area * 0.5
    to_face = center - cc[mesh.owner]
    flip = (normal * to_face).sum(axis=1) < 0
    normal[flip] = -normal[flip]
    mesh.fcenter, mesh.normal, mesh.area = center, normal, area
    # volumes (_compute_cell_geometry_3d :116-138), faces in cell.faces order
    cf = mesh.cell_faces
    vol = np.zeros(n)
    for k in range(cf.shape[1]):
        f = cf[:, k]
        has = f >= 0
        fc, fnrm, fa = center[f[has]], normal[f[has]], area[f[has]]
        tf = fc - cc[has]
        sign = np.where((fnrm * tf).sum(axis=1) < 0, -1.0, 1.0)
        d = fc[:, 0] * fnrm[:, 0] + fc[:, 1] * fnrm[:, 1] + fc[:, 2] * fnrm[:, 2]
        vol[has] = vol[has] + sign * d * fa
    vol = np.abs(vol) / 3.0
    vol[vol < 1e-30] = 1e-30
    mesh.volume = vol
    names, brows = _flatten_bdict(boundary_faces_dict, len(nodes), 3)
    # a boundary face longer than every cell face can never match one: drop it
    keep = [i for i, r in enumerate(brows) if len(r) <= rows.shape[1]]
    if keep:
        B = -np.ones((len(keep), rows.shape[1]), dtype=np.int64)
        for i, j in enumerate(keep):
            B[i, :len(brows[j])] = brows[j]
        bh, bl = _sorted_face_keys(B, None, NN)
        names = [names[j] for j in keep]
    else:
        bh = bl = np.zeros(0, dtype=np.int64)
        names = []

    def keyfun(bf):
        return _sorted_face_keys(fn[bf], None, NN)

    _tag_boundary(mesh, keyfun, (bh, bl), np.array(names, dtype=object))
    return mesh


def build(node_coords, cell_node_list, boundary_faces_dict, ndim=2, cell_face_node_list=None):
    """Dispatch like build_fvmesh_from_arrays (mesh/mesh_reader.py:141-171)."""
    if ndim == 3 and cell_face_node_list is not None:
        return build_3d(node_coords, cell_node_list, cell_face_node_list, boundary_faces_dict)
    return build_2d(node_coords, cell_node_list, boundary_faces_dict)


def csr_pattern(mesh):
    """Canonical CSR pattern of an FVM matrix on this mesh: diagonal + both sides of
    every internal face, duplicates merged, columns sorted (scipy coo->csr)."""
    n = mesh.n_cells
    internal = mesh.neighbour >= 0
    o, nb = mesh.owner[internal], mesh.neighbour[internal]
    rows = np.concatenate([np.arange(n), o, nb])
    cols = np.concatenate([np.arange(n), nb, o])
    key = np.unique(rows * n + cols)
    r, c = key // n, key % n
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(r, minlength=n), out=indptr[1:])
    return indptr.astype(np.int32), c.astype(np.int32)

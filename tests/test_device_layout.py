"""Device face layout (kcfd_mesh_device_layout via kcfd.device_mesh.device_layout) on the
host: every array the device mesh uploads equals, bit for bit, the numpy statement of the
same layout below (faces sorted stably by colour; gathers; gc = dN/(dO+dN),
dlen = |d_PN| or |x_f - x_P|, dorth = max(|d_PN . n|, 0.1 |d_PN|) as in
models/single_phase.py:166-175,197,380-388; per-cell faces in ascending reference id).
No device call."""
import numpy as np
import pytest

from conftest import golden_inputs, load_golden
from kcfd import mesh as km, meshgen
from kcfd.device_mesh import device_layout


def _norm_rows(v):
    return np.sqrt((v * v).sum(axis=1))


def numpy_layout(mesh):
    F, Fi = mesh.n_faces, mesh.n_internal_faces
    col = mesh.face_color.astype(np.int64)
    order = np.lexsort((np.arange(F), col))
    nc = mesh.n_int_colors + mesh.n_bnd_colors
    color_ptr = np.searchsorted(col[order], np.arange(nc + 1)).astype(np.int32)
    o = mesh.owner[order]
    nb = mesh.neighbour[order][:Fi]
    cc = mesh.ccenter
    fc = mesh.fcenter[order]
    nrm = mesh.normal[order]
    nb_full = np.concatenate([nb, o[Fi:]])
    dvec = cc[nb_full] - cc[o]
    d_int = _norm_rows(dvec[:Fi])
    d_bnd = _norm_rows(fc[Fi:] - cc[o[Fi:]])
    dn = (dvec[:Fi] * nrm[:Fi]).sum(axis=1)
    dorth = np.maximum(np.abs(dn), 0.1 * d_int)
    dO = _norm_rows(fc[:Fi] - cc[o[:Fi]])
    dN = _norm_rows(fc[:Fi] - cc[nb])
    t = dO + dN
    gc = np.where(t > 1e-30, dN / np.where(t > 1e-30, t, 1.0), 0.5)
    dev_of_ref = np.empty(F, dtype=np.int64)
    dev_of_ref[order] = np.arange(F)
    cf = np.sort(np.where(mesh.cell_faces >= 0, mesh.cell_faces, np.iinfo(np.int64).max), axis=1)
    valid = cf != np.iinfo(np.int64).max
    cf_ptr = np.concatenate([[0], np.cumsum(valid.sum(axis=1))])
    return {"order": order, "color_ptr": color_ptr, "owner": o.astype(np.int32), "neigh": nb.astype(np.int32),
            "area": mesh.area[order], "normal": nrm, "fcenter": fc, "gc": gc,
            "dlen": np.concatenate([d_int, d_bnd]), "dorth": dorth,
            "slot_on": mesh.slot_on[order][:Fi], "slot_no": mesh.slot_no[order][:Fi],
            "cf_ptr": cf_ptr.astype(np.int32), "cf_face": dev_of_ref[cf[valid]].astype(np.int32)}


def _meshes():
    out = []
    for name in ["quad", "cavity", "tri", "hex", "hybrid"]:
        d = load_golden("mesh_" + name)
        nodes, cells, bd, cfl = golden_inputs(d)
        out.append(("fixture_" + name, lambda a=(nodes, cells, bd, int(d["ndim"]), cfl):
                    km.build_mesh(a[0], a[1], a[2], ndim=a[3], cell_face_node_list=a[4])))
    out.append(("quad_97x61", lambda: km.build_mesh(*meshgen.quad_box_arrays(0, 0, 1, 0.7, 97, 61))))
    out.append(("delaunay_tri", lambda: km.build_mesh(*meshgen.delaunay_tri_arrays(3000, np.random.default_rng(2)))))

    def jittered_hex():
        n, c, f, b = meshgen.hex_box_arrays(1, 1, 1, 23, 19, 17, meshgen.CAVITY_3D_NAMES)
        n = meshgen.jitter_interior(n, (23, 19, 17), (1 / 23, 1 / 19, 1 / 17), 0.2, seed=4)
        return km.build_mesh(n, c, b, ndim=3, cell_face_node_list=f)

    def tets():
        n, c, f, b = meshgen.delaunay_tet_arrays((0.2, 0.2, 1.0), 20000, np.random.default_rng(1))
        return km.build_mesh(n, c, b, ndim=3, cell_face_node_list=f)

    def hybrid():
        n, c, f, b = meshgen.hybrid_hex_tet_arrays(nx=14, ny=6, nz=5)
        return km.build_mesh(n, c, b, ndim=3, cell_face_node_list=f)

    out += [("jittered_hex", jittered_hex), ("delaunay_tets", tets), ("hybrid", hybrid)]
    return out


@pytest.mark.parametrize("name,make", _meshes(), ids=[m[0] for m in _meshes()])
def test_layout_bitwise_equals_numpy(name, make):
    m = make()
    got, want = device_layout(m), numpy_layout(m)
    assert set(got) == set(want)
    for k in want:
        assert got[k].shape == want[k].shape, k
        assert np.array_equal(got[k].view(np.uint8), np.ascontiguousarray(want[k]).astype(got[k].dtype).view(np.uint8)), k
    Fi = m.n_internal_faces
    assert got["color_ptr"][m.n_int_colors] == Fi and got["color_ptr"][-1] == m.n_faces


def test_layout_rejects_bad_input():
    from kcfd._lib import KcfdError
    m = km.build_mesh(*meshgen.quad_box_arrays(0, 0, 1, 1, 4, 3))
    m.face_color = m.face_color.copy()
    m.face_color[0] = m.n_int_colors + m.n_bnd_colors  # colour out of range
    with pytest.raises(KcfdError, match="colour"):
        device_layout(m)
    m = km.build_mesh(*meshgen.quad_box_arrays(0, 0, 1, 1, 4, 3))
    m.face_color = m.face_color.copy()
    b = int(np.nonzero(m.neighbour < 0)[0][0])
    m.face_color[b] = 0  # a boundary face in an internal colour
    with pytest.raises(KcfdError, match="internal faces"):
        device_layout(m)

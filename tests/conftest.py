"""Shared pytest set-up: the gpu marker, import paths and golden-fixture helpers."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "k-cfd_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False)


def golden_inputs(d):
    """Rebuild the generator inputs (nodes, cells, boundary dict, cell faces) recorded
    in a mesh fixture."""
    nodes = d["in_nodes"]
    cp, cn = d["in_cell_ptr"], d["in_cell_nodes"]
    cells = [cn[cp[i]:cp[i + 1]] for i in range(len(cp) - 1)]
    names = [str(x) for x in d["in_bnames"]]
    bp, bl, bn = d["in_bptr"], d["in_bface_len"], d["in_bface_nodes"]
    boff = np.concatenate([[0], np.cumsum(bl)])
    bdict = {}
    for i, nm in enumerate(names):
        bdict[nm] = [bn[boff[j]:boff[j + 1]] for j in range(bp[i], bp[i + 1])]
    cfl = None
    if "in_cface_ptr" in d.files:
        fp, fl, fn = d["in_cface_ptr"], d["in_face_len"], d["in_face_nodes"]
        foff = np.concatenate([[0], np.cumsum(fl)])
        cfl = [[fn[foff[j]:foff[j + 1]] for j in range(fp[i], fp[i + 1])] for i in range(len(fp) - 1)]
    return nodes, cells, bdict, cfl


def golden_patches(d):
    names = [str(x) for x in d["patch_names"]]
    ptr, fids = d["patch_ptr"], d["patch_fids"]
    return {nm: fids[ptr[i]:ptr[i + 1]] for i, nm in enumerate(names)}


@pytest.fixture(scope="session")
def golden():
    return load_golden

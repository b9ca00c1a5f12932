"""The oracle's ILU(k) (oracle/linsolve.py: distance-(k+1) colouring, level-of-fill
pattern, IKJ factorisation), checked on the CPU before it serves as the device's
checker: the factor pattern holds A's pattern, no factor entry joins two rows of one
colour (so the colours are valid parallel levels), a level-0 colour row carries no
fill, and the preconditioned loop converges faster as k grows on a Laplacian."""
import numpy as np
import pytest
from scipy import sparse

from case16 import channel_mesh, convdiff_system
from oracle import linsolve as ol


def _laplacian(N, shift=0.1):
    n = N * N
    A = sparse.lil_matrix((n, n))
    for i in range(N):
        for j in range(N):
            r = i * N + j
            A[r, r] = 4.0 + shift
            for di, dj in ((1, 0), (-1, 0), (0, 1), (0, -1)):
                a, b = i + di, j + dj
                if 0 <= a < N and 0 <= b < N:
                    A[r, a * N + b] = -1.0
    return A.tocsr()


@pytest.mark.parametrize("k", [1, 2])
def test_iluk_pattern_and_colours(k):
    A, _ = convdiff_system(channel_mesh(12, 10))
    F, perm, colour = ol.iluk_factor(A, k)
    B = sparse.csr_matrix(A)[perm][:, perm].tocsr()
    rows, cols = np.repeat(np.arange(F.shape[0]), np.diff(F.indptr)), F.indices
    pattern = set(zip(rows.tolist(), cols.tolist()))
    for i, j in zip(*B.nonzero()):
        assert (int(i), int(j)) in pattern
    cp = colour[perm]
    off = rows != cols
    assert not np.any(cp[rows[off]] == cp[cols[off]])
    first = cp == 0
    assert np.all(np.diff(F.indptr)[first] == np.diff(B.indptr)[first])
    assert np.all(np.diff(np.flatnonzero(np.diff(cp) != 0)) >= 0)  # rows grouped by colour


def test_iluk_converges_faster_with_more_fill():
    A = _laplacian(16)
    b = np.random.default_rng(0).standard_normal(A.shape[0])
    its = []
    for k in (0, 1, 2):
        F, perm, _ = ol.iluk_factor(A, k)
        x, info, it = ol.bicgstab_scipy(A, b, rtol=1e-10, M=lambda z: ol.ilu0_apply(F, perm, z))
        assert info == 0 and np.linalg.norm(A @ x - b) / np.linalg.norm(b) < 1.5e-10
        its.append(it)
    assert its[2] <= its[1] < its[0]

"""The partitioned solve's device path on one GPU (one rank over NCCL): the local
product runs on kcfd_spmv_f64 with the rank's CSR, the scalars go through NCCL
all_reduce, and the halo exchange has no peers. Ranks that wait on each other are not
run on one GPU; the exchange itself is covered by the two-rank gloo test."""
import os

import numpy as np
import pytest
import scipy.sparse.linalg as spla
from scipy import sparse

from case16 import channel_mesh, convdiff_system

pytestmark = pytest.mark.gpu


def test_one_rank_device_solve():
    import torch
    import torch.distributed as dist
    from kcfd.parallel import DistributedBiCGSTAB, HaloPlan
    from oracle.linsolve import bicgstab_scipy, jacobi
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", str(29900 + os.getpid() % 500))
    own = not dist.is_initialized()
    if own:
        dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        A, b = convdiff_system(channel_mesh(40, 30))
        A = sparse.csr_matrix(A)
        p = HaloPlan(A.indptr, A.indices, np.zeros(A.shape[0], dtype=int), 0)
        assert p.n_ghost == 0 and p.n_own == A.shape[0]
        vals = torch.from_numpy(A.data[p.src].copy()).cuda()
        s = DistributedBiCGSTAB(p, vals)
        x, info, its = s.solve(torch.from_numpy(b).cuda(), rtol=1e-10, maxiter=3000)
        assert info == 0
        xd = spla.spsolve(A.tocsc(), b)
        assert np.linalg.norm(x.cpu().numpy() - xd) / np.linalg.norm(xd) < 1e-8
        _, info_o, its_o = bicgstab_scipy(A, b, np.zeros(len(b)), rtol=1e-10, atol=0.0, maxiter=3000, M=jacobi(A))
        assert abs(its - its_o) <= max(2, its_o // 10), (its, its_o)
        # the block ILU(0) on the device (one rank: the block is the whole matrix)
        s2 = DistributedBiCGSTAB(p, vals, precond="block_ilu0")
        x2, info2, its2 = s2.solve(torch.from_numpy(b).cuda(), rtol=1e-10, maxiter=3000)
        assert info2 == 0 and its2 < its, (its2, its)
        assert np.linalg.norm(x2.cpu().numpy() - xd) / np.linalg.norm(xd) < 1e-8
    finally:
        if own:
            dist.destroy_process_group()

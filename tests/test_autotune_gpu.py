"""The launch-shape autotuner (kcfd.autotune): it picks the fastest (lanes, block) per
Krylov iteration among the candidates, caches the choice in the process and in the
KCFD_TUNE_CACHE file, and the tuned handle solves to the requested tolerance."""
import json

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from case16 import channel_mesh, convdiff_system

pytestmark = pytest.mark.gpu


def test_tune_caches_and_solves(tmp_path, monkeypatch):
    import torch
    from kcfd import autotune
    from kcfd.solver import DeviceCSR
    cache = tmp_path / "tune.json"
    monkeypatch.setenv("KCFD_TUNE_CACHE", str(cache))
    monkeypatch.setattr(autotune, "_CACHE", {})
    A, b = convdiff_system(channel_mesh(32, 24))
    d = DeviceCSR.from_scipy(A)
    bd = torch.from_numpy(b).cuda()
    x0 = torch.zeros_like(bd)
    r = autotune.tune(d, bd, x0, precond="jacobi", team=1, lanes=(1, 2), blocks=(256, 512))
    assert r["lanes"] in (1, 2) and r["block"] in (256, 512)
    assert len(r["candidates"]) == 4
    per_it = [t / max(it, 1) for _, _, t, it in r["candidates"]]
    assert r["ms"] / max(r["iters"], 1) == min(per_it)
    assert autotune.tune(d, bd, x0, precond="jacobi", team=1, lanes=(1, 2), blocks=(256, 512)) is r
    saved = json.loads(cache.read_text())
    assert list(saved.values())[0]["lanes"] == r["lanes"]
    monkeypatch.setattr(autotune, "_CACHE", {})
    s = autotune.tuned_solver(d, bd, x0, precond="jacobi", team=1, rtol=1e-10, lanes=(1, 2), blocks=(256, 512))
    info = s.info()
    assert (info["lanes"], info["block"]) == (r["lanes"], r["block"])
    s.setup(d)
    x = x0.clone()
    it, rr, st = s.solve(d, bd, x)
    assert int(st[0]) == 0
    xd = spla.spsolve(A.tocsc(), b)
    assert np.linalg.norm(x.cpu().numpy() - xd) / np.linalg.norm(xd) < 1e-8

"""Autotuner for the BiCGSTAB launch shape: SpMV lanes per row and CTA size.

For a given matrix, preconditioner, precision and right-hand-side count it times one
solve per candidate (CUDA events on the launching stream, after a warm-up solve) and
keeps the fastest. Results are cached per (n, nnz, nrhs, precond, mode, team) for the
life of the process, and in a JSON file when KCFD_TUNE_CACHE names one, so the SIMPLE
driver, the batched engine and the request loop tune a shape once.
"""
from __future__ import annotations

import json
import os

from . import _lib
from .solver import Solver

_CACHE = {}
LANES = (1, 2, 4, 8)
BLOCKS = {1: (256, 512, 1024), 2: (256, 512, 1024), 3: (256, 512)}


def _key(csr, precond, mode, nrhs, team):
    return f"{csr.n}:{csr.nnz}:{nrhs}:{precond}:{mode}:{team}"


def _load():
    p = os.environ.get("KCFD_TUNE_CACHE")
    if p and os.path.exists(p):
        try:
            with open(p) as f:
                _CACHE.update(json.load(f))
        except (OSError, ValueError):
            pass


def _save():
    """Write the cache next to its final name, then rename it into place, so that a
    reader (another process tuning the same shapes) never sees a partial file."""
    p = os.environ.get("KCFD_TUNE_CACHE")
    if p:
        tmp = f"{p}.{os.getpid()}.tmp"
        try:
            with open(tmp, "w") as f:
                json.dump(_CACHE, f)
            os.replace(tmp, p)
        except OSError:
            pass


def tune(csr, b, x0, precond="jacobi", mode=_lib.MODE_FP64, nrhs=1, team=0, levels=None, rtol=1e-8,
         maxiter=5000, lanes=LANES, blocks=None, reps=1, verbose=False, **kw):
    """Return {'lanes', 'block', 'ms'} for the fastest candidate (cached)."""
    torch = _lib.require_cuda()
    if not _CACHE:
        _load()
    k = _key(csr, precond, mode, nrhs, team)
    if k in _CACHE:
        return _CACHE[k]
    blocks = blocks or BLOCKS[nrhs]
    best = None
    results = []
    for L in lanes:
        for B in blocks:
            try:
                s = Solver(csr, precond=precond, mode=mode, nrhs=nrhs, team=team, lanes=L, block=B,
                           levels=levels, rtol=rtol, maxiter=maxiter, **kw)
            except _lib.KcfdError:
                continue
            s.setup(csr)
            x = x0.clone()
            s.solve(csr, b, x)  # warm-up
            ts = []
            for _ in range(reps):
                x.copy_(x0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                s.solve(csr, b, x)
                e1.record()
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
            t = min(ts)
            it = int(s.iters.max())
            results.append((L, B, t, it))
            if verbose:
                print(f"  lanes={L:2d} block={B:4d}: {t:9.3f} ms ({it} iterations, {1e3 * t / max(it, 1):.1f} us/it)")
            # compare per iteration: counts wobble by a few with the reduction shape
            per_it = t / max(it, 1)
            if best is None or per_it < best[2] / max(best[3], 1):
                best = (L, B, t, it)
            del s
    out = {"lanes": best[0], "block": best[1], "ms": best[2], "iters": best[3],
           "candidates": [list(r) for r in results]}
    _CACHE[k] = out
    _save()
    return out


def tuned_solver(csr, b, x0, precond="jacobi", mode=_lib.MODE_FP64, nrhs=1, team=0, levels=None, rtol=1e-8,
                 maxiter=5000, **kw):
    """A Solver with the launch shape tune() picks for this pattern (tuned once per
    process, or read from the KCFD_TUNE_CACHE file)."""
    shape = tune(csr, b, x0, precond=precond, mode=mode, nrhs=nrhs, team=team, levels=levels, rtol=rtol,
                 maxiter=maxiter, **kw)
    return Solver(csr, precond=precond, mode=mode, nrhs=nrhs, team=team, lanes=shape["lanes"], block=shape["block"],
                  levels=levels, rtol=rtol, maxiter=maxiter)

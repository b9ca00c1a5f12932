"""Host logic of the ctypes layer: a handle dropped while a CUDA graph is being captured on
this thread is queued and destroyed at the next release outside a capture (a device free
inside the capture would invalidate it). Checked with a stand-in library and a stand-in
capture flag, so it runs without a GPU. Also: the device path has no host fallback."""
import types


def test_release_defers_inside_a_capture(monkeypatch):
    import torch
    from kcfd import _lib
    destroyed = []
    fake = types.SimpleNamespace(kcfd_solver_destroy=lambda h: destroyed.append(("solver", h)),
                                 kcfd_amg_destroy=lambda h: destroyed.append(("amg", h)))
    monkeypatch.setattr(_lib, "lib", lambda: fake)
    monkeypatch.setattr(_lib, "_deferred", [])
    capturing = {"on": True}
    monkeypatch.setattr(torch.cuda, "is_available", lambda: True)
    monkeypatch.setattr(torch.cuda, "is_current_stream_capturing", lambda: capturing["on"])
    _lib.release("kcfd_solver_destroy", 1)
    _lib.release("kcfd_amg_destroy", 2)
    assert destroyed == [] and len(_lib._deferred) == 2
    capturing["on"] = False
    _lib.release("kcfd_solver_destroy", 3)          # outside: the queued ones go first
    assert destroyed == [("solver", 1), ("amg", 2), ("solver", 3)]
    assert _lib._deferred == []


def test_release_survives_a_failing_destroy(monkeypatch):
    import torch
    from kcfd import _lib

    def boom(h):
        raise RuntimeError("destroy failed")
    monkeypatch.setattr(_lib, "lib", lambda: types.SimpleNamespace(kcfd_batch_destroy=boom))
    monkeypatch.setattr(_lib, "_deferred", [])
    monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
    _lib.release("kcfd_batch_destroy", 7)            # no exception escapes a destructor path
    assert _lib._deferred == []


def test_no_cpu_fallback_without_a_device(monkeypatch):
    """Without a CUDA device the drop-in raises; it never solves on the host."""
    import numpy as np
    import pytest
    import torch
    from scipy import sparse
    from kcfd import _lib
    from kcfd.linear_solver import solve_linear_system
    monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
    system = types.SimpleNamespace(to_sparse=lambda: sparse.identity(4, format="csr"), rhs=np.ones(4))
    with pytest.raises(_lib.KcfdError, match="no CPU fallback"):
        solve_linear_system(system, method="bicgstab")
    with pytest.raises(ValueError, match="device only"):
        solve_linear_system(system, method="bicgstab", backend="cpu")


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    """A libkcfd.so that is absent and cannot be built is an error at the first call."""
    import pytest
    from kcfd import _lib, build

    def no_toolchain(*a, **k):
        raise RuntimeError("nvcc not found")
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "libkcfd.so"))
    monkeypatch.setattr(build, "build", no_toolchain)
    with pytest.raises(RuntimeError, match="nvcc not found"):
        _lib.lib()
    assert _lib._lib is None

"""Host logic of the ctypes layer: a handle dropped while a CUDA graph is being captured on
this thread is queued and destroyed at the next release outside a capture (a device free
inside the capture would invalidate it). Checked with a stand-in library and a stand-in
capture flag, so it runs without a GPU."""
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

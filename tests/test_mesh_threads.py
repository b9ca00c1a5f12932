"""The native mesh builder's output does not depend on its host thread count
(KCFD_HOST_THREADS = 1, 3 or 16): every array of a 3D jittered-hex mesh and of a 2D
Delaunay mesh, both large enough to be split into chunks, and the device face layout,
hash the same. Each count runs in its own process, since the count is read once per
process. Host only."""
import os
import subprocess
import sys

from conftest import ROOT

PROBE = r"""
import hashlib, sys
import numpy as np
sys.path.insert(0, {pkg!r})
from kcfd import mesh as km, meshgen
from kcfd.device_mesh import device_layout
h = hashlib.sha256()
n, c, f, b = meshgen.hex_box_arrays(1, 1, 1, 36, 34, 32, meshgen.CAVITY_3D_NAMES)
n = meshgen.jitter_interior(n, (36, 34, 32), (1 / 36, 1 / 34, 1 / 32), 0.2, seed=1)
m3 = km.build_mesh(n, c, b, ndim=3, cell_face_node_list=f)
m2 = km.build_mesh(*meshgen.delaunay_tri_arrays(60000, np.random.default_rng(4)))
for m in (m3, m2):
    for k in sorted(vars(m)):
        v = getattr(m, k)
        if isinstance(v, np.ndarray):
            h.update(k.encode()); h.update(np.ascontiguousarray(v).tobytes())
    lay = device_layout(m)
    for k in sorted(lay):
        h.update(k.encode()); h.update(lay[k].tobytes())
print(h.hexdigest())
"""


def test_output_independent_of_thread_count():
    code = PROBE.format(pkg=os.path.join(ROOT, "k-cfd_b200"))
    digests = []
    for t in ("1", "3", "16"):
        env = dict(os.environ, KCFD_HOST_THREADS=t)
        r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        digests.append(r.stdout.strip())
    assert len(set(digests)) == 1, digests

"""Device-side box mesh setup (vlm_box_create: generateBox, RawMesh.cpp:391-502, and the serial
Mesh::build geometry, Mesh.cpp:21-48, 135-153, 239-320, 600-626, as kernels) against the host
restatement voluma_b200.mesh.box_mesh, whose arrays tests/test_mesh.py pins to the reference's own
(golden fixtures): every array bit for bit, on uniform, graded, periodic, 2D, jittered and
one-cell-thick boxes; then a registered device-built mesh solves like the host-built one."""
import numpy as np
import pytest

import voluma_b200 as vb
from voluma_b200 import cases, mesh as vm

pytestmark = pytest.mark.gpu

ARRAYS = ("owner", "neighbour", "V", "C", "Sf", "magSf", "Cf", "d", "w", "ndc", "corrVecs", "skewVecs",
          "patch_start", "patch_size")

SPECS = {
    "uniform": dict(n=(7, 5, 4)),
    "graded": dict(n=(9, 8, 6), lo=(-1.0, 0.5, 0.0), hi=(2.0, 1.5, 3.0), beta=(0.9, 0.0, 1.3)),
    "periodic_xz": dict(n=(6, 5, 4), periodic=(True, False, True), beta=(0.0, 1.1, 0.0)),
    "periodic_all": dict(n=(4, 3, 5), hi=(2 * np.pi,) * 3, periodic=(True, True, True)),
    "two_d": dict(n=(12, 9, 1), hi=(1.0, 1.0, 0.1), two_d=True, beta=(0.7, 0.4, 0.0)),
    "two_d_periodic": dict(n=(8, 6, 1), hi=(1.0, 1.0, 0.1), two_d=True, periodic=(True, False, True)),
    "thin": dict(n=(1, 6, 3)),
    "line": dict(n=(9, 1, 1)),
}


@pytest.mark.parametrize("name", sorted(SPECS))
def test_device_box_equals_host(name):
    s = dict(SPECS[name])
    host = vm.box_mesh(**s)
    dev = vb.box_mesh_device(**s)
    for k in ARRAYS:
        assert np.array_equal(np.asarray(dev[k]), np.asarray(host[k])), k
    assert dev["patch_names"] == list(host["patch_names"])
    assert (dev["two_d"], dev["empty_dir"], dev["skewed"]) == (host["two_d"], host["empty_dir"], host["skewed"])


def test_device_box_with_points_equals_host():
    n = (10, 7, 5)
    pts = vm.jitter_interior(vm.box_points(n, beta=(0.5, 0.0, 0.8)), n, 0.2, 17)
    pts[:, 0] += 0.2 * pts[:, 1]
    host = vm.box_mesh(n, periodic=(False, True, False), points=pts)
    dev = vb.box_mesh_device(n, periodic=(False, True, False), points=pts)
    for k in ARRAYS:
        assert np.array_equal(np.asarray(dev[k]), np.asarray(host[k])), k
    assert dev["skewed"] and host["skewed"]


def test_device_box_rejects_bad_specs():
    with pytest.raises(vb.VlmError):
        vb.box_mesh_device((4, 4, 2), two_d=True)
    with pytest.raises(vb.VlmError):
        vb.box_mesh_device((1, 4, 4), periodic=(True, False, False))


def test_device_built_mesh_solves_like_host_mesh():
    m_h, case = cases.lid_cavity(24, 100.0)
    m_d = vb.box_mesh_device((24, 24, 1), hi=(1.0, 1.0, 0.1), two_d=True)
    out = []
    for m in (m_h, m_d):
        fl = vb.Flow(vb.Mesh.from_arrays(m), dict(case, reproducible=True))
        fl.set_state(None, None)
        for _ in range(3):
            fl.step(1.0)
        out.append(fl.state())
        fl.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)

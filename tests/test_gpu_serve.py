"""Serving runtime on the device: continuous batching keeps each result identical to its solo run,
admission follows the HBM budget, and admitted requests overlap on the device."""
import numpy as np
import pytest

import voluma_b200 as vb
from voluma_b200 import cases

pytestmark = pytest.mark.gpu

SPECS = [(12, 100.0), (16, 250.0), (20, 400.0)]


def drain(s, n, timeout=120.0):
    out = []
    for _ in range(int(timeout / 0.5)):
        out += s.collect(timeout=0.5)
        if len(out) >= n:
            break
    assert len(out) == n
    return {r["id"]: r for r in out}


def submit_all(s, arrival=0.0, max_iter=60):
    ids = []
    for n, re in SPECS:
        m, case = cases.lid_cavity(n, re)
        ids.append(s.submit(m, case, arrival=arrival, max_iter=max_iter, residual_tol=1e-12))
    return ids


def test_results_identical_alone_and_in_the_mix():
    alone = []
    for n, re in SPECS:
        s = vb.Server(max_active=1)
        m, case = cases.lid_cavity(n, re)
        rid = s.submit(m, case, max_iter=60, residual_tol=1e-12)
        r = drain(s, 1)[rid]
        assert r["status"] == 0 and r["iterations"] == 60
        alone.append(s.fields(rid))
        s.close()
    s = vb.Server(max_active=3)
    ids = submit_all(s)
    res = drain(s, 3)
    for rid, ref in zip(ids, alone):
        assert res[rid]["status"] == 0
        got = s.fields(rid)
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)
    s.close()
    # and the same as a Flow run without the server
    n, re = SPECS[1]
    m, case = cases.lid_cavity(n, re)
    fl = vb.Flow(vb.Mesh.from_arrays(m), case)
    fl.set_state(None, None)
    for _ in range(60):
        fl.step()
    for a, b in zip(fl.state(), alone[1]):
        assert np.array_equal(a, b)
    fl.close()


def test_budget_serialises_and_slots_overlap():
    m, case = cases.lid_cavity(SPECS[-1][0], 100.0)
    one = vb.request_bytes(m["n_cells"], m["n_faces"])
    # budget for one request at a time: no two requests are ever resident together
    s = vb.Server(hbm_budget=int(one * 1.5), max_active=3)
    ids = submit_all(s)
    res = drain(s, 3)
    s.close()
    spans = sorted((res[i]["admitted"], res[i]["finished"]) for i in ids)
    for (a0, f0), (a1, f1) in zip(spans, spans[1:]):
        assert a1 >= f0 - 1e-6
    # ample budget, three slots: requests run at the same time
    s = vb.Server(hbm_budget=one * 10, max_active=3)
    ids = submit_all(s, max_iter=150)
    res = drain(s, 3)
    s.close()
    spans = sorted((res[i]["admitted"], res[i]["finished"]) for i in ids)
    assert spans[1][0] < spans[0][1] and spans[2][0] < spans[0][1]
    assert all(res[i]["status"] == 0 for i in ids)


def test_device_agglomeration_requests_alone_and_in_the_mix():
    """Requests whose meshes build their GAMG hierarchy on the device (mesh_flags): the same result
    alone, in a mix with host-agglomerated requests, and as a Flow on a mesh registered the same way."""
    n, re = SPECS[2]
    m, case = cases.lid_cavity(n, re)
    s = vb.Server(max_active=1)
    rid = s.submit(m, case, max_iter=60, residual_tol=1e-12, agglomeration="device")
    assert drain(s, 1)[rid]["status"] == 0
    alone = s.fields(rid)
    s.close()
    s = vb.Server(max_active=3)
    ids = submit_all(s)
    did = s.submit(m, case, max_iter=60, residual_tol=1e-12, agglomeration="device")
    res = drain(s, 4)
    assert all(r["status"] == 0 for r in res.values())
    for a, b in zip(s.fields(did), alone):
        assert np.array_equal(a, b)
    s.close()
    fl = vb.Flow(vb.Mesh.from_arrays(m, agglomeration="device"), case)
    fl.set_state(None, None)
    for _ in range(60):
        fl.step()
    for a, b in zip(fl.state(), alone):
        assert np.array_equal(a, b)
    fl.close()

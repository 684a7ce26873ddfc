"""Admission logic of the serving runtime (vlm_server_*), on the host: with no GPU every admitted
request fails at context creation (NO_DEVICE) at once, so the order and times of admission, the
arrival gating and the out-of-memory rejection are observable without a device."""
import numpy as np
import pytest

import voluma_b200 as vb
from voluma_b200 import cases


def _nogpu():
    import torch
    return not torch.cuda.is_available()


@pytest.fixture(scope="module")
def cavity():
    return cases.lid_cavity(8, 100.0)


def test_request_bytes_grow_with_the_mesh():
    assert vb.request_bytes(4096, 8192) < vb.request_bytes(65536, 131072)


@pytest.mark.skipif(not _nogpu(), reason="host-only admission check (workers fail without a device)")
def test_admission_order_arrival_and_budget(cavity):
    m, case = cavity
    s = vb.Server(hbm_budget=vb.request_bytes(m["n_cells"], m["n_faces"]) * 3, max_active=2)
    ids = [s.submit(m, case, arrival=a) for a in (0.30, 0.0, 0.10)]
    big = s.submit(m, case, arrival=0.05, device_bytes=1 << 50)  # larger than the budget
    out = []
    for _ in range(50):
        out += s.collect(timeout=0.2)
        if len(out) == 4:
            break
    s.close()
    byid = {r["id"]: r for r in out}
    assert byid[big]["status"] == 3  # VLM_ERR_OOM
    for rid, a in zip(ids, (0.30, 0.0, 0.10)):
        r = byid[rid]
        assert r["status"] == 8  # VLM_ERR_NO_DEVICE: admitted, then no device
        assert r["admitted"] >= a - 1e-6  # never before its arrival
    # admitted in arrival order
    adm = sorted(ids, key=lambda i: byid[i]["admitted"])
    assert adm == [ids[1], ids[2], ids[0]]


def test_trace_is_seeded_and_in_range():
    t1 = cases.serving_trace(20, seed=3)
    assert t1 == cases.serving_trace(20, seed=3)
    assert all(32 <= q["n"] <= 256 and 100 <= q["Re"] <= 1000 for q in t1)
    assert all(b["arrival"] >= a["arrival"] for a, b in zip(t1, t1[1:]))

"""Serving loop host logic that needs no GPU: registration, queueing, request state, errors."""
import ctypes

import numpy as np
import pytest

from safire_b200 import capi, synthetic
from safire_b200.serve import Server


def test_server_queue_without_gpu():
    srv = Server(hbm_budget_gb=1.0, max_inflight=2)
    s = synthetic.make_system(synthetic.CFG_SMALL)
    a = srv.add_system(s, 8, seed=1)
    b = srv.add_system(s, 8, seed=2)
    assert (a, b) == (0, 1)
    r0 = srv.submit(a, steps=10)
    r1 = srv.submit(b, steps=10)
    assert (r0, r1) == (0, 1)
    for r in (r0, r1):
        info = srv.request(r)
        assert info["status"] == 1  # queued: progress() has not run
        assert info["t_submit"] >= 0.0
    st = srv.stats()
    assert st == {"used_bytes": 0, "resident": 0, "running": 0, "queued": 2}
    srv.close()


def test_server_argument_errors():
    L = capi.lib()
    h = ctypes.c_void_p()
    bad = capi.ServerParams(0, 1, 0)
    assert L.sfq_server_create(ctypes.byref(h), ctypes.byref(bad)) == 2  # SFQ_ERR_ARG: empty budget
    srv = Server(hbm_budget_gb=1.0, max_inflight=1)
    with pytest.raises(capi.SafireError):
        srv.submit(3, steps=5)  # no such system
    s = synthetic.make_system(synthetic.CFG_SMALL)
    sid = srv.add_system(s, 4)
    with pytest.raises(capi.SafireError):
        srv.submit(sid, steps=0)
    with pytest.raises(capi.SafireError):
        srv.request(99)
    srv.close()

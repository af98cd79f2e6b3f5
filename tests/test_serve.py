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


def test_server_refuses_multideterminant_systems():
    """The serving loop builds single-determinant engines; a multi-determinant system is refused
    before any library call (no GPU needed)."""
    import numpy as np
    from safire_b200 import capi, synthetic
    from safire_b200.serve import Server
    s = synthetic.System(synthetic.SystemSpec(M=4, N=1, Nc=4, decay=1.0), np.eye(4), np.zeros((4, 4, 4)),
                         np.zeros((2, 1, 4), np.complex128), 0.0, ci=np.array([1.0, 0.5], np.complex128))
    srv = Server.__new__(Server)  # the check precedes the server handle
    srv.walkers = {}
    with pytest.raises(capi.SafireError) as ex:
        Server.add_system(srv, s, 8)
    assert ex.value.code == 3

"""Continuous-batching server: admission, retirement, fault handling, and the
result of every request being the same alone and in the mix (bit-identical:
the batched kernel gives each domain the same arithmetic whatever runs next
to it)."""
import numpy as np
import pytest

import mrlbm

pytestmark = pytest.mark.gpu


def mix():
    return [mrlbm.make_request(mrlbm.REQ_LID_CAVITY, 24, re=100.0),
            mrlbm.make_request(mrlbm.REQ_DUCT, 28, nnf_n=0.7, solid_fraction=0.05, seed=3),
            mrlbm.make_request(mrlbm.REQ_LID_CAVITY, 36, re=400.0),
            mrlbm.make_request(mrlbm.REQ_DUCT, 32, nnf_n=1.1, solid_fraction=0.05, seed=4),
            mrlbm.make_request(mrlbm.REQ_LID_CAVITY, 30, re=900.0)]


def run_server(reqs, max_steps=300, tick=50, budget=150e9, max_active=64, inject=None, capacity=0):
    srv = mrlbm.Server(storage=mrlbm.F16, hbm_budget=budget, max_active=max_active, steps_per_tick=tick,
                       residual_tol=1e-12, max_steps=max_steps, keep_results=True, capacity_nodes=capacity)
    ids = [srv.submit(r) for r in reqs]
    first = True
    while True:
        active = srv.tick()
        if first and inject is not None:
            srv.inject_nan(ids[inject])
        first = False
        st = srv.stats()
        if active == 0 and st["queued"] == 0:
            break
    out = {}
    for rid, r in zip(ids, reqs):
        res = srv.result(rid)
        m = srv.moments(rid, r.n, 11 if r.kind == mrlbm.REQ_DUCT else 10) if res["status"] == 0 else None
        out[rid] = (res, m)
    stats = srv.stats()
    srv.close()
    return ids, out, stats


def test_results_same_alone_and_in_mix():
    reqs = mix()
    ids, mixed, stats = run_server(reqs)
    assert stats["done"] == len(reqs) and stats["failed"] == 0
    assert stats["p99_latency"] >= stats["p50_latency"] > 0
    for rid, r in zip(ids, reqs):
        _, alone, _ = run_server([r])
        res_m, m_mix = mixed[rid]
        res_a, m_alone = list(alone.values())[0]
        assert res_m["steps"] == res_a["steps"] == 300
        np.testing.assert_array_equal(m_mix, m_alone)


def test_injected_nan_retires_only_that_request():
    reqs = mix()
    ids, out, stats = run_server(reqs, inject=1)
    assert out[ids[1]][0]["status"] == 5      # MRLBM_EDIVERGED
    assert stats["failed"] == 1 and stats["done"] == len(reqs) - 1
    _, ref, _ = run_server(reqs)
    for k in (0, 2, 3, 4):
        np.testing.assert_array_equal(out[ids[k]][1], ref[ids[k]][1])


def test_budget_admission_and_cancel():
    a = mrlbm.make_request(mrlbm.REQ_LID_CAVITY, 40, re=100.0)
    desc_bytes = mrlbm.domain_bytes(mrlbm.lid_cavity_desc(40, storage=mrlbm.F16))
    # room for one 40^3 request at a time
    srv = mrlbm.Server(storage=mrlbm.F16, hbm_budget=1.5 * desc_bytes, max_active=8, steps_per_tick=20,
                       residual_tol=1e-12, max_steps=60)
    big = mrlbm.make_request(mrlbm.REQ_LID_CAVITY, 64, re=100.0)
    with pytest.raises(mrlbm.MrlbmError):
        srv.submit(big)                        # can never fit: refused
    r0, r1, r2 = srv.submit(a), srv.submit(a), srv.submit(a)
    srv.tick()
    st = srv.stats()
    assert st["active"] == 1 and st["queued"] == 2
    srv.cancel(r2)                             # queued: cancelled at once
    assert srv.result(r2)["status"] == 9
    while srv.tick() or srv.stats()["queued"]:
        pass
    res0, res1 = srv.result(r0), srv.result(r1)
    assert res0["status"] == 0 and res1["status"] == 0
    assert res1["admitted"] >= res0["finished"]  # admitted only after the first freed its bytes
    srv.close()


def test_cancel_running_request():
    srv = mrlbm.Server(storage=mrlbm.F16, steps_per_tick=10, residual_tol=1e-12, max_steps=10000)
    rid = srv.submit(mrlbm.make_request(mrlbm.REQ_LID_CAVITY, 24, re=100.0))
    srv.tick()
    srv.cancel(rid)
    srv.tick()
    assert srv.result(rid)["status"] == 9
    assert srv.stats()["active"] == 0
    srv.close()


def test_capacity_admits_in_arrival_order_within_the_node_limit():
    """With a compute limit of 60,000 nodes: the 24^3 and 28^3 requests
    (13,824 + 21,952 nodes) run together, the 36^3 one (46,656) waits until
    they leave, and every result is still the one the request gets alone."""
    reqs = mix()
    srv = mrlbm.Server(storage=mrlbm.F16, hbm_budget=150e9, max_active=64, steps_per_tick=50,
                       residual_tol=1e-12, max_steps=300, keep_results=True, capacity_nodes=60000)
    ids = [srv.submit(r) for r in reqs]
    srv.tick()
    st = srv.stats()
    assert st["active"] == 2 and st["queued"] == 3
    while True:
        active = srv.tick()
        if active == 0 and srv.stats()["queued"] == 0:
            break
    res = [srv.result(i) for i in ids]
    assert all(r["status"] == 0 and r["steps"] == 300 for r in res)
    # later arrivals start no earlier than the requests before them
    admitted = [r["admitted"] for r in res]
    assert admitted == sorted(admitted) and admitted[2] >= max(res[0]["finished"], res[1]["finished"]) - 1e-9
    with pytest.raises(mrlbm.MrlbmError):
        mrlbm.check(srv.L.mrlbm_server_set_capacity(srv.h, -1.0))
    _, ref, _ = run_server(reqs)
    for rid, k in zip(ids, range(len(reqs))):
        np.testing.assert_array_equal(srv.moments(rid, reqs[k].n, 11 if reqs[k].kind == mrlbm.REQ_DUCT else 10),
                                      list(ref.values())[k][1])
    srv.close()

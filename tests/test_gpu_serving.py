"""The device-resident request server (jfg_server_*).

Requests for three small families (plate, stiffened panel, barrel with an
RBE2 end) are submitted as one burst, so that the batched policy runs them
in batches on overlapping family streams; every request's K and KG must
equal, bit for bit, the same request assembled alone on a fresh handle with
that thickness vector.  The serial policy must give the same bits.
"""
import ctypes as C
import time

import numpy as np
import pytest

from jf_2026_05_19_b200 import decks, native

pytestmark = pytest.mark.gpu


def _d2h(ptr, n):
    from cuda.bindings import runtime as rt
    out = np.empty(n, np.float64)
    err, = rt.cudaMemcpy(out.ctypes.data, ptr, 8 * n, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert int(err) == 0
    return out


def _families():
    return [decks.plate_c1(n=12),
            decks.stiffened_panel_c2(seed=1, lx=300.0, ly=200.0, stringer_every=4, stringer_offset=0.0),
            decks.barrel_small(seed=2, n_circ=48, n_axial=16)]


def _requests(fams, n, seed=3):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        f = int(rng.integers(len(fams)))
        m = fams[f]
        out.append((f, rng.uniform(0.8, 3.0, m.q4_nodes.shape[0]), rng.uniform(0.8, 3.0, m.t3_nodes.shape[0])))
    return out


def _alone(m, hq, ht, u):
    with native.GpuModel(m.with_thickness(hq, ht)) as g:
        return g.assemble_k()[0], g.assemble_kg(u)


def _serve(fams, us, reqs, policy):
    models = [native.GpuModel(m) for m in fams]
    got = []
    try:
        with native.Server(models, us, hbm_budget_bytes=8 * 10**9, max_batch=8, policy=policy) as srv:
            srv.hold(True)
            tickets = [srv.submit(f, np.concatenate([hq, ht])) for f, hq, ht in reqs]
            srv.hold(False)
            for t, (f, _, _) in zip(tickets, reqs):
                assert srv.wait(t, timeout=120.0)
                pk, pkg, _, times = srv.result(t)
                assert times[0] <= times[1] <= times[2]
                nnz = models[f].nnz
                got.append((_d2h(pk, nnz), _d2h(pkg, nnz)))
                srv.release(t)
            stats = srv.stats()
    finally:
        for g in models:
            g.close()
    return got, stats


def test_batched_server_results_equal_requests_alone(cuda_device):
    fams = _families()
    us = [decks.smooth_displacement(m, seed=10 + i) for i, m in enumerate(fams)]
    reqs = _requests(fams, 18)
    got, stats = _serve(fams, us, reqs, native.SERVE_BATCHED)
    assert stats["completed"] == len(reqs) and stats["queued"] == 0
    assert stats["max_batch"] > 1 and stats["batches"] < len(reqs)     # the burst was batched
    for (f, hq, ht), (k, kg) in zip(reqs, got):
        k1, kg1 = _alone(fams[f], hq, ht, us[f])
        assert np.array_equal(k, k1) and np.array_equal(kg, kg1)


def test_serial_server_matches_batched(cuda_device):
    fams = _families()
    us = [decks.smooth_displacement(m, seed=10 + i) for i, m in enumerate(fams)]
    reqs = _requests(fams, 6, seed=4)
    a, sa = _serve(fams, us, reqs, native.SERVE_BATCHED)
    b, sb = _serve(fams, us, reqs, native.SERVE_SERIAL)
    assert sb["batches"] == len(reqs) and sb["max_batch"] == 1
    for (ka, kga), (kb, kgb) in zip(a, b):
        assert np.array_equal(ka, kb) and np.array_equal(kga, kgb)


def test_server_rejects_bad_requests(cuda_device):
    fams = _families()[:1]
    models = [native.GpuModel(m) for m in fams]
    try:
        with native.Server(models, None, hbm_budget_bytes=10**9, max_batch=4) as srv:
            h = np.full(fams[0].q4_nodes.shape[0], 2.0)
            h[3] = 0.0
            with pytest.raises(native.JfgError):
                srv.submit(0, h)                       # thickness must be positive
            with pytest.raises(ValueError):
                srv.submit(0, h[:-1])                  # wrong length
            t = srv.submit(0, np.full(fams[0].q4_nodes.shape[0], 2.0))
            assert srv.wait(t, timeout=60.0)
            pk, pkg, _, _ = srv.result(t)
            assert pk and pkg is None                  # K only: no displacement field given
            srv.release(t)
            with pytest.raises(native.JfgError):
                srv.release(t)                         # already released
    finally:
        for g in models:
            g.close()


def test_grouped_families_share_batches(cuda_device):
    """Three small families as members of one group handle: a burst runs as
    batches that mix families, and every request still equals itself alone."""
    fams = _families()
    us = [decks.smooth_displacement(m, seed=10 + i) for i, m in enumerate(fams)]
    reqs = _requests(fams, 15, seed=6)
    g = native.GpuGroup(fams)
    try:
        with native.Server([g], [np.concatenate(us)], hbm_budget_bytes=8 * 10**9, max_batch=8,
                           family_map=[(0, i) for i in range(len(fams))]) as srv:
            srv.hold(True)
            tickets = [srv.submit(f, np.concatenate([hq, ht])) for f, hq, ht in reqs]
            srv.hold(False)
            got = []
            for t, (f, _, _) in zip(tickets, reqs):
                assert srv.wait(t, timeout=120.0)
                pk, pkg, _, _ = srv.result(t)
                nnz = g.member(f)["nnz"]
                got.append((_d2h(pk, nnz), _d2h(pkg, nnz)))
                srv.release(t)
            st = srv.stats()
    finally:
        g.close()
    counts = np.bincount([f for f, _, _ in reqs], minlength=len(fams))
    assert st["completed"] == len(reqs) and st["batches"] <= int(np.ceil(counts.max() / 8)) + 1
    for (f, hq, ht), (k, kg) in zip(reqs, got):
        k1, kg1 = _alone(fams[f], hq, ht, us[f])
        assert np.array_equal(k, k1) and np.array_equal(kg, kg1)


def test_pool_admits_requests_as_memory_frees(cuda_device):
    """A budget that holds about two variants of the largest family: a burst
    is served in batches that fit (two at most for that family) as batches
    finish and results are released, the pool never exceeds the budget, and
    the results stay exact."""
    fams = _families()
    us = [decks.smooth_displacement(m, seed=10 + i) for i, m in enumerate(fams)]
    models = [native.GpuModel(m) for m in fams]
    big = max(range(len(fams)), key=lambda i: models[i].nnz)
    per = models[big].batch_workspace_bytes(1) + 8 * (2 * models[big].nnz + 1 + models[big].counts[1] + models[big].counts[2])
    budget = int(2.5 * per)
    reqs = [r for r in _requests(fams, 12, seed=8)]
    try:
        with native.Server(models, us, hbm_budget_bytes=budget, max_batch=8) as srv:
            assert srv.batch_limit(big) == 2
            limits = [srv.batch_limit(f) for f in range(len(fams))]
            srv.hold(True)
            tickets = [srv.submit(f, np.concatenate([hq, ht])) for f, hq, ht in reqs]
            srv.hold(False)
            # results in completion order: a batch's result memory returns to
            # the pool once all of its requests are released
            got, todo = {}, dict(enumerate(tickets))
            deadline = time.monotonic() + 300.0
            while todo and time.monotonic() < deadline:
                for i, t in list(todo.items()):
                    if srv.wait(t, timeout=0.0):
                        f = reqs[i][0]
                        pk, pkg, _, _ = srv.result(t)
                        got[i] = (_d2h(pk, models[f].nnz), _d2h(pkg, models[f].nnz))
                        srv.release(t)
                        del todo[i]
                time.sleep(0.001)
            assert not todo
            got = [got[i] for i in range(len(reqs))]
            st = srv.stats()
    finally:
        for m in models:
            m.close()
    assert st["completed"] == len(reqs) and st["pool_peak_bytes"] <= budget
    assert st["max_batch"] <= max(limits)          # each family within what the budget allows it
    for (f, hq, ht), (k, kg) in zip(reqs, got):
        k1, kg1 = _alone(fams[f], hq, ht, us[f])
        assert np.array_equal(k, k1) and np.array_equal(kg, kg1)

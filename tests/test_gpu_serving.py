"""Serving loop (config 5 shape, scaled down): requests arriving while others
run are batched and overlapped; every result equals the same operation run
alone; admission respects the HBM budget."""
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import pyfideslib_b200 as F


@pytest.fixture(scope="module")
def env():
    cc = F.CryptoContext(log_n=13, num_q=8, dnum=3)
    sk = cc.KeyGen(seed=3, hamming_weight=32)
    cc.EvalMultKeyGen(sk)
    idx = [1, 2, 5, -3]
    cc.EvalRotateKeyGen(sk, idx)
    rng = np.random.default_rng(0)
    cts = []
    for i in range(6):
        z = rng.uniform(-1, 1, cc.N // 2) + 1j * rng.uniform(-1, 1, cc.N // 2)
        lv = [7, 7, 6, 5, 7, 6][i]
        cts.append(cc.Encrypt(sk, z, level=lv, seed=10 + i))
    return cc, sk, cts, idx


def _requests(rng, cts, idx, n):
    reqs = []
    for _ in range(n):
        if rng.uniform() < 0.6:
            lv = int(rng.integers(0, 3))
            same = [c for c in cts if c.level == cts[lv].level]
            reqs.append((F.Server.HMULT, same[int(rng.integers(0, len(same)))], same[int(rng.integers(0, len(same)))], 0))
        else:
            reqs.append((F.Server.ROTATE, cts[int(rng.integers(0, len(cts)))], None, idx[int(rng.integers(0, len(idx)))]))
    return reqs


def test_mixed_requests_equal_alone(env):
    cc, sk, cts, idx = env
    srv = F.Server(cc, hbm_budget=8 << 30, max_batch=8, num_streams=2)
    rng = np.random.default_rng(1)
    reqs = _requests(rng, cts, idx, 48)
    results = [None] * len(reqs)

    def client(part):
        lr = np.random.default_rng(100 + part)
        for k in range(part, len(reqs), 2):
            op, a, b, r = reqs[k]
            time.sleep(float(lr.exponential(0.0005)))  # Poisson arrivals
            rid, out = srv.submit(op, a, b, r)
            results[k] = (rid, out)

    th = [threading.Thread(target=client, args=(p,)) for p in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for rid, _ in results:
        srv.wait(rid)
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["p99_ms"] >= st["p50_ms"] > 0
    for (op, a, b, r), (_, out) in zip(reqs, results):
        alone = cc.EvalMult(a, b, rescale=True) if op == F.Server.HMULT else cc.EvalRotate(a, r)
        g, w = out.download(), alone.download()
        assert np.array_equal(g[0], w[0]) and np.array_equal(g[1], w[1])
    srv.close()


def test_budget_admission_and_rejection(env):
    cc, sk, cts, idx = env
    ws_one = 2 * (8 * 4 + 3 * 11 + 2 * 11 + 2 * 8 + 2) * cc.N * 8  # workspace words of max_batch=2, 1 stream
    out_bytes = 2 * 8 * cc.N * 8
    srv = F.Server(cc, hbm_budget=ws_one + out_bytes + 1, max_batch=2, num_streams=1)
    rids = [srv.submit(F.Server.ROTATE, cts[0], None, 1) for _ in range(5)]
    for rid, _ in rids:
        srv.wait(rid)  # admitted one at a time under the budget
    assert srv.stats()["completed"] == 5
    srv.close()
    with pytest.raises(F.FidesError):
        F.Server(cc, hbm_budget=1 << 20, max_batch=2, num_streams=1)  # smaller than its workspaces

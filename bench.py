"""Benchmark of the CKKS evaluation hot path: key-switched HMult/s.

Workload (one step): HMult + relinearisation + rescale of B = 32 resident
ciphertext pairs at N=2^16, 30 moduli (one 60-bit + 29 x 50-bit), K=10
special 60-bit moduli, dnum=3, top level (29).  Inputs are seeded synthetic
residues (uniform in [0, q)), which is all the kernels see; the pairs occupy
2 GB (> the 126 MB L2), so no L2 flush is needed between steps.

  value  = HMult/s of the batched path (fides_hmult_batch: all pairs share
           every launch and the relinearisation key reads), inputs resident in
           HBM (device time, CUDA events on the library's stream, max over
           ranks).  per_op_value = the same pairs through B fides_hmult calls.
  e2e    = the batched metric through the C ABI with host buffers: per step
           the pinned-host upload of the B pairs, the batched HMult and the
           download of the B results are inside the timed region.
  roofline = the forward NTT (two kernels) as the key-switch pipeline
           launches it, batched over 32 polynomials x 30 limbs, timed live:
           algorithmic bytes 16*N*30*32 (one read + one write of each limb);
           the single 30-limb polynomial is reported beside it.
  cpu_baseline = the CPU oracle (C, OpenMP over limbs) on one HMult of the
           same shape on this host's cores.

`--impl reference` times the CPU implementation of the path (the oracle port:
FIDESlib's own CPU path is OpenFHE, which is not available) on rank 0.
Multi-GPU: independent replicas, one per rank (the path has no exchange).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "key-switched HMult/s at N=2^16 L=30 (batched vs per-op), bootstrap ms, NTT HBM GB/s"
LOGN, L, K, DNUM = 16, 30, 10, 3
# DRAM bytes (read + write) of one batched forward NTT (32 polynomials x 30
# limbs at N=2^16): a constant taken from one ncu capture of that launch pair
# (dram__bytes_read.sum + dram__bytes_write.sum of k_ntt_fwd_cols and
# k_ntt_fwd_rows, forward variant 9, caches flushed before each kernel), stale
# after any change to those kernels; --ntt-traffic-csv reads a fresh capture
# instead.  About twice the algorithmic bytes: the column pass writes the 960
# intermediate limbs (480 MB, more than L2) and the row pass reads them back;
# twiddles add 32 MB (read once per prime for the whole batch).
NTT_BATCH_TRAFFIC_BYTES = 1922.8e6  # 503.5 + 443.3 (cols) + 535.0 + 441.0 (rows) MB
NTT_BATCH_TRAFFIC_SOURCE = "constant from one ncu capture of the launch pair (variant 9, caches flushed)"
_UNITS = {"byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "Tbyte": 1e12}


def ntt_traffic_from_csv(path):
    """DRAM bytes of the last k_ntt_fwd_cols + k_ntt_fwd_rows launch pair in
    an ncu --csv log of dram__bytes_read.sum and dram__bytes_write.sum."""
    import csv

    per = {}
    for r in csv.DictReader(line for line in open(path) if line.startswith('"')):
        name = r.get("Metric Name", "")
        if not name.startswith("dram__bytes_"):
            continue
        kern = r["Kernel Name"].split("(")[0].split("<")[0].split()[-1]
        if kern not in ("k_ntt_fwd_cols", "k_ntt_fwd_rows"):
            continue
        v = float(r["Metric Value"].replace(",", "")) * _UNITS.get(r["Metric Unit"], 1.0)
        per.setdefault((int(r["ID"]), kern), 0.0)
        per[(int(r["ID"]), kern)] += v
    cols = [v for (i, k), v in sorted(per.items()) if k == "k_ntt_fwd_cols"]
    rows = [v for (i, k), v in sorted(per.items()) if k == "k_ntt_fwd_rows"]
    if not cols or not rows:
        raise SystemExit("no k_ntt_fwd_cols / k_ntt_fwd_rows DRAM metrics in " + path)
    return cols[-1] + rows[-1]


def measure_h2d_link(nbytes=1 << 30, reps=3):
    """Host-to-device bandwidth of one pinned copy of nbytes (GB/s, best of
    reps, CUDA events on a side stream): the link the end-to-end step's
    uploads cross."""
    import torch

    src = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    dst = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    s = torch.cuda.Stream()
    best = 0.0
    with torch.cuda.stream(s):
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            dst.copy_(src, non_blocking=True)
            e1.record(s)
            e1.synchronize()
            best = max(best, nbytes / (e0.elapsed_time(e1) * 1e-3) / 1e9)
    del src, dst
    return best


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, dev):
        self.dev = dev
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline_hmult(max_seconds=30.0):
    """One HMult+Relin+Rescale of the workload's shape on the host cores (oracle port)."""
    import numpy as np

    from oracle import oracle as O

    # moduli from the oracle's own search (the same list the library
    # generates), so this process loads oracle/ code only
    q, p = O.moduli(LOGN, L, K, DNUM)
    oc = O.Ctx(LOGN, q, p, DNUM)
    lv = L - 1
    pid = list(range(lv + 1))
    np_ = L + K
    kb = oc.random(list(range(np_)) * DNUM, 1).reshape(DNUM, np_, oc.N)
    ka = oc.random(list(range(np_)) * DNUM, 2).reshape(DNUM, np_, oc.N)
    a0, a1, b0, b1 = (oc.random(pid, s) for s in (3, 4, 5, 6))
    n, t0 = 0, time.perf_counter()
    while True:
        oc.hmult(lv, a0, a1, b0, b1, kb, ka, rescale=True)
        n += 1
        el = time.perf_counter() - t0
        if el > max_seconds / 3 or n >= 3:
            break
    return n / el, O.get_threads(), "%d HMult+Relin+Rescale at N=2^16 L=30 K=10 dnum=3 (%.1f s)" % (n, el)


def measure_c4(cc, lib, st, n=256, reps=3, seed=4):
    """Config 4: n pairs at levels uniform in 4..29 (5..30 limbs), HMult+Relin+
    Rescale then one rotation by a random index in [1, 2^15) (one key per
    pair), captured once as a CUDA graph and replayed; compared with the same
    work through per-operation calls."""
    import numpy as np
    import torch

    import pyfideslib_b200 as F

    rng = np.random.default_rng(seed)
    levels = [int(x) for x in rng.integers(4, 30, size=n)]
    idx = [int(x) for x in rng.integers(1, 2 ** 15, size=n)]
    sk = cc.KeyGen(seed=77, hamming_weight=192)
    cc.EvalRotateKeyGen(sk, idx)
    A = [cc.random_ct(lv, 2 * i + 1) for i, lv in enumerate(levels)]
    B = [cc.random_ct(lv, 2 * i + 2) for i, lv in enumerate(levels)]
    plan, outs = cc.plan_hmult_rotate(A, B, idx, rescale=True)
    plan.launch()
    cc.Synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        plan.launch()
    e1.record(st)
    e1.synchronize()
    graph_ms = e0.elapsed_time(e1) / reps
    # the same work, one operation per call
    tmp = [F.Ciphertext(cc) for _ in range(n)]
    outs2 = [F.Ciphertext(cc) for _ in range(n)]
    # one untimed pass, so that the memory pool already holds buffers of every
    # size (the plan allocates all of its buffers when it is created)
    for i in range(n):
        cc.EvalRotate(cc.EvalMult(A[i], B[i], rescale=True, out=tmp[i]), idx[i], out=outs2[i])
    cc.Synchronize()
    e0.record(st)
    for i in range(n):
        cc.EvalMult(A[i], B[i], rescale=True, out=tmp[i])
        cc.EvalRotate(tmp[i], idx[i], out=outs2[i])
    e1.record(st)
    e1.synchronize()
    op_ms = e0.elapsed_time(e1)
    same = all(np.array_equal(outs[i].download()[0], outs2[i].download()[0]) for i in (0, n // 2, n - 1))
    del plan
    return {"pairs": n, "levels": "uniform 4..29", "rotations": "one per pair, random index in [1, 2^15)",
            "graph_ms": graph_ms, "graph_pairs_per_s": n / (graph_ms * 1e-3),
            "per_op_ms": op_ms, "per_op_pairs_per_s": n / (op_ms * 1e-3), "results_equal": bool(same)}


def measure_c3(reps=5, seed=3, ntt_variant=-1, ks_variant=-1, key_compression=1, profile=False):
    """Config 3: N=2^16, 20 moduli (60 + 19 x 40-bit, scale 2^40), dnum=3, one
    ciphertext; 32 hoisted rotations (+-2^k, k < 15, and 3, 5) sharing one
    ModUp, and a 64-diagonal plaintext matrix (offsets 0..63, entries uniform
    in [-1, 1]) applied by baby-step giant-step with 8 baby steps; the
    transform's error is taken against the FP64 product."""
    import numpy as np
    import torch

    import pyfideslib_b200 as F

    from pyfideslib_b200._capi import lib

    cc = F.CryptoContext(log_n=16, num_q=20, dnum=3, qi_bits=40)
    if ntt_variant >= 0:
        lib.fides_set_ntt_variant(cc._h, ntt_variant)
    if ks_variant >= 0:
        lib.fides_set_keyswitch_variant(cc._h, ks_variant)
    lib.fides_set_key_compression(cc._h, key_compression)
    slots = cc.N // 2
    rng = np.random.default_rng(seed)
    idx = sorted({s * (1 << k) for k in range(15) for s in (1, -1)} | {3, 5})
    offsets, bstep = list(range(64)), 8
    sk = cc.KeyGen(seed=21, hamming_weight=192)
    cc.EvalRotateKeyGen(sk, sorted(set(idx) | set(F.CryptoContext.linear_transform_rotations(offsets, bstep))))
    x = rng.uniform(-1, 1, slots) + 1j * rng.uniform(-1, 1, slots)
    ct = cc.Encrypt(sk, x, slots=slots)
    diags = {o: rng.uniform(-1, 1, slots) for o in offsets}
    offs, pts = cc.prepare_linear_transform(diags, bstep, level=ct.level, slots=slots)
    st = torch.cuda.ExternalStream(cc.stream_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        fn()
        cc.Synchronize()
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    keep = [None]

    def hoist():
        keep[0] = cc.EvalFastRotation(ct, idx)

    hoist_ms = timed(hoist)
    if profile:
        # one more hoisted call between the profiler marks, for an ncu
        # capture started with --profile-from-start off
        cc.Synchronize()
        torch.cuda.profiler.start()
        hoist()
        cc.Synchronize()
        torch.cuda.profiler.stop()
    lt_ms = timed(lambda: cc.EvalLinearTransform(ct, offs, pts, bstep, rescale=True))
    y = cc.EvalLinearTransform(ct, offs, pts, bstep, rescale=True)
    want = np.zeros(slots, dtype=np.complex128)
    for o, d in diags.items():
        want += d * np.roll(x, -o)
    err = float(np.max(np.abs(cc.Decrypt(sk, y, slots=slots) - want)))
    del keep
    cc.close()
    return {"params": "N=2^16 L=20 (60+19x40-bit) K=%d dnum=3, scale 2^40, level 19" % cc.K,
            "hoisted_rotations": len(idx), "hoisted_ms": hoist_ms, "rotations_per_s": len(idx) / (hoist_ms * 1e-3),
            "bsgs_diagonals": len(offs), "bsgs_baby_step": bstep, "bsgs_ms": lt_ms,
            "bsgs_max_abs_err_vs_fp64": err}


def measure_bootstrap(cc, reps=3, seed=101, degree=119):
    """Config 5's bootstrap: N=2^16, L=30, dnum=3, full packing (2^15 slots),
    sparse ternary secret h=32, level budget {3,3}, degree-119 Chebyshev
    EvalMod with 3 double-angle steps.  Time of one EvalBootstrap (host
    orchestration included, CUDA events on the context stream) and its
    precision in bits against the FP64 message.  Returns (result, sk, inputs)."""
    import numpy as np
    import torch

    sk = cc.KeyGen(seed=seed, hamming_weight=32)
    cc.EvalMultKeyGen(sk)
    t0 = time.perf_counter()
    cc.EvalBootstrapSetup(level_budget=(3, 3), cheb_degree=degree)
    cc.EvalBootstrapKeyGen(sk)
    cc.Synchronize()
    setup_s = time.perf_counter() - t0
    out_level, rots = cc.bootstrap_info()
    slots = cc.N // 2
    rng = np.random.default_rng(seed)
    msgs = [rng.uniform(-1, 1, slots) + 1j * rng.uniform(-1, 1, slots) for _ in range(2)]
    cts = [cc.Encrypt(sk, m, slots=slots, level=0, seed=7 + i) for i, m in enumerate(msgs)]
    bt = cc.EvalBootstrap(cts[0])
    cc.Synchronize()
    st = torch.cuda.ExternalStream(cc.stream_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    e0.record(st)
    for r in range(reps):
        bt = cc.EvalBootstrap(cts[r % 2])
    e1.record(st)
    e1.synchronize()
    wall_ms = (time.perf_counter() - w0) * 1e3 / reps
    ms = e0.elapsed_time(e1) / reps
    got = cc.Decrypt(sk, bt, slots=slots)
    err = float(np.max(np.abs(got - msgs[(reps - 1) % 2])))
    # the same with one ModDown per giant-step rotation in the transforms
    # (fides_set_giant_step_moddown scope 0) instead of one per input
    from pyfideslib_b200._capi import lib
    lib.fides_set_giant_step_moddown(cc._h, 0)
    cc.EvalBootstrap(cts[0])
    cc.Synchronize()
    e0.record(st)
    for r in range(reps):
        cc.EvalBootstrap(cts[r % 2])
    e1.record(st)
    e1.synchronize()
    ms_per_rot = e0.elapsed_time(e1) / reps
    lib.fides_set_giant_step_moddown(cc._h, 1)
    # the same with the message scaled by 2^6 through EvalMod (correction
    # factor; valid for these messages, whose coefficients are below 2^-5)
    cc.EvalBootstrapSetup(level_budget=(3, 3), cheb_degree=degree, correction=6)
    bt6 = cc.EvalBootstrap(cts[0])
    err6 = float(np.max(np.abs(cc.Decrypt(sk, bt6, slots=slots) - msgs[0])))
    cc.EvalBootstrapSetup(level_budget=(3, 3), cheb_degree=degree)
    # two iterations (the error of the first bootstrapped again at 2^12): the
    # input at the bootstrap's output level, where its residual is formed
    hi = cc.Encrypt(sk, msgs[0], slots=slots, level=out_level, seed=17)
    cc.EvalBootstrap(hi, num_iterations=2)
    cc.Synchronize()
    e0.record(st)
    bt2 = cc.EvalBootstrap(hi, num_iterations=2)
    e1.record(st)
    e1.synchronize()
    ms2 = e0.elapsed_time(e1)
    err2 = float(np.max(np.abs(cc.Decrypt(sk, bt2, slots=slots) - msgs[0])))
    del hi, bt2
    # several bootstraps in one batched call (EvalMod lanes and giant-step
    # rotations shared): time per call
    batch_ms = {}
    for nb in (2, 4):
        ins = [cts[i % 2] for i in range(nb)]
        cc.EvalBootstrapBatch(ins)
        cc.Synchronize()
        e0.record(st)
        outs_b = cc.EvalBootstrapBatch(ins)
        e1.record(st)
        e1.synchronize()
        batch_ms[nb] = e0.elapsed_time(e1)
        del outs_b
    # client side, all on the device: encode + encrypt at level 29 and
    # decrypt + decode of 2^15 slots (blocking host calls, wall clock, median
    # of 5)
    def wall(fn):
        ts = []
        for _ in range(6):
            t = time.perf_counter()
            fn()
            ts.append((time.perf_counter() - t) * 1e3)
        return float(np.median(ts[1:]))

    top = cc.Encrypt(sk, msgs[0], slots=slots, seed=19)
    client = {"encrypt_ms": wall(lambda: cc.Encrypt(sk, msgs[1], slots=slots, seed=23)),
              "decrypt_ms": wall(lambda: cc.Decrypt(sk, top, slots=slots)),
              "level": top.level, "slots": slots}
    del top
    res = {"bootstrap_ms": ms, "wall_ms": wall_ms, "client": client,
           "bootstrap_ms_moddown_per_giant_rotation": ms_per_rot, "precision_bits": -float(np.log2(err)), "max_abs_err": err,
           "precision_bits_correction6": -float(np.log2(err6)),
           "two_iterations": {"ms": ms2, "precision_bits": -float(np.log2(err2)), "input_level": out_level,
                              "output_level": out_level - 1},
           "batched_bootstrap_ms": {str(k): v for k, v in batch_ms.items()},
           "output_level": out_level, "rotation_keys": len(rots), "setup_s": setup_s,
           "params": "N=2^16 L=30 K=%d dnum=3, 2^15 slots, h=32, budget {3,3}, Chebyshev degree %d, K=16, "
                     "3 double-angle steps" % (cc.K, degree)}
    # serving's bootstrap requests: inputs at levels spread over the valid
    # range below the bootstrap's output level (ModRaise reads limb 0 only)
    boot_inputs = [cc.Encrypt(sk, msgs[lv % 2], slots=slots, level=lv, seed=31 + lv) for lv in range(0, out_level)]
    return res, sk, boot_inputs


def measure_serving(cc, rates, duration, rot_indices, seed=5, max_batch=16, num_streams=2, boot_share=0.0,
                    boot_inputs=None):
    """Poisson arrivals at each rate for `duration` seconds on resident
    ciphertexts at random levels: HMult+Relin+Rescale, Rotate and (share
    `boot_share`) EvalBootstrap.  A waiter thread retires requests in arrival
    order and drops their outputs, so device memory stays bounded by the
    requests in flight."""
    import queue

    import numpy as np

    import pyfideslib_b200 as F

    rng = np.random.default_rng(seed)
    # inputs at every level of the valid range (1..L-1: HMult consumes one),
    # two resident ciphertexts per level; requests draw a level uniformly
    pool = {}
    for lv in range(1, cc.L):
        pool[lv] = [cc.random_ct(lv, 1000 * lv + i) for i in range(2)]
    out = []
    srv = F.Server(cc, hbm_budget=40 << 30, max_batch=max_batch, num_streams=num_streams)
    p_rot = (1.0 - boot_share) / 3.0
    # the first pass warms the server's pool and the output allocations; not reported
    for k, rate in enumerate([rates[0]] + list(rates)):
        srv.reset_stats()
        q = queue.Queue()
        failures = []

        def waiter():
            while True:
                item = q.get()
                if item is None:
                    return
                try:
                    srv.wait(item[0], 300.0)
                except Exception as e:  # reported, not raised from the thread
                    failures.append(str(e))

        th = threading.Thread(target=waiter)
        th.start()
        n_sub = 0
        t_end = time.perf_counter() + duration
        t_next = time.perf_counter()
        while True:
            now = time.perf_counter()
            if now >= t_end:
                break
            if now < t_next:
                time.sleep(min(t_next - now, 0.002))
                continue
            t_next += float(rng.exponential(1.0 / rate))
            u = rng.uniform()
            if u < boot_share:
                q.put(srv.submit(F.Server.BOOTSTRAP, boot_inputs[int(rng.integers(0, len(boot_inputs)))]))
            else:
                lv = list(pool)[int(rng.integers(0, len(pool)))]
                a = pool[lv][int(rng.integers(0, 2))]
                if u < 1.0 - p_rot:
                    q.put(srv.submit(F.Server.HMULT, a, pool[lv][int(rng.integers(0, 2))]))
                else:
                    q.put(srv.submit(F.Server.ROTATE, a, None,
                                     rot_indices[int(rng.integers(0, len(rot_indices)))]))
            n_sub += 1
        q.put(None)
        th.join()
        if failures:
            raise RuntimeError("serving request failed: " + failures[0])
        st = srv.stats()
        if k == 0:
            continue
        out.append({"rate": rate, "offered": n_sub / duration, "throughput": st["throughput"],
                    "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_queue_ms": st["mean_queue_ms"],
                    "batches": st["batches"], "completed": st["completed"]})
    srv.close()
    mix = "%.0f%% HMult+Relin+Rescale, %.0f%% Rotate, %.0f%% EvalBootstrap" % (
        100 * (1 - boot_share - p_rot), 100 * p_rot, 100 * boot_share)
    params = "N=2^16 L=30 K=10 dnum=3, HMult/Rotate inputs at levels uniform in 1..29"
    if boot_share > 0 and boot_inputs:
        params += ", bootstrap inputs at levels uniform in 0..%d" % (len(boot_inputs) - 1)
    return {"mix": mix, "params": params,
            "streams": num_streams, "max_batch": max_batch, "sweep": out}


def run_reference(args):
    """The CPU implementation of the path on this host's cores (the oracle
    port, oracle/ only: FIDESlib's own CPU path is OpenFHE, not available).
    Each step is the GPU arm's workload (args.batch pairs at level 29), or a
    bounded sample of it when the whole run would take more than about four
    minutes; the pair count per step is recorded in the config."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O

    q, p = O.moduli(LOGN, L, K, DNUM)
    oc = O.Ctx(LOGN, q, p, DNUM)
    lv = L - 1
    pid = list(range(lv + 1))
    np_ = L + K
    kb = oc.random(list(range(np_)) * DNUM, 1).reshape(DNUM, np_, oc.N)
    ka = oc.random(list(range(np_)) * DNUM, 2).reshape(DNUM, np_, oc.N)
    a0, a1, b0, b1 = (oc.random(pid, s) for s in (3, 4, 5, 6))
    t0 = time.perf_counter()
    oc.hmult(lv, a0, a1, b0, b1, kb, ka, rescale=True)
    one = time.perf_counter() - t0
    pairs = max(1, min(args.batch, int(240.0 / (max(1, args.steps + args.warmup) * one))))

    def step():
        for _ in range(pairs):
            oc.hmult(lv, a0, a1, b0, b1, kb, ka, rescale=True)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    el = time.perf_counter() - t0
    val = pairs * args.steps / el
    out = {"impl": "reference", "metric": METRIC, "value": val, "unit": "HMult/s", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
           "data": "synthetic", "config": {"workload": "HMult+Relin+Rescale N=2^16 L=30 (60+29x50-bit) K=10 dnum=3, "
                                                       "level 29",
                                           "batch_pairs": pairs, "gpu_arm_batch_pairs": args.batch,
                                           "parallelism": "host threads"},
           "cpu_baseline": {"value": val, "unit": "HMult/s", "cores": O.get_threads(), "kind": "port",
                            "sample": "%d HMult+Relin+Rescale per step (the GPU arm's step has %d); FIDESlib's CPU "
                                      "path is OpenFHE (not available), so the C restatement of the path "
                                      "(oracle/oracle.c) is timed" % (pairs, args.batch)},
           "e2e": {"value": val, "unit": "HMult/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def max_over_ranks(ms, pg, device="cuda"):
    """The job's time for one timed region: the slowest rank's (an all-reduce
    MAX over the process group; the identity on one rank)."""
    if pg is None:
        return ms
    import torch

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank, world, ms):
    """Whole-job throughput: the units every rank processed over the job's
    (max-over-ranks) time in ms.  Ranks are independent replicas with the
    same per-rank work, so the job processes world x units_per_rank."""
    return units_per_rank * world / (ms * 1e-3)


def run_ours(args):
    import ctypes as C

    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist

    import pyfideslib_b200 as F
    from pyfideslib_b200._capi import lib

    cc = F.CryptoContext(log_n=LOGN, num_q=L, dnum=DNUM, num_p=K, device=local)
    lib.fides_set_key_compression(cc._h, args.key_compression)
    tv, nv = C.c_int(), C.c_int()
    tms = (C.c_float * 16)()
    lib.fides_autotune(cc._h, C.byref(tv), tms, C.byref(nv))
    cacc = C.c_int()
    cms = (C.c_float * 8)()
    lib.fides_autotune_conv_info(cc._h, C.byref(cacc), cms)
    autotune = {"ntt_variant": tv.value,
                "fwd_inv_us_3x40_limbs": [round(1e3 * tms[i], 2) for i in range(nv.value)],
                "conv_variant": ["2 coefficients/thread, 128-bit sums", "2 coefficients/thread, split 32-bit products",
                                 "1 coefficient/thread, 128-bit sums", "tensor cores (int8 split), 32 targets/MMA",
                                 "tensor cores (int8 split), 16 targets/MMA"][cacc.value],
                "modup_conv_4_elements_us": [round(1e3 * cms[i], 2) for i in range(5)]}
    # forced choices (reproducible profiler runs, where the serialised
    # launches would skew the autotuner's timings)
    if args.ntt_variant >= 0:
        lib.fides_set_ntt_variant(cc._h, args.ntt_variant)
        autotune["forced_ntt_variant"] = args.ntt_variant
    if args.conv_variant >= 0:
        lib.fides_set_conv_accumulator(cc._h, args.conv_variant)
        autotune["forced_conv_variant"] = args.conv_variant
    if args.ks_variant >= 0:
        lib.fides_set_keyswitch_variant(cc._h, args.ks_variant)
        autotune["forced_keyswitch_variant"] = args.ks_variant
    stream_ptr = C.c_void_p()
    lib.fides_ctx_stream(cc._h, C.byref(stream_ptr))
    st = torch.cuda.ExternalStream(stream_ptr.value, device=local)
    N = cc.N
    lv = L - 1
    B = args.batch
    rng = np.random.default_rng(1234 + rank)
    qs = np.array(cc.q, dtype=np.uint64)

    def rand_poly(nl, primes):
        x = rng.integers(0, 2 ** 63, size=(nl, N), dtype=np.uint64)
        return (x % np.asarray(primes, dtype=np.uint64)[:, None]).astype(np.uint64)

    np_ = L + K
    allp = cc.primes()
    kb = np.stack([rand_poly(np_, allp) for _ in range(DNUM)])
    ka = np.stack([rand_poly(np_, allp) for _ in range(DNUM)])
    cc.upload_relin_key(kb, ka)
    # pinned host inputs (e2e) and resident device inputs (value)
    host_in = []
    for i in range(B):
        pair = []
        for _ in range(2):
            t0 = torch.empty((2, lv + 1, N), dtype=torch.int64, pin_memory=True)
            arr = t0.numpy().view(np.uint64)
            arr[0] = rand_poly(lv + 1, qs[:lv + 1])
            arr[1] = rand_poly(lv + 1, qs[:lv + 1])
            pair.append((t0, arr))
        host_in.append(pair)
    host_out = [torch.empty((2, lv, N), dtype=torch.int64, pin_memory=True) for _ in range(B)]
    dev_a = [cc.upload(p[0][1][0], p[0][1][1]) for p in host_in]
    dev_b = [cc.upload(p[1][1][0], p[1][1][1]) for p in host_in]
    outs = [F.Ciphertext(cc) for _ in range(B)]

    vp = C.c_void_p
    u64p = C.POINTER(C.c_uint64)
    A_h = (vp * B)(*[x._h for x in dev_a])
    B_h = (vp * B)(*[x._h for x in dev_b])
    O_h = (vp * B)(*[o._h for o in outs])

    def step_batched():
        lib.fides_hmult_batch(cc._h, B, A_h, B_h, O_h, 1)

    def step_per_op():
        for i in range(B):
            lib.fides_hmult(cc._h, dev_a[i]._h, dev_b[i]._h, outs[i]._h, 1)

    def step_e2e():
        ha = [vp() for _ in range(B)]
        hb = [vp() for _ in range(B)]
        for i in range(B):
            a, b = host_in[i]
            lib.fides_ct_upload(cc._h, a[1][0].ctypes.data_as(u64p), a[1][1].ctypes.data_as(u64p), lv, cc.scale, 1,
                                N // 2, C.byref(ha[i]))
            lib.fides_ct_upload(cc._h, b[1][0].ctypes.data_as(u64p), b[1][1].ctypes.data_as(u64p), lv, cc.scale, 1,
                                N // 2, C.byref(hb[i]))
        lib.fides_hmult_batch(cc._h, B, (vp * B)(*[h.value for h in ha]), (vp * B)(*[h.value for h in hb]), O_h, 1)
        for i in range(B):
            ho = host_out[i].numpy().view(np.uint64)
            lib.fides_ct_download_async(cc._h, outs[i]._h, ho[0].ctypes.data_as(u64p), ho[1].ctypes.data_as(u64p))
            lib.fides_ct_free(cc._h, ha[i])
            lib.fides_ct_free(cc._h, hb[i])

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        cc.Synchronize()
        if pg:
            pg.barrier()
        n0 = lib.fides_kernel_launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(st):
            e0.record(st)
        for _ in range(steps):
            fn()
        with torch.cuda.stream(st):
            e1.record(st)
        e1.synchronize()
        cc.Synchronize()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        launches = lib.fides_kernel_launches() - n0
        return max_over_ranks(ms, pg), launches

    with ClockSampler(local) as clk:
        ms, launches = timed(step_batched, args.steps, args.warmup)
    if args.profile_step:
        # one more batched step between profiler marks: what an ncu capture
        # started with --profile-from-start off sees
        cc.Synchronize()
        torch.cuda.profiler.start()
        step_batched()
        cc.Synchronize()
        torch.cuda.profiler.stop()
    ms_op, _ = timed(step_per_op, max(1, args.steps // 2), 2)
    ms_e2e, _ = timed(step_e2e, max(1, args.steps // 2), 1)
    h2d_link_gbs = measure_h2d_link()

    # roofline: the forward NTT as the key-switch pipeline launches it, batched
    # over 32 polynomials of 30 limbs (one launch pair, 1.0 GB algorithmic
    # traffic), alternating between two resident batches (2 x 1 GB > L2); and
    # the single 30-limb polynomial for reference
    nl, nb_ntt = 30, 32
    # values below 2^40 are canonical residues of every modulus
    bufs = [torch.randint(0, 2 ** 40, (nb_ntt, nl, N), dtype=torch.int64, device="cuda") for _ in range(2)]
    stride = nl * N
    reps = 20
    for b in bufs:
        lib.fides_ntt_batch(cc._h, b.data_ptr(), stride, nb_ntt, 0, nl, 0)
    cc.Synchronize()
    # with --profile-roofline the region between the profiler marks is what an
    # ncu capture started with --profile-from-start off sees
    if args.profile_roofline:
        torch.cuda.profiler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(st):
        e0.record(st)
    for r in range(reps):
        lib.fides_ntt_batch(cc._h, bufs[r % 2].data_ptr(), stride, nb_ntt, 0, nl, 0)
    with torch.cuda.stream(st):
        e1.record(st)
    e1.synchronize()
    if args.profile_roofline:
        torch.cuda.profiler.stop()
    ntt_ms = e0.elapsed_time(e1) / reps
    traffic, traffic_source = NTT_BATCH_TRAFFIC_BYTES, NTT_BATCH_TRAFFIC_SOURCE
    if args.ntt_traffic_csv:
        traffic = ntt_traffic_from_csv(args.ntt_traffic_csv)
        traffic_source = "ncu capture " + os.path.basename(args.ntt_traffic_csv)
    # single polynomial, 30 limbs, cycling through 10 polynomials (157 MB)
    single = bufs[0].view(-1)
    cc.Synchronize()
    with torch.cuda.stream(st):
        e0.record(st)
    for r in range(40):
        lib.fides_ntt(cc._h, single.data_ptr() + (r % 10) * stride * 8, 0, nl, 0)
    with torch.cuda.stream(st):
        e1.record(st)
    e1.synchronize()
    single_us = e0.elapsed_time(e1) / 40 * 1e3
    del bufs, single
    ntt_bytes = 16.0 * N * nl * nb_ntt
    hbm, peak_kind = peaks()
    achieved = ntt_bytes / (ntt_ms * 1e-3) / 1e9

    c4 = None
    serving = None
    c3 = None
    if not args.no_c4:
        c4 = measure_c4(cc, lib, st)
    boot = None
    boot_sk, boot_cts = None, None
    if not args.no_boot:
        boot, boot_sk, boot_cts = measure_bootstrap(cc)
    if not args.no_serve:
        rot_idx = [1, 2, 4, 8, 16, 33]
        cc.EvalRotateKeyGen(boot_sk or cc.KeyGen(seed=91, hamming_weight=192), rot_idx)
        rates = [1000.0, 3000.0, 5000.0]
        serving = {"hmult_rotate": {
            "continuous_batching": measure_serving(cc, rates, 2.0, rot_idx, max_batch=8, num_streams=3),
            "per_op": measure_serving(cc, rates, 2.0, rot_idx, max_batch=1, num_streams=1)}}
        if boot is not None:
            # rates at 20 / 40 / 70% of the bootstrap lane's capacity
            cap = 1.0 / (0.1 * boot["bootstrap_ms"] * 1e-3)
            brates = [round(f * cap, 1) for f in (0.2, 0.4, 0.7)]
            serving["c5_mix_with_bootstrap"] = {
                "continuous_batching": measure_serving(cc, brates, 4.0, rot_idx, max_batch=8, num_streams=3,
                                                       boot_share=0.1, boot_inputs=boot_cts),
                "per_op": measure_serving(cc, brates, 4.0, rot_idx, max_batch=1, num_streams=1, boot_share=0.1,
                                          boot_inputs=boot_cts)}
    if not args.no_c3:
        c3 = measure_c3(ntt_variant=args.ntt_variant, ks_variant=args.ks_variant, key_compression=args.key_compression,
                        profile=args.profile_c3)
    value = job_throughput(B * args.steps, world, ms)
    per_op_value = job_throughput(B * max(1, args.steps // 2), world, ms_op)
    e2e_steps = max(1, args.steps // 2)
    e2e_val = job_throughput(B * e2e_steps, world, ms_e2e)
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            v, cores, sample = cpu_baseline_hmult(max_seconds=20.0)
            cpu = {"value": v, "unit": "HMult/s", "cores": cores, "kind": "port", "sample": sample}
        out = {"metric": METRIC, "value": value, "unit": "HMult/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "u64", "data": "synthetic",
               "per_op_value": per_op_value,
               "config": {"workload": "HMult+Relin+Rescale N=2^16 L=30 (60+29x50-bit) K=10 dnum=3, level 29",
                          "batch_pairs": B, "path": "batched (fides_hmult_batch)",
                          "l2": "inputs larger than L2 (%d MB resident)" %
                          int(B * 2 * 2 * (lv + 1) * N * 8 / 1e6), "parallelism": "replicas%d" % world},
               "e2e": {"value": e2e_val, "unit": "HMult/s",
                       "h2d_bytes_per_step": int(B * 2 * 2 * (lv + 1) * N * 8),
                       "d2h_bytes_per_step": int(B * 2 * lv * N * 8),
                       # the step's host-to-device bytes over its time, against one plain
                       # pinned 1 GiB copy on the same link
                       "h2d_link_gbs": h2d_link_gbs,
                       "h2d_frac": (B * 2 * 2 * (lv + 1) * N * 8 * e2e_steps / (ms_e2e * 1e-3) / 1e9)
                       / h2d_link_gbs if h2d_link_gbs else None},
               "roofline": {"kernel": "ntt_forward batched (32 polynomials x 30 limbs, k_ntt_fwd_cols + k_ntt_fwd_rows)",
                            "bound": "hbm", "achieved": achieved,
                            "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind,
                            "traffic": traffic, "traffic_source": traffic_source,
                            "algorithmic_bytes": ntt_bytes, "us_per_launch": ntt_ms * 1e3,
                            "single_30limb_us": single_us,
                            "single_30limb_gbs": 16.0 * N * nl / (single_us * 1e-6) / 1e9},
               "ntt_gbs": achieved,
               "gpu_launches": int(launches),
               "autotune": autotune,
               "batched_uneven_c4": c4,
               "hoisted_bsgs_c3": c3,
               "bootstrap_c5": boot,
               "serving_c5": serving,
               "clocks": clk.summary(),
               "cpu_baseline": cpu}
        print(json.dumps(out), flush=True)
    for o in outs:
        del o
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-c4", action="store_true", help="skip the config-4 graph-plan measurement")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving measurement")
    ap.add_argument("--no-c3", action="store_true", help="skip the config-3 hoisted/BSGS measurement")
    ap.add_argument("--no-boot", action="store_true", help="skip the bootstrap measurement")
    ap.add_argument("--ntt-variant", type=int, default=-1, help="force a forward NTT variant (default: tuned)")
    ap.add_argument("--conv-variant", type=int, default=-1, help="force a base-conversion variant (default: tuned)")
    ap.add_argument("--ks-variant", type=int, default=-1,
                    help="force the key-switch inner product: bit 0 FP64 sums, bit 1 fused into the NTT row pass, "
                         "bit 2 fused for batches of 8+, bit 3 the fused row pass in two launches (default: the context's, 13)")
    ap.add_argument("--profile-roofline", action="store_true",
                    help="mark the roofline NTT loop for ncu --profile-from-start off")
    ap.add_argument("--key-compression", type=int, default=1, choices=[0, 1, 2, 3],
                    help="keys generated store b and the seed of a, a bit mask: bit 0 rotation keys "
                         "(1, the default), bit 1 the relinearisation key; 0 stores both halves")
    ap.add_argument("--ntt-traffic-csv", default=None,
                    help="ncu --csv log with dram__bytes_read.sum and dram__bytes_write.sum of the roofline "
                         "NTT pair (--profile-roofline); its last pair gives roofline.traffic")
    ap.add_argument("--profile-c3", action="store_true",
                    help="mark one call of config 3's 32 hoisted rotations for ncu --profile-from-start off")
    ap.add_argument("--profile-step", action="store_true",
                    help="mark one batched HMult step (after the timed region) for ncu --profile-from-start off")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

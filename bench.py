#!/usr/bin/env python
"""Benchmark of the Spartan+WHIR prover on B200.

Default (the headline line): whole proofs of a synthetic 2^20-constraint R1CS
(2^18 inputs, witness padded to 2^21) -- the WHIR commitment of the witness
(RS encode at rate 1/4 + Skyscraper Merkle tree, OOD sample), the Spartan
zk-sumcheck, the covector evaluations and WHIR's prove rounds -- bit-exact
with the CPU restatement; proofs/s and p50/p99 latency.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload prove|commit|batched|served|ntt|whir_ops|poseidon2|dual]

N > 1 runs under torchrun: every rank proves its own instance (independent
replicas, no data-path collective); time = max over ranks.  Prints one JSON
line on rank 0.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PROVE_METRIC = ("Spartan+WHIR proofs/s & p99 latency @2^20-constraint R1CS (whole proof: WHIR-ZK "
                "commit, zk-sumcheck, covector evaluations, WHIR rounds; plain GPU; bit-exact "
                "with the C restatement of the prover)")
PROVE_UNIT = "proofs/s"
METRIC = ("WHIR commit throughput, Spartan+WHIR prover hot path: 2^20 Fr coefficients -> "
          "RS rate-1/4 coset NTT -> 2^22 evaluations -> Skyscraper Merkle tree (bit-exact)")
UNIT = "commits/s"
IMAD_PER_MONT = 264  # mad.lo/madc.hi/mul.lo per 8x32 CIOS product (fr.cuh: 8 x (16 + 16 + 1))
# binary64 instructions per Fr operation of the FP64-pipe routines (fr_f64.cuh):
# digit conversion 11 per operand, digit products (121 general, 66 + 10
# doublings for a square), ten 24-bit Montgomery steps of 14, and the 16-bit
# step plus normalisation (69).
F64_PER_MUL = 22 + 121 + 140 + 69      # 352
F64_PER_SQR = 11 + 66 + 10 + 140 + 69  # 296
# integer multiply-adds of one Montgomery->canonical REDC (fr.cuh
# fr_from_mont: 8 x (1 + 16)); B200 runs them on the same throughput as the
# binary64 fmas (a kernel mixing the two runs at the rate of either alone),
# so the leaf kernel's multiply work is its squarings plus these.
IMAD_PER_REDC = 8 * (1 + 16)  # 136
# dram__bytes_read.sum + dram__bytes_write.sum of one leaf_fold_fr_kernel launch
# from an ncu capture of this workload (the leaf kernel's WHIR-commit profile
# summary under profiles/), keyed by (log2 coeffs, folding factor, log inv rate).
LEAF_TRAFFIC_BYTES = {(20, 4, 2): 134.264064e6 + 6.855168e6}
# the same for the whole proof's witness commitment (whir-ZK: 2^20 leaves of
# 16 Fr, the witness and blinding polynomials of m = 21 at rate 1/4), from an
# ncu capture of the default command (the leaf kernel's whole-proof profile
# summary under profiles/).
LEAF_TRAFFIC_PROVE_BYTES = 537195264 + 33959680


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--log-coeffs", type=int, default=20)
    p.add_argument("--folding-factor", type=int, default=4)
    p.add_argument("--log-inv-rate", type=int, default=2)
    p.add_argument("--seed", type=int, default=2)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-plugin-e2e", action="store_true")
    p.add_argument("--no-targets", action="store_true",
                   help="prove: skip the 2^24 NTT, batched, two-commitment and served "
                        "measurements after the headline")
    p.add_argument("--workload", choices=["commit", "prove", "batched", "served", "ntt", "whir_ops",
                                          "poseidon2", "dual"],
                   default="prove",
                   help="prove (default, the headline line): whole proofs of a 2^20-constraint "
                        "R1CS; commit: WHIR commit of 2^20 coefficients; batched: 256 uneven "
                        "jobs as one CUDA graph vs the same jobs one at a time; served: Poisson "
                        "stream of whole proofs; dual: two-commitment proofs of a 2^20-constraint "
                        "R1CS with 16 verifier challenges")
    p.add_argument("--jobs", type=int, default=256)
    p.add_argument("--tune", action="store_true", help="batched: run the NTT radix autotuner first")
    p.add_argument("--requests", type=int, default=32, help="served: requests per arrival rate")
    p.add_argument("--clock-ms", type=int, default=200, help="nvidia-smi sampling interval")
    return p.parse_args()


def workload_config(a):
    return {"workload": "whir_commit", "log2_coeffs": a.log_coeffs,
            "folding_factor": a.folding_factor, "log_inv_rate": a.log_inv_rate,
            "leaf_fr": 1 << a.folding_factor,
            "num_leaves": (1 << (a.log_coeffs - a.folding_factor)) << a.log_inv_rate,
            "leaf_encoding": "canonical", "seed": a.seed,
            "l2": "flushed: 256 MiB device write between timed steps (outside the step events)",
            "parallelism": f"replicas x{a.gpus}"}


# ---------------------------------------------------------------------------
# CPU arm: the oracle restatement (the reference is Rust and cannot be built
# here), OpenMP over all host threads.
# ---------------------------------------------------------------------------
def cpu_commit_once(O, coeffs_np, a):
    import numpy as np
    M = 1 << a.folding_factor
    L = coeffs_np.shape[0] // M
    cw_len = L << a.log_inv_rate
    out = np.zeros((M * cw_len, 4), np.uint64)
    rc = O.lib().pko_rs_interleaved_encode(O.p64(coeffs_np), M, L, O.p64(coeffs_np), 0, cw_len,
                                           O.p64(out))
    assert rc == 0
    O.lib().pko_from_mont_many(O.p64(out), out.shape[0])
    layers = np.zeros(32 * (2 * cw_len - 1), np.uint8)
    rc = O.lib().pko_merkle_tree(O.p8(out.view(np.uint8).reshape(-1)), 32 * M, cw_len, O.p8(layers))
    assert rc == 0
    return layers[-32:]


def cpu_baseline_measure(a, samples=1):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    coeffs = O.sample_fr(a.seed, 1 << a.log_coeffs)
    t0 = time.perf_counter()
    cpu_commit_once(O, coeffs, a)
    dt = (time.perf_counter() - t0) / 1.0
    times = [dt]
    for _ in range(samples - 1):
        t0 = time.perf_counter()
        cpu_commit_once(O, coeffs, a)
        times.append(time.perf_counter() - t0)
    return statistics.median(times), O.lib().pko_num_threads()


def commit_products(log_coeffs, ff, lr):
    """Montgomery products of one commit: NTT butterflies + leaf hashing
    (14 squarings per compression, one conversion per Fr) + tree levels."""
    n = 1 << log_coeffs
    M = 1 << ff
    cw_len = (n >> ff) << lr
    ntt = (cw_len * M // 2) * (log_coeffs - ff)
    leaves = cw_len * ((M - 1) * 14 + M)
    levels = (cw_len - 1) * 14
    return ntt + leaves + levels


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import copy
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    coeffs = O.sample_fr(a.seed, 1 << a.log_coeffs)
    t0 = time.perf_counter()
    cpu_commit_once(O, coeffs, a)
    t_full = time.perf_counter() - t0
    budget_s = 180.0
    shrink = 0
    while t_full / (1 << shrink) * (a.steps + a.warmup) > budget_s and shrink < a.log_coeffs - a.folding_factor - 2:
        shrink += 1
    s = copy.copy(a)
    s.log_coeffs = a.log_coeffs - shrink
    scale = commit_products(s.log_coeffs, a.folding_factor, a.log_inv_rate) / commit_products(
        a.log_coeffs, a.folding_factor, a.log_inv_rate)
    sample_coeffs = coeffs[: 1 << s.log_coeffs]
    for _ in range(max(a.warmup - 1, 0)):
        cpu_commit_once(O, sample_coeffs, s)
    times = []
    for _ in range(a.steps):
        t0 = time.perf_counter()
        cpu_commit_once(O, sample_coeffs, s)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = scale * a.steps / total
    cores = O.lib().pko_num_threads()
    if shrink:
        sample = (f"each step commits a 2^{s.log_coeffs}-coefficient polynomial (same folding factor "
                  f"and rate); throughput scaled to the 2^{a.log_coeffs} workload by Montgomery-"
                  f"product count (x{scale:.5f}); one full commit took {t_full:.2f} s")
    else:
        sample = "full workload per step"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64 (BN254 Fr)",
        "data": "synthetic (ChaCha20-seeded Fr)", "config": workload_config(a),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample + "; C restatement of RSFr::interleaved_encode + the "
                                   "SkyscraperHashEngine tree, OpenMP, not the reference binary "
                                   "(no Rust toolchain)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Clock sampling during the timed region.
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index, interval_ms=200):
        self.gpu_index = gpu_index
        self.interval_ms = interval_ms
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu_index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", str(self.interval_ms)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def physical_gpu_index(local_rank):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x.strip() for x in vis.split(",") if x.strip()]
        if local_rank < len(ids) and ids[local_rank].isdigit():
            return int(ids[local_rank])
    return local_rank


# ---------------------------------------------------------------------------
# GPU arm.
# ---------------------------------------------------------------------------
def run_b200(a):
    import numpy as np
    import torch

    from provekit_b200 import _lib
    from provekit_b200._lib import PKG_LEAF_CANONICAL, check
    from provekit_b200.replicas import max_over_ranks

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world != a.gpus:
        raise SystemExit(f"--gpus {a.gpus} but WORLD_SIZE={world}")
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    L = _lib.lib()
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream

    M = 1 << a.folding_factor
    n = 1 << a.log_coeffs
    msg_len = n // M
    cw_len = msg_len << a.log_inv_rate
    total_fr = cw_len * M

    h_coeffs = np.zeros((n, 4), np.uint64)
    check(L.pkg_sample_fr(a.seed + 1000 * rank, n, h_coeffs.ctypes.data, 1))
    pinned = torch.from_numpy(h_coeffs.view(np.int64)).pin_memory()
    d_coeffs = pinned.to(f"cuda:{local_rank}")
    d_cw = torch.empty((total_fr, 4), dtype=torch.int64, device=d_coeffs.device)
    d_layers = torch.empty(32 * (2 * cw_len - 1), dtype=torch.uint8, device=d_coeffs.device)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=d_coeffs.device)
    root_host = torch.empty(32, dtype=torch.uint8).pin_memory()
    check(L.pkg_ntt_engine_reserve(cw_len))

    def step():
        check(L.pkg_rs_interleaved_encode(d_coeffs.data_ptr(), M, msg_len, None, 0, cw_len,
                                          d_cw.data_ptr(), sh))
        ev[1].record(stream)
        check(L.pkg_merkle_leaves_fr(d_cw.data_ptr(), M, cw_len, PKG_LEAF_CANONICAL,
                                     d_layers.data_ptr(), sh))
        ev[2].record(stream)
        check(L.pkg_merkle_levels(d_layers.data_ptr(), cw_len, sh))

    # warm-up
    with torch.cuda.stream(stream):
        for _ in range(max(a.warmup, 0)):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            flush.zero_()
            step()
    stream.synchronize()

    events = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(a.steps)]
    clocks = ClockSampler(physical_gpu_index(local_rank))
    clocks.start()
    time.sleep(0.3)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = L.pkg_kernel_launches()
    with torch.cuda.stream(stream):
        for i in range(a.steps):
            ev = events[i]
            flush.zero_()
            ev[0].record(stream)
            step()
            ev[3].record(stream)
    stream.synchronize()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    launches = L.pkg_kernel_launches() - launches0
    clk = clocks.stop()

    step_ms = [e[0].elapsed_time(e[3]) for e in events]
    enc_ms = [e[0].elapsed_time(e[1]) for e in events]
    leaf_ms = [e[1].elapsed_time(e[2]) for e in events]
    lvl_ms = [e[2].elapsed_time(e[3]) for e in events]
    total_ms = sum(step_ms)
    total_ms_max = max_over_ranks(total_ms, device=d_coeffs.device)

    # ---- end to end through the C ABI: pinned host coefficients in, root out
    e2e_events = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(a.steps)]
    with torch.cuda.stream(stream):
        for i in range(a.warmup + a.steps):
            flush.zero_()
            if i >= a.warmup:
                e2e_events[i - a.warmup][0].record(stream)
            d_coeffs.copy_(pinned, non_blocking=True)
            check(L.pkg_whir_commit(d_coeffs.data_ptr(), n, a.folding_factor, a.log_inv_rate, None,
                                    0, PKG_LEAF_CANONICAL, d_cw.data_ptr(), d_layers.data_ptr(), sh))
            root_host.copy_(d_layers[-32:], non_blocking=True)
            if i >= a.warmup:
                e2e_events[i - a.warmup][1].record(stream)
    stream.synchronize()
    e2e_ms = sum(e[0].elapsed_time(e[1]) for e in e2e_events)
    e2e_ms_max = max_over_ranks(e2e_ms, device=d_coeffs.device)

    # ---- the same calls pipelined over two streams and two buffer sets, as a
    # prover serving a stream of commitments runs them: step i+1's H2D copy
    # and first kernels overlap step i's tree; every step still copies its
    # own coefficients in and its own root out.
    dev = d_coeffs.device
    sets = [(d_coeffs, d_cw, d_layers, root_host, stream)]
    sets.append((torch.empty_like(d_coeffs), torch.empty_like(d_cw), torch.empty_like(d_layers),
                 torch.empty(32, dtype=torch.uint8).pin_memory(), torch.cuda.Stream(device=dev)))

    def pipelined_step(i):
        dc, dcw, dl, rh, st = sets[i % 2]
        with torch.cuda.stream(st):
            dc.copy_(pinned, non_blocking=True)
            check(L.pkg_whir_commit(dc.data_ptr(), n, a.folding_factor, a.log_inv_rate, None, 0,
                                    PKG_LEAF_CANONICAL, dcw.data_ptr(), dl.data_ptr(),
                                    st.cuda_stream))
            rh.copy_(dl[-32:], non_blocking=True)

    for i in range(a.warmup):
        pipelined_step(i)
    torch.cuda.synchronize()
    p_start = torch.cuda.Event(enable_timing=True)
    p_start.record(sets[0][4])
    sets[1][4].wait_event(p_start)
    for i in range(a.steps):
        pipelined_step(i)
    p_end = [torch.cuda.Event(enable_timing=True) for _ in sets]
    for ev, st in zip(p_end, sets):
        ev.record(st[4])
    torch.cuda.synchronize()
    pipe_ms = max(p_start.elapsed_time(ev) for ev in p_end)
    pipe_ms_max = max_over_ranks(pipe_ms, device=dev)
    root_ok = bytes(sets[0][3].numpy()) == bytes(sets[1][3].numpy()) == bytes(root_host.numpy())

    # ---- device-resident, pipelined: the same commits with the coefficients
    # already in HBM (one copy per buffer set before timing), alternating
    # streams so that one step's latency-bound tree overlaps the next step's
    # transform.  Reported beside `value`, which stays the one-step-at-a-time
    # figure with an L2 flush between steps.
    for dc, _, _, _, st in sets:
        with torch.cuda.stream(st):
            dc.copy_(pinned, non_blocking=True)
    torch.cuda.synchronize()

    def resident_step(i):
        dc, dcw, dl, _, st = sets[i % 2]
        check(L.pkg_whir_commit(dc.data_ptr(), n, a.folding_factor, a.log_inv_rate, None, 0,
                                PKG_LEAF_CANONICAL, dcw.data_ptr(), dl.data_ptr(), st.cuda_stream))

    for i in range(a.warmup):
        resident_step(i)
    torch.cuda.synchronize()
    r_start = torch.cuda.Event(enable_timing=True)
    r_start.record(sets[0][4])
    sets[1][4].wait_event(r_start)
    for i in range(a.steps):
        resident_step(i)
    r_end = [torch.cuda.Event(enable_timing=True) for _ in sets]
    for ev, st in zip(r_end, sets):
        ev.record(st[4])
    torch.cuda.synchronize()
    res_ms_max = max_over_ranks(max(r_start.elapsed_time(ev) for ev in r_end), device=dev)

    # ---- the trait-shaped drop-in: host slices through RSFr / HashEngine
    plugin = None
    if not a.no_plugin_e2e:
        msgs = [np.ascontiguousarray(h_coeffs[j * msg_len:(j + 1) * msg_len]) for j in range(M)]
        ptrs = (ctypes.c_void_p * M)(*[m.ctypes.data for m in msgs])
        out_cw = np.zeros((total_fr, 4), np.uint64)
        digests = np.zeros(32 * cw_len, np.uint8)

        def plugin_commit():
            check(L.pkg_host_rs_interleaved_encode(ctypes.cast(ptrs, ctypes.c_void_p), M, msg_len,
                                                   None, 0, cw_len, out_cw.ctypes.data))
            check(L.pkg_host_skyscraper_hash_many(32 * M, out_cw.ctypes.data, cw_len,
                                                  digests.ctypes.data))
            level = digests
            while level.size > 32:
                nxt = np.zeros(level.size // 2, np.uint8)
                check(L.pkg_host_skyscraper_hash_many(64, level.ctypes.data, level.size // 64,
                                                      nxt.ctypes.data))
                level = nxt
            return level

        plugin_commit()
        pt = []
        for _ in range(min(a.steps, 5)):
            t0 = time.perf_counter()
            plugin_commit()
            pt.append(time.perf_counter() - t0)
        plugin = {"value": len(pt) / sum(pt), "unit": UNIT,
                  "h2d_bytes_per_step": 32 * n + 32 * total_fr + 32 * cw_len,
                  "d2h_bytes_per_step": 32 * total_fr + 32 * cw_len + 32 * (cw_len - 1),
                  "note": "wall clock, host-slice plugin calls (pkg_host_rs_interleaved_encode + "
                          "pkg_host_skyscraper_hash_many per level), raw Montgomery leaf bytes"}

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    # ---- roofline of the dominant kernel (Merkle leaf fold): its Fr
    # arithmetic runs on the FP64 pipe, so the bound is the measured fma rate
    # over the binary64 instructions the squarings and conversions need.
    imad = ctypes.c_double(0)
    check(L.pkg_measure_imad_rate(ctypes.byref(imad)))
    dfma = ctypes.c_double(0)
    check(L.pkg_measure_dfma_rate(ctypes.byref(dfma)))
    mont_peak = imad.value / IMAD_PER_MONT
    num_leaves = cw_len
    mont_per_leaf_launch = num_leaves * ((M - 1) * 14 + M)
    # the squarings' binary64 instructions plus the M Montgomery->canonical
    # REDCs per leaf (integer multiply-adds on the same shared throughput)
    f64_per_leaf_launch = num_leaves * ((M - 1) * 14 * F64_PER_SQR + M * IMAD_PER_REDC)
    leaf_avg_s = statistics.mean(leaf_ms) * 1e-3
    achieved = mont_per_leaf_launch / leaf_avg_s
    f64_achieved = f64_per_leaf_launch / leaf_avg_s
    ntt_stages = (msg_len << a.log_inv_rate).bit_length() - 1 - a.log_inv_rate
    ntt_mont = (total_fr // 2) * ntt_stages
    enc_avg_s = statistics.mean(enc_ms) * 1e-3

    cpu = None
    if not a.no_cpu_baseline:
        cpu_s, cores = cpu_baseline_measure(a)
        cpu = {"value": 1.0 / cpu_s, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": "one full 2^20-coefficient commit on the host (C restatement, OpenMP); "
                         "not the reference binary (no Rust toolchain)"}

    value = a.gpus * a.steps / (total_ms_max * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": total_ms_max / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32 (BN254 Fr, 8x32-bit limbs)",
        "data": "synthetic (ChaCha20-seeded uniform Fr, Montgomery form)",
        "config": workload_config(a),
        "roofline": {
            "kernel": "leaf_fold_fr_kernel (Skyscraper leaf hashing)", "bound": "fp64",
            "achieved": f64_achieved / 1e12, "peak": dfma.value / 1e12, "unit": "T multiply-op/s",
            "frac": f64_achieved / dfma.value,
            "traffic": LEAF_TRAFFIC_BYTES.get((a.log_coeffs, a.folding_factor, a.log_inv_rate)),
            "traffic_algorithmic": 32 * total_fr + 32 * num_leaves,
            "peak_source": f"measured binary64 fma rate {dfma.value / 1e12:.3f} T/s "
                           "(pkg_measure_dfma_rate, this GPU, this run)",
            "algorithmic": f"{num_leaves} leaves x ({M - 1} compressions x 14 squarings x "
                           f"{F64_PER_SQR} binary64 instructions + {M} Montgomery->canonical "
                           f"REDCs x {IMAD_PER_REDC} integer multiply-adds) = "
                           f"{f64_per_leaf_launch} multiply-pipe instructions per launch "
                           f"({mont_per_leaf_launch} Fr products and REDCs); the integer "
                           "multiply-adds share the binary64 fma throughput on B200",
            "achieved_gmont_per_s": achieved / 1e9,
            "int_pipe_alt": {"peak_gmont_per_s": mont_peak / 1e9, "frac": achieved / mont_peak,
                             "note": f"the same products against the IMAD roofline (measured "
                                     f"{imad.value / 1e12:.3f} T/s / {IMAD_PER_MONT} per CIOS "
                                     "product), the bound of the integer-pipe routines"},
        },
        "kernels": {
            "rs_encode_ms": statistics.mean(enc_ms), "merkle_leaves_ms": statistics.mean(leaf_ms),
            "merkle_levels_ms": statistics.mean(lvl_ms),
            "share": {"rs_encode": sum(enc_ms) / total_ms, "merkle_leaves": sum(leaf_ms) / total_ms,
                      "merkle_levels": sum(lvl_ms) / total_ms},
            "ntt_gmont_per_s": ntt_mont / enc_avg_s / 1e9,
            "encode_hbm_gbs": 32 * (n + 2 * total_fr) / enc_avg_s / 1e9,
        },
        "cpu_baseline": cpu,
        "e2e": {"value": a.gpus * a.steps / (pipe_ms_max * 1e-3), "unit": UNIT,
                "h2d_bytes_per_step": 32 * n, "d2h_bytes_per_step": 32,
                "note": "every step copies its 2^20 coefficients from pinned host memory, calls "
                        "pkg_whir_commit and reads its root back; steps alternate between two "
                        "streams and buffer sets, so copies overlap the previous step's kernels; "
                        "device-timed from the first copy to the last root; no L2 flush (inputs "
                        "arrive over PCIe, the two buffer sets span 2 x 176 MiB)",
                "roots_agree": root_ok,
                "serial": {"value": a.gpus * a.steps / (e2e_ms_max * 1e-3),
                           "note": "the same calls one step at a time on one stream, L2 flushed "
                                   "between steps (outside the timed region)"}},
        "value_pipelined": {"value": a.gpus * a.steps / (res_ms_max * 1e-3), "unit": UNIT,
                            "note": "inputs resident in HBM, steps alternating over two streams "
                                    "and buffer sets (2 x 176 MiB, larger than L2), no flush; "
                                    "one step's tree overlaps the next step's transform"},
        "e2e_plugin": plugin,
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# The headline: whole proofs of a synthetic 2^20-constraint R1CS.
# ---------------------------------------------------------------------------
PROVE_NC, PROVE_NI = 1 << 20, 1 << 18


def prove_config(a, h, wp, proof_bytes=None):
    return {"workload": "prove_r1cs", "num_constraints": PROVE_NC, "num_inputs": PROVE_NI,
            "num_witnesses": h.num_witnesses, "whir_num_variables": wp.num_variables,
            "folding_factor": wp.folding_factor, "log_inv_rate": wp.log_inv_rate,
            "security_bits": 128, "pow_bits": wp.pow_bits, "whir_rounds": wp.num_rounds,
            "whir_zk": wp.batch_size == 2,
            "whir_batch": f"{wp.batch_size} (the witness with a blinding polynomial)"
            if wp.batch_size == 2 else "1",
            "queries": list(wp.queries[:wp.num_rounds + 1]), "proof_bytes": proof_bytes,
            "seed": a.seed, "parallelism": f"replicas x{a.gpus}",
            "l2": "flushed: 256 MiB device write between timed steps (outside the step events); "
                  "a proof's working set (~1 GB) is larger than L2 as well"}


def run_prove(a):
    import numpy as np
    import torch

    from provekit_b200 import _lib
    from provekit_b200._lib import PKG_LEAF_CANONICAL, check
    from provekit_b200.prover import HostR1CS, prove_r1cs, spartan_prove, whir_params_for
    from provekit_b200.replicas import max_over_ranks

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world != a.gpus:
        raise SystemExit(f"--gpus {a.gpus} but WORLD_SIZE={world}")
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    L = _lib.lib()
    dev = torch.device("cuda", local_rank)
    t0 = time.perf_counter()
    h = HostR1CS(a.seed + 1000 * rank, PROVE_NC, PROVE_NI)
    gen_s = time.perf_counter() - t0
    d = h.to_device(dev)
    wp = whir_params_for(d)  # ff 3, rate 1/4, 128 bits, 10 PoW bits: m = 21
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    w_pinned = torch.from_numpy(h.witness.view(np.int64)).pin_memory()
    w_dev = torch.empty_like(d.witness)

    with torch.cuda.stream(stream):
        for _ in range(a.warmup):
            flush.zero_()
            prove_r1cs(d, wp, stream=stream)
    stream.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(a.steps)]
    clocks = ClockSampler(physical_gpu_index(local_rank), a.clock_ms)
    clocks.start()
    time.sleep(0.3)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = L.pkg_kernel_launches()
    with torch.cuda.stream(stream):
        for i in range(a.steps):
            flush.zero_()
            evs[i][0].record(stream)
            last = prove_r1cs(d, wp, stream=stream)
            evs[i][1].record(stream)
    stream.synchronize()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    launches = L.pkg_kernel_launches() - launches0
    clk = clocks.stop()
    ms = [e[0].elapsed_time(e[1]) for e in evs]
    total_max = max_over_ranks(sum(ms), device=dev)
    p50_max = max_over_ranks(statistics.median(ms), device=dev)
    p99_max = max_over_ranks(sorted(ms)[min(len(ms) - 1, int(np.ceil(0.99 * len(ms))) - 1)],
                             device=dev)
    stages = (ctypes.c_double * 6)()
    L.pkg_last_prove_stages(stages)
    stage_ms = dict(zip(["commit", "witness_bounds", "zk_sumcheck", "eq_alpha",
                         "transposed_products", "whir_rounds"], list(stages)))
    wst = (ctypes.c_double * 8)()
    L.pkg_last_whir_stages(wst)
    whir_ms = dict(zip(["setup", "sumcheck", "fold_commit", "ood", "pow", "stir_openings",
                        "weight_updates", "final_poly"], list(wst)))

    # the Spartan part alone (the work before whir's prove call)
    core = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(min(a.steps, 5))]
    with torch.cuda.stream(stream):
        for c in core:
            c[0].record(stream)
            spartan_prove(d, stream=stream)
            c[1].record(stream)
    stream.synchronize()
    core_ms = statistics.mean(c[0].elapsed_time(c[1]) for c in core)

    # e2e through the public call: the witness copied from pinned host memory
    # every step, the proof written back to host memory by the call
    e2e_ev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(a.steps)]
    with torch.cuda.stream(stream):
        for i in range(a.steps):
            flush.zero_()
            e2e_ev[i][0].record(stream)
            w_dev.copy_(w_pinned, non_blocking=True)
            prove_r1cs(d, wp, witness=w_dev, stream=stream)
            e2e_ev[i][1].record(stream)
    stream.synchronize()
    e2e_serial_max = max_over_ranks(sum(e[0].elapsed_time(e[1]) for e in e2e_ev), device=dev)

    # the same calls with the next witness's copy (pinned host memory, a copy
    # stream, two device buffers) running under the current proof: every
    # step still copies its witness in and its proof out inside the timed
    # region, which runs from the first copy's start to the last proof's end
    copy_stream = torch.cuda.Stream(device=dev)
    w2 = [w_dev, torch.empty_like(d.witness)]
    copied = [torch.cuda.Event() for _ in range(2)]
    p_start, p_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    flush.zero_()
    torch.cuda.synchronize()
    p_start.record(copy_stream)
    with torch.cuda.stream(copy_stream):
        w2[0].copy_(w_pinned, non_blocking=True)
    copied[0].record(copy_stream)
    for i in range(a.steps):
        if i + 1 < a.steps:  # proof i - 1 has returned: its buffer is free
            with torch.cuda.stream(copy_stream):
                w2[(i + 1) % 2].copy_(w_pinned, non_blocking=True)
            copied[(i + 1) % 2].record(copy_stream)
        stream.wait_event(copied[i % 2])
        with torch.cuda.stream(stream):
            prove_r1cs(d, wp, witness=w2[i % 2], stream=stream)
    p_end.record(stream)
    torch.cuda.synchronize()
    e2e_max = max_over_ranks(p_start.elapsed_time(p_end), device=dev)

    # the batched comparison of the metric: one resident circuit, many
    # witnesses -- 4 host threads, each with its own stream and witness
    # buffer, prove concurrently (witness copied from pinned host memory and
    # proof written back per proof, as in e2e), so that one proof's host
    # round trips overlap the others' kernels
    nthr, per = 4, max(a.steps // 4, 2)
    check(L.pkg_reserve_memory(nthr * (3 << 30)))  # four proofs' working sets, mapped up front
    bstreams = [torch.cuda.Stream(device=dev) for _ in range(nthr)]
    bw = [torch.empty_like(d.witness) for _ in range(nthr)]
    blat = [[] for _ in range(nthr)]
    bdone = [[] for _ in range(nthr)]  # completion times from the common start
    t_common = [0.0]

    def batch_worker(j, count):
        torch.cuda.set_device(dev)
        for i in range(count):
            t1 = time.perf_counter()
            with torch.cuda.stream(bstreams[j]):
                bw[j].copy_(w_pinned, non_blocking=True)
                prove_r1cs(d, wp, witness=bw[j], blinding_seed=1 + i, stream=bstreams[j])
            t2 = time.perf_counter()
            blat[j].append((t2 - t1) * 1e3)
            bdone[j].append((t2 - t_common[0]) * 1e3)

    th = [threading.Thread(target=batch_worker, args=(j, 1)) for j in range(nthr)]  # warm-up
    for t in th:
        t.start()
    for t in th:
        t.join()
    blat = [[] for _ in range(nthr)]
    bdone = [[] for _ in range(nthr)]
    torch.cuda.synchronize()
    # the same requests (all arriving at once) proved one at a time by one
    # thread: completion times from the common start
    nreq = nthr * per
    seq_done = []
    t0 = time.perf_counter()
    with torch.cuda.stream(bstreams[0]):
        for i in range(nreq):
            bw[0].copy_(w_pinned, non_blocking=True)
            prove_r1cs(d, wp, witness=bw[0], blinding_seed=1 + i, stream=bstreams[0])
            seq_done.append((time.perf_counter() - t0) * 1e3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    t_common[0] = t0
    th = [threading.Thread(target=batch_worker, args=(j, per)) for j in range(nthr)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    torch.cuda.synchronize()
    batched_s = time.perf_counter() - t0
    batched_max = max_over_ranks(batched_s, device=dev)
    lat = sorted(x for v in blat for x in v)
    done_b = [x for v in bdone for x in v]

    # the dominant kernel (Merkle leaf hashing of the witness commitment:
    # 2^20 leaves of 8 Fr) timed on its own with CUDA events, L2 flushed
    M = (1 << wp.folding_factor) * wp.batch_size  # Fr per leaf of the witness commitment
    msg_len = (wp.batch_size << wp.num_variables) // M
    rows = msg_len << wp.log_inv_rate
    coeffs = torch.empty((wp.batch_size << wp.num_variables, 4), dtype=torch.int64, device=dev)
    hc = np.zeros((coeffs.shape[0], 4), np.uint64)
    check(L.pkg_sample_fr(a.seed + 7, hc.shape[0], hc.ctypes.data, 1))
    coeffs.copy_(torch.from_numpy(hc.view(np.int64)))
    cw = torch.empty((rows * M, 4), dtype=torch.int64, device=dev)
    layers = torch.empty(32 * (2 * rows - 1), dtype=torch.uint8, device=dev)
    sh = stream.cuda_stream
    check(L.pkg_rs_interleaved_encode(coeffs.data_ptr(), M, msg_len, None, 0, rows,
                                      cw.data_ptr(), sh))
    leaf_ev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(8)]
    with torch.cuda.stream(stream):
        for i in range(2 + len(leaf_ev)):
            flush.zero_()
            if i >= 2:
                leaf_ev[i - 2][0].record(stream)
            check(L.pkg_merkle_leaves_fr(cw.data_ptr(), M, rows, PKG_LEAF_CANONICAL,
                                         layers.data_ptr(), sh))
            if i >= 2:
                leaf_ev[i - 2][1].record(stream)
    stream.synchronize()
    leaf_s = statistics.mean(e[0].elapsed_time(e[1]) for e in leaf_ev) * 1e-3
    del coeffs, cw, layers

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    dfma = ctypes.c_double(0)
    check(L.pkg_measure_dfma_rate(ctypes.byref(dfma)))
    f64_per_launch = rows * ((M - 1) * 14 * F64_PER_SQR + M * IMAD_PER_REDC)
    f64_achieved = f64_per_launch / leaf_s

    cpu = None
    parity = {"result": "not checked in this run (the oracle leg runs on rank 0 at N=1 only)"}
    if not a.no_cpu_baseline and a.gpus == 1:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib as O
        owp = O.whir_params(wp.num_variables, wp.folding_factor, wp.log_inv_rate, 128, wp.pow_bits,
                            batch_size=wp.batch_size)
        t0 = time.perf_counter()
        esp, ecw, eproof = O.prove_r1cs(h, 1, 3, owp)
        cpu_s = time.perf_counter() - t0
        cpu = {"value": 1.0 / cpu_s, "unit": PROVE_UNIT, "cores": O.lib().pko_num_threads(),
               "kind": "port",
               "sample": "one whole proof of the same 2^20-constraint instance on the host (C "
                         "restatement, OpenMP); not the reference binary (no Rust toolchain)"}
        # the last timed proof (blinding seed 1, domain 3) against the
        # oracle's proof of the same instance, field by field and word by word
        gsp, gcw, gproof = last
        same = (all(np.array_equal(gsp[k], esp[k]) if isinstance(gsp[k], np.ndarray)
                    else gsp[k] == esp[k] for k in esp)
                and np.array_equal(gcw, ecw) and np.array_equal(gproof, eproof))
        parity = {"result": "bit-exact" if same else "MISMATCH",
                  "against": "the oracle's whole proof of the same instance and seeds (C "
                             "restatement; whir's and spongefish's own bytes cannot be built "
                             "here, so this is equality with the restatement)",
                  "words": int(gproof.shape[0] + gcw.shape[0])}
    proof = last[2]
    proof_bytes = 8 * proof.shape[0]

    # the project's other targets, measured in the same run: the 2^24 NTT
    # against both rooflines, the batched form on the 256-job mix against
    # the same jobs one at a time, and the served form under an open-loop
    # Poisson stream against sequential plain proving
    north = None
    if a.gpus == 1 and not a.no_targets:
        north = {}
        imad = ctypes.c_double(0)
        check(L.pkg_measure_imad_rate(ctypes.byref(imad)))
        with torch.cuda.device(dev):
            north["ntt_2p24"] = ntt_measure(L, stream, flush, 24, 10, 3, dfma.value, imad.value)
        torch.cuda.empty_cache()
        t0 = time.perf_counter()
        b = batched_compare(batched_sizes(a.seed, 256), a.seed, 3, 3)
        b["wall_s"] = time.perf_counter() - t0
        b["config"] = ("256 jobs, NTT sizes log-uniform on 2^10..2^22, each: NTT, WHIR commit "
                       "(ff 3, rate 1/4), zk-sumcheck; one CUDA graph, replayed")
        north["batched_256_jobs"] = b
        torch.cuda.empty_cache()
        north["dual_2p20"] = dual_measure(L, stream, flush, a.seed, 5, 2)
        torch.cuda.empty_cache()
        t0 = time.perf_counter()
        logs, reqs, rng = make_requests(a.seed, 32, 14, 20)
        sgen_s = time.perf_counter() - t0
        free_b, _ = torch.cuda.mem_get_info()
        budget = int(min(free_b * 0.5, 48e9))
        cap, sweeps = served_compare(reqs, (1.0, 2.0), budget, rng)
        north["served_short_stream"] = {
            "config": f"{len(reqs)} whole-proof requests, log2 constraints uniform on [14, 20] "
                      f"(the full sweep to 2^22: --workload served), whir-ZK ff 3, rate 1/4, "
                      f"128 bits, 10 PoW bits; budget {budget / 1e9:.0f} GB, 8 slots",
            "log2_constraints": logs, "generation_s": sgen_s,
            "sequential_capacity_per_s": cap, "sweeps": sweeps,
            "wall_s": time.perf_counter() - t0}
    line = {"metric": PROVE_METRIC,
            "value": a.gpus * a.steps / (total_max * 1e-3), "unit": PROVE_UNIT,
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": total_max / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32/f64 (BN254 Fr: 8x32-bit limbs, products on the FP64 pipe)",
            "data": "synthetic R1CS (pkg_synthetic_r1cs, seeded)",
            "config": prove_config(a, h, wp, proof_bytes),
            "host_generation_s": gen_s,
            "parity": parity,
            "latency_ms": {"p50": p50_max, "p99": p99_max,
                           "note": "per-proof device time, worst rank"},
            "roofline": {
                "kernel": f"leaf_fold_fr_kernel (Skyscraper leaf hashing of the witness "
                          f"commitment: {rows} leaves of {M} Fr)",
                "bound": "fp64", "achieved": f64_achieved / 1e12, "peak": dfma.value / 1e12,
                "unit": "T multiply-op/s", "frac": f64_achieved / dfma.value,
                "traffic": LEAF_TRAFFIC_PROVE_BYTES,
                "traffic_algorithmic": 32 * rows * M + 32 * rows,
                "peak_source": f"measured binary64 fma rate {dfma.value / 1e12:.3f} T/s "
                               "(pkg_measure_dfma_rate, this GPU, this run)",
                "algorithmic": f"{rows} leaves x ({M - 1} compressions x 14 squarings x "
                               f"{F64_PER_SQR} binary64 instructions + {M} Montgomery->"
                               f"canonical REDCs x {IMAD_PER_REDC} integer multiply-adds) = "
                               f"{f64_per_launch} multiply-pipe instructions per launch; the "
                               "integer multiply-adds share the binary64 fma throughput on B200",
                "launch_ms": leaf_s * 1e3,
            },
            "stages_ms_last_step": stage_ms, "whir_phases_ms_last_step": whir_ms,
            "spartan_core_ms": core_ms,
            "cpu_baseline": cpu,
            "e2e": {"value": a.gpus * a.steps / (e2e_max * 1e-3), "unit": PROVE_UNIT,
                    "h2d_bytes_per_step": 32 * h.num_witnesses,
                    "d2h_bytes_per_step": proof_bytes + 32 * (3 + 4 * 20 + 2 * 20 + 8) + 32 * 5,
                    "note": "pkg_prove_r1cs with the witness copied from pinned host memory "
                            "every step and the proof written back to host memory by the call; "
                            "the next step's witness copy (copy stream, two device buffers) "
                            "runs under the current proof; device-timed from the first copy's "
                            "start to the last proof's end",
                    "serial": {"value": a.gpus * a.steps / (e2e_serial_max * 1e-3),
                               "note": "one step at a time: copy, then the call, on one "
                                       "stream; device-timed around copy + call"}},
            "batched": {"value": a.gpus * nreq / batched_max, "unit": PROVE_UNIT,
                        "proofs": nreq, "concurrent": nthr,
                        "latency_ms": {"p50": statistics.median(lat),
                                       "p99": lat[min(len(lat) - 1,
                                                      int(np.ceil(0.99 * len(lat))) - 1)]},
                        "vs_plain_e2e": (a.gpus * nreq / batched_max) /
                                        (a.gpus * a.steps / (e2e_max * 1e-3)),
                        "same_requests_at_once": {
                            "note": f"the same {nreq} requests arriving together: completion "
                                    "time of each from the common start, batched (4 in flight) "
                                    "against plain proving one at a time (measured, one thread)",
                            "batched_ms": {"p50": _pct(done_b, 0.5), "p99": _pct(done_b, 0.99)},
                            "plain_sequential_ms": {"p50": _pct(seq_done, 0.5),
                                                    "p99": _pct(seq_done, 0.99)},
                            "plain_sequential_proofs_per_s": nreq / (seq_done[-1] * 1e-3)},
                        "note": "one resident circuit, many witnesses: 4 host threads with their "
                                "own streams call pkg_prove_r1cs concurrently (witness from "
                                "pinned host memory, proof back to host per proof); wall clock "
                                "from the first call to the last proof"},
            "gpu_launches": int(launches),
            "clocks": clk,
            "targets": north}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_reference_prove(a):
    """The CPU arm: the oracle restatement's whole proof on the same
    instance (the reference is Rust and cannot be built here), OpenMP over
    all host threads; rank 0 only.  Nothing of the CUDA library is loaded:
    the instance comes from the oracle's own generator (pko_synthetic_r1cs,
    equal entry for entry to the library's, tests/test_capi_host.py)."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O

    t0 = time.perf_counter()
    h = O.SyntheticR1CS(a.seed, PROVE_NC, PROVE_NI)
    gen_s = time.perf_counter() - t0
    m, _ = O.r1cs_sizing(h.num_constraints, h.num_witnesses)
    wp = O.whir_params(m, 3, 2, 128, 10, batch_size=2)  # whir-ZK, as the default line
    t0 = time.perf_counter()
    _, _, full_proof = O.prove_r1cs(h, 1, 3, wp)
    t_full = time.perf_counter() - t0
    # keep the whole run within a few minutes: smaller instances of the same
    # shape when one full proof is too slow for steps + warmup of them
    budget_s, shrink = 180.0, 0
    while t_full / (1 << shrink) * (a.steps + a.warmup) > budget_s and shrink < 6:
        shrink += 1
    hs = h if shrink == 0 else O.SyntheticR1CS(a.seed, PROVE_NC >> shrink, PROVE_NI >> shrink)
    ms_, _ = O.r1cs_sizing(hs.num_constraints, hs.num_witnesses)
    wps = wp if shrink == 0 else O.whir_params(ms_, 3, 2, 128, 10, batch_size=2)
    for _ in range(max(a.warmup - 1, 0)):
        O.prove_r1cs(hs, 1, 3, wps)
    times = []
    for _ in range(a.steps):
        t0 = time.perf_counter()
        O.prove_r1cs(hs, 1, 3, wps)
        times.append(time.perf_counter() - t0)
    value = a.steps / sum(times) / (1 << shrink)
    cores = O.lib().pko_num_threads()
    sample = ("whole proof of the 2^20-constraint instance per step" if shrink == 0 else
              f"each step proves a 2^{20 - shrink}-constraint instance of the same shape; "
              f"throughput scaled to 2^20 constraints by the constraint ratio (/2^{shrink}); "
              f"one full proof took {t_full:.2f} s")
    line = {"impl": "reference", "metric": PROVE_METRIC, "value": value, "unit": PROVE_UNIT,
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u64 (BN254 Fr)",
            "data": "synthetic R1CS (seeded; the oracle's generator, equal to pkg_synthetic_r1cs)",
            "config": prove_config(a, h, wp, 8 * full_proof.shape[0]),
            "host_generation_s": gen_s,
            "cpu_baseline": {"value": value, "unit": PROVE_UNIT, "cores": cores, "kind": "port",
                             "sample": sample + "; C restatement of the whole prover (Spartan "
                                       "zk-sumcheck + WHIR rounds), OpenMP, not the reference "
                                       "binary (no Rust toolchain)"},
            "e2e": {"value": value, "unit": PROVE_UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# The batched form (256 uneven jobs) vs the plain path.
# ---------------------------------------------------------------------------
def batched_sizes(seed, jobs, lo=10, hi=22):
    import numpy as np
    rng = np.random.default_rng(seed)
    return [int(x) for x in rng.integers(lo, hi + 1, size=jobs)]


def batched_compare(sizes, seed, steps, warmup, tune=False):
    """The batched form (every phase one grouped launch over all jobs, the
    whole batch one CUDA graph, replayed) against the same jobs one at a time
    through the plain entry points (pkg_ntt_nr, pkg_whir_commit,
    pkg_spartan_sumcheck), inputs resident; spot parity of every 32nd job."""
    import numpy as np
    import torch

    from provekit_b200 import _lib
    from provekit_b200.batch import Batch
    from provekit_b200.merkle import whir_commit
    from provekit_b200.ntt import ntt_nr
    from provekit_b200.spartan import Transcript, spartan_sumcheck

    L = _lib.lib()
    total_fr = sum(1 << k for k in sizes)
    t0 = time.perf_counter()
    b = Batch(sizes, seed=seed)
    setup_s = time.perf_counter() - t0
    stream = torch.cuda.Stream()
    tuned = None
    if tune:
        k, e, ms = b.tune(stream)
        tuned = {"kmax": k, "log_elems_per_cta": e,
                 "log_butterflies_per_thread": b.params()[2], "ms": ms}
    b.run(use_graph=True, stream=stream)  # capture
    for _ in range(warmup):
        b.run(use_graph=True, stream=stream)
    stream.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(steps)]
    launches0 = L.pkg_kernel_launches()
    for i in range(steps):
        evs[i][0].record(stream)
        b.run(use_graph=True, stream=stream)
        evs[i][1].record(stream)
    stream.synchronize()
    launches = L.pkg_kernel_launches() - launches0
    ms = [e[0].elapsed_time(e[1]) for e in evs]
    plain_ms = 0.0
    mismatches = 0
    with torch.cuda.stream(stream):
        for j in range(len(sizes)):
            job = b.job(j)
            n = job.n
            coeffs = torch.from_numpy(Batch.read_fr(job.coeffs, n).view(np.int64)).cuda()
            g = np.array(job.g[: 16 * job.log_n], np.uint64).reshape(-1, 4)
            wb = np.array(job.w1_blinding[: 16 * job.log_n], np.uint64).reshape(-1, 4)
            ntt = torch.empty_like(coeffs)
            cwb = torch.empty((4 * n, 4), dtype=torch.int64, device="cuda")
            lay = torch.empty(32 * (2 * job.num_leaves - 1), dtype=torch.uint8, device="cuda")
            ta, tb, tc = (torch.empty_like(coeffs) for _ in range(3))
            stream.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ntt.copy_(coeffs)
            ntt_nr(ntt, n, 1, stream=stream)
            whir_commit(coeffs, 3, 2, codeword=cwb, layers=lay, stream=stream)
            ta.copy_(coeffs)
            tb.copy_(ntt)
            tc.copy_(cwb[:n])
            t = Transcript.new(job.transcript_domain)
            sc = spartan_sumcheck(ta, tb, tc, job.log_n, g, wb, t, stream=stream)
            e1.record(stream)
            stream.synchronize()
            plain_ms += e0.elapsed_time(e1)
            if j % 32 == 0:  # spot parity (the full check is in tests/test_gpu_batch.py)
                got = b.sumcheck_result(j)
                if not (np.array_equal(got["alpha"], sc["alpha"])
                        and Batch.read(job.layers, 32 * (2 * job.num_leaves - 1))
                        == lay.cpu().numpy().tobytes()):
                    mismatches += 1
    b.close()
    batch_ms = statistics.mean(ms)
    return {"jobs": len(sizes), "log_sizes": sizes, "total_fr": total_fr,
            "log2_total_fr": float(np.log2(total_fr)), "setup_s": setup_s, "tuned": tuned,
            "batch_ms": batch_ms, "jobs_per_s": len(sizes) / (batch_ms * 1e-3),
            "fr_per_s": total_fr / (batch_ms * 1e-3),
            "plain_ms": plain_ms, "plain_jobs_per_s": len(sizes) / (plain_ms * 1e-3),
            "speedup_vs_plain": plain_ms / batch_ms, "spot_parity_mismatches": mismatches,
            "launches_per_batch": int(launches) // max(steps, 1)}


def run_batched(a):
    import torch

    torch.cuda.set_device(0)
    sizes = batched_sizes(a.seed, a.jobs)
    clocks = ClockSampler(physical_gpu_index(0))
    clocks.start()
    r = batched_compare(sizes, a.seed, a.steps, a.warmup, a.tune)
    clk = clocks.stop()
    line = {"metric": "batched form: 256 uneven jobs (NTT + WHIR commit + zk-sumcheck each) as one "
                      "CUDA graph vs the same jobs one at a time",
            "value": r["jobs_per_s"], "unit": "jobs/s", "n_gpus": 1,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": r["batch_ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32 (BN254 Fr, 8x32-bit limbs)", "data": "synthetic (ChaCha20-seeded Fr)",
            "config": {"workload": "batched", "jobs": r["jobs"], "log_sizes": r["log_sizes"],
                       "total_fr": r["total_fr"], "log2_total_fr": r["log2_total_fr"],
                       "setup_s": r["setup_s"], "tuned": r["tuned"]},
            "fr_per_s": r["fr_per_s"],
            "plain": {"value": r["plain_jobs_per_s"], "unit": "jobs/s", "ms": r["plain_ms"]},
            "speedup_vs_plain": r["speedup_vs_plain"],
            "spot_parity_mismatches": r["spot_parity_mismatches"],
            "gpu_launches": r["launches_per_batch"] * a.steps, "clocks": clk}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# The served form under open-loop Poisson arrivals.
# ---------------------------------------------------------------------------
def _pct(v, p):
    import numpy as np
    v = sorted(v)
    return v[min(len(v) - 1, max(0, int(np.ceil(p * len(v))) - 1))]


def served_compare(reqs, mults, budget, rng, max_inflight=8):
    """Sequential plain proving (one request at a time on the server's one
    slot) gives each request's service time and the sequential capacity; then
    for every arrival-rate multiple of that capacity, an open-loop Poisson
    stream of the same requests goes to one long-lived server with
    max_inflight slots (warmed once), against sequential proving under the
    same arrivals (FIFO, the measured service times).  Latency is from submit
    to completion; proofs/s is the stream's requests over its first submit
    to its last completion.  Every served proof is compared with the same
    request's sequential proof (same seeds, so the same words)."""
    import hashlib

    import numpy as np

    from provekit_b200.server import ProofServer

    def digest(res):  # every field of a whole proof, in key order
        h = hashlib.sha256()
        for k in sorted(res):
            v = res[k]
            h.update(k.encode())
            if isinstance(v, np.ndarray):
                v = np.ascontiguousarray(v).tobytes()
            h.update(v if isinstance(v, bytes) else repr(v).encode())
        return h.digest()

    srv = ProofServer(budget, max_inflight=1)
    srv.wait(srv.submit(reqs[0], whole_proof=True, blinding_seed=0, transcript_domain=0))  # warm-up
    service, want = [], []
    for i, h in enumerate(reqs):
        res, tm = srv.wait(srv.submit(h, whole_proof=True, blinding_seed=i, transcript_domain=i))
        service.append((tm["done_ns"] - tm["submit_ns"]) * 1e-9)
        want.append(digest(res))
    srv.close()
    cap = len(service) / sum(service)
    sweeps = []
    # one long-lived server for every rate, as a service runs: warmed first
    # by one request per slot at once (the largest of the stream)
    srv = ProofServer(budget, max_inflight=max_inflight)
    big = sorted(range(len(reqs)), key=lambda i: reqs[i].num_constraints)[-max_inflight:]
    for rid in [srv.submit(reqs[i], whole_proof=True, blinding_seed=0, transcript_domain=0)
                for i in big]:
        srv.wait(rid)
    for mult in mults:
        lam = cap * mult
        arrivals = np.cumsum(rng.exponential(1.0 / lam, size=len(reqs)))
        fin, seq_lat = 0.0, []
        for t_arr, sv in zip(arrivals, service):
            start = max(t_arr, fin)
            fin = start + sv
            seq_lat.append(fin - t_arr)
        ids = [None] * len(reqs)
        t_start = time.perf_counter()
        for i, (t_arr, h) in enumerate(zip(arrivals, reqs)):
            delay = t_start + t_arr - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            ids[i] = srv.submit(h, whole_proof=True, blinding_seed=i, transcript_domain=i)
        lat, qwait, svc, t_sub, t_done = [], [], [], [], []
        mismatches = 0
        for i, rid in enumerate(ids):
            res, tm = srv.wait(rid)
            mismatches += digest(res) != want[i]
            lat.append((tm["done_ns"] - tm["submit_ns"]) * 1e-9)
            qwait.append((tm["admit_ns"] - tm["submit_ns"]) * 1e-9)
            svc.append((tm["done_ns"] - tm["admit_ns"]) * 1e-9)
            t_sub.append(tm["submit_ns"])
            t_done.append(tm["done_ns"])
        st = srv.stats()
        sweeps.append({
            "rate_per_s": lam, "rate_vs_sequential_capacity": mult,
            "served": {"proofs_per_s": len(ids) / ((max(t_done) - min(t_sub)) * 1e-9),
                       "p50_ms": 1e3 * _pct(lat, 0.5),
                       "p99_ms": 1e3 * _pct(lat, 0.99), "p999_ms": 1e3 * _pct(lat, 0.999),
                       "peak_reserved_gb": st["peak_reserved_bytes"] / 1e9,
                       "queue_wait_ms": {"p50": 1e3 * _pct(qwait, 0.5),
                                         "p99": 1e3 * _pct(qwait, 0.99)},
                       "service_ms": {"p50": 1e3 * _pct(svc, 0.5), "p99": 1e3 * _pct(svc, 0.99),
                                      "max": 1e3 * max(svc)}},
            "sequential": {"proofs_per_s": len(reqs) / fin, "p50_ms": 1e3 * _pct(seq_lat, 0.5),
                           "p99_ms": 1e3 * _pct(seq_lat, 0.99),
                           "p999_ms": 1e3 * _pct(seq_lat, 0.999)},
            "proofs_differing_from_sequential": mismatches,
        })
        s = sweeps[-1]
        s["served_beats_sequential"] = bool(
            s["served"]["proofs_per_s"] >= s["sequential"]["proofs_per_s"]
            and s["served"]["p99_ms"] <= s["sequential"]["p99_ms"])
    srv.close()
    return cap, sweeps


def make_requests(seed, count, lo, hi):
    """count synthetic R1CS requests, log2 constraints uniform on [lo, hi],
    a quarter as many inputs, per-request seeds; generated on all host
    threads."""
    import concurrent.futures as cf

    import numpy as np

    from provekit_b200.prover import HostR1CS
    rng = np.random.default_rng(seed)
    logs = [int(x) for x in rng.integers(lo, hi + 1, size=count)]
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        reqs = list(ex.map(lambda i: HostR1CS(10_000 + i, 1 << logs[i], 1 << (logs[i] - 2)),
                           range(count)))
    return logs, reqs, rng


def run_served(a):
    import torch

    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    logs, reqs, rng = make_requests(a.seed, a.requests, 14, 22)
    gen_s = time.perf_counter() - t0
    free_b, _ = torch.cuda.mem_get_info()
    budget = int(min(free_b * 0.9, 180e9))
    cap, sweeps = served_compare(reqs, (0.5, 1.0, 1.5, 2.0, 3.0), budget, rng)
    line = {"metric": "served form: open-loop Poisson prove requests (whole proofs: Spartan + WHIR), "
                      "log2 constraints uniform on [14, 22]; proofs/s and p50/p99/p99.9 latency vs "
                      "sequential plain-GPU proving",
            "value": max(s["served"]["proofs_per_s"] for s in sweeps), "unit": "proofs/s",
            "n_gpus": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32/f64 (BN254 Fr: 8x32-bit limbs, products on the FP64 pipe)",
            "data": "synthetic R1CS (pkg_synthetic_r1cs)",
            "config": {"workload": "served", "whir": "ff 3, rate 1/4, 128 bits, 10 PoW bits",
                       "requests": len(reqs), "log2_constraints": logs,
                       "hbm_budget_gb": budget / 1e9, "max_inflight": 8, "generation_s": gen_s},
            "sequential_capacity_per_s": cap, "sweeps": sweeps}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Two commitments: an R1CS with verifier challenges of the headline's size
# ---------------------------------------------------------------------------
def dual_measure(L, stream, flush, seed, steps, warmup):
    """pkg_dual_prove_begin + _finish on a 2^20-constraint R1CS with 16
    challenges (w1: 2^19 rows over 2^18 inputs; w2: the challenges and
    2^19 - 16 challenge products; 1 310 721 witnesses, as the headline's),
    whir-ZK ff 3, rate 1/4, 128 bits, 10 PoW bits on both commitments.  w2
    is solved once on the host before the timed steps (the caller's witness
    solving is not this path); each step is device-timed from begin's first
    copy to finish's last proof word, L2 flushed before each."""
    import numpy as np
    import torch

    from provekit_b200._lib import check
    from provekit_b200.prover import (DualProofC, HostDualR1CS, dual_statement_counts,
                                      r1cs_sizing_split)
    from provekit_b200.whir import WhirParams
    t0 = time.perf_counter()
    nchal = 16
    h = HostDualR1CS(seed + 11, 1 << 19, 1 << 18, nchal, (1 << 19) - nchal)
    gen_s = time.perf_counter() - t0
    d = h.to_device()
    m, m0 = r1cs_sizing_split(h.num_constraints, h.num_witnesses, h.w1_size)
    p = WhirParams.new(m, 3, 2, 128, 10, batch_size=2)
    n1, n2 = dual_statement_counts(0, nchal)
    offs = np.ascontiguousarray(h.challenge_offsets, dtype=np.uint64)
    ch = np.zeros((nchal, 4), np.uint64)
    cw1, cw2 = np.zeros(p.commit_words(), np.uint64), np.zeros(p.commit_words(), np.uint64)
    pr1, pr2 = np.zeros(p.proof_words(n1), np.uint64), np.zeros(p.proof_words(n2), np.uint64)
    out = DualProofC()
    sh = stream.cuda_stream
    w2 = None
    proofs, times = [], []
    for i in range(warmup + steps):
        st = ctypes.c_void_p()
        with torch.cuda.stream(stream):
            flush.zero_()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            ev[0].record(stream)
            check(L.pkg_dual_prove_begin(ctypes.byref(d.c), h.w1_size, offs.ctypes.data, nchal,
                                         d.witness.data_ptr(), 1, 3, ctypes.byref(p),
                                         cw1.ctypes.data, ch.ctypes.data, ctypes.byref(st), sh))
            try:
                if w2 is None:  # the caller's solve, once (the challenges repeat)
                    w2 = torch.from_numpy(h.solve(ch).view(np.int64)).to(d.witness.device)
                check(L.pkg_dual_prove_finish(st, w2.data_ptr(), ctypes.byref(out),
                                              cw2.ctypes.data, pr1.ctypes.data, pr2.ctypes.data))
            finally:
                L.pkg_dual_prove_free(st)
            ev[1].record(stream)
        stream.synchronize()
        if i >= warmup:
            times.append(ev[0].elapsed_time(ev[1]))
            proofs.append(np.concatenate([cw1, cw2, pr1, pr2]))
    ms = statistics.mean(times)
    return {"config": "2^20 constraints (w1: 2^19 rows over 2^18 inputs; w2: 16 challenges and "
                      "2^19 - 16 challenge products), 1310721 witnesses, m = %d per commitment, "
                      "whir-ZK ff 3, rate 1/4, 128 bits, 10 PoW bits" % m,
            "ms": ms, "proofs_per_s": 1e3 / ms, "p99_ms": max(times), "steps": steps,
            "generation_s": gen_s, "proof_words": int(proofs[0].shape[0]),
            "deterministic": all(np.array_equal(x, proofs[0]) for x in proofs),
            "note": "CUDA events around begin + finish (the host solve of w2 is the caller's and "
                    "runs once before the timed steps); parity with the oracle is tested "
                    "(tests/test_gpu_dual.py), not repeated here"}


# ---------------------------------------------------------------------------
# NTT: 2^24 (the size whose FP64-roofline fraction is the transform's target)
# and the 2^16 single-vector transform.
# ---------------------------------------------------------------------------
def ntt_measure(L, stream, flush, logn, steps, warmup, dfma_rate, imad_rate):
    """ntt_nr at 2^logn (one vector, L2 flushed between steps, CUDA events on
    the launching stream) and intt_rn on its output with the round trip
    checked; throughput against the FP64-pipe roofline (measured DFMA rate /
    binary64 instructions per product) and the integer-pipe one (measured
    IMAD rate / 264 per 8x32 CIOS product)."""
    import numpy as np
    import torch

    from provekit_b200._lib import check
    n = 1 << logn
    h = np.zeros((n, 4), np.uint64)
    check(L.pkg_sample_fr(1 if logn == 16 else logn, n, h.ctypes.data, 1))
    src_t = torch.from_numpy(h.view(np.int64)).cuda()
    d = torch.empty_like(src_t)
    check(L.pkg_ntt_engine_reserve(n))
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            d.copy_(src_t)
            check(L.pkg_ntt_nr(d.data_ptr(), n, n, 1, stream.cuda_stream))
    stream.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(steps)]
    with torch.cuda.stream(stream):
        for i in range(steps):
            d.copy_(src_t)
            flush.zero_()
            evs[i][0].record(stream)
            check(L.pkg_ntt_nr(d.data_ptr(), n, n, 1, stream.cuda_stream))
            evs[i][1].record(stream)
    stream.synchronize()
    ms = statistics.mean(e[0].elapsed_time(e[1]) for e in evs)
    evi = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(steps)]
    with torch.cuda.stream(stream):
        for i in range(steps):
            d.copy_(src_t)
            check(L.pkg_ntt_nr(d.data_ptr(), n, n, 1, stream.cuda_stream))
            flush.zero_()
            evi[i][0].record(stream)
            check(L.pkg_intt_rn(d.data_ptr(), n, stream.cuda_stream))
            evi[i][1].record(stream)
        ok = bool(torch.equal(d, src_t))
    stream.synchronize()
    ms_inv = statistics.mean(e[0].elapsed_time(e[1]) for e in evi)
    products = (n // 2) * logn
    rate = products / (ms * 1e-3)
    del d, src_t
    return {"log2_n": logn, "ms": ms, "fr_per_s": n / (ms * 1e-3), "gmont_per_s": rate / 1e9,
            "frac_fp64": rate / (dfma_rate / F64_PER_MUL),
            "frac_int": rate / (imad_rate / IMAD_PER_MONT),
            "peak_gmont_fp64": dfma_rate / F64_PER_MUL / 1e9,
            "peak_gmont_int": imad_rate / IMAD_PER_MONT / 1e9,
            "hbm_gbs": 2 * 32 * n * ((logn + 8) // 9) / (ms * 1e-3) / 1e9,
            "intt_rn_ms": ms_inv, "round_trip_ok": ok,
            "note": "CUDA events around one ntt_nr launch sequence, L2 flushed (256 MiB write) "
                    "before each; frac_fp64 against the measured binary64 fma rate / "
                    f"{F64_PER_MUL} per product (the butterflies multiply on the FP64 pipe), "
                    f"frac_int against the measured IMAD rate / {IMAD_PER_MONT} per 8x32 CIOS "
                    "product (the integer-pipe roofline)"}


def run_ntt(a):
    import torch

    from provekit_b200 import _lib
    from provekit_b200._lib import check

    L = _lib.lib()
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    imad = ctypes.c_double(0)
    check(L.pkg_measure_imad_rate(ctypes.byref(imad)))
    dfma = ctypes.c_double(0)
    check(L.pkg_measure_dfma_rate(ctypes.byref(dfma)))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    out = {logn: ntt_measure(L, stream, flush, logn, a.steps, a.warmup, dfma.value, imad.value)
           for logn in (24, 16)}
    line = {"metric": "BN254 Fr ntt_nr throughput, 2^24 (roofline target) and 2^16 (single vector)",
            "value": out[24]["fr_per_s"], "unit": "Fr/s", "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": out[24]["ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32 (BN254 Fr, 8x32-bit limbs)",
            "data": "synthetic (ChaCha20-seeded Fr)",
            "config": {"workload": "ntt", "log2_n": 24, "l2": "flushed between steps"},
            "roofline": {"kernel": "ntt_pass_kernel", "bound": "fp64",
                         "achieved": out[24]["gmont_per_s"],
                         "peak": out[24]["peak_gmont_fp64"],
                         "unit": "Gmont/s", "frac": out[24]["frac_fp64"],
                         "algorithmic": f"(n/2) log2 n Montgomery products per transform, "
                                        f"{F64_PER_MUL} binary64 instructions each",
                         "peak_source": f"measured binary64 fma rate {dfma.value / 1e12:.3f} T/s "
                                        f"(pkg_measure_dfma_rate) / {F64_PER_MUL}",
                         "int_pipe_alt": {"peak_gmont_per_s": out[24]["peak_gmont_int"],
                                          "frac": out[24]["frac_int"]}},
            "ntt_2p24": out[24], "ntt_2p16": out[16]}
    print(json.dumps(line), flush=True)


def run_dual(a):
    """The two-commitment proof of an R1CS with verifier challenges on its own
    line (dual_measure: 2^20 constraints, 16 challenges, whir-ZK)."""
    import torch

    from provekit_b200 import _lib

    L = _lib.lib()
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    r = dual_measure(L, stream, flush, a.seed, a.steps, a.warmup)
    line = {"metric": "two-commitment proofs/s (R1CS with verifier challenges: w1 committed, "
                      "challenges drawn, w2 committed, zk-sumcheck, two WHIR proofs)",
            "value": r["proofs_per_s"], "unit": "proofs/s", "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": r["ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "u32/f64 (BN254 Fr: 8x32-bit limbs, products on the FP64 pipe)",
            "data": "synthetic R1CS with challenges (pkg_synthetic_r1cs_dual, seeded)",
            "config": {"workload": "dual", "description": r["config"],
                       "l2": "flushed: 256 MiB device write before each step"},
            "dual_2p20": r}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# WHIR prove-round operations at the prove core's first-round sizes
# (m = 21 variables, folding factor 3, rate 1/4).
# ---------------------------------------------------------------------------
def run_whir_ops(a):
    import numpy as np
    import torch

    from provekit_b200 import _lib, whir
    from provekit_b200._lib import check
    from provekit_b200.merkle import whir_commit

    L = _lib.lib()
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    dfma = ctypes.c_double(0)
    check(L.pkg_measure_dfma_rate(ctypes.byref(dfma)))
    m, k, lr = 21, 3, 2
    n = 1 << m

    def sample(seed, cnt):
        h = np.zeros((cnt, 4), np.uint64)
        check(L.pkg_sample_fr(seed, cnt, h.ctypes.data, 1))
        return h

    coeffs = torch.from_numpy(sample(1, n).view(np.int64)).cuda()
    alpha = sample(2, k)
    cw, layers = whir_commit(coeffs, k, lr)
    nl = (n >> k) << lr
    f = torch.from_numpy(sample(3, n).view(np.int64)).cuda()
    w = torch.from_numpy(sample(4, n).view(np.int64)).cuda()
    pts = sample(5, 2)
    eq_pts = sample(6, 40 * 18)
    eq_cf = sample(7, 40)
    w18 = torch.from_numpy(sample(8, 1 << 18).view(np.int64)).cuda()
    idx = np.arange(0, nl, nl // 64, dtype=np.uint64)[:64]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    out_fold = torch.empty((n >> k, 4), dtype=torch.int64, device="cuda")
    out_rows = torch.empty((nl, 4), dtype=torch.int64, device="cuda")
    ops = {
        "fold_coeffs_2p21_k3": (lambda: whir.fold_coeffs(coeffs, k, alpha, out=out_fold, stream=stream),
                                n, 32 * (n + (n >> k))),
        "fold_rows_2p21_rows": (lambda: whir.fold_rows(cw, k, alpha, out=out_rows, stream=stream),
                                cw.shape[0], 32 * (cw.shape[0] + nl)),
        "sumcheck_round_2p21": (lambda: whir.sumcheck_round(f, w, n, None, stream=stream),
                                3 * (n // 2), 32 * 2 * n),
        "poly_eval_2p21_x2": (lambda: whir.poly_eval_many(coeffs, pts, stream=stream),
                              2 * n, 32 * 2 * n),
        "eq_accumulate_2p18_x40": (lambda: whir.eq_accumulate(w18, 18, eq_pts, eq_cf, stream=stream),
                                   40 << 18, 64 << 18),
        "merkle_open_64_of_2p20": (lambda: whir.merkle_open(layers, nl, idx, stream=stream),
                                   0, 64 * 20 * 32),
    }
    res = {}
    for name, (fn, products, nbytes) in ops.items():
        with torch.cuda.stream(stream):
            for _ in range(a.warmup):
                fn()
            stream.synchronize()
            evs = []
            for _ in range(a.steps):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fn()
                e1.record(stream)
                evs.append((e0, e1))
        stream.synchronize()
        ms = statistics.mean(e0.elapsed_time(e1) for e0, e1 in evs)
        res[name] = {"ms": ms, "gmont_per_s": products / (ms * 1e-3) / 1e9,
                     "fp64_frac": products * F64_PER_MUL / (ms * 1e-3) / dfma.value,
                     "hbm_gbs": nbytes / (ms * 1e-3) / 1e9}
    line = {"metric": "WHIR prove-round operations (device), first-round sizes of the 2^20-"
                      "constraint prove core: m = 21, folding factor 3, rate 1/4",
            "value": 1e3 / sum(r["ms"] for r in res.values()), "unit": "op-sets/s", "n_gpus": 1,
            "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": sum(r["ms"] for r in res.values()), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32 (BN254 Fr, 8x32-bit limbs)",
            "data": "synthetic (ChaCha20-seeded Fr)",
            "config": {"workload": "whir_ops", "m": m, "folding_factor": k, "log_inv_rate": lr,
                       "l2": "flushed between steps"},
            "ops": res, "dfma_rate_tops": dfma.value / 1e12,
            "note": "synchronous ops (poly_eval, sumcheck_round, eq_accumulate, merkle_open) "
                    "include their host read-back"}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Poseidon2 (t = 4, rf = 8, rp = 56) permutations and hashes over 2^22 states.
# ---------------------------------------------------------------------------
def run_poseidon2(a):
    import numpy as np
    import torch

    from provekit_b200 import _lib
    from provekit_b200._lib import check
    from provekit_b200.poseidon2 import poseidon2_hash_many, poseidon2_permutation_many

    L = _lib.lib()
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    dfma = ctypes.c_double(0)
    check(L.pkg_measure_dfma_rate(ctypes.byref(dfma)))
    n = 1 << 22
    h = np.zeros((4 * n, 4), np.uint64)
    check(L.pkg_sample_fr(17, 4 * n, h.ctypes.data, 1))
    src = torch.from_numpy(h.view(np.int64)).cuda()
    st = torch.empty_like(src)
    out = torch.empty(((4 * n) // 3, 4), dtype=torch.int64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def timed(fn):
        with torch.cuda.stream(stream):
            for _ in range(a.warmup):
                fn()
            evs = []
            for _ in range(a.steps):
                st.copy_(src)
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fn()
                e1.record(stream)
                evs.append((e0, e1))
        stream.synchronize()
        return statistics.mean(x.elapsed_time(y) for x, y in evs)

    ms_perm = timed(lambda: poseidon2_permutation_many(st, stream=stream))
    ms_hash = timed(lambda: poseidon2_hash_many(src[: 3 * ((4 * n) // 3)], 3, out=out, stream=stream))
    # products per permutation: full rounds 8 x 4 s-boxes (x^5: 2 squares + 1
    # product), partial rounds 56 x 1 s-box, plus the internal layer's 4
    # diagonal products in each of the 56 partial rounds
    prod_perm = 8 * 4 * 3 + 56 * 3 + 56 * 4
    fp64 = prod_perm * F64_PER_MUL
    line = {"metric": "Poseidon2 (BN254, t = 4) permutations/s over 2^22 states",
            "value": n / (ms_perm * 1e-3), "unit": "permutations/s", "n_gpus": 1,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_perm,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32 (BN254 Fr, 8x32-bit limbs)", "data": "synthetic (ChaCha20-seeded Fr)",
            "config": {"workload": "poseidon2", "states": n, "l2": "flushed between steps"},
            "roofline": {"kernel": "poseidon2 permutation kernel", "bound": "fp64",
                         "achieved": n * fp64 / (ms_perm * 1e-3) / 1e12,
                         "peak": dfma.value / 1e12, "unit": "T fp64-op/s",
                         "frac": n * fp64 / (ms_perm * 1e-3) / dfma.value,
                         "algorithmic": f"{prod_perm} Fr products per permutation at "
                                        f"{F64_PER_MUL} binary64 instructions (squares counted as "
                                        "products: an upper bound on the work)"},
            "hash_rate_per_s": ((4 * n) // 3) / (ms_hash * 1e-3),
            "hash_note": "poseidon2_hash of 3-element inputs (one permutation each)"}
    print(json.dumps(line), flush=True)


def main():
    a = parse_args()
    if a.impl == "reference":
        if a.workload == "prove":
            run_reference_prove(a)
        elif a.workload == "commit":
            run_reference(a)
        elif int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps({"impl": "reference", "unavailable":
                              f"no CPU reference arm for the {a.workload} workload"}), flush=True)
    elif a.workload == "prove":
        run_prove(a)
    elif a.workload == "batched":
        run_batched(a)
    elif a.workload == "served":
        run_served(a)
    elif a.workload == "ntt":
        run_ntt(a)
    elif a.workload == "whir_ops":
        run_whir_ops(a)
    elif a.workload == "poseidon2":
        run_poseidon2(a)
    elif a.workload == "dual":
        run_dual(a)
    else:
        run_b200(a)


if __name__ == "__main__":
    main()

"""BLS12-381 batch verification bench (one JSON line on rank 0).

Workload (the headline configuration): 4,096 verifications against 40
distinct public keys whose G2 line tables are computed once on the device and
kept resident; 1 in 8 items corrupted (half message flip, half wrong key), so
the expected accept bits are known and checked after timing.

  value  verifies/s with inputs resident in HBM: one verify launch per step,
         timed with CUDA events on the library's stream; L2 flushed (256 MiB
         write) between steps, outside the timed interval.
  e2e    verifies/s through the C ABI call (bls_verify_batch) from host
         buffers: host->device copies, kernel, result copy-back per step.
  roofline  INT32 IMAD pipe: algorithmic IMAD-pipe instructions per verify
         (the reference's 16,941 Fp multiplies x 588) / kernel time, against
         SMs x 64 IMAD/clk x the SM clock sampled during the timed region;
         this implementation's own count is reported beside it.
  cpu_baseline  the oracle (C++ restatement of the reference CPU verifier)
         on all host cores, bounded sample of the same workload.

--impl reference runs the reference's CPU verifier (the oracle port; the
reference's Rust crates cannot be built here) on the same workload.
Multi-GPU (torchrun): every rank verifies its own 4,096 items (weak scaling);
the step time is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "icp-gpu_b200"))

import numpy as np  # noqa: E402

N_ITEMS = 4096
N_KEYS = 40
SEED = 2
METRIC = "BLS12-381 verifies/s, batched vs plain launch, bit-exact; serve p50/p99 ms"

# Multiply instructions per verification in this implementation (the
# six-lane kernels' generated op sequence, counted by gen_fp2ops.py over the
# 646 programs of one verification): 20,684 products of 12 x 12 limbs, each by
# one level of limb Karatsuba (three 6 x 6 products: 216 mul.lo / mul.hi), and
# 7,284 Montgomery reductions (12 rows x 25) = 6,652,944.
OWN_PRODUCTS_PER_VERIFY = 20684
OWN_REDC_PER_VERIFY = 7284
IMAD_PER_VERIFY = OWN_PRODUCTS_PER_VERIFY * 216 + OWN_REDC_PER_VERIFY * 300
IMAD_PER_CLK_PER_SM = 64
# Algorithmic work per verification, the fixed roofline numerator: the
# reference's operation count (gpu-crypto/cuda/api.cu:22-91 over
# field_sppark.cuh), 16,941 Fp multiplies x 588 IMAD each.  Work this
# implementation saves (lazy reduction, a cheaper inverse) raises the achieved
# fraction; work it adds lowers it.
ALGO_FP_MULS_PER_VERIFY = 16941
IMAD_PER_FP_MUL = 588   # the reference CIOS multiply: 12 rows x (24 for a b_i + 1 for m + 24 for m p)
ALGO_IMAD_PER_VERIFY = ALGO_FP_MULS_PER_VERIFY * IMAD_PER_FP_MUL
# DRAM bytes of one 4,096-verify launch of the verify kernel (k_verify_w),
# measured with ncu (1.76 MB read, 0 written): the kernel is not memory-bound.
DRAM_BYTES_PER_LAUNCH = 1762560


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons, samples = [], None, set(), 0
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            samples += 1
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": samples}


def max_over_ranks(pg, value, device):
    """the largest `value` over all ranks (every rank gets it); `pg` is
    torch.distributed or None for one process"""
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], device=device, dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(items_per_rank, world, steps, seconds):
    """verifies/s of the whole job: every rank verifies its own shard each step,
    and the job takes as long as its slowest rank"""
    return items_per_rank * world * steps / seconds


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


# ---------------------------------------------------------------- CPU (oracle) legs

def cpu_verifier():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cpu as C  # the checker / reference CPU verifier restated (oracle/)
    return C


def cpu_rate(C, wl, g2, count, threads):
    """verify `count` items of the workload (cycling through it) on the CPU"""
    ix = np.arange(count) % len(wl["expect"])
    sigs, nhms, pki = wl["sigs"][ix], wl["nhms"][ix], wl["pk_index"][ix]
    t = time.perf_counter()
    r = C.verify_batch(sigs, nhms, g2, wl["pk_tables"], pk_index=pki, nthreads=threads)
    dt = time.perf_counter() - t
    assert (r == wl["expect"][ix]).all(), "CPU verifier disagrees with the expected accept bits"
    return count / dt, dt


# The reference's own CPU figure for one verification (ic_bls12_381 0.10.1 on
# the authors' CPU, not named; cuda/bench_bls_verify.cu:167,228): context for
# reading the port's rate, not a measurement on this host.
REF_CPU_US_PER_VERIFY = 348.0


def host_cores():
    """(physical cores, logical CPUs) of this host"""
    logical = os.cpu_count() or 1
    try:
        import psutil
        phys = psutil.cpu_count(logical=False) or logical
    except Exception:
        phys = logical
    return phys, logical


def cpu_model():
    """the host CPU's model name and, where the kernel reports one, its
    highest clock (MHz)"""
    name, mhz = None, None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name") and name is None:
                    name = line.split(":", 1)[1].strip()
    except OSError:
        pass
    try:
        with open("/sys/devices/system/cpu/cpu0/cpufreq/cpuinfo_max_freq") as f:
            mhz = round(int(f.read().strip()) / 1000.0)
    except (OSError, ValueError):
        pass
    return name, mhz


def cpu_context(rate, threads):
    """what a reader needs to place the CPU rate: cores, threads, the CPU
    model, time per verification per thread, and the reference's own
    single-thread figure"""
    phys, logical = host_cores()
    us = 1e6 * threads / rate
    name, mhz = cpu_model()
    return {"physical_cores": phys, "logical_cpus": logical, "threads": threads,
            "cpu_model": name, "cpu_max_mhz": mhz,
            "us_per_verify_per_thread": round(us, 1),
            "reference_us_per_verify": REF_CPU_US_PER_VERIFY,
            "reference_us_basis": "ic_bls12_381 0.10.1 single verify on the reference authors' CPU "
                                  "(cuda/bench_bls_verify.cu:167,228; the machine its README names, README.md:246, "
                                  "is a Ryzen 9 9900X desktop part), not measured here",
            "rate_at_reference_speed": round(threads * 1e6 / REF_CPU_US_PER_VERIFY, 1)}


def cpu_baseline(wl, g2, target_s=12.0):
    C = cpu_verifier()
    threads = C.num_threads()
    calib = min(N_ITEMS, max(64, 4 * threads))
    rate, dt = cpu_rate(C, wl, g2, calib, threads)
    count = int(max(calib, rate * target_s))
    rate, dt = cpu_rate(C, wl, g2, count, threads)
    return {"value": rate, "unit": "verifies/s", "cores": threads, "kind": "port",
            "sample": "%d items cycling through the %d-item workload, oracle/cpu_verifier.cpp on %d host "
                      "threads, %.1f s" % (count, N_ITEMS, threads, dt),
            **cpu_context(rate, threads)}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import workload as WL
    wl = WL.config_keyset(N_ITEMS, N_KEYS, seed=SEED)
    g2 = generator_table(WL)
    C = cpu_verifier()
    threads = C.num_threads()
    rate, _ = cpu_rate(C, wl, g2, min(N_ITEMS, max(64, 4 * threads)), threads)
    per_step = int(max(threads, rate * 3.0))  # about 3 s of CPU work per step
    for _ in range(args.warmup):
        cpu_rate(C, wl, g2, min(per_step, threads), threads)
    times = []
    for _ in range(args.steps):
        _, dt = cpu_rate(C, wl, g2, per_step, threads)
        times.append(dt)
    total = sum(times)
    value = per_step * args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "verifies/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": "keyset-4096-40: 4,096 verifications over 40 public keys",
                   "step_sample": per_step, "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": "verifies/s", "cores": threads, "kind": "port",
                         "sample": "%d items per step, cycling through the 4,096-item workload" % per_step,
                         **cpu_context(value, threads)},
        "e2e": {"value": value, "unit": "verifies/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference CPU verifier = oracle/cpu_verifier.cpp (restatement of ic_bls12_381's verify as the "
                "reference's GPU code mirrors it); the reference's Rust crates are not buildable offline",
    }
    print(json.dumps(line), flush=True)


def generator_table(WL):
    g = np.array([[0xf5f28fa202940a10, 0xb3f5fb2687b4961a, 0xa1a893b53e2ae580, 0x9894999d1a3caee9,
                   0x6f67b7631863366b, 0x058191924350bcd7, 0xa5a9c0759e23f606, 0xaaa0c59dbccd60c3,
                   0x3bb17e18e2867806, 0x1b1ab6cc8541b367, 0xc2b6ed0ef2158547, 0x11922a097360edf3,
                   0x4c730af860494c4a, 0x597cfa1f5e369c5a, 0xe7e6856caa0a635a, 0xbbefb5e96e0d495f,
                   0x07d3a975f0ef25a2, 0x0083fd8e7e80dae5, 0xadc0fc92df64b05d, 0x18aa270a2b1461dc,
                   0x86adac6a3be4eba0, 0x79495c4ec93da33a, 0xe7175850a43ccaed, 0x0b2bc2a163de1bf2]],
                 dtype=np.uint64)
    return WL.g2_prepare(g)[0]


# ---------------------------------------------------------------- GPU arm

def run_gpu(args):
    import torch
    import bls_gpu as G
    import workload as WL

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist

    wl = WL.config_keyset(N_ITEMS, N_KEYS, seed=SEED + rank)
    ctx = G.Context(device=local, lanes=args.lanes, threads_per_block=args.threads_per_block)
    t_keys = time.perf_counter()
    ids = ctx.register_pk_affine_batch(wl["pk_affine"])
    key_setup_ms = 1e3 * (time.perf_counter() - t_keys)
    for i in (0, N_KEYS - 1):  # device tables == caller-built tables
        assert (ctx.pk_table(int(ids[i])) == wl["pk_tables"][i]).all()
    pk_ids = ids[wl["pk_index"]]

    dev = torch.device("cuda", local)
    d_sigs = torch.from_numpy(wl["sigs"].view(np.int64)).to(dev)
    d_nhms = torch.from_numpy(wl["nhms"].view(np.int64)).to(dev)
    d_ids = torch.from_numpy(pk_ids).to(dev)
    d_res = torch.zeros(N_ITEMS, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    torch.cuda.synchronize()

    def step():
        ctx.verify_device(N_ITEMS, d_sigs.data_ptr(), d_nhms.data_ptr(), d_ids.data_ptr(), d_res.data_ptr())

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            flush.zero_()
            step()
    ctx.sync()
    res = d_res.cpu().numpy()
    assert (res == wl["expect"]).all(), "GPU accept bits differ from the expected ones"

    props = torch.cuda.get_device_properties(dev)
    sms = props.multi_processor_count
    sampler = ClockSampler(local)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.zero_()
            starts[k].record(stream)
            step()
            ends[k].record(stream)
    ctx.sync()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    if pg:
        pg.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = max_over_ranks(pg, sum(step_ms), dev)
    res = d_res.cpu().numpy()
    assert (res == wl["expect"]).all(), "GPU accept bits differ from the expected ones (timed run)"
    value = whole_job_rate(N_ITEMS, world, args.steps, total_ms / 1e3)
    kernel_ms = statistics.mean(step_ms)

    # e2e through the C ABI from host buffers
    e2e_times = []
    for k in range(args.warmup + args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        ctx.sync()
        t0 = time.perf_counter()
        r = ctx.verify(wl["sigs"], wl["nhms"], pk_ids)
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            e2e_times.append(dt)
    assert (r == wl["expect"]).all()
    e2e_s = max_over_ranks(pg, sum(e2e_times), dev)
    e2e_value = whole_job_rate(N_ITEMS, world, args.steps, e2e_s)

    # the same items through the reference's own entry point, unchanged callers'
    # view: per-item line tables from host memory (19,584 B each), no resident
    # keys.  That entry point uses device 0, as the reference's does, so only a
    # one-GPU run times it.
    ref_abi = None
    if world == 1:
        item_tables = np.ascontiguousarray(wl["pk_tables"][wl["pk_index"]])
        g2_table = generator_table(WL)
        ref_abi_times = []
        for k in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            r = G.batch_bls_verify(wl["sigs"], wl["nhms"], g2_table, item_tables)
            dt = time.perf_counter() - t0
            if k >= args.warmup:
                ref_abi_times.append(dt)
        assert [int(x) for x in r] == list(wl["expect"])
        ref_abi = {"value": round(N_ITEMS * args.steps / sum(ref_abi_times), 1), "unit": "verifies/s",
                   "api": "gpu_batch_bls_verify (the reference's entry point: per-item line tables from host "
                          "buffers, no resident keys)",
                   "h2d_bytes_per_step": int(wl["sigs"].nbytes + wl["nhms"].nbytes + item_tables.nbytes
                                             + g2_table.nbytes),
                   "d2h_bytes_per_step": int(N_ITEMS * 4)}

    full_chip = run_full_chip(ctx, wl, pk_ids, stream, flush, sms, args) if args.lanes == 6 and \
        args.threads_per_block in (0, 384) else None
    chain_timad = ctx.imad_chain_rate() / 1e12
    lo_rate, hi_rate = ctx.imad_pipe_rates()
    batching = serving = serving_compressed = ingest = hashing = rlc = compressed = None
    # the single-GPU sections (ingest, hashing, compressed signatures, random
    # linear combinations, batching, serving) run on one GPU only; under torchrun every rank times
    # the headline step alone
    if not args.no_extras and world == 1:
        sizes = [int(v) for v in args.ingest_keys.split(",") if int(v) > 0]
        ingest = [run_ingest(G, WL, local, args.lanes, k) for k in sizes] or None
        hashing = run_hash(G, WL, ctx, wl, pk_ids)
        compressed = run_compressed(G, WL, ctx, n=args.compressed_items) if args.compressed_items > 0 else None
        rlc = run_rlc(G, WL, ctx, wl, pk_ids, n=args.rlc_items) if args.rlc_items > 0 else None
        batching = run_batching(G, WL, ctx, wl)
        if args.serve_seconds > 0:
            serving = run_serving(G, WL, ctx, args.serve_seconds, slots=args.serve_slots,
                                  max_batch=args.serve_max_batch, mode=args.serve_mode,
                                  ring_blocks_per_sm=args.serve_ring_blocks,
                                  wide=args.lanes == 6 and args.threads_per_block in (0, 384))
        if args.serve_compressed_seconds > 0:
            serving_compressed = run_serving(G, WL, ctx, args.serve_compressed_seconds, slots=args.serve_slots,
                                             max_batch=args.serve_max_batch, mode=args.serve_mode,
                                             ring_blocks_per_sm=args.serve_ring_blocks,
                                             wide=args.lanes == 6 and args.threads_per_block in (0, 384),
                                             compressed=True)

    result = None
    if rank == 0:
        clk = clocks["sm_mhz"] or float(load_peaks().get("sm_max_mhz", 1965.0))
        peak_timad = sms * IMAD_PER_CLK_PER_SM * clk * 1e6 / 1e12
        achieved_timad = ALGO_IMAD_PER_VERIFY * N_ITEMS / (kernel_ms / 1e3) / 1e12
        roofline = {
            "bound": "int32-imad", "achieved": round(achieved_timad, 3), "peak": round(peak_timad, 3),
            "unit": "TIMAD/s", "frac": round(achieved_timad / peak_timad, 4), "traffic": DRAM_BYTES_PER_LAUNCH,
            "traffic_basis": "dram__bytes_read.sum + dram__bytes_write.sum of one 4,096-verify launch from an "
                             "ncu capture of this kernel (line tables and points; the bound is the IMAD pipe, "
                             "not DRAM)",
            "peak_basis": "%d SMs x 64 IMAD/clk x %.0f MHz (median SM clock sampled during the timed region)"
                          % (sms, clk),
            "algorithmic_imad_per_verify": ALGO_IMAD_PER_VERIFY,
            "own_imad_per_verify": IMAD_PER_VERIFY, "own_products_per_verify": OWN_PRODUCTS_PER_VERIFY,
            "own_reductions_per_verify": OWN_REDC_PER_VERIFY,
            "kernel": (("k_verify_fp2" if args.threads_per_block == 64 else "k_verify_w") if args.lanes == 6
                       else "k_verify_lanes<%d>" % args.lanes) if args.lanes > 1
            else "k_verify",
            "kernel_ms": round(kernel_ms, 4),
            "chain_ceiling": round(chain_timad, 3),
            "frac_of_chain_ceiling": round(achieved_timad / chain_timad, 4),
            "chain_ceiling_basis": "measured: 12 x 12-limb carry-chain products (288 IMAD each) in a loop with the "
                                   "verify kernel's block shape and occupancy (bls_imad_chain_rate)",
            # The nominal peak counts every IMAD at the full rate, but only the
            # low-word multiply issues at that rate: the high word (mul.hi /
            # mul.wide) is measured at half of it.  The reference's CIOS
            # multiply (and this kernel's products) are half low-word and half
            # high-word multiplies, so the most the pipe can retire of that mix is
            # the harmonic mean of the two rates.
            "imad_lo_rate": round(lo_rate / 1e12, 3),
            "imad_hi_rate": round(hi_rate / 1e12, 3),
            "mix_peak": round(2.0 / (1e12 / lo_rate + 1e12 / hi_rate), 3),
            "frac_of_mix_peak": round(achieved_timad / (2.0 / (1e12 / lo_rate + 1e12 / hi_rate)), 4),
            "mix_peak_basis": "measured (bls_imad_pipe_rates): independent mad.lo.u32 and mad.hi.u32 with every "
                              "latency covered; a half-low, half-high multiply mix retires at most at their "
                              "harmonic mean",
        }
        if full_chip:
            fc_timad = ALGO_IMAD_PER_VERIFY * full_chip["items"] / (full_chip["kernel_ms"] / 1e3) / 1e12
            full_chip.update({"achieved": round(fc_timad, 3), "frac": round(fc_timad / peak_timad, 4),
                              "frac_of_mix_peak": roofline["mix_peak"] and
                              round(fc_timad / roofline["mix_peak"], 4)})
            roofline["full_chip"] = full_chip
        result = {
            "metric": METRIC, "value": round(value, 1), "unit": "verifies/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded keys, RFC 9380 hash-to-G1, signatures; 1 in 8 corrupted)",
            "config": {"workload": "keyset-4096-40: 4,096 verifications over 40 device-resident public keys",
                       "items_per_gpu": N_ITEMS, "keys": N_KEYS,
                       "parallelism": "replicas: independent shards per GPU, no collective",
                       "l2": "flushed between steps (256 MiB write), outside the timed interval"},
            "e2e": {"value": round(e2e_value, 1), "unit": "verifies/s",
                    "h2d_bytes_per_step": int(wl["sigs"].nbytes + wl["nhms"].nbytes + pk_ids.nbytes),
                    "d2h_bytes_per_step": int(N_ITEMS * 4), "api": "bls_verify_batch (C ABI, host buffers)"},
            "roofline": roofline,
            "clocks": clocks,
            "gpu_launches": args.steps,
            "bit_exact": True,
            "key_setup": {"keys": N_KEYS, "api": "bls_pk_register_affine_batch (line tables and their "
                          "normalisation for every key, one launch each)", "ms": round(key_setup_ms, 2)},
        }
        if ref_abi:
            result["e2e"]["reference_abi"] = ref_abi
        if ingest:
            result["ingest"] = ingest
        if hashing:
            result["hash"] = hashing
        if compressed:
            result["compressed"] = compressed
        if rlc:
            result["rlc"] = rlc
        if batching:
            result["batching"] = batching
        if serving:
            result["serving"] = serving
        if serving_compressed:
            result["serving_compressed"] = serving_compressed
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(wl, generator_table(WL))
    ctx.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if result is not None:
        print(json.dumps(result), flush=True)


def run_full_chip(ctx, wl, pk_ids, stream, flush, sms, args):
    """The headline kernel with every SM busy.  The twelve-warp kernel holds an
    SM with one block of 32 items, so the 4,096-item keyset workload is 128
    blocks and leaves sms - 128 SMs idle for its one wave.  Here the same
    kernel verifies sms x 32 items (the keyset items, cycled) in one launch:
    one block per SM, inputs resident, L2 flushed between launches, CUDA
    events on the library's stream, mean of args.steps launches after
    args.warmup; the accept bits are checked against the expected ones."""
    import torch
    n = sms * 32
    ix = np.arange(n) % N_ITEMS
    dev = torch.device("cuda", torch.cuda.current_device())
    d_sigs = torch.from_numpy(np.ascontiguousarray(wl["sigs"][ix]).view(np.int64)).to(dev)
    d_nhms = torch.from_numpy(np.ascontiguousarray(wl["nhms"][ix]).view(np.int64)).to(dev)
    d_ids = torch.from_numpy(np.ascontiguousarray(pk_ids[ix])).to(dev)
    d_res = torch.zeros(n, dtype=torch.int32, device=dev)
    times = []
    for k in range(args.warmup + args.steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            flush.zero_()
            a.record(stream)
            ctx.verify_device(n, d_sigs.data_ptr(), d_nhms.data_ptr(), d_ids.data_ptr(), d_res.data_ptr())
            b.record(stream)
        ctx.sync()
        if k >= args.warmup:
            times.append(a.elapsed_time(b))
    assert (d_res.cpu().numpy() == wl["expect"][ix]).all(), "full-chip launch: accept bits differ"
    ms = statistics.mean(times)
    return {"items": n, "blocks": sms, "kernel_ms": round(ms, 4), "verifies_per_s": round(n / (ms / 1e3), 1),
            "basis": "the same kernel with one 32-item block on each of the %d SMs (the keyset items cycled); "
                     "the headline's %d items fill %d of them" % (sms, N_ITEMS, (N_ITEMS + 31) // 32)}


def run_compressed(G, WL, ctx, n=65536, reps=3):
    """Compressed workload: n 48-byte signatures over 40 keys, 2% of them
    invalid encodings (bad flags, x >= p, off the curve, outside the subgroup)
    with the reason per index known.  Decode, checks and verify in one launch
    (bls_verify_batch with BLS_SIG_COMPRESSED) from host buffers, and the same
    through two calls (bls_g1_decompress_status, then the affine verify of the
    decoded points, statuses merged: the reference's decompress-then-verify
    flow, ic-integration/gpu_crypto/lib.rs:189-223 then :124-160).  Host-timed,
    best of reps; every result checked against the known one."""
    import torch
    wl = WL.config_compressed(n, 40, seed=3)
    ids = np.array([ctx.register_pk_affine(q) for q in wl["pk_affine"]], dtype=np.int32)[wl["pk_index"]]
    enc = wl["sigs_compressed"]
    expect = wl["expect"]

    def fused():
        return ctx.verify(enc, wl["nhms"], ids, compressed=True)

    def two_calls():
        st, xy = ctx.g1_decompress(enc.tobytes())
        r = ctx.verify(xy, wl["nhms"], ids)
        return np.where(st != 0, -st, r)

    out = {"items": n, "keys": 40, "invalid": int((expect < 0).sum()),
           "api": "bls_verify_batch, BLS_SIG_COMPRESSED (host buffers): decode, checks and verify in one launch"}
    for name, fn in (("fused", fused), ("decompress_then_verify", two_calls)):
        assert (fn() == expect).all(), name + ": results differ from the expected ones"
        best = 1e30
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            best = min(best, time.perf_counter() - t0)
        out[name + "_verifies_per_s"] = round(n / best, 1)
    # the fused launch alone, inputs resident (CUDA events on the library's stream)
    dev = torch.device("cuda", torch.cuda.current_device())
    d_enc = torch.from_numpy(np.ascontiguousarray(enc).reshape(-1)).to(dev)
    d_nhms = torch.from_numpy(wl["nhms"].view(np.int64)).to(dev)
    d_ids = torch.from_numpy(ids).to(dev)
    d_res = torch.zeros(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    times = []
    for k in range(reps + 1):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            a.record(stream)
            ctx.verify_device(n, d_enc.data_ptr(), d_nhms.data_ptr(), d_ids.data_ptr(), d_res.data_ptr(),
                              compressed=True)
            b.record(stream)
        ctx.sync()
        if k:
            times.append(a.elapsed_time(b))
    assert (d_res.cpu().numpy() == expect).all(), "device-resident compressed verify differs"
    out["kernel_ms"] = round(min(times), 3)
    out["verifies_per_s"] = round(n / (min(times) / 1e3), 1)
    return out


def run_batching(G, WL, ctx, wl_headline, reps=2):
    """Batching workload: 256 requests, sizes log-uniform in [1, 2048], 1-40 keys each.
    First the autotuner (bls_autotune: lanes per verification x block shape x
    blocks per SM) on a device-resident 16,384-item slice of this mix, in a
    context of its own that keeps the fastest point; then, with that point,
    one launch per request against one persistent graph-replayed launch, both
    through bls_verify_requests from host buffers (host-timed, best of reps)."""
    import torch
    wl = WL.config_requests(256, 2048, N_KEYS, seed=4)
    bctx = G.Context()
    try:
        ids = bctx.register_pk_affine_batch(wl["pk_affine"])
        m = min(16384, len(wl["expect"]))
        dev = torch.device("cuda", torch.cuda.current_device())
        ds = torch.from_numpy(wl["sigs"][:m].view(np.int64)).to(dev)
        dn = torch.from_numpy(wl["nhms"][:m].view(np.int64)).to(dev)
        di = torch.from_numpy(ids[wl["pk_index"][:m]]).to(dev)
        pts = bctx.autotune(m, ds.data_ptr(), dn.data_ptr(), di.data_ptr(), repeats=2)
        layout_rates = bctx.limb_layout_rates()
        off = wl["offsets"]
        reqs = [(wl["sigs"][a:b], wl["nhms"][a:b], ids[wl["pk_index"][a:b]]) for a, b in zip(off[:-1], off[1:])]
        n = int(off[-1])
        out = {"requests": len(reqs), "items": n, "sizes": "log-uniform [1, 2048]"}
        for mode, name in ((G.MODE_PLAIN, "plain"), (G.MODE_PERSISTENT, "persistent")):
            r = bctx.verify_requests(reqs, mode=mode)
            assert (np.concatenate(r) == wl["expect"]).all(), "batched accept bits differ"
            best = 1e30
            for _ in range(reps):
                t0 = time.perf_counter()
                bctx.verify_requests(reqs, mode=mode)
                best = min(best, time.perf_counter() - t0)
            out[name + "_verifies_per_s"] = round(n / best, 1)
            out[name + "_ms"] = round(best * 1e3, 2)
        out["speedup"] = round(out["persistent_verifies_per_s"] / out["plain_verifies_per_s"], 2)
    finally:
        bctx.close()
    kernel = {1: "k_verify (thread per verification)", 2: "k_verify_lanes<2>", 4: "k_verify_lanes<4>",
              8: "k_verify_lanes<8>"}

    def name(l, tpb):
        if l == 6:
            return "k_verify_w (32 items / 12 warps)" if tpb == 384 else "k_verify_fp2 (5 items / 2 warps)"
        return kernel.get(l, "%d lanes" % l)
    best = min(pts, key=lambda p: p[3])
    out["autotune"] = {
        "sample": "first %d items of this mix (mixed keys), inputs resident (bls_autotune, best of 2 per point); "
                  "the chosen point runs both request modes above" % m,
        "points": [{"lanes": l, "threads_per_block": t, "kernel": name(l, t), "blocks_per_sm": b, "ms": round(ms, 3)}
                   for l, t, b, ms in pts],
        "chosen": {"lanes": best[0], "threads_per_block": best[1], "kernel": name(best[0], best[1]),
                   "blocks_per_sm": best[2], "ms": round(best[3], 3)}}
    # the limb-layout dimension: product throughput of each layout in the
    # twelve-warp kernel's setting (bls_limb_layout_rates); the verify kernels
    # are built for the first, and the sweep shows whether it is still the fastest
    layouts = ["12 x 32-bit limbs, limb Karatsuba, carry-chain rows (216 multiplies)",
               "15 x 26-bit signed limbs, 225 mad.wide.s32 into 64-bit columns",
               "14 x 28-bit limbs, 196 mad.wide.u32 into 64-bit columns"]
    lpts = [{"layout": nm, "g_products_per_s": round(r / 1e9, 2)} for nm, r in zip(layouts, layout_rates)]
    out["autotune"]["limb_layout_points"] = lpts
    out["autotune"]["limb_layout_chosen"] = max(lpts, key=lambda q: q["g_products_per_s"])["layout"]
    out["autotune"]["limb_layout_basis"] = (
        "products/s on the whole device, one block of 384 threads per SM, operands from lane-interleaved shared "
        "memory (bls_limb_layout_rates); every verify kernel uses the first layout")
    return out


def run_ingest(G, WL, device, lanes, n_keys, reps=3):
    """Key ingest: n_keys 96-byte compressed public keys decoded, validated,
    prepared and normalised on the GPU by one bls_pk_register_compressed call
    (host-timed, best of reps, each on a fresh context), against the CPU line-table
    precompute alone (the caller's per-key G2Prepared::from) on all host threads."""
    rng = WL.SplitMix64(SEED + 17)
    sks = np.array([WL.scalar_limbs(rng.scalar()) for _ in range(n_keys)], dtype=np.uint64)
    q = WL.g2_mul_gen(sks)
    enc = WL.g2_compress(q).tobytes()
    best = 1e30
    for _ in range(reps):
        c = G.Context(device=device, lanes=lanes, max_pks=n_keys)
        t0 = time.perf_counter()
        ids, st = c.register_pk_compressed(enc)
        best = min(best, time.perf_counter() - t0)
        assert (st == 0).all()
        check = [0, n_keys - 1]
        want = WL.g2_prepare(q[check])
        for j, i in enumerate(check):
            assert (c.pk_table(int(ids[i])) == want[j]).all(), "ingested table differs"
        c.close()
    t0 = time.perf_counter()
    WL.g2_prepare(q)
    cpu_s = time.perf_counter() - t0
    return {"keys": n_keys, "api": "bls_pk_register_compressed (decode + checks + tables + normalise)",
            "gpu_keys_per_s": round(n_keys / best, 1), "gpu_ms": round(best * 1e3, 2),
            "cpu_prepare_keys_per_s": round(n_keys / cpu_s, 1), "cpu_threads": WL.nthreads(),
            "cpu_note": "CPU line-table precompute only (no decode or subgroup check)"}


def run_hash(G, WL, ctx, wl, pk_ids, reps=3):
    """Verification from message bytes: -H(m) on the GPU (bls_verify_messages)
    against the same verify with -H(m) precomputed by the caller on the CPU
    (the reference's flow), and the hash alone on the GPU against the CPU
    workload hash on all host threads (host-timed, best of reps)."""
    msgs = wl["msgs"]
    n = len(msgs)
    r = ctx.verify_messages(wl["sigs"], msgs, pk_ids, WL.DST)
    assert (r == wl["expect"]).all(), "verify from messages differs"
    assert (ctx.neg_hash_to_g1(msgs[:64], WL.DST) == wl["nhms"][:64]).all(), "GPU hash differs"

    def best(fn):
        t = 1e30
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            t = min(t, time.perf_counter() - t0)
        return t
    t_msgs = best(lambda: ctx.verify_messages(wl["sigs"], msgs, pk_ids, WL.DST))
    t_gpu_hash = best(lambda: ctx.neg_hash_to_g1(msgs, WL.DST))
    t_cpu_hash = best(lambda: WL.g1_neg(WL.hash_to_g1(msgs)))
    t_verify = best(lambda: ctx.verify(wl["sigs"], wl["nhms"], pk_ids))
    return {"items": n, "suite": "RFC 9380 hash_to_curve, expand_message_xmd SHA-256, SSWU map + 11-isogeny",
            "verify_messages_per_s": round(n / t_msgs, 1),
            "verify_messages_api": "bls_verify_messages (hash + verify on the GPU, host buffers)",
            "cpu_hash_then_verify_per_s": round(n / (t_cpu_hash + t_verify), 1),
            "gpu_hash_per_s": round(n / t_gpu_hash, 1),
            "cpu_hash_per_s": round(n / t_cpu_hash, 1), "cpu_threads": WL.nthreads()}


def run_rlc(G, WL, ctx, wl4096, pk_ids4096, n=65536, reps=3):
    """Random-linear-combination batches (bls_verify_batch_rlc) from host
    buffers: an all-valid batch (the corrupted items of a keyset-n-40 draw
    removed) against the same batch item by item (bls_verify_batch); and the
    headline 4,096-item workload, whose 1-in-8 corrupted items make the combined
    check fail, to show the cost of the fallback (host-timed, best of reps)."""
    wl = WL.config_keyset(n, N_KEYS, seed=SEED + 5)
    keep = np.nonzero(wl["expect"] == 1)[0]
    ids = np.array([ctx.register_pk_affine(q) for q in wl["pk_affine"]], dtype=np.int32)[wl["pk_index"][keep]]
    sigs, nhms = wl["sigs"][keep], wl["nhms"][keep]

    def best(fn):
        t, out = 1e30, None
        for _ in range(reps):
            t0 = time.perf_counter()
            out = fn()
            t = min(t, time.perf_counter() - t0)
        return t, out
    t_item, r_item = best(lambda: ctx.verify(sigs, nhms, ids))
    t_rlc, (r_rlc, comb) = best(lambda: ctx.verify_rlc(sigs, nhms, ids))
    assert comb == 1 and (r_rlc == 1).all() and (r_item == 1).all(), "all-valid batch not accepted"
    t_fb, (r_fb, comb_fb) = best(lambda: ctx.verify_rlc(wl4096["sigs"], wl4096["nhms"], pk_ids4096))
    assert comb_fb == 0 and (r_fb == wl4096["expect"]).all(), "fallback results differ"
    t_fb_item, _ = best(lambda: ctx.verify(wl4096["sigs"], wl4096["nhms"], pk_ids4096))
    m = len(keep)
    return {"items": m, "keys": N_KEYS, "api": "bls_verify_batch_rlc vs bls_verify_batch (host buffers)",
            "per_item_verifies_per_s": round(m / t_item, 1), "rlc_verifies_per_s": round(m / t_rlc, 1),
            "speedup": round(t_item / t_rlc, 2), "rlc_ms": round(t_rlc * 1e3, 2),
            "fallback_4096_ms": round(t_fb * 1e3, 2), "per_item_4096_ms": round(t_fb_item * 1e3, 2)}


def run_serving(G, WL, ctx, seconds, load=0.8, slots=3, max_batch=8192, mode="ring", ring_blocks_per_sm=0,
                ring_blocks=0, wide=True, compressed=False):
    """Serving workload: seeded Poisson stream of requests (sizes log-uniform in
    [1, 512]) over a pool of 40 resident keys, through the continuous-batching
    server (bls_server_*) under a 4 GiB device-memory cap: `mode` "ring" (one
    persistent kernel claiming items from a device ring as they are published)
    or "slots" (`slots` launches of up to `max_batch` items in flight);
    `compressed`: the signatures arrive as 48-byte encodings and are decoded on
    the device.  The arrival rate is `load` x the server's measured saturated
    throughput; latency is submit to completion on the library's steady clock."""
    import threading
    pool = WL.config_pool(8192, N_KEYS, seed=5)
    ids = ctx.register_pk_affine_batch(pool["pk_affine"])
    pk_ids = ids[pool["pk_index"]]
    npool = len(pool["expect"])
    sig_src = WL.g1_compress(pool["sigs"]) if compressed else pool["sigs"]

    def materialise(starts, sizes):
        out = []
        for a, s in zip(starts, sizes):
            ix = (int(a) + np.arange(int(s))) % npool
            out.append((ix, np.ascontiguousarray(sig_src[ix]), np.ascontiguousarray(pool["nhms"][ix]),
                        np.ascontiguousarray(pk_ids[ix])))
        return out

    if mode == "ring":
        server = G.Server(ctx, compressed=compressed, max_batch_items=512, mem_cap_bytes=4 << 30,
                          mode=G.SERVE_RING, ring_blocks_per_sm=ring_blocks_per_sm, ring_blocks=ring_blocks)
    else:
        server = G.Server(ctx, compressed=compressed, slots=slots, max_batch_items=max_batch,
                          mem_cap_bytes=4 << 30)
    with server as srv:
        # saturated throughput: a backlog of requests submitted at once
        _, sizes, starts = WL.poisson_stream(1.0, 4000.0, max_size=512, pool_size=npool, seed=7)
        burst = materialise(starts, sizes)
        for rep in range(2):
            t0 = time.perf_counter()
            tk = [srv.submit(s, h, i) for _, s, h, i in burst]
            for t, _, _ in tk:
                srv.wait(t, timeout_ms=120000)
            dt = time.perf_counter() - t0
        sat = sum(len(b[0]) for b in burst) / dt

        mean_size = float(np.mean(sizes))
        rate = load * sat / mean_size
        arrivals, sizes, starts = WL.poisson_stream(seconds, rate, max_size=512, pool_size=npool, seed=6)
        reqs = materialise(starts, sizes)
        tickets = [None] * len(reqs)
        lat = np.zeros(len(reqs))
        mismatches = [0]

        def waiter():
            for k in range(len(reqs)):
                while tickets[k] is None:
                    time.sleep(0.0002)
                t, ts, res = tickets[k]
                td = srv.wait(t, timeout_ms=120000)
                lat[k] = (td - ts) / 1e6
                if not (res == pool["expect"][reqs[k][0]]).all():
                    mismatches[0] += 1

        th = threading.Thread(target=waiter)
        th.start()
        stats0 = srv.stats()
        t0 = time.perf_counter()
        for k, (ix, s, h, i) in enumerate(reqs):
            while True:
                d = arrivals[k] - (time.perf_counter() - t0)
                if d <= 0:
                    break
                time.sleep(min(d, 0.001) if d > 0.0015 else 0)
            tickets[k] = srv.submit(s, h, i)
        th.join()
        wall = time.perf_counter() - t0
        stats1 = srv.stats()
    items = int(sum(sizes))
    assert mismatches[0] == 0, "served results differ from the expected accept bits"
    return {
        "requests": len(reqs), "items": items, "seconds": round(wall, 2), "offered_load": load,
        "saturated_verifies_per_s": round(sat, 1), "arrival_rate_req_per_s": round(rate, 1),
        "throughput_verifies_per_s": round(items / wall, 1),
        "p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
        "p999_ms": round(float(np.percentile(lat, 99.9)), 3), "max_ms": round(float(lat.max()), 3),
        "launches": int(stats1["launches"] - stats0["launches"]),
        "mem_cap_bytes": 4 << 30, "sizes": "log-uniform [1, 512]", "bit_exact": True,
        "signatures": "48-byte compressed, decoded on the device before publication" if compressed
                      else "affine (96 bytes)",
        "mode": (("ring: one persistent twelve-warp block per SM claiming up to 32 published items at a time "
                  "from a device ring" if wide else
                  "ring: one persistent kernel (%d five-item blocks per SM) claiming items five at a time from a "
                  "device ring" % (ring_blocks_per_sm or 4)) if mode == "ring"
                 else "slots: %d launches of up to %d items in flight" % (slots, max_batch)),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the batching and serving sections")
    ap.add_argument("--lanes", type=int, default=6, help="lanes per verification (6: Fp2-lane kernel; 1, 2, 4, 8)")
    ap.add_argument("--threads-per-block", type=int, default=0,
                    help="six lanes: 384 (32 items per block, twelve warps; the default), 64 (five items, two warps)")
    ap.add_argument("--ingest-keys", default="1024,16384",
                    help="comma-separated key counts ingested compressed on the GPU (0 = skip)")
    ap.add_argument("--rlc-items", type=int, default=65536, help="random-linear-combination batch draw (0 = skip)")
    ap.add_argument("--compressed-items", type=int, default=65536,
                    help="compressed workload: 48-byte signatures, 2%% invalid encodings (0 = skip)")
    ap.add_argument("--serve-seconds", type=float, default=30.0, help="length of the serving stream (0 = skip)")
    ap.add_argument("--serve-compressed-seconds", type=float, default=10.0,
                    help="length of a second serving stream with 48-byte signatures (0 = skip)")
    ap.add_argument("--serve-mode", choices=["ring", "slots"], default="ring", help="serving: server mode")
    ap.add_argument("--serve-ring-blocks", type=int, default=4,
                    help="serving, ring mode: resident verify blocks per SM")
    ap.add_argument("--serve-slots", type=int, default=8, help="serving: launches in flight")
    ap.add_argument("--serve-max-batch", type=int, default=740, help="serving: items per launch")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()

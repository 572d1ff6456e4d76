"""Benchmark of the gate-bootstrapping hot path on B200.

Workload (one "step"): 4096 independent bootsNAND gates in one batch at the default 128-bit
parameters (n=630, N=1024, k=1, l=3, Bgbit=7, ks t=8 basebit=2): gate prologue + mod-switch,
blind rotation (630 CMUX steps), sample extraction and keyswitch, on GPU-resident ciphertexts.
The headline `value` is the split-FP32 form; the plain FP64 form is measured in the same run
(`fp64`).  Multi-GPU runs are independent replicas (one key set per GPU, no collective on the data
path); value = all gates of all ranks / the slowest rank's device time.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--form split|fp64]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "bootstrapped gates/s on 1 B200: split-FP32 vs FP64 FFT, 0 errors in 1e6 gates"
UNIT = "gates/s"
PARAMS = "n=630,N=1024,k=1,l=3,Bgbit=7,ks_t=8,ks_basebit=2"

# Algorithmic work per gate (FFT of size M complex = 5 M log2 M flops, twist 6M, complex MAC 8):
# per CMUX step FP64 = 8 transforms + 12*512 MACs = 258,048 flops; split = 10 transforms + 24*512 MACs
# = 359,424 flops; x 630 steps.
FLOPS_PER_GATE = {"fp64": 162.57e6, "split": 226.44e6}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--form", choices=["split", "fp64"], default="split")
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--error-gates", type=int, default=1_003_520,
                    help="gates per form of the decryption-error count after the timed steps (0: skip)")
    ap.add_argument("--workload", choices=["nand", "netlist", "mux2048", "errors", "keyswitch", "dropin", "dft"],
                    default="nand",
                    help="nand: the headline line (4096 NAND batches); the others print their own line: "
                         "netlist = seeded 200-level random circuit through a CUDA graph, mux2048 = 1024 MUX "
                         "at N=2048, errors = decryption-error count over 10^6 split-FP32 NAND gates, "
                         "keyswitch = the three keyswitch kernels on --batch extracted samples, dropin = "
                         "one bootsNAND per call through include/tfhe.h from 1, 16 and 64 threads, dft = a "
                         "radix-8 DFT stage on CUDA cores vs tensor cores (tfheb_measure_dft8)")
    ap.add_argument("--gates", type=int, default=1_000_000, help="gate count of --workload errors")
    ap.add_argument("--ring", type=int, choices=[1024, 2048], default=1024,
                    help="--workload errors: 1024 = NAND at the default parameters in the --form form "
                         "(batches of 4096); 2048 = MUX at n=800, N=2048 in both forms (batches of 1024)")
    return ap.parse_args()


def replica_throughput(local_ms, units_per_rank, world, dist=None, device="cpu"):
    """Replicas-only aggregation: every rank evaluates its own batch with its own keys, no collective
    on the data path.  Returns (slowest rank's time in ms, all ranks' units / that time in seconds)."""
    import torch
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    if dist is not None and world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    slowest = float(t.item())
    return slowest, units_per_rank * world / (slowest / 1e3)


def run_extra_workload(args):
    """Secondary measurements (not the headline line): one JSON line each."""
    import ctypes

    import numpy as np
    import torch

    import tfhe_b200 as tb
    from tfhe_b200.api import Netlist, eval_plain, random_netlist

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    out = {"workload": args.workload}
    if args.workload == "netlist":
        p = tb.default_params()
        sk, ck = tb.keygen(p, seed=4)
        ck.to_device(0)
        rng = np.random.default_rng(2024)
        ni, gates, ia, ib, ic = random_netlist(rng, levels=200, width_lo=16, width_hi=4096)
        bits = rng.integers(0, 2, ni)
        truth = eval_plain(ni, gates, ia, ib, ic, bits)
        wires = torch.zeros((ni + len(gates), p.n + 1), dtype=torch.int32, device="cuda")
        wires[:ni] = torch.from_numpy(sk.encrypt(bits, seed=3))
        for prec, name in ((tb.SPLIT_FP32, "split"), (tb.FP64, "fp64")):
            ck.autotune(prec, boots=2048)
            nl = Netlist(ck, ni, gates, ia, ib, ic)
            nl.run(wires, precision=prec, use_graph=True, stream=sptr)  # eager run + capture
            torch.cuda.synchronize()
            times = []
            for _ in range(max(1, args.steps)):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                nl.run(wires, precision=prec, use_graph=True, stream=sptr)
                e1.record(stream)
                torch.cuda.synchronize()
                times.append(e0.elapsed_time(e1))
            got, _ = sk.decrypt(wires.cpu().numpy())
            ms = float(np.median(times))
            out[name] = {"gates_per_s": len(gates) / (ms / 1e3), "ms_per_run": ms,
                         "wrong_wires": int((got != truth).sum()), "levels": nl.info()[0]}
            nl.free()
        out.update({"gates": int(len(gates)), "inputs": int(ni),
                    "mix": "NAND .40 XOR .20 AND .15 OR .15 MUX .10; widths U[16,4096]; 200 levels; "
                           "operands uniform over the previous two levels",
                    "timing": "median device time of one CUDA-graph replay (CUDA events)"})
    elif args.workload == "mux2048":
        p = tb.large_params()
        sk, ck = tb.keygen(p, seed=5)
        ck.to_device(0)
        B = 1024
        rng = np.random.default_rng(3)
        a, b, c = rng.integers(0, 2, (3, B))
        d = [torch.from_numpy(sk.encrypt(x, seed=i + 1)).cuda() for i, x in enumerate((a, b, c))]
        dout = torch.zeros_like(d[0])
        for prec, name in ((tb.SPLIT_FP32, "split"), (tb.FP64, "fp64")):
            tune = ck.autotune(prec, boots=2 * B)
            for _ in range(args.warmup):
                ck.gate_device(tb.api.MUX, d[0], d[1], d[2], dout, B, precision=prec, stream=sptr)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                ck.gate_device(tb.api.MUX, d[0], d[1], d[2], dout, B, precision=prec, stream=sptr)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / args.steps
            got, _ = sk.decrypt(dout.cpu().numpy())
            out[name] = {"gates_per_s": B / (ms / 1e3), "ms_per_batch": ms,
                         "errors": int((got != np.where(a == 1, b, c)).sum()), "autotune": tune}
        out.update({"params": "n=800,N=2048,k=1,l=3,Bgbit=8,ks_t=8,ks_basebit=2", "batch": B,
                    "split_shift": int(tb.api.lib().tfheb_default_split_shift(ctypes.byref(p)))})
    elif args.workload == "errors" and args.ring == 2048:
        # config 5: bootsMUX at n=800, N=2048, decryption errors over --gates gates per form
        p = tb.large_params()
        sk, ck = tb.keygen(p, seed=8)
        ck.to_device(0)
        B = 1024
        rng = np.random.default_rng(12)
        dout = torch.zeros((B, p.n + 1), dtype=torch.int32, device="cuda")
        for prec, name in ((tb.SPLIT_FP32, "split"), (tb.FP64, "fp64")):
            ck.autotune(prec, boots=2 * B)
            t0, errors, done, batch = time.perf_counter(), 0, 0, 0
            while done < args.gates:
                bits = rng.integers(0, 2, (3, B))
                d = [torch.from_numpy(sk.encrypt(bits[i], seed=3 * batch + i + 1)).cuda() for i in range(3)]
                ck.gate_device(tb.api.MUX, d[0], d[1], d[2], dout, B, precision=prec, stream=sptr)
                got, _ = sk.decrypt(dout.cpu().numpy())
                errors += int((got != np.where(bits[0] == 1, bits[1], bits[2])).sum())
                done += B
                batch += 1
            out[name] = {"gates": done, "decryption_errors": errors, "batches": batch,
                         "wall_s": time.perf_counter() - t0}
        out.update({"gate": "MUX", "params": "n=800,N=2048,k=1,l=3,Bgbit=8,ks_t=8,ks_basebit=2"})
    elif args.workload == "errors":
        p = tb.default_params()
        sk, ck = tb.keygen(p, seed=6)
        ck.to_device(0)
        prec = tb.SPLIT_FP32 if args.form == "split" else tb.FP64
        ck.autotune(prec, boots=4096)
        B, total, errors, done = 4096, args.gates, 0, 0
        rng = np.random.default_rng(11)
        dout = torch.zeros((B, p.n + 1), dtype=torch.int32, device="cuda")
        t0 = time.perf_counter()
        batch = 0
        while done < total:
            bits = rng.integers(0, 2, (2, B))
            da = torch.from_numpy(sk.encrypt(bits[0], seed=2 * batch + 1)).cuda()
            db = torch.from_numpy(sk.encrypt(bits[1], seed=2 * batch + 2)).cuda()
            ck.gate_device(tb.api.NAND, da, db, None, dout, B, precision=prec, stream=sptr)
            got, _ = sk.decrypt(dout.cpu().numpy())
            errors += int((got != 1 - (bits[0] & bits[1])).sum())
            done += B
            batch += 1
        out.update({"form": "split-FP32" if args.form == "split" else "FP64", "gates": done,
                    "decryption_errors": errors, "batches": batch, "wall_s": time.perf_counter() - t0})
    elif args.workload == "keyswitch":
        # default parameters, --batch random extracted samples (dimension kN + 1); each kernel runs
        # --warmup untimed then --steps timed calls on this stream; outputs must agree bit for bit
        p = tb.default_params()
        sk, ck = tb.keygen(p, seed=3)
        ck.to_device(0, precisions=(tb.FP64,))
        B = args.batch
        rng = np.random.default_rng(B)
        x = torch.from_numpy(rng.integers(-2**31, 2**31, (B, p.k * p.N + 1), dtype=np.int64).astype(np.int32)).cuda()
        ref_out, times = None, {}
        for which, name in ((1, "per_sample"), (2, "tiled"), (3, "regkey"), (4, "tensor_core")):
            ck.set_keyswitch_kernel(which)
            dout = torch.zeros((B, p.n + 1), dtype=torch.int32, device="cuda")
            for _ in range(args.warmup):
                ck.keyswitch_device(x, dout, B, stream=sptr)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(args.steps):
                ck.keyswitch_device(x, dout, B, stream=sptr)
            e1.record(stream)
            torch.cuda.synchronize()
            times[name] = e0.elapsed_time(e1) / args.steps
            got = dout.cpu().numpy()
            if ref_out is None:
                ref_out = got
            elif not (got == ref_out).all():
                raise RuntimeError(f"keyswitch kernel {name} disagrees with the per-sample kernel")
        ck.set_keyswitch_kernel(0)
        out.update({"samples": B, "ms_per_call": times, "bit_identical": True,
                    "params": "n=630,N=1024,k=1,ks_t=8,ks_basebit=2"})
    elif args.workload == "dropin":
        # the reference's calling pattern: a C client (tests/c/dropin_bench.c) compiled against
        # include/tfhe.h calls bootsNAND once per gate, from several threads on one keyset
        libdir = os.path.join(ROOT, "tfhe_b200")
        with tempfile.TemporaryDirectory() as tmp:
            exe = os.path.join(tmp, "dropin_bench")
            subprocess.check_call(["gcc", "-std=c99", "-D_POSIX_C_SOURCE=200809L", "-O2", "-I",
                                   os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "c", "dropin_bench.c"),
                                   "-o", exe, "-L", libdir, "-ltfhe_b200", f"-Wl,-rpath,{libdir}", "-lpthread"])
            runs = []
            for threads, per_thread in ((1, 40), (16, 40), (64, 24), (256, 16)):
                res = subprocess.run([exe, "1", str(threads), str(per_thread)], capture_output=True, text=True,
                                     timeout=900)
                if res.returncode != 0:
                    raise RuntimeError(f"dropin_bench failed: {res.stdout}{res.stderr}")
                runs.append(json.loads(res.stdout.strip().splitlines()[-1]))
        out.update({"form": "split-FP32", "api": "bootsNAND (include/tfhe.h), one gate per call", "runs": runs})
    elif args.workload == "dft":
        # one radix-8 stage of the blind rotation's FFT: CUDA-core codelet vs TF32x3 mma.sync
        L = tb.api.lib()
        L.tfheb_measure_dft8.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]
        names = {0: "cuda_core_dft8", 1: "mma_tf32x3_compute_only", 2: "mma_tf32x3_with_relayout"}
        for method, name in names.items():
            ns, err = ctypes.c_double(), ctypes.c_double()
            st = L.tfheb_measure_dft8(0, method, ctypes.byref(ns), ctypes.byref(err))
            if st != 0:
                raise RuntimeError(L.tfheb_last_error().decode())
            out[name] = {"ns_per_dft8_whole_gpu": ns.value, "max_rel_err_vs_fp64": err.value}
        out["faster"] = min(names.values(), key=lambda k: out[k]["ns_per_dft8_whole_gpu"])
    print(json.dumps(out), flush=True)


def count_errors(ck, sk, form, total, stream, sptr, seed=90):
    """Decryption errors over `total` bootsNAND gates in batches of 4096 on fresh encryptions (new
    bits, new seeds per batch), device buffers through tfheb_gate_batch_device.  Host encryption and
    decryption of the next and previous batches run in a worker thread while the GPU evaluates the
    current one (the library's host calls release the GIL)."""
    from concurrent.futures import ThreadPoolExecutor

    import numpy as np
    import torch

    import tfhe_b200 as tb
    prec = tb.SPLIT_FP32 if form == "split" else tb.FP64
    B, p = 4096, sk.params
    batches = -(-total // B)
    rng = np.random.default_rng(seed)
    dout = torch.zeros((B, p.n + 1), dtype=torch.int32, device="cuda")

    def make(i):
        bits = rng.integers(0, 2, (2, B))
        return bits, sk.encrypt(bits[0], seed=seed * 100003 + 2 * i + 1), sk.encrypt(bits[1], seed=seed * 100003 + 2 * i + 2)

    def check(bits, out):
        got, _ = sk.decrypt(out)
        return int((got != 1 - (bits[0] & bits[1])).sum())

    t0 = time.perf_counter()
    errors, pending = 0, None
    with ThreadPoolExecutor(max_workers=2) as pool:
        nxt = pool.submit(make, 0)
        for i in range(batches):
            bits, ha, hb = nxt.result()
            if i + 1 < batches:
                nxt = pool.submit(make, i + 1)
            da, db = torch.from_numpy(ha).cuda(), torch.from_numpy(hb).cuda()
            ck.gate_device(tb.api.NAND, da, db, None, dout, B, precision=prec, stream=sptr)
            out = dout.cpu().numpy()  # synchronises with the stream's work
            if pending is not None:
                errors += pending.result()
            pending = pool.submit(check, bits, out)
        errors += pending.result()
    return {"gates": batches * B, "errors": errors, "batches": batches,
            "wall_s": round(time.perf_counter() - t0, 2)}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait(timeout=5)
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        under_load = [s for s in sm if s > 0.3 * max(sm)] if sm else []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(under_load) if under_load else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def cpu_baseline(seconds, batch_hint):
    """The reference library (oracle/_ref, spqlios-fma) on this host's cores, one gate per thread;
    the C oracle port (exact products) if the reference build is absent."""
    import numpy as np
    from tfhe_ref import RefLib
    threads = os.cpu_count() or 1
    ref = RefLib.load()
    if ref is not None:
        keys = ref.keygen(custom=None, seed=4242)
        try:
            per = 1
            rng = np.random.default_rng(0)

            def run(per_thread):
                total = threads * per_thread
                bits = rng.integers(0, 2, (2, total)).astype(np.int32)
                a, b = keys.encrypt(bits[0]), keys.encrypt(bits[1])
                out = np.zeros_like(a)
                dt = keys.bench_gates(0, threads, per_thread, a, b, None, out)
                got, _ = keys.decrypt(out)
                return total, dt, int((got != 1 - (bits[0] & bits[1])).sum())

            total, dt, _ = run(per)  # calibration
            per = max(1, int(seconds / max(dt, 1e-3)))
            total, dt, errors = run(per)
            return {"value": total / dt, "unit": UNIT, "cores": threads, "kind": "reference",
                    "sample": f"{total} bootsNAND (default params) on {threads} threads, one gate per thread, "
                              f"{dt:.1f} s, {errors} decryption errors"}
        finally:
            keys.free()
    from tfhe_oracle import DEFAULT, Oracle
    o = Oracle.get()
    lk, tk, ksk, bsk = o.keygen(DEFAULT, seed=3)
    rng = np.random.default_rng(0)
    bits = rng.integers(0, 2, (2, 4))
    a, b = o.encrypt_bits(lk, bits[0], seed=1), o.encrypt_bits(lk, bits[1], seed=2)
    t0 = time.perf_counter()
    o.gate(DEFAULT, bsk, ksk, 0, a, b)
    dt = time.perf_counter() - t0
    return {"value": 4 / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"4 bootsNAND through the C oracle (exact products), 1 thread, {dt:.1f} s"}


def run_reference(args, rank):
    if rank != 0:
        return
    t0 = time.perf_counter()
    vals = []
    base = None
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(max(2.0, args.cpu_seconds / max(1, args.steps)), args.batch)
        if i >= args.warmup:
            vals.append(r["value"])
            base = r
    value = sum(vals) / len(vals)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "bootsNAND at the default 128-bit parameters on the host cores, "
                                   "one gate per thread (tfhe v1.1 spqlios-fma)", "params": PARAMS},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": base["cores"], "kind": base["kind"],
                             "sample": base["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": time.perf_counter() - t0}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload != "nand":
        if rank == 0:
            run_extra_workload(args)
        return

    import ctypes

    import numpy as np
    import torch

    import tfhe_b200 as tb

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    p = tb.default_params()
    sk, ck = tb.keygen(p, seed=1000 + rank)
    ck.to_device(local_rank)
    B = args.batch
    rng = np.random.default_rng(rank)
    bits = rng.integers(0, 2, (2, B))
    ha, hb = sk.encrypt(bits[0], seed=11 + rank), sk.encrypt(bits[1], seed=12 + rank)
    d_a = torch.from_numpy(ha).cuda()
    d_b = torch.from_numpy(hb).cuda()
    d_out = torch.zeros_like(d_a)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device="cuda")  # 256 MiB > 126 MB L2
    stream = torch.cuda.Stream()  # a real stream: the engine's kernels and the timing events share it
    torch.cuda.set_stream(stream)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    L = tb.api.lib()

    def barrier():
        if dist is not None:
            dist.barrier()

    def measure(form):
        precision = tb.SPLIT_FP32 if form == "split" else tb.FP64
        for _ in range(args.warmup):
            ck.gate_device(tb.api.NAND, d_a, d_b, None, d_out, B, precision=precision, stream=sptr)
        torch.cuda.synchronize()
        got, _ = sk.decrypt(d_out.cpu().numpy())
        errors = int((got != 1 - (bits[0] & bits[1])).sum())
        L.tfheb_profile(ck.h, 1)
        L.tfheb_profile_read(ck.h, None, None, 1)
        barrier()
        torch.cuda.synchronize()
        launches0 = tb.kernel_launches()
        evs = []
        for i in range(args.steps):
            flush.fill_(i)  # evict the L2 between timed steps (outside the events)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ck.gate_device(tb.api.NAND, d_a, d_b, None, d_out, B, precision=precision, stream=sptr)
            e1.record(stream)
            evs.append((e0, e1))
        torch.cuda.synchronize()
        barrier()
        launches = tb.kernel_launches() - launches0
        total_ms = sum(a.elapsed_time(b) for a, b in evs)
        kms = (ctypes.c_double * 4)()
        kn = (ctypes.c_int64 * 4)()
        L.tfheb_profile_read(ck.h, kms, kn, 1)
        L.tfheb_profile(ck.h, 0)
        slowest_ms, _ = replica_throughput(total_ms, B * args.steps, world, dist, "cuda")
        return {"total_ms": slowest_ms, "errors": errors, "launches": launches,
                "kernel_ms": [kms[i] / max(1, kn[i]) for i in range(4)], "kernel_n": [kn[i] for i in range(4)]}

    # pick the fastest compiled blind-rotation launch variant for this batch (both precisions)
    tuning = {}
    for name, prec in (("split", tb.SPLIT_FP32), ("fp64", tb.FP64)):
        tuning[name] = ck.autotune(prec, boots=B)

    # FMA throughput probe (roofline denominator at the current clocks)
    peak = {}
    for name, prec in (("fp32", tb.SPLIT_FP32), ("fp64", tb.FP64)):
        v = ctypes.c_double()
        L.tfheb_measure_fma_peak(local_rank, prec, ctypes.byref(v))
        peak[name] = v.value

    other = "fp64" if args.form == "split" else "split"
    clocks = ClockSampler(local_rank)
    clocks.start()
    main_r = measure(args.form)
    clk = clocks.stop()
    other_r = measure(other)

    gates = B * args.steps * world
    value = gates / (main_r["total_ms"] / 1e3)
    other_value = gates / (other_r["total_ms"] / 1e3)

    # end to end through the public host API: pinned host inputs in, host outputs back, every step
    pa = torch.from_numpy(ha).pin_memory()
    pb = torch.from_numpy(hb).pin_memory()
    po = torch.empty_like(pa).pin_memory()
    precision = tb.SPLIT_FP32 if args.form == "split" else tb.FP64
    L.tfheb_gate_batch(ck.h, tb.api.NAND, precision, B, ctypes.c_void_p(pa.data_ptr()),
                       ctypes.c_void_p(pb.data_ptr()), None, ctypes.c_void_p(po.data_ptr()))
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        st = L.tfheb_gate_batch(ck.h, tb.api.NAND, precision, B, ctypes.c_void_p(pa.data_ptr()),
                                ctypes.c_void_p(pb.data_ptr()), None, ctypes.c_void_p(po.data_ptr()))
        assert st == 0
    e2e_s = time.perf_counter() - t0
    e2e_ms, e2e_value = replica_throughput(e2e_s * 1e3, B * args.e2e_steps, world, dist, "cuda")
    got, _ = sk.decrypt(po.numpy())
    e2e_errors = int((got != 1 - (bits[0] & bits[1])).sum())

    # decryption-error count over >= 10^6 fresh gates per form, outside every timed region
    errors_1e6 = None
    if args.error_gates > 0:
        errors_1e6 = {form: count_errors(ck, sk, form, args.error_gates, stream, sptr, seed=90 + rank)
                      for form in (args.form, other)}

    if rank == 0:
        br_ms = main_r["kernel_ms"][1]
        flops = FLOPS_PER_GATE[args.form] * B
        achieved = flops / (br_ms / 1e3) / 1e12
        pk = peak["fp32" if args.form == "split" else "fp64"]
        # DRAM traffic of the default blind-rotation variant per launch of this batch, from a one-kernel
        # ncu capture (profiles/traffic.json names the variant and the command)
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tpath):
            traffic = json.load(open(tpath)).get(f"blind_rotate_{args.form}")
        # nominal CUDA-core peak at the highest SM clock seen: SMs x lanes x 2 flops x clock
        sms = torch.cuda.get_device_properties(local_rank).multi_processor_count
        lanes = 128 if args.form == "split" else 64
        nominal = sms * lanes * 2 * (clk.get("sm_max_mhz") or 1965.0) * 1e6 / 1e12
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": main_r["total_ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.form == "split" else "f64",
            "data": "synthetic",
            "config": {"workload": f"{B} independent bootsNAND per step (one batch), default 128-bit params, "
                                   f"{'split-FP32' if args.form == 'split' else 'FP64'} external product",
                       "params": PARAMS, "global_batch": B * world, "parallelism": f"replicas x{world}",
                       "l2": "256 MiB buffer written between timed steps (outside the events)"},
            "errors": main_r["errors"],
            "fp64" if args.form == "split" else "split": {
                "value": other_value, "ms_per_step": other_r["total_ms"] / args.steps, "errors": other_r["errors"],
                "kernel_ms": other_r["kernel_ms"]},
            "kernel_ms": {"prologue": main_r["kernel_ms"][0], "blind_rotate": main_r["kernel_ms"][1],
                          "extract": main_r["kernel_ms"][2], "keyswitch": main_r["kernel_ms"][3]},
            "roofline": {"bound": "fp32" if args.form == "split" else "fp64", "kernel": "blind_rotate_kernel",
                         "achieved": achieved, "peak": pk, "unit": "TFLOP/s", "frac": achieved / pk,
                         "peak_source": "measured FMA-chain probe on this GPU (tfheb_measure_fma_peak)",
                         "peak_nominal": nominal, "frac_nominal": achieved / nominal,
                         "nominal_source": f"{sms} SMs x {lanes} lanes x 2 flops x max SM clock",
                         "traffic": traffic.get("bytes_per_launch") if traffic else None,
                         "traffic_variant": traffic.get("variant") if traffic else None,
                         "traffic_source": traffic.get("source") if traffic else None,
                         "algorithmic": f"{FLOPS_PER_GATE[args.form] / 1e6:.2f} MFLOP/gate x {B} gates per launch"},
            "peaks_measured": peak,
            "autotune": tuning,
            "plans": {"0": "radix-8 team FFT, one transform per thread",
                      "1": "radix-8 team FFT, two transforms per thread on packed f32x2, digit spectra in TMEM "
                           "(candidates differ in ring depth and in how many transform pairs run interleaved)"},
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * B * (p.n + 1) * 4,
                    "d2h_bytes_per_step": B * (p.n + 1) * 4, "errors": e2e_errors,
                    "api": "tfheb_gate_batch (host buffers, pinned)"},
            "gpu_launches": main_r["launches"],
            "errors_1e6": errors_1e6,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args.cpu_seconds, B)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Benchmark: HBM GB/s per state pass on the 30-qubit complex<double> brick
circuit (H layer + 20 layers of U3 on every qubit and CNOT pairs, seeded
angles, written with BEGIN/END FUSION blocks of <= 5 qubits), on one B200.

A step applies the whole circuit to the state held in HBM.  value = state
passes executed x bytes per pass (2 * 2^30 * 16 B = 34.36 GB) / step time,
summed over ranks; the time is taken with CUDA events on the library's own
stream (rbk_state_device_ms), max over ranks.  `e2e` repeats the measurement
through the C ABI as a bra run sees it: reset to |0...0>, the gate calls,
DO MEASUREMENT (all spins) and its read-back, all inside the timed region.

--impl reference times the reference's own CPU code (ket + bra fused gates,
release flags -Ofast -fopenmp, all host cores) on a bounded sample of the
same circuit: its 4-qubit fusion blocks (4 U3 + 2 CNOT each), one reference
pass per block, the same blocks the GPU arm's cpu_baseline leg times.  Both
arms also report a circuit time: the GPU's measured, the reference's
extrapolated from its mean block time to the circuit's 156 passes.

Multi-GPU: the path does not shard in this tier, so --gpus N runs N
independent replicas (one process per GPU, launched by torchrun).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_QUBITS = 30
DEPTH = 20
FUSE_K = 5
SEED = 1
METRIC = "HBM GB/s per state pass (30q c128 brick, depth 20, fusion k<=5)"
WORKLOAD = "brick circuit: 30 qubits, complex<double>, H layer + 20 layers of U3 (seeded) and CNOT pairs, BEGIN/END FUSION blocks of <= 5 qubits"


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic():
    """dram bytes per launch of the pass kernel, from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def host_mem_available():
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except Exception:
        pass
    return 0


def reference_blocks(ops):
    """Splits the instruction list into the reference's state passes: one per
    fusion block, one per gate outside a block."""
    blocks, cur, inside = [], [], False
    for op in ops:
        if op[0] == "BEGIN FUSION":
            inside, cur = True, [op]
        elif op[0] == "END FUSION":
            cur.append(op)
            blocks.append(cur)
            inside, cur = False, []
        elif inside:
            cur.append(op)
        else:
            blocks.append([op])
    return blocks


def sample_blocks(ops):
    """The blocks both CPU legs time: the 4-qubit fusion blocks of the brick
    layers (each 4 U3 and 2 CNOT on 4 consecutive qubits), in circuit order.  They share one structure, so a few of them give the same mean as
    many; the circuit's other blocks hold 2-5 qubits and 2-7 gates."""
    out = []
    for b in reference_blocks(ops):
        gates = [op for op in b if op[0] not in ("BEGIN FUSION", "END FUSION")]
        qubits = {q for op in gates for q in op[1]}
        kinds = sorted(op[0] for op in gates)
        if len(qubits) == 4 and kinds == ["CNOT", "CNOT", "U3", "U3", "U3", "U3"]:
            out.append(b)
    return out


class CpuReference:
    """The reference's own ket/bra code, release build (oracle/_ref/libketref_fast.so)."""

    def __init__(self, n, threads):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        self.kind = "reference"
        self.state = oracle.KetRef(n, threads=threads, fast=True)
        self.n, self.threads = n, threads

    def run_blocks(self, blocks):
        t = 0.0
        for b in blocks:
            t += self.state.apply_timed(b)
        return t


def cpu_sample(ops, threads, budget_s, n=N_QUBITS):
    """Times reference passes of the workload on the host, the blocks of
    sample_blocks() in order (the ones the reference arm's timed steps start
    with), until budget_s of CPU time is spent.  Returns (passes, seconds,
    description)."""
    need = (16 << n) * 1.1
    if host_mem_available() < need:
        return None, None, f"host has {host_mem_available() / 2**30:.0f} GiB free, a {n}-qubit state needs {need / 2**30:.0f} GiB"
    ref = CpuReference(n, threads)
    blocks = sample_blocks(ops)
    done, secs = 0, 0.0
    while done < len(blocks) and secs < budget_s:
        secs += ref.run_blocks([blocks[done]])
        done += 1
    desc = (f"first {done} of the {len(blocks)} 4-qubit fusion blocks (4 U3 + 2 CNOT) of the {n}-qubit circuit, "
            f"one reference pass each")
    return done, secs, desc


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world == 1:
        return world, rank, local, None
    import datetime

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local, dist


def dist_max(dist, value, local):
    """The maximum over ranks (NCCL reduces on the rank's GPU; gloo on the host)."""
    if dist is None:
        return value
    import torch
    device = f"cuda:{local}" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, local):
    if dist is not None:
        import torch
        if dist.get_backend() == "nccl":
            dist.barrier(device_ids=[local])
            torch.cuda.synchronize(local)
        else:
            dist.barrier()


def run_gpu(args):
    world, rank, local, dist = dist_setup()
    from __graft_entry__ import load_package
    pkg = load_package()
    C = pkg.circuits
    ops = C.brick(N_QUBITS, DEPTH, seed=SEED, fuse_k=FUSE_K)
    ref_passes = C.reference_passes(ops)
    bytes_pass = 2 * (1 << N_QUBITS) * 16

    s = pkg.State(N_QUBITS, pkg.C128, device=local)
    if args.shape is not None:
        s.set_tile_shape(args.shape)
    if args.budget is not None:
        s.set_pass_budget(args.budget)
    for _ in range(args.warmup):
        s.apply(ops)
        s.synchronize()

    # ---- device-resident throughput: the circuit applied K times to the state in HBM
    barrier(dist, local)
    s.synchronize()
    s.reset_stats()
    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(args.steps):
        s.apply(ops)
    ms = s.device_ms()  # CUDA events on the library's stream, first launch .. last completion
    clk = clocks.stop()
    st = s.stats()
    ms_max = dist_max(dist, ms, local)
    passes_per_step = st["passes"] / args.steps
    value = world * st["passes"] * bytes_pass / (ms_max * 1e-3) / 1e9
    launch_ms = ms / max(1, st["passes"])
    achieved = bytes_pass / (launch_ms * 1e-3) / 1e9
    peak, peak_kind = load_peaks()

    # ---- end to end through the C ABI: reset, gate calls, DO MEASUREMENT, read-back
    barrier(dist, local)
    s.synchronize()
    s.reset_stats()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s.reset(0)
        s.apply(ops)
        spins = s.spins()  # flush + reduction passes + device->host copy of 3n doubles
    e2e_s = time.perf_counter() - t0
    e2e_max = dist_max(dist, e2e_s, local)
    st_e = s.stats()
    e2e_passes = st_e["passes"] / args.steps
    e2e_value = world * args.steps * e2e_passes * bytes_pass / e2e_max / 1e9
    assert math.isfinite(float(spins.sum()))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        done, secs, desc = cpu_sample(ops, threads, budget_s=args.cpu_budget, n=N_QUBITS)
        if done:
            cpu = {"value": done * bytes_pass / secs / 1e9, "unit": "GB/s", "cores": threads, "kind": "reference",
                   "sample": desc + f", {secs:.1f} s, reference release build (-Ofast -fopenmp)",
                   "circuit_ms_extrapolated": secs / done * ref_passes * 1e3,
                   "circuit_ms_basis": f"mean time of the sampled blocks x {ref_passes} reference passes (extrapolated)"}
        else:
            cpu = {"value": None, "unit": "GB/s", "cores": threads, "kind": "reference", "sample": desc}

    traffic = load_traffic()
    desc_bytes = pkg.rbk.pass_descriptor_bytes()
    line = {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "qubits": N_QUBITS, "depth": DEPTH, "fusion_k": FUSE_K, "seed": SEED,
                   "passes_per_step": passes_per_step, "reference_passes_per_step": ref_passes,
                   "circuit_ms": ms_max / args.steps,
                   "bytes_per_pass": bytes_pass, "l2": "inputs larger than L2 (16 GiB state)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind,
                     "traffic": traffic.get("bytes_per_launch") if traffic else None,
                     "kernel": "rbk::tile_pass_kernel<double>"},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "GB/s", "h2d_bytes_per_step": int(e2e_passes * desc_bytes),
                "d2h_bytes_per_step": 8 * 3 * N_QUBITS, "circuit_ms": e2e_max / args.steps * 1e3,
                "h2d_basis": f"{e2e_passes:g} fused passes x {desc_bytes} B pass descriptor (rbk_pass_descriptor_bytes), "
                             "the kernel parameter block each pass launch carries; other launches' parameters "
                             "(under 100 B each) are not counted",
                "step": "reset |0..0>, gate calls through the C ABI, DO MEASUREMENT (all spins), read-back"},
        "gpu_launches": st["kernel_launches"],
        "clocks": clk,
    }
    s.close()
    if rank == 0 and world == 1 and not args.no_secondary:
        line["secondary"] = secondary_workloads(pkg)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier(device_ids=[local])
        dist.destroy_process_group()


def secondary_workloads(pkg):
    """Configs 3, 4 and 5 measured after the headline's timed region, so that
    the default run records them too:
    * the QFT + brick circuit: 33 qubits complex<double> (128 GiB) and
      32 qubits complex<float> in both fusion modes, one warm-up and one timed
      circuit each, CUDA events on the state's stream (rbk_state_device_ms);
    * the 20-qubit adjoint gradient on a kept context (rbk_adjoint_run;
      3 warm-up, 10 timed) and the 4096-instance complex<double> batch
      (rbk_batch_run; 1 warm-up, 1 timed): host wall clock around calls that
      return their results to the host."""
    A, C = pkg.adjoint, pkg.circuits
    out = {}

    def circuit_ms(n, prec, mode):
        ops = C.qft_brick(n, 5, seed=SEED, fuse_k=6)
        s = pkg.State(n, prec)
        s.set_fusion_mode(mode)
        s.apply(ops)
        s.synchronize()
        s.reset(0)
        s.synchronize()
        s.reset_stats()
        s.apply(ops)
        s.synchronize()
        ms, passes = s.device_ms(), s.stats()["passes"]
        s.close()
        return {"ms": ms, "passes": passes}

    out["qft_brick"] = {"workload": "H j + U m j (m-j+1) for all m > j, then 5 seeded brick layers, fusion blocks of 6",
                        "c128_33q": circuit_ms(33, pkg.C128, 0),
                        "c64_32q_gate_by_gate": circuit_ms(32, pkg.C64, 0),
                        "c64_32q_tensor_core_blocks": circuit_ms(32, pkg.C64, 1)}
    n, layers = 20, 16
    terms = C.ansatz_hamiltonian(n)
    _, theta = C.ansatz(n, layers, seed=SEED)
    spec, _ = A.ansatz_spec(n, layers)
    ctx = A.AdjointContext(n)
    for _ in range(3):
        ctx.gradient(spec, theta, terms)
    t0 = time.perf_counter()
    for _ in range(10):
        ctx.gradient(spec, theta, terms)
    out["adjoint_20q_640_params"] = {"ms_per_gradient": (time.perf_counter() - t0) / 10 * 1e3,
                                     "workload": "energy + gradient, 20-qubit ansatz, 16 layers, 640 parameters"}
    ctx.close()
    inst, thetas = [], []
    for nq, lay, th in C.batch_instances(4096):
        sp, k = A.ansatz_spec(nq, lay)
        inst.append((nq, sp, k, C.ansatz_hamiltonian(nq)))
        thetas.append(th)
    b = A.Batch(inst, precision=pkg.C128)
    b.run(thetas)
    t0 = time.perf_counter()
    b.run(thetas)
    secs = time.perf_counter() - t0
    out["batch_4096_c128"] = {"seconds": secs, "instances_per_s": len(inst) / secs,
                              "workload": "4096 ansatz instances, n log-uniform in [10, 24], depth U{4..16}, "
                                          "energies + adjoint gradients"}
    b.close()
    return out


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from __graft_entry__ import load_package
    C = load_package().circuits
    ops = C.brick(N_QUBITS, DEPTH, seed=SEED, fuse_k=FUSE_K)
    bytes_pass = 2 * (1 << N_QUBITS) * 16
    threads = os.cpu_count() or 1
    need = (16 << N_QUBITS) * 1.1
    if host_mem_available() < need:
        print(json.dumps({"impl": "reference", "unavailable": f"host RAM: {host_mem_available() / 2**30:.0f} GiB free, "
                                                             f"the 30-qubit state needs {need / 2**30:.0f} GiB"}))
        return
    ref = CpuReference(N_QUBITS, threads)
    blocks = sample_blocks(ops)
    per_step = max(1, args.ref_blocks_per_step)
    # Warm-up steps take the blocks just before the sample's start (cyclically),
    # so that the timed steps begin with its first block, as the GPU arm's
    # cpu_baseline leg does.
    pos = -args.warmup * per_step

    def step():
        nonlocal pos
        chunk = [blocks[(pos + i) % len(blocks)] for i in range(per_step)]
        pos += per_step
        return ref.run_blocks(chunk)

    for _ in range(args.warmup):
        step()
    secs = sum(step() for _ in range(args.steps))
    value = args.steps * per_step * bytes_pass / secs / 1e9
    ref_passes = C.reference_passes(ops)
    sample = (f"{per_step} reference pass(es) per step from the {len(blocks)} 4-qubit fusion blocks (4 U3 + 2 CNOT) "
              f"of the 30-qubit circuit, in circuit order from the first; "
              f"reference release build (-Ofast -fopenmp), {threads} threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "qubits": N_QUBITS, "depth": DEPTH, "fusion_k": FUSE_K, "seed": SEED,
                   "reference_passes_per_step": ref_passes,
                   "circuit_ms_extrapolated": secs / (args.steps * per_step) * ref_passes * 1e3,
                   "circuit_ms_basis": f"mean time of the timed blocks x {ref_passes} reference passes (extrapolated)"},
        "cpu_baseline": {"value": value, "unit": "GB/s", "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_adjoint(args):
    """Config 4: energy + adjoint gradient of the 20-qubit ansatz (16 layers of
    RY, RZ and a CZ ring; 640 parameters; H = sum Z_i Z_i+1 + 0.5 sum X_i),
    against per-parameter plain GPU evaluation (parameter shift, 2 energies per
    parameter) and the reference's CPU code doing the same."""
    from __graft_entry__ import load_package
    pkg = load_package()
    C = pkg.circuits
    n, layers = 20, 16
    terms = C.ansatz_hamiltonian(n)
    _, theta = C.ansatz(n, layers, seed=SEED)
    spec, nparams = pkg.adjoint.ansatz_spec(n, layers)
    ctx = pkg.adjoint.AdjointContext(n)  # an optimiser loop keeps its two state vectors
    for _ in range(args.warmup):
        ctx.gradient(spec, theta, terms)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e, g = ctx.gradient(spec, theta, terms)
    t_adj = (time.perf_counter() - t0) / args.steps
    ctx.close()

    # Per-parameter plain GPU evaluation: E(theta +- pi/2 e_k) through the fused engine.
    s = pkg.State(n, pkg.C128)
    sample = list(range(0, nparams, max(1, nparams // 16)))[:16]

    def energy_gpu(th):
        s.reset(0)
        s.apply(C.ansatz(n, layers, thetas=th)[0])
        return s.expectation(terms).real

    energy_gpu(theta)
    t0 = time.perf_counter()
    shift = []
    for k in sample:
        tp, tm = theta.copy(), theta.copy()
        tp[k] += math.pi / 2
        tm[k] -= math.pi / 2
        shift.append(0.5 * (energy_gpu(tp) - energy_gpu(tm)))
    t_shift = (time.perf_counter() - t0) / len(sample) * nparams
    err = max(abs(a - g[k]) for a, k in zip(shift, sample))

    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        threads = os.cpu_count() or 1
        ops, _ = C.ansatz(n, layers, thetas=theta)
        r = oracle.KetRef(n, threads=threads, fast=True)
        secs = r.apply_timed(ops)
        t1 = time.perf_counter()
        r.expectation(terms)
        secs += time.perf_counter() - t1
        cpu = {"value": 1.0 / (secs * 2 * nparams), "unit": "gradients/s", "cores": threads, "kind": "reference",
               "sample": f"one energy evaluation (ket forward + expectation, release build) = {secs:.3f} s, "
                         f"times 2 x {nparams} parameter-shift evaluations"}
    peak, peak_kind = load_peaks()
    line = {
        "metric": "adjoint gradients/s (20q ansatz, 640 parameters)", "value": 1.0 / t_adj, "unit": "gradients/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_adj * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "energy + adjoint gradient, 20-qubit hardware-efficient ansatz, 16 layers, 640 parameters",
                   "per_parameter_gpu_ms": t_shift * 1e3, "speedup_vs_per_parameter_gpu": t_shift / t_adj,
                   "max_abs_diff_vs_parameter_shift": err, "energy": e,
                   "timing": "host wall clock per gradient on a reused context (rbk_adjoint_run): parameters in, energy and gradient out"},
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def run_batch(args):
    """Config 5: energies + adjoint gradients of a batch of independent ansatz
    instances (n log-uniform in [10, 24], depth U{4..16}, per-instance seeds
    1 + index) in complex<double> and complex<float>; the complex<float> results
    are compared instance by instance with the complex<double> ones."""
    from __graft_entry__ import load_package
    pkg = load_package()
    A, C = pkg.adjoint, pkg.circuits
    draws = C.batch_instances(args.instances)
    inst, thetas = [], []
    for n, layers, th in draws:
        spec, k = A.ansatz_spec(n, layers)
        inst.append((n, spec, k, C.ansatz_hamiltonian(n)))
        thetas.append(th)
    results, stats, times = {}, {}, {}
    for prec, name in ((pkg.C128, "c128"), (pkg.C64, "c64")):
        b = A.Batch(inst, precision=prec)
        for _ in range(args.warmup):
            b.run(thetas)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e, g = b.run(thetas)
        times[name] = (time.perf_counter() - t0) / args.steps
        results[name] = (e, g)
        stats[name] = b.stats()
        stats[name]["tuned_tile_shapes"] = {str(k): v for k, v in b.tuned_shapes([d[0] for d in draws]).items()}
        b.close()
    e64, g64 = results["c128"]
    e32, g32 = results["c64"]
    e_err = float(np.max(np.abs(e32 - e64)))
    g_err = float(max(np.abs(a - b).max() for a, b in zip(g32, g64)))
    ns = np.array([d[0] for d in draws])
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        threads = os.cpu_count() or 1
        # parameter-shift gradient on the reference's CPU code for a sample: 2 energies per parameter
        secs, done = 0.0, 0
        for i in range(0, len(draws), max(1, len(draws) // 8)):
            n, layers, th = draws[i]
            ops, _ = C.ansatz(n, layers, thetas=th)
            r = oracle.KetRef(n, threads=threads, fast=True)
            t = r.apply_timed(ops)
            t1 = time.perf_counter()
            r.expectation(C.ansatz_hamiltonian(n))
            t += time.perf_counter() - t1
            secs += t * 2 * len(th)
            done += 1
        cpu = {"value": done / secs, "unit": "instances/s", "cores": threads, "kind": "reference",
               "sample": f"{done} instances spread over the batch, each one energy evaluation with the reference ket "
                         f"code (release build) times 2 x parameters (parameter shift)"}
    line = {
        "metric": "batched energy + adjoint gradient, instances/s", "value": len(inst) / times["c128"],
        "unit": "instances/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": times["c128"] * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{len(inst)} ansatz instances, n log-uniform in [10, 24] (round), depth U{{4..16}}, "
                               "H = sum Z_i Z_i+1 + 0.5 sum X_i",
                   "qubit_histogram": {str(k): int(v) for k, v in zip(*np.unique(ns, return_counts=True))},
                   "c128": {"seconds": times["c128"], **stats["c128"]},
                   "c64": {"seconds": times["c64"], "instances_per_s": len(inst) / times["c64"], **stats["c64"]},
                   "c64_vs_c128_max_abs_energy_diff": e_err, "c64_vs_c128_max_abs_gradient_diff": g_err,
                   "timing": "host wall clock per batch run (parameters in, energies and gradients out)"},
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def run_qft(args):
    """Config 3: H on qubit j then U m j (m-j+1) for every m > j (all n(n-1)/2
    controlled phases), then 5 seeded brick layers, in fusion blocks of 6 qubits.
    complex<float> at 32 qubits (gate-by-gate fused passes, and the tensor-core
    mode that runs 5-6 qubit blocks as 3xTF32 GEMMs), complex<double> at 33
    qubits (128 GiB), and the complex<float> accuracy against complex<double> at
    30 qubits."""
    from __graft_entry__ import load_package
    pkg = load_package()
    C = pkg.circuits
    out = {}

    def timed(n, prec, mode, ops):
        s = pkg.State(n, prec)
        s.set_fusion_mode(mode)
        for _ in range(args.warmup):
            s.reset(0)
            s.apply(ops)
            s.synchronize()
        times, st = [], None
        for _ in range(args.steps):
            s.reset(0)
            s.synchronize()
            s.reset_stats()
            s.apply(ops)
            s.synchronize()
            times.append(s.device_ms())
            st = s.stats()
        return s, statistics.median(times), st

    n = 30
    ops = C.qft_brick(n, 5, seed=SEED, fuse_k=6)
    s, ms, st = timed(n, pkg.C128, 0, ops)
    ref = s.amplitudes()
    s.close()
    acc = {}
    for mode, name in ((0, "fused passes"), (1, "tensor-core blocks")):
        s, ms32, st32 = timed(n, pkg.C64, mode, ops)
        got = s.amplitudes().astype(np.complex128)
        s.close()
        fid = abs(np.vdot(ref, got)) ** 2 / (np.vdot(got, got).real * np.vdot(ref, ref).real)
        acc[name] = {"max_abs_error": float(np.abs(got - ref).max()), "one_minus_fidelity": float(1 - fid),
                     "ms": ms32}
    del ref, got
    big = {}
    ops32 = C.qft_brick(32, 5, seed=SEED, fuse_k=6)
    for mode, name in ((0, "fused passes"), (1, "tensor-core blocks")):
        s, ms32, st32 = timed(32, pkg.C64, mode, ops32)
        s.close()
        big[name] = {"ms": ms32, "passes": st32["passes"], "relabel_passes": st32["relabel_passes"]}
    ops33 = C.qft_brick(33, 5, seed=SEED, fuse_k=6)
    s, ms33, st33 = timed(33, pkg.C128, 0, ops33)
    s.close()
    bytes33 = 2 * (1 << 33) * 16
    line = {
        "metric": "circuit time, 33-qubit complex<double> QFT + 5 brick layers", "value": ms33, "unit": "ms",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms33, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "H j + U m j (m-j+1) for all m > j, then 5 seeded brick layers, fusion blocks of 6",
                   "c128_33q": {"ms": ms33, "passes": st33["passes"],
                                "gb_per_s_per_pass": st33["passes"] * bytes33 / ms33 / 1e6},
                   "c64_32q": big, "c64_vs_c128_at_30q": acc,
                   "timing": "CUDA events on the state's stream (rbk_state_device_ms), median of steps"},
        "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="rbk", choices=["rbk", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=25.0, help="seconds of CPU reference work for cpu_baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true", help="skip the config-4 / config-5 timings after the headline")
    ap.add_argument("--ref-blocks-per-step", type=int, default=1)
    ap.add_argument("--qubits", type=int, default=N_QUBITS, help="smaller cases for profiling only")
    ap.add_argument("--depth", type=int, default=DEPTH)
    ap.add_argument("--shape", type=int, default=None, help="tile shape (rbk_state_set_tile_shape)")
    ap.add_argument("--budget", type=int, default=None, help="dense gates per pass (rbk_state_set_pass_budget)")
    ap.add_argument("--workload", default="brick", choices=["brick", "adjoint", "batch", "qft"],
                    help="brick: the 30-qubit circuit (default); adjoint: energy + gradient of the 20-qubit ansatz; "
                         "batch: energies + gradients of a batch of ansatz instances; "
                         "qft: the QFT + brick circuit at 32 (c64) and 33 (c128) qubits")
    ap.add_argument("--instances", type=int, default=4096, help="batch workload: number of instances")
    args = ap.parse_args()
    globals()["N_QUBITS"], globals()["DEPTH"] = args.qubits, args.depth
    if args.workload == "adjoint":
        run_adjoint(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "qft":
        run_qft(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()

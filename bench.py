"""Benchmark of the symmetry-sector matvec and its Lanczos recurrence on B200.

Workload: the periodic XXZ chain N = 32 (J = 1, Delta = 0.7) in the sector S^z = 0, k = 0, reflection-even,
spin-flip-even (group D_32 x Z_2, 128 elements; 4,707,969 representatives found on the device). Synthetic
input: a seeded complex Gaussian vector. One step = one H.v on device-resident vectors with FP32 storage
(FP64 arithmetic) through the lane the engine picks for a sector whose merged CSR fits the device: the
reduced CSR, built once on the device from the row walk (its build time is reported). The on-the-fly walk,
the FP64-storage applies and time-to-E0 (FP64 plain vs FP32 storage + FP64 refinement) are reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs N independent replicas (one process per GPU, launched by torchrun): the path has no
cross-GPU exchange, so the metric is the sum over replicas and the time the max over ranks.
`--impl reference` times the reference engine's own CPU matvec (oracle/_ref) on the host cores: its
default host lane, the merged reduced CSR (built once, outside the timed region) and its OpenMP spmv.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def peaks():
    try:
        with open(MEASURED_PEAKS) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def workload():
    from qed_spin_b200 import lattice as lat
    from qed_spin_b200 import operators as ops
    N = 32
    spec = lat.chain_a1_flip_sector(N)
    prods = ops.xxz_products(lat.chain_bonds(N), 1.0, 0.7)
    prog = ops.row_program(ops.from_products(N, prods))
    return spec, prog, prods


# DRAM bytes (read + write) of one spmv1<complex64> launch on this workload, measured by ncu
# (dram__bytes_read.sum + dram__bytes_write.sum of one launch, cold L2).
SPMV1_CHAIN32_DRAM_BYTES = 596.873472e6 + 38.907392e6

CONFIG = {"workload": "XXZ chain N=32 J=1 Delta=0.7, Sz=0 k=0 reflection-even flip-even (D32 x Z2)",
          "n_sites": 32, "group_size": 128}


class Clocks:
    """SM clock, power and clock-event-reason samples (NVML, read only) taken every 10 ms while the timed
    region runs, plus one sample just before it and one just after, so a short region still has samples."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown"}

    def __init__(self, cuda_index: int):
        self.cuda_index = cuda_index
        self.samples = []
        self.stop = None
        self.thread = None
        self.h = None
        d = os.environ.get("QB_CLOCKS_DIR")   # keeps the raw samples when set
        self.path = os.path.join(d, f"clocks_gpu{cuda_index}.csv") if d and os.path.isdir(d) else None

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            p = torch.cuda.get_device_properties(self.cuda_index)
            bus = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
            return pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.cuda_index)

    def _sample(self):
        import pynvml
        h = self.h
        sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
        try:
            reasons = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
        except AttributeError:
            reasons = pynvml.nvmlDeviceGetCurrentClocksThrottleReasons(h)
        try:
            power = pynvml.nvmlDeviceGetPowerUsage(h) / 1000.0
        except Exception:
            power = None
        self.samples.append((time.time(), sm, reasons, power))

    def __enter__(self):
        import threading
        try:
            self.h = self._handle()
            import pynvml
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self._sample()
            self.stop = threading.Event()

            def run():
                while not self.stop.wait(0.01):
                    self._sample()

            self.thread = threading.Thread(target=run, daemon=True)
            self.thread.start()
        except Exception as e:
            self.h = None
            self.error = str(e)
        return self

    def __exit__(self, *a):
        if self.h is None:
            return
        self.stop.set()
        self.thread.join()
        self._sample()
        if self.path:
            with open(self.path, "w") as fh:
                fh.write("unix_time,sm_mhz,reasons_mask,power_w\n")
                for t, sm, r, pw in self.samples:
                    fh.write(f"{t:.3f},{sm},{r:#x},{pw}\n")

    def summary(self):
        if self.h is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0,
                    "unavailable": getattr(self, "error", "no NVML")}
        sm = [x[1] for x in self.samples]
        reasons = set()
        for _, _, r, _ in self.samples:
            for bit, name in self.REASONS.items():
                if r & bit:
                    reasons.add(name)
        pw = [x[3] for x in self.samples if x[3] is not None]
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": self.max_mhz, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_median": statistics.median(pw) if pw else None, "source": "NVML"}


def dist_init():
    from qed_spin_b200 import replicas
    return replicas.init("nccl")


def dist_max(x: float, world: int) -> float:
    from qed_spin_b200 import replicas
    return replicas.max_over_ranks(x, world)


def barrier(world):
    from qed_spin_b200 import replicas
    replicas.barrier(world)


def _reference_lane(threads):
    """The reference engine on the workload: its sector, its row program and its merged reduced CSR (the
    host lane RepSectorMatVec applies through), with the build times."""
    from oracle import ref as R
    spec, prog, prods = workload()
    R.set_threads(threads)
    t0 = time.time()
    rs = R.Sector(spec.n_sites, spec.n_up, spec.perms, spec.chars, flips=spec.flips, slc_mode=-1)
    sector_s = time.time() - t0
    rp = R.Operator(spec.n_sites, prods).row_program()
    t0 = time.time()
    csr = R.Csr(rs, rp)
    csr_s = time.time() - t0
    return rs, rp, csr, sector_s, csr_s


def run_reference(args, world, rank):
    """The reference engine's own CPU matvec (oracle/_ref) on the host cores: H.v/s on the same workload,
    through its default host lane (ReducedSymmetryCsr::spmv over the CSR build_sector_csr made)."""
    if rank != 0:
        return None
    from oracle import ref as R
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "the reference CPU engine was not built into oracle/_ref"}))
        return None
    threads = os.cpu_count() or 1
    rs, rp, csr, sector_s, csr_s = _reference_lane(threads)
    x = R.staged_seed(1, rs.dim)
    y = np.zeros(rs.dim, np.complex128)
    for _ in range(args.warmup):
        csr.spmv(x, y)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        csr.spmv(x, y)
        times.append(time.perf_counter() - t)
    tot = sum(times)
    v = args.steps / tot
    line = {"impl": "reference", "metric": "H.v/s", "value": v, "unit": "H.v/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(CONFIG, dim=rs.dim, nnz=csr.nnz, csr_bytes=csr.bytes,
                           lane="reduced CSR (build_sector_csr + ReducedSymmetryCsr::spmv, OpenMP)"),
            "cpu_baseline": {"value": v, "unit": "H.v/s", "cores": threads, "kind": "reference",
                             "sample": f"{args.steps} full H.v on the {rs.dim}-state sector"},
            "e2e": {"value": v, "unit": "H.v/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_sector_build_s": sector_s, "reference_csr_build_s": csr_s}
    print(json.dumps(line))
    return line


def cpu_baseline_sample(dim_gpu):
    """The reference engine's CPU matvec on a bounded sample: full H.v through its reduced CSR for about
    10 s, plus a few through its on-the-fly host walk (sector_gather)."""
    from oracle import ref as R
    if not R.available():
        return None
    threads = os.cpu_count() or 1
    rs, rp, csr, sector_s, csr_s = _reference_lane(threads)
    assert rs.dim == dim_gpu
    x = R.staged_seed(1, rs.dim)
    y = np.zeros(rs.dim, np.complex128)
    csr.spmv(x, y)
    n, t0 = 0, time.perf_counter()
    while n < 3 or (time.perf_counter() - t0 < 10.0 and n < 200):
        csr.spmv(x, y)
        n += 1
    dt = time.perf_counter() - t0
    t = time.perf_counter()
    rs.gather(rp, x)
    walk_s = time.perf_counter() - t
    return {"value": n / dt, "unit": "H.v/s", "cores": threads, "kind": "reference",
            "sample": f"{n} full H.v through the reference's reduced CSR (its default host lane) on the "
                      f"{rs.dim}-state sector",
            "csr_build_s": csr_s, "sector_build_s": sector_s, "walk_hv_per_s": 1.0 / walk_s}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ftlm", action="store_true", help="leave the batched FTLM measurement out of the line")
    ap.add_argument("--ftlm", action="store_true",
                    help="batched FTLM over the 600 blocks of the XXZ chain N=24 (every S^z x 24 momenta), one "
                         "JSON line: samples/s against the plain single-sample path and the reference CPU engine")
    ap.add_argument("--serve", action="store_true",
                    help="the served request stream (Poisson arrivals of eigs / S^z(q) dynamics requests on chains "
                         "N = 16..30): p50/p99 latency and solves/s of the server against one solve at a time")
    ap.add_argument("--serve-requests", type=int, default=60)
    ap.add_argument("--no-serve", action="store_true", help="leave the served-stream measurement out of the line")
    ap.add_argument("--e0-6x6", action="store_true",
                    help="time-to-E0 on the 6x6 J1-J2 k=(0,0) sector: the plain FP64 walk against the CSR lane "
                         "(FP64, and FP32 storage + FP64 refinement), one JSON line")
    ap.add_argument("--profile-case", choices=["chain32", "sq30", "sq36", "ftlm4", "chain20"], default=None,
                    help="profiling run: build one sector and apply H (complex64) warmup + steps times, print timing; "
                         "ftlm4: batched FTLM (40 samples, depth 100) on the four largest N = 24 XXZ blocks")
    ap.add_argument("--profile-lane", choices=["walk", "csr", "c64", "c128"], default="walk",
                    help="the lane of the profiling run: the on-the-fly walk or the device reduced CSR; for ftlm4 "
                         "the storage type")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.profile_case:
        profile_case(args)
        return
    if args.e0_6x6:
        e0_6x6(args)
        return
    if args.ftlm:
        ftlm_config(args)
        return
    if args.serve:
        print(json.dumps(serve_measure(args)))
        return

    world, rank, local = dist_init() if args.impl == "b200" else (int(os.environ.get("WORLD_SIZE", "1")),
                                                                   int(os.environ.get("RANK", "0")), 0)
    if args.impl == "reference":
        run_reference(args, world, rank)
        return

    import torch

    from qed_spin_b200 import build
    from qed_spin_b200 import device as D
    build.build()
    torch.cuda.set_device(local)
    dev = torch.cuda.current_device()
    stream = torch.cuda.current_stream()

    spec, prog, prods = workload()
    t0 = time.perf_counter()
    S = D.Sector(spec)
    torch.cuda.synchronize()
    enum_s = time.perf_counter() - t0
    P = D.Program(prog)
    n = S.dim
    info = S.info()

    rng = np.random.default_rng(1)
    x64 = torch.from_numpy(rng.normal(size=n) + 1j * rng.normal(size=n)).to(dev)
    x32 = x64.to(torch.complex64)
    y32 = torch.empty_like(x32)
    y64 = torch.empty_like(x64)
    e_bar = emitted_per_row(S.reps()[0], prog)
    hbm, peak_kind = peaks()

    def time_apply(x, y, dt, steps, warm):
        for _ in range(warm):
            D.matvec(S, S, P, [x], [y], dtype=dt, stream=stream)
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            D.matvec(S, S, P, [x], [y], dtype=dt, stream=stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        barrier(world)
        return dist_max(ms, world) / steps

    # the on-the-fly walk: 8 rep + 8 inv_norm + S_out per row, S_in per emitted entry
    def walk_bytes(sb):
        return n * (8 + 8 + sb) + n * e_bar * sb

    walk_steps = max(5, args.steps // 10)
    walk32 = time_apply(x32, y32, "c64", walk_steps, 3)
    walk64 = time_apply(x64, y64, "c128", walk_steps, 3)

    # time to E0 on the plain FP64 lane (the walk), before the CSR exists
    torch.cuda.synchronize()
    t = time.perf_counter()
    r_plain = D.eigs_lowest(S, P, dtype="c128")
    t_plain = time.perf_counter() - t

    # the reduced CSR, built on the device from the walk, attached to the program
    torch.cuda.synchronize()
    t = time.perf_counter()
    A = D.Csr(S, S, P)
    torch.cuda.synchronize()
    csr_build_s = time.perf_counter() - t
    A.attach(P)
    cinfo = A.info()

    # the CSR matvec: the CSR streamed once, x read (each element at least once) and y written
    def csr_bytes(sb):
        return cinfo["bytes"] + 2 * n * sb

    with Clocks(dev) as clk:
        per32 = time_apply(x32, y32, "c64", args.steps, args.warmup)
    per64 = time_apply(x64, y64, "c128", max(10, args.steps // 2), 3)
    ach32 = csr_bytes(8) / (per32 * 1e-3) / 1e9
    ach64 = csr_bytes(16) / (per64 * 1e-3) / 1e9

    # end to end through the public C-ABI: host start vector in, alpha/beta out, K Lanczos steps
    v0 = (rng.normal(size=n) + 1j * rng.normal(size=n)).astype(np.complex128)
    D.lanczos(S, P, v0, 8, dtype="c64")
    torch.cuda.synchronize()
    barrier(world)
    t = time.perf_counter()
    a, b = D.lanczos(S, P, v0, args.steps, dtype="c64")
    e2e_s = time.perf_counter() - t
    e2e_s = dist_max(e2e_s, world)

    # time to E0 on the CSR lane: FP64 storage, and FP32 storage + FP64 refinement
    torch.cuda.synchronize()
    t = time.perf_counter()
    r64 = D.eigs_lowest(S, P, dtype="c128")
    t64 = time.perf_counter() - t
    t = time.perf_counter()
    r32 = D.eigs_lowest(S, P, dtype="c64", refine=True)
    t32 = time.perf_counter() - t

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline_sample(n)
        except Exception as e:  # the baseline is reported, never required
            cpu = {"unavailable": str(e)}
    # config 2's two lowest levels (the k > 1 lane on the CSR lane, FP64) and config 1 (chain-20, four levels)
    levels = None
    if rank == 0 and world == 1:
        try:
            levels = levels_measure(S, P, args)
        except Exception as e:
            levels = {"unavailable": str(e)}
    # the served request stream, rank 0 at N = 1
    serve = None
    if rank == 0 and world == 1 and not args.no_serve:
        try:
            serve = serve_measure(args)
        except Exception as e:
            serve = {"unavailable": str(e)}
    # the batched FTLM workload (every block of the N = 24 chain), rank 0 at N = 1
    ftlm = None
    if rank == 0 and world == 1 and not args.no_ftlm:
        try:
            ftlm = ftlm_measure(args, with_cpu=not args.no_cpu_baseline)
        except Exception as e:
            ftlm = {"unavailable": str(e)}

    from qed_spin_b200 import replicas
    if rank != 0:
        A.close()
        replicas.finish(world)
        return
    value = replicas.whole_job_rate(1.0, world, per32 * 1e-3)
    line = {
        "metric": "H.v/s", "value": value, "unit": "H.v/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per32, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(CONFIG, dim=n, lane="device reduced CSR (built from the row walk)", nnz=cinfo["nnz"],
                       csr_bytes=cinfo["bytes"], n_dict=cinfo["n_dict"], emitted_per_row=e_bar,
                       storage="complex64 vectors, FP64 arithmetic", lookup=info["lookup"],
                       sublattice=[info["slc_L"], info["slc_m"]],
                       l2=f"inputs larger than the 126 MB L2 (CSR {cinfo['bytes'] / 1e6:.0f} MB streamed per step), "
                          "no flush",
                       parallelism=f"replicas x{world}"),
        "roofline": {"bound": "hbm", "achieved": ach32, "peak": hbm, "unit": "GB/s", "frac": ach32 / hbm,
                     "traffic": SPMV1_CHAIN32_DRAM_BYTES, "traffic_source": "ncu capture of one spmv1 launch on this workload",
                     "peak_kind": peak_kind, "kernel": "spmv1<complex64>",
                     "alg_bytes_per_launch": csr_bytes(8)},
        "fp64": {"ms_per_hv": per64, "hv_per_s": 1e3 / per64, "achieved_gbs": ach64, "frac": ach64 / hbm},
        "csr_build_s": csr_build_s,
        "walk": {"ms_per_hv_fp32": walk32, "hv_per_s_fp32": 1e3 / walk32, "ms_per_hv_fp64": walk64,
                 "achieved_gbs_fp32": walk_bytes(8) / (walk32 * 1e-3) / 1e9,
                 "frac_fp32": walk_bytes(8) / (walk32 * 1e-3) / 1e9 / hbm},
        "e2e": {"value": world * args.steps / e2e_s, "unit": "H.v/s", "h2d_bytes_per_step": 16 * n / args.steps,
                "d2h_bytes_per_step": 16, "path": "qb_lanczos (host v0 in, alpha/beta out, FP32 storage, CSR lane)"},
        "time_to_e0": {"plain_fp64_walk_s": t_plain, "plain_e0": r_plain["e0"], "plain_iters": r_plain["iters"],
                       "csr_build_s": csr_build_s,
                       "csr_fp64_s": t64, "csr_fp64_e0": r64["e0"],
                       "csr_fp32_refined_s": t32, "csr_fp32_refined_e0": r32["e0"], "fp32_matvecs": r32["matvecs"],
                       "rel_err_vs_plain": abs(r32["e0"] - r_plain["e0"]) / abs(r_plain["e0"]),
                       "speedup_vs_plain_incl_build": t_plain / (t32 + csr_build_s)},
        "enumeration_s": enum_s,
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
        "levels": levels,
        "ftlm": ftlm,
        "serve": serve,
    }
    print(json.dumps(line), flush=True)
    A.close()
    replicas.finish(world)


FTLM_N, FTLM_SAMPLES, FTLM_DEPTH, FTLM_SEED = 24, 40, 100, 20240601


def ftlm_workload():
    """XXZ chain N = 24 (J = 1, Delta = 0.5, field h = 0.1 as -h sum S^z): every S^z sector x the 24
    translation momenta (the non-empty ones), 40 temperatures linspace(0.1, 4)."""
    from qed_spin_b200 import lattice as lat
    from qed_spin_b200 import operators as ops
    N = FTLM_N
    prods = ops.xxz_products(lat.chain_bonds(N), 1.0, 0.5) + ops.zeeman_z_products(N, 0.1)
    specs = [lat.chain_sector(N, n_up, k) for n_up in range(N + 1) for k in range(N)]
    betas = 1.0 / np.linspace(0.1, 4.0, 40)
    return specs, prods, ops.row_program(ops.from_products(N, prods)), betas


def ftlm_reference_sample(threads):
    """The reference engine's sampled thermal blocks on the host cores, on a bounded stratified sample: the
    k = 0 block of every S^z sector with 4 samples each at depth 100 (a sample's cost depends only on its
    block, so samples/s carries over to the whole 600-block workload)."""
    from oracle import ref as R
    _, prods, _, betas = ftlm_workload()
    R.set_threads(threads)
    from qed_spin_b200 import lattice as lat
    blocks = [lat.chain_sector(FTLM_N, n_up, 0) for n_up in range(FTLM_N + 1)]
    rs = [R.Sector(s.n_sites, s.n_up, s.perms, s.chars, flips=s.flips, slc_mode=-1) for s in blocks]
    rp = R.Operator(FTLM_N, prods).row_program()
    dims = [r.dim for r in rs]
    t = time.perf_counter()
    R.ftlm_blocks(rs, rp, 4, FTLM_DEPTH, FTLM_SEED, betas)
    dt = time.perf_counter() - t
    # whole-workload estimate: each S^z sector's 24 blocks have about its k = 0 block's dimension
    return {"value": 4 * len(rs) / dt, "unit": "samples/s", "cores": threads, "kind": "reference",
            "sample": f"k=0 block of each of the 25 S^z sectors (dims {min(dims)}..{max(dims)}), 4 samples, depth "
                      f"{FTLM_DEPTH}, CSR lane, the reference's block scheduling; {dt:.1f} s"}


def ftlm_config(args):
    print(json.dumps(ftlm_measure(args, with_cpu=not args.no_cpu_baseline)))


def ftlm_measure(args, with_cpu=True):
    """Batched FTLM over the 554 non-empty blocks of the N = 24 chain: samples/s of the FP64 and FP32-storage
    lanes, the plain single-sample path on a stratified subset, and the reference engine on the host cores."""
    import torch

    from qed_spin_b200 import build
    from qed_spin_b200 import device as D
    build.build()
    specs, prods, prog, betas = ftlm_workload()
    t = time.perf_counter()
    secs = [D.Sector(s) for s in specs]
    secs = [s for s in secs if s.dim > 0]
    torch.cuda.synchronize()
    enum_s = time.perf_counter() - t
    P = D.Program(prog)
    n_blocks = len(secs)
    dims = np.array([s.dim for s in secs])
    out = {"workload": "XXZ chain N=24 J=1 Delta=0.5 h=0.1, every Sz x 24 momenta, 40 samples, depth 100, 40 T",
           "blocks": n_blocks, "dim_total": int(dims.sum()), "dim_max": int(dims.max()), "enumeration_s": enum_s}
    res = {}
    for dtype in ("c128", "c64"):
        D.ftlm_blocks(secs[-8:], P, FTLM_SAMPLES, FTLM_DEPTH, FTLM_SEED, betas, dtype=dtype)   # warm-up
        torch.cuda.synchronize()
        t = time.perf_counter()
        r = D.ftlm_blocks(secs, P, FTLM_SAMPLES, FTLM_DEPTH, FTLM_SEED, betas, dtype=dtype)
        dt = time.perf_counter() - t
        res[dtype] = r
        out[f"batched_{dtype}"] = {"s": dt, "samples_per_s": n_blocks * FTLM_SAMPLES / dt, "phases": r["stats"]}
    tot64, tot32 = res["c128"]["total"], res["c64"]["total"]
    out["fp32_vs_fp64_max_rel"] = {k: float(np.max(np.abs(tot32[k] - tot64[k]) / np.maximum(np.abs(tot64[k]), 1e-12)))
                                   for k in ("lnZ", "E", "C")}
    i1 = int(np.argmin(np.abs(1.0 / betas - 1.0)))
    out["thermo_T1"] = {"T": float(1.0 / betas[i1]), "E_per_site": float(tot64["E"][i1] / FTLM_N),
                        "C_per_site": float(tot64["C"][i1] / FTLM_N), "S_per_site": float(tot64["S"][i1] / FTLM_N)}
    # the plain path: one sample at a time, FP64, the on-the-fly walk, on a stratified subset (the k = 0 block
    # of every S^z sector, one sample each)
    from qed_spin_b200 import lattice as lat
    sub = [D.Sector(lat.chain_sector(FTLM_N, n_up, 0)) for n_up in range(FTLM_N + 1)]
    torch.cuda.synchronize()
    t = time.perf_counter()
    for s in sub:
        D.ftlm_blocks([s], P, 1, FTLM_DEPTH, FTLM_SEED, betas, use_csr=False)
    dt = time.perf_counter() - t
    out["plain_fp64_walk"] = {"samples_per_s": len(sub) / dt,
                              "sample": "k=0 block of each S^z sector, 1 sample each, one call per sample"}
    out["speedup_batched_fp64_vs_plain"] = out["batched_c128"]["samples_per_s"] / out["plain_fp64_walk"]["samples_per_s"]
    if with_cpu:
        try:
            out["cpu_baseline"] = ftlm_reference_sample(os.cpu_count() or 1)
        except Exception as e:
            out["cpu_baseline"] = {"unavailable": str(e)}
    return out


def levels_measure(S, P, args):
    """The k > 1 lane: config 2's two lowest levels on the attached CSR (FP64), and config 1 (the Heisenberg chain
    N = 20, Sz = 0, k = 0, lowest four) on the device against the reference engine's krylov_schur_kernel on the
    host cores."""
    import torch

    from qed_spin_b200 import device as D
    from qed_spin_b200 import lattice as lat
    from qed_spin_b200 import operators as ops
    out = {}
    torch.cuda.synchronize()
    t = time.perf_counter()
    r2 = D.eigs(S, P, 2)
    out["chain32_k2"] = {"s": time.perf_counter() - t, "values": list(map(float, r2["values"])),
                         "converged": r2["converged"], "matvecs": r2["matvecs"], "lane": "Krylov-Schur on the CSR"}
    spec = lat.chain_sector(20, 10, 0)
    prods = ops.heisenberg_products(lat.chain_bonds(20))
    prog = ops.row_program(ops.from_products(20, prods))
    S20, P20 = D.Sector(spec), D.Program(prog)
    D.eigs(S20, P20, 4)   # warm
    t = time.perf_counter()
    r4 = D.eigs(S20, P20, 4)
    dev_s = time.perf_counter() - t
    out["chain20_k4"] = {"device_s": dev_s, "values": list(map(float, r4["values"])), "converged": r4["converged"],
                         "matvecs": r4["matvecs"], "dim": S20.dim}
    if not args.no_cpu_baseline:
        try:
            from oracle import ref as R
            if R.available():
                R.set_threads(os.cpu_count() or 1)
                rs = R.Sector(20, 10, spec.perms, spec.chars, flips=spec.flips, slc_mode=-1)
                rp = R.Operator(20, prods).row_program()
                t = time.perf_counter()
                ev, cv, ap = rs.ks_lowest(rp, 4, use_csr=True)
                out["chain20_k4"]["reference_cpu_s"] = time.perf_counter() - t
                out["chain20_k4"]["reference_values"] = list(map(float, ev))
                out["chain20_k4"]["max_abs_diff"] = float(np.max(np.abs(np.array(ev) - r4["values"])))
        except Exception as e:
            out["chain20_k4"]["reference_unavailable"] = str(e)
    out["graphs_chain20"] = graphs_measure(S20, P20)
    return out


def graphs_measure(S, P):
    """The lanes that batch their steps into captured CUDA graphs on a small sector (chain-20, 9,252 states),
    with graphs and launched step by step (QB_GRAPHS=0): the certified ground-state vector and a 200-step
    continued fraction; and, as a control, the k = 1 lane, which runs step by step either way. Median seconds of
    5 calls each after a warm-up call."""
    from qed_spin_b200 import device as D
    rng = np.random.default_rng(1)
    phi = rng.standard_normal(S.dim) + 1j * rng.standard_normal(S.dim)
    omega = np.linspace(-0.5, 6.0, 400)
    calls = {"k1_lane": lambda: D.eigs_lowest(S, P),
             "ground_state_vector": lambda: D.ground_state(S, P),
             "continued_fraction_200": lambda: D.cf(S, P, phi, 200, omega, 0.05)}
    out = {}
    saved = os.environ.get("QB_GRAPHS")
    try:
        for flag, key in (("1", "graphs_s"), ("0", "step_by_step_s")):
            os.environ["QB_GRAPHS"] = flag
            for name, fn in calls.items():
                fn()
                ts = []
                for _ in range(5):
                    t = time.perf_counter()
                    fn()
                    ts.append(time.perf_counter() - t)
                out.setdefault(name, {})[key] = float(np.median(ts))
    finally:
        if saved is None:
            os.environ.pop("QB_GRAPHS", None)
        else:
            os.environ["QB_GRAPHS"] = saved
    for v in out.values():
        v["speedup"] = v["step_by_step_s"] / v["graphs_s"]
    return out


def serve_requests(n: int, seed: int = 7):
    """The served stream's requests: periodic chains with N uniform in 16..30 and n_up = N // 2 (S^z = 0 for
    even N, -1/2 for odd), H = J sum S_i.S_{i+1} + K sum S_i.(S_{i+1} x S_{i+2}) with J ~ U[0.5, 1.5] and
    K ~ U[0, 0.3] drawn per request (uniform over the bonds, so translations stay a symmetry); half eigs (k
    uniform in 1..4 in a uniform momentum sector), half T = 0 dynamics of S^z(q) from the lowest state of the
    k = 0 sector, q = 2 pi m / N with m uniform, Krylov 200, 400 frequencies in [-0.5, 6], eta = 0.05."""
    from qed_spin_b200 import lattice as lat
    from qed_spin_b200 import operators as ops
    rng = np.random.default_rng(seed)
    omega = np.linspace(-0.5, 6.0, 400)
    out = []
    for _ in range(n):
        N = int(rng.integers(16, 31))
        J = float(rng.uniform(0.5, 1.5))
        K = float(rng.uniform(0.0, 0.3))
        prods = ops.heisenberg_products(lat.chain_bonds(N), J) + ops.chiral_products(
            [(i, (i + 1) % N, (i + 2) % N) for i in range(N)], K)
        h = ops.row_program(ops.from_products(N, prods))
        if rng.random() < 0.5:
            k = int(rng.integers(1, 5))
            mom = int(rng.integers(0, N))
            out.append({"kind": "eigs", "N": N, "spec": lat.chain_sector(N, N // 2, mom), "h": h, "k": k})
        else:
            m = int(rng.integers(0, N))
            src, tgt = lat.chain_sector(N, N // 2, 0), lat.chain_sector(N, N // 2, m)
            op = ops.cross_row_program(ops.from_products(N, ops.sz_q_products(N, 2 * np.pi * m / N)), tgt, src)
            out.append({"kind": "dynamics", "N": N, "src": src, "tgt": tgt, "h": h, "op": op, "omega": omega})
    return out


def serve_run(reqs, arrivals, max_active):
    """Submits each request at its arrival time (seconds from the start) to a server with max_active slots;
    returns the per-request latencies (done - arrival) and the makespan."""
    import threading

    from qed_spin_b200 import device as D
    srv = D.Server(max_active=max_active)
    t0 = srv.clock()
    tickets = [None] * len(reqs)

    def submitter():
        for i, (r, ta) in enumerate(zip(reqs, arrivals)):
            dt = ta - (srv.clock() - t0)
            if dt > 0:
                time.sleep(dt)
            if r["kind"] == "eigs":
                tickets[i] = srv.submit_eigs(r["spec"], r["h"], r["k"])
            else:
                tickets[i] = srv.submit_dynamics(r["src"], r["tgt"], r["h"], r["op"], 200, r["omega"], 0.05)

    th = threading.Thread(target=submitter)
    th.start()
    results = []
    for i in range(len(reqs)):
        while tickets[i] is None:
            time.sleep(0.0005)
        results.append(srv.wait(tickets[i]))
    th.join()
    lat_s = np.array([res["t_done"] - t0 - ta for res, ta in zip(results, arrivals)])
    span = max(res["t_done"] for res in results) - t0
    srv.close()
    return lat_s, span, results


def serve_measure(args):
    import torch

    from qed_spin_b200 import build
    build.build()
    n = args.serve_requests
    reqs = serve_requests(n)
    # warm-up: one of each kind
    serve_run(reqs[:2], [0.0, 0.0], 2)
    # the service time of one solve at a time, back to back
    lat1, span1, _ = serve_run(reqs, [0.0] * n, 1)
    mean_service = span1 / n
    rate = 0.9 / mean_service   # 90% offered load for one solve at a time
    rng = np.random.default_rng(11)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n))
    out = {"workload": "served stream: chains N=16..30, J~U[0.5,1.5], K~U[0,0.3]; half eigs k=1..4, half S^z(q) "
                       "T=0 dynamics (Krylov 200, 400 omega, eta 0.05); Poisson arrivals",
           "requests": n, "mean_service_s_one_at_a_time": mean_service, "arrival_rate_per_s": rate}
    for name, slots in (("plain_one_at_a_time", 1), ("served_continuous_batching", 8)):
        lat, span, res = serve_run(reqs, arrivals, slots)
        torch.cuda.synchronize()
        out[name] = {"slots": slots, "p50_ms": 1e3 * float(np.percentile(lat, 50)),
                     "p99_ms": 1e3 * float(np.percentile(lat, 99)), "solves_per_s": n / span,
                     "makespan_s": span, "unconverged": int(sum(1 for r in res if not r["converged"]))}
    # capacity: the whole stream submitted at once
    lat8, span8, _ = serve_run(reqs, [0.0] * n, 8)
    out["saturated_solves_per_s"] = {"one_at_a_time": n / span1, "served": n / span8}
    return out


def e0_6x6(args):
    """Time to E0 on the 6x6 periodic J1-J2 lattice (J1 = 1, J2 = 0.5), S^z = 0, momentum (0, 0) under the 36
    translations (252,091,362 representatives): the plain FP64 lane (the on-the-fly walk, no CSR) against the
    device reduced CSR with FP64 storage and with FP32 storage + FP64 refinement; the CSR build is counted."""
    import torch

    from qed_spin_b200 import build
    from qed_spin_b200 import device as D
    from qed_spin_b200 import lattice as lat
    from qed_spin_b200 import operators as ops
    build.build()
    nn, nnn = lat.square_j1j2_bonds(6, 6)
    spec = lat.square_k0_sector(6, 6, 18)
    prog = ops.row_program(ops.from_products(36, ops.heisenberg_products(nn, 1.0) + ops.heisenberg_products(nnn, 0.5)))
    t = time.perf_counter()
    S = D.Sector(spec)
    torch.cuda.synchronize()
    enum_s = time.perf_counter() - t
    P = D.Program(prog)
    n = S.dim
    out = {"workload": "6x6 J1-J2 (J2/J1 = 0.5) Sz=0 k=(0,0), translations only", "dim": n, "enumeration_s": enum_s}
    stream = torch.cuda.current_stream()

    def per_apply(dt, steps):
        x = torch.randn(n, dtype=torch.complex64 if dt == "c64" else torch.complex128, device="cuda")
        y = torch.empty_like(x)
        D.matvec(S, S, P, [x], [y], dtype=dt, stream=stream)
        torch.cuda.synchronize()
        e0_, e1_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0_.record(stream)
        for _ in range(steps):
            D.matvec(S, S, P, [x], [y], dtype=dt, stream=stream)
        e1_.record(stream)
        torch.cuda.synchronize()
        del x, y
        return e0_.elapsed_time(e1_) / steps

    out["walk_ms_per_hv_fp64"] = per_apply("c128", 2)
    torch.cuda.synchronize()
    t = time.perf_counter()
    r = D.eigs_lowest(S, P, dtype="c128")
    out["plain_fp64_walk"] = {"s": time.perf_counter() - t, "e0": r["e0"], "iters": r["iters"],
                              "matvecs": r["matvecs"], "converged": r["converged"]}
    t = time.perf_counter()
    A = D.Csr(S, S, P)
    torch.cuda.synchronize()
    out["csr_build_s"] = time.perf_counter() - t
    out["csr"] = A.info()
    A.attach(P)
    out["csr_ms_per_hv_fp32"] = per_apply("c64", 5)
    out["csr_ms_per_hv_fp64"] = per_apply("c128", 5)
    hbm, kind = peaks()
    for dt, sb in (("fp32", 8), ("fp64", 16)):
        ms = out[f"csr_ms_per_hv_{dt}"]
        alg = out["csr"]["bytes"] + 2 * n * sb
        # each x load fetches a whole 32-byte DRAM sector when x is far larger than L2
        sectors = out["csr"]["bytes"] + out["csr"]["nnz"] * 32 + n * sb
        out[f"roofline_{dt}"] = {"alg_bytes": alg, "alg_frac": alg / (ms * 1e-3) / 1e9 / hbm,
                                 "sector_bytes_model": sectors, "sector_frac": sectors / (ms * 1e-3) / 1e9 / hbm,
                                 "peak_gbs": hbm, "peak_kind": kind}
    t = time.perf_counter()
    r = D.eigs_lowest(S, P, dtype="c128")
    out["csr_fp64"] = {"s": time.perf_counter() - t, "e0": r["e0"], "iters": r["iters"], "matvecs": r["matvecs"]}
    t = time.perf_counter()
    r = D.eigs_lowest(S, P, dtype="c64", refine=True)
    out["csr_fp32_refined"] = {"s": time.perf_counter() - t, "e0": r["e0"], "iters": r["iters"],
                               "matvecs": r["matvecs"], "converged": r["converged"]}
    e_ref = out["plain_fp64_walk"]["e0"]
    out["rel_err_fp32_refined_vs_plain"] = abs(out["csr_fp32_refined"]["e0"] - e_ref) / abs(e_ref)
    out["speedup_fp32_refined_incl_build_vs_plain"] = out["plain_fp64_walk"]["s"] / (out["csr_fp32_refined"]["s"]
                                                                                      + out["csr_build_s"])
    print(json.dumps(out))
    A.close()


def profile_case(args):
    """The small profiling workloads of the ncu summaries under profiles/: the sector is built on the device,
    then H is applied to one complex64 vector `warmup + steps` times."""
    import torch

    from qed_spin_b200 import build
    from qed_spin_b200 import device as D
    from qed_spin_b200 import lattice as lat
    from qed_spin_b200 import operators as ops
    build.build()
    if args.profile_case == "ftlm4":
        N = FTLM_N
        prods = ops.xxz_products(lat.chain_bonds(N), 1.0, 0.5) + ops.zeeman_z_products(N, 0.1)
        P = D.Program(ops.row_program(ops.from_products(N, prods)))
        secs = [D.Sector(lat.chain_sector(N, n, k)) for n, k in [(12, 0), (11, 1), (13, 2), (12, 5)]]
        betas = 1.0 / np.linspace(0.1, 4.0, 40)
        dt = args.profile_lane if args.profile_lane in ("c64", "c128") else "c64"
        D.ftlm_blocks(secs, P, FTLM_SAMPLES, FTLM_DEPTH, FTLM_SEED, betas, dtype=dt)
        torch.cuda.synchronize()
        t = time.perf_counter()
        r = D.ftlm_blocks(secs, P, FTLM_SAMPLES, FTLM_DEPTH, FTLM_SEED, betas, dtype=dt)
        print(json.dumps({"profile_case": "ftlm4", "dtype": dt, "dims": [s.dim for s in secs],
                          "s": time.perf_counter() - t, "phases": r["stats"]}))
        return
    if args.profile_case == "chain20":
        # a small sector (9,252 states) in FP64, the tuner on: the shape one vector takes on a small sector
        spec = lat.chain_sector(20, 10, 0)
        prog = ops.row_program(ops.from_products(20, ops.heisenberg_products(lat.chain_bonds(20))))
        S, P = D.Sector(spec), D.Program(prog)
        x = torch.randn(S.dim, dtype=torch.complex128, device="cuda")
        y = torch.empty_like(x)
        for _ in range(args.warmup):
            D.matvec(S, S, P, [x], [y])
        torch.cuda.synchronize()
        t = time.perf_counter()
        for _ in range(args.steps):
            D.matvec(S, S, P, [x], [y])
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": "chain20", "dim": S.dim, "ms_per_matvec": (time.perf_counter() - t) /
                          args.steps * 1e3, "tuned_shapes": D.tune_entries()}))
        return
    if args.profile_case == "chain32":
        spec, prog, _ = workload()
    else:
        Ly = 5 if args.profile_case == "sq30" else 6
        nn, nnn = lat.square_j1j2_bonds(6, Ly)
        spec = lat.square_k0_sector(6, Ly, 3 * Ly)
        prog = ops.row_program(ops.from_products(6 * Ly, ops.heisenberg_products(nn, 1.0)
                                                 + ops.heisenberg_products(nnn, 0.5)))
    S = D.Sector(spec)
    P = D.Program(prog)
    A = None
    build_s = None
    if args.profile_lane == "csr":
        torch.cuda.synchronize()
        t = time.perf_counter()
        A = D.Csr(S, S, P)
        torch.cuda.synchronize()
        build_s = time.perf_counter() - t
        A.attach(P)
    x = torch.randn(S.dim, dtype=torch.complex64, device="cuda")
    y = torch.empty_like(x)
    for _ in range(args.warmup):
        D.matvec(S, S, P, [x], [y], dtype="c64")
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(args.steps):
        D.matvec(S, S, P, [x], [y], dtype="c64")
    torch.cuda.synchronize()
    print(json.dumps({"profile_case": args.profile_case, "lane": args.profile_lane, "dim": S.dim,
                      "ms_per_matvec": (time.perf_counter() - t) / args.steps * 1e3, "sector": S.info(),
                      "csr": A.info() if A is not None else None, "csr_build_s": build_s,
                      "tuned_shapes": D.tune_entries()}))


def emitted_per_row(reps: np.ndarray, prog) -> float:
    """Mean number of program groups that act on a representative (each reads one x element): the
    exact count over the sector's representatives."""
    total = 0
    for g in range(prog.n_groups):
        F = np.uint64(prog.group_flip[g])
        vals = prog.vsub_val[prog.group_vbegin[g]:prog.group_vbegin[g + 1]].astype(np.uint64)
        total += int(np.count_nonzero(np.isin(reps & F, vals)))
    return total / len(reps)


if __name__ == "__main__":
    main()

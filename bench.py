"""Benchmark of the symmetry-sector matvec and its Lanczos recurrence on B200.

Workload (the default line): the 6x6 periodic square lattice, J1-J2 Heisenberg (J1 = 1 on the 72 nearest-
neighbour bonds, J2 = 0.5 on the 72 diagonal bonds), sector S^z = 0, momentum (0, 0) under the 36 translations
(252,091,362 representatives, uint64 states, found on the device). Synthetic input: a seeded complex Gaussian
vector. One step = one H.v on device-resident vectors with FP32 storage (FP64 arithmetic) through the lane the
engine picks for a sector whose merged CSR fits the device: the reduced CSR, built once on the device from the row
walk (its build time is reported). Reported beside it: the FP64-storage apply, the on-the-fly walk, e2e through
qb_lanczos with host buffers, time-to-E0 (FP64 CSR, FP32 CSR + FP64 refinement, the plain FP64 walk), and the
XXZ chain N = 32 sector (4,707,969 states) as a secondary workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs N independent replicas (one process per GPU, launched by torchrun): the path has no
cross-GPU exchange, so the metric is the sum over replicas and the time the max over ranks.
`--impl reference` times the reference engine's own CPU matvec (oracle/_ref) on the host cores on the same
sector: its host lane for a real sector whose CSR fits host memory (the merged reduced CSR, applied to real
vectors), on a bounded sample of the rows (four contiguous blocks of 1/256 of the rows each, built outside the
timed region), scaled to one whole H.v.
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


def sq36_workload():
    """6x6 J1-J2 (J1 = 1, J2 = 0.5), S^z = 0 (18 up), momentum (0, 0) under the 36 translations."""
    from qed_spin_b200 import lattice as lat
    from qed_spin_b200 import operators as ops
    nn, nnn = lat.square_j1j2_bonds(6, 6)
    spec = lat.square_k0_sector(6, 6, 18)
    prods = ops.heisenberg_products(nn, 1.0) + ops.heisenberg_products(nnn, 0.5)
    return spec, ops.row_program(ops.from_products(36, prods)), prods


def workload():
    """XXZ chain N = 32 (J = 1, Delta = 0.7), S^z = 0, k = 0, reflection-even, flip-even (D32 x Z2)."""
    from qed_spin_b200 import lattice as lat
    from qed_spin_b200 import operators as ops
    N = 32
    spec = lat.chain_a1_flip_sector(N)
    prods = ops.xxz_products(lat.chain_bonds(N), 1.0, 0.7)
    prog = ops.row_program(ops.from_products(N, prods))
    return spec, prog, prods


CONFIG = {"workload": "6x6 periodic square J1-J2 Heisenberg, J1=1 J2=0.5, Sz=0, momentum (0,0) under the 36 "
                      "translations", "n_sites": 36, "n_up": 18, "group_size": 36}
CHAIN32 = "XXZ chain N=32 J=1 Delta=0.7, Sz=0 k=0 reflection-even flip-even (D32 x Z2)"

# The reference arm's sample of the 6x6 sector: SQ36_BLOCKS contiguous blocks of dim / SQ36_BLOCK_DIV rows each,
# centred at (2i + 1) / (2 SQ36_BLOCKS) of the row range.
SQ36_BLOCKS, SQ36_BLOCK_DIV = 4, 256



# DRAM bytes (read + write) of one spmv1<complex64> launch on the 6x6 workload, from ncu: dram__bytes_read.sum +
# dram__bytes_write.sum of one launch (a one-pass metric set, captured on this workload after two warm-up applies).
SPMV1_SQ36_DRAM_BYTES_PER_LAUNCH = 418.38e9 + 2.02e9
SPMV1_SQ36_TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one spmv1<complex64> launch on this "
                             "workload (profiles/spmv1_sq36_csr_dram.md): the thread-per-row kernel, which makes the "
                             "same x gathers and reads the same CSR bytes as the timed four-lanes-per-row kernel; the "
                             "timed kernel's full capture is of the 6.5 GB small case (profiles/spmv1_team32_sq36n11.md)")

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


def reference_sq36(steps: int, warmup: int, threads: int) -> dict:
    """The reference engine's host lane on the 6x6 sector, on the host cores: its own orbit scan builds the sector,
    its build_cross_csr the merged rows of SQ36_BLOCKS contiguous row blocks (outside the timed region), and each
    step applies those rows to a real vector through RealCsrView::spmv -- the lane RepSectorMatVec takes for a real
    sector of a real H (is_real, with_backend). A step's time scaled by dim / (rows sampled) is one whole H.v."""
    from oracle import ref as R
    spec, _, prods = sq36_workload()
    R.set_threads(threads)
    t0 = time.perf_counter()
    rs = R.Sector(spec.n_sites, spec.n_up, spec.perms, spec.chars, flips=spec.flips, slc_mode=-1)
    scan_s = time.perf_counter() - t0
    n = rs.dim
    rp = R.Operator(spec.n_sites, prods).row_program()
    B = n // SQ36_BLOCK_DIV
    t0 = time.perf_counter()
    blocks = []
    for i in range(SQ36_BLOCKS):
        r0 = (2 * i + 1) * n // (2 * SQ36_BLOCKS) - B // 2
        blocks.append(R.Csr(rs, rp, rows=(r0, B)))
    build_s = time.perf_counter() - t0
    nnz = sum(b.nnz for b in blocks)
    x = np.random.default_rng(1).normal(size=n)
    ys = [np.zeros(B) for _ in blocks]
    real = all(b.spmv_real(x, y) for b, y in zip(blocks, ys))
    assert real, "the 6x6 k=0 sector of the J1-J2 model is real"
    for _ in range(warmup):
        for b, y in zip(blocks, ys):
            b.spmv_real(x, y)
    times = []
    for _ in range(steps):
        t = time.perf_counter()
        for b, y in zip(blocks, ys):
            b.spmv_real(x, y)
        times.append(time.perf_counter() - t)
    rows = SQ36_BLOCKS * B
    per_hv = sum(times) / steps * n / rows
    # the complex lane on the same rows (the reference's device-less lane for a complex sector), for context
    xc = (x + 1j * np.random.default_rng(2).normal(size=n)).astype(np.complex128)
    yc = [np.zeros(B, np.complex128) for _ in blocks]
    t = time.perf_counter()
    for b, y in zip(blocks, yc):
        b.spmv(xc, y)
    per_hv_c = (time.perf_counter() - t) * n / rows
    for b in blocks:
        b.close()
    return {"value": 1.0 / per_hv, "unit": "H.v/s", "cores": threads, "kind": "reference",
            "sample": f"{SQ36_BLOCKS} contiguous blocks of {B} rows ({rows} of {n} rows, {nnz} merged entries), "
                      f"{steps} timed applies through RealCsrView::spmv (real vectors), scaled by dim / rows",
            "dim": n, "ms_per_hv": 1e3 * per_hv, "complex_lane_hv_per_s": 1.0 / per_hv_c,
            "scan_s": scan_s, "block_csr_build_s": build_s, "sample_nnz": nnz}


def run_reference(args, world, rank):
    """The reference engine's own CPU matvec (oracle/_ref) on the host cores, rank 0 only: H.v/s on the 6x6
    sector through its host CSR lane, on the row sample described in reference_sq36."""
    if rank != 0:
        return None
    from oracle import ref as R
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "the reference CPU engine was not built into oracle/_ref"}))
        return None
    threads = os.cpu_count() or 1
    r = reference_sq36(args.steps, args.warmup, threads)
    v = r["value"]
    line = {"impl": "reference", "metric": "H.v/s", "value": v, "unit": "H.v/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_hv"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(CONFIG, dim=r["dim"], lane="host reduced CSR on real vectors (build_cross_csr + "
                                                        "RealCsrView::spmv, OpenMP), sampled rows"),
            "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": v, "unit": "H.v/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_detail": {k: r[k] for k in ("complex_lane_hv_per_s", "scan_s", "block_csr_build_s",
                                                   "sample_nnz")}}
    print(json.dumps(line))
    return line


def reference_chain32(threads: int) -> dict:
    """The reference engine's host lane on the chain-32 sector: its merged CSR built whole, applied to real vectors
    (RealCsrView::spmv) for about 10 s, and once to complex ones."""
    from oracle import ref as R
    spec, _, prods = workload()
    R.set_threads(threads)
    rs = R.Sector(spec.n_sites, spec.n_up, spec.perms, spec.chars, flips=spec.flips, slc_mode=-1)
    rp = R.Operator(spec.n_sites, prods).row_program()
    t0 = time.perf_counter()
    csr = R.Csr(rs, rp)
    csr_s = time.perf_counter() - t0
    x = np.random.default_rng(1).normal(size=rs.dim)
    y = np.zeros(rs.dim)
    assert csr.spmv_real(x, y)
    n, t0 = 0, time.perf_counter()
    while n < 3 or (time.perf_counter() - t0 < 10.0 and n < 200):
        csr.spmv_real(x, y)
        n += 1
    dt = time.perf_counter() - t0
    xc = (x + 1j * x[::-1]).astype(np.complex128)
    yc = np.zeros(rs.dim, np.complex128)
    t = time.perf_counter()
    csr.spmv(xc, yc)
    c_s = time.perf_counter() - t
    csr.close()
    return {"value": n / dt, "unit": "H.v/s", "cores": threads, "kind": "reference",
            "sample": f"{n} whole H.v through the reference's reduced CSR on real vectors (its host lane for a real "
                      f"sector) on the {rs.dim}-state sector", "csr_build_s": csr_s,
            "complex_lane_hv_per_s": 1.0 / c_s}


def time_applies(fn, steps, warm, stream, world):
    """Device time per call of fn (CUDA events on `stream`, after `warm` untimed calls), max over ranks."""
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        fn()
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    barrier(world)
    return dist_max(ms, world) / steps


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e0", action="store_true", help="leave the 6x6 time-to-E0 runs out of the line")
    ap.add_argument("--no-secondary", action="store_true",
                    help="leave the chain-32, k > 1, FTLM and served-stream measurements out of the line")
    ap.add_argument("--no-ftlm", action="store_true", help="leave the batched FTLM measurement out of the line")
    ap.add_argument("--ftlm", action="store_true",
                    help="batched FTLM over the 600 blocks of the XXZ chain N=24 (every S^z x 24 momenta), one "
                         "JSON line: samples/s against the plain single-sample path and the reference CPU engine")
    ap.add_argument("--serve", action="store_true",
                    help="the served request stream (Poisson arrivals of eigs / S^z(q) dynamics requests on chains "
                         "N = 16..30): p50/p99 latency and solves/s of the server against one solve at a time")
    ap.add_argument("--serve-requests", type=int, default=60)
    ap.add_argument("--no-serve", action="store_true", help="leave the served-stream measurement out of the line")
    ap.add_argument("--profile-case", choices=["chain32", "sq30", "sq36", "sq36n11", "sq36n12", "ftlm4", "chain20"],
                    default=None,
                    help="profiling run: build one sector and apply H (complex64) warmup + steps times, print timing; "
                         "sq36n11 / sq36n12: the 6x6 J1-J2 k=0 sector at 11 / 12 up spins; ftlm4: batched FTLM (40 "
                         "samples, depth 100) on the four largest N = 24 XXZ blocks")
    ap.add_argument("--profile-lane", choices=["walk", "csr", "c64", "c128"], default="walk",
                    help="the lane of the profiling run: the on-the-fly walk or the device reduced CSR; for ftlm4 "
                         "the storage type")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.profile_case:
        profile_case(args)
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
    from qed_spin_b200 import replicas
    build.build()
    torch.cuda.set_device(local)
    dev = torch.cuda.current_device()
    stream = torch.cuda.current_stream()
    hbm, peak_kind = peaks()

    spec, prog, prods = sq36_workload()
    t0 = time.perf_counter()
    S = D.Sector(spec)
    torch.cuda.synchronize()
    enum_s = time.perf_counter() - t0
    P = D.Program(prog)
    n = S.dim
    info = S.info()
    reps, _ = S.reps()
    sample = reps[::64].copy()
    del reps
    e_bar = emitted_per_row(sample, prog)

    # the reduced CSR, built on the device from the walk, attached to the program
    torch.cuda.synchronize()
    t = time.perf_counter()
    A = D.Csr(S, S, P)
    torch.cuda.synchronize()
    csr_build_s = time.perf_counter() - t
    A.attach(P)
    cinfo = A.info()

    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    x32 = torch.randn(n, dtype=torch.complex64, device="cuda", generator=g)
    y32 = torch.empty_like(x32)

    def apply32():
        D.matvec(S, S, P, [x32], [y32], dtype="c64", stream=stream)

    with Clocks(dev) as clk:
        per32 = time_applies(apply32, args.steps, args.warmup, stream, world)
    x64 = x32.to(torch.complex128)
    y64 = torch.empty_like(x64)
    per64 = time_applies(lambda: D.matvec(S, S, P, [x64], [y64], dtype="c128", stream=stream),
                         max(3, args.steps // 4), 2, stream, world)

    def b_alg(sb):   # the per-H.v algorithmic bytes: rep + 1/norm + y per row, one x element per emitted entry
        return n * (8 + 8 + sb) + n * e_bar * sb

    def csr_stream(sb):   # the CSR streamed once, x read once, y written once
        return cinfo["bytes"] + 2 * n * sb

    ach32 = b_alg(8) / (per32 * 1e-3) / 1e9
    ach64 = b_alg(16) / (per64 * 1e-3) / 1e9

    # end to end through the public C-ABI: a host complex128 start vector in, alpha / beta out, K Lanczos steps on
    # FP32 storage through the attached CSR
    v0 = x64.cpu().numpy()
    D.lanczos(S, P, v0, 4, dtype="c64")
    torch.cuda.synchronize()
    barrier(world)
    t = time.perf_counter()
    D.lanczos(S, P, v0, args.steps, dtype="c64")
    e2e_s = dist_max(time.perf_counter() - t, world)
    del v0

    # the on-the-fly walk (the CSR detached)
    D.detach_csr(P)
    walk32 = time_applies(apply32, 1, 1, stream, world)
    walk64 = time_applies(lambda: D.matvec(S, S, P, [x64], [y64], dtype="c128", stream=stream), 1, 1, stream,
                          world)
    del x32, y32, x64, y64
    torch.cuda.synchronize()

    e0 = None
    if not args.no_e0 and world == 1:   # the time-to-E0 runs are per-GPU facts: measured on a single replica
        e0 = {}
        A.attach(P)
        # each solve starts from an empty block cache (the library keeps released device blocks for reuse; blocks
        # of another solve's sizes would otherwise be freed one by one inside the next solve's timing)
        D.memory_trim(0)
        t = time.perf_counter()
        r = D.eigs_lowest(S, P, dtype="c128")
        e0["csr_fp64"] = {"s": time.perf_counter() - t, "e0": r["e0"], "iters": r["iters"], "matvecs": r["matvecs"]}
        D.memory_trim(0)
        t = time.perf_counter()
        r = D.eigs_lowest(S, P, dtype="c64", refine=True)
        e0["csr_fp32_refined"] = {"s": time.perf_counter() - t, "e0": r["e0"], "iters": r["iters"],
                                  "matvecs": r["matvecs"], "converged": r["converged"]}
        A.close()
        torch.cuda.synchronize()
        D.memory_trim(0)
        t = time.perf_counter()
        r = D.eigs_lowest(S, P, dtype="c128")
        e0["plain_fp64_walk"] = {"s": time.perf_counter() - t, "e0": r["e0"], "iters": r["iters"],
                                 "matvecs": r["matvecs"]}
        e_ref = e0["csr_fp64"]["e0"]
        e0["csr_build_s"] = csr_build_s
        e0["rel_err_fp32_refined_vs_fp64"] = abs(e0["csr_fp32_refined"]["e0"] - e_ref) / abs(e_ref)
        e0["rel_err_plain_walk_vs_csr_fp64"] = abs(e0["plain_fp64_walk"]["e0"] - e_ref) / abs(e_ref)
        e0["speedup_fp32_refined_vs_fp64_same_lane"] = e0["csr_fp64"]["s"] / e0["csr_fp32_refined"]["s"]
        e0["speedup_fp32_refined_incl_build_vs_plain_walk"] = e0["plain_fp64_walk"]["s"] / (
            e0["csr_fp32_refined"]["s"] + csr_build_s)
    A.close()
    S.close()
    P.close()
    torch.cuda.synchronize()
    D.memory_trim(0)   # the 6x6 buffers back to the device before the smaller workloads below

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = reference_sq36(10, 1, os.cpu_count() or 1)
        except Exception as e:  # the baseline is reported, never required
            cpu = {"unavailable": str(e)}

    secondary = {}
    if rank == 0 and world == 1 and not args.no_secondary:
        for key, fn in (("chain32", lambda: chain32_measure(args, stream)), ("levels", lambda: levels_measure(args)),
                        ("ftlm", lambda: None if args.no_ftlm else ftlm_measure(args, not args.no_cpu_baseline)),
                        ("serve", lambda: None if args.no_serve else serve_measure(args))):
            try:
                secondary[key] = fn()
            except Exception as e:
                secondary[key] = {"unavailable": str(e)}

    if rank != 0:
        replicas.finish(world)
        return
    value = replicas.whole_job_rate(1.0, world, per32 * 1e-3)
    line = {
        "metric": "H.v/s", "value": value, "unit": "H.v/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per32, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 arithmetic, complex64 (FP32) vector storage", "data": "synthetic",
        "config": dict(CONFIG, dim=n, lane="device reduced CSR (built from the row walk)", nnz=cinfo["nnz"],
                       csr_bytes=cinfo["bytes"], n_dict=cinfo["n_dict"],
                       emitted_per_row=e_bar, emitted_per_row_sample="every 64th representative",
                       storage="complex64 vectors, FP64 arithmetic", lookup=info["lookup"],
                       sublattice=[info["slc_L"], info["slc_m"]],
                       l2=f"inputs larger than the 126 MB L2 (CSR {cinfo['bytes'] / 1e9:.1f} GB streamed per step, "
                          f"x {8 * n / 1e9:.2f} GB), no flush",
                       parallelism=f"replicas x{world}"),
        "roofline": {"bound": "hbm", "achieved": ach32, "peak": hbm, "unit": "GB/s", "frac": ach32 / hbm,
                     "traffic": SPMV1_SQ36_DRAM_BYTES_PER_LAUNCH, "traffic_source": SPMV1_SQ36_TRAFFIC_SOURCE,
                     "peak_kind": peak_kind, "kernel": "spmv1_team32 (complex64 in and out, 4 lanes per row)",
                     "traffic_kernel": "spmv1<complex64>",
                     "alg_bytes_per_launch": b_alg(8),
                     "alg_bytes_rule": "D*(8 rep + 8 inv_norm + 8 y) + D*e_bar*8 (one complex64 x element per "
                                       "emitted entry)",
                     "csr_stream_bytes_per_launch": csr_stream(8),
                     "csr_stream_frac": csr_stream(8) / (per32 * 1e-3) / 1e9 / hbm},
        "fp64": {"ms_per_hv": per64, "hv_per_s": 1e3 / per64, "achieved_gbs": ach64, "frac": ach64 / hbm},
        "csr_build_s": csr_build_s,
        "enumeration_s": enum_s,
        "walk": {"ms_per_hv_fp32": walk32, "ms_per_hv_fp64": walk64, "hv_per_s_fp32": 1e3 / walk32,
                 "frac_fp32": b_alg(8) / (walk32 * 1e-3) / 1e9 / hbm},
        "e2e": {"value": world * args.steps / e2e_s, "unit": "H.v/s", "h2d_bytes_per_step": 16 * n / args.steps,
                "d2h_bytes_per_step": 16, "path": "qb_lanczos (host complex128 v0 in, alpha/beta out, FP32 storage, "
                                                  "CSR lane)"},
        "time_to_e0": e0,
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
    }
    line.update(secondary)
    print(json.dumps(line), flush=True)
    replicas.finish(world)


def chain32_measure(args, stream):
    """The XXZ chain N = 32 sector (4,707,969 states): FP32 / FP64 CSR applies, the walk, e2e, time-to-E0 and the
    reference engine's host lane on the whole sector."""
    import torch

    from qed_spin_b200 import device as D
    spec, prog, prods = workload()
    t0 = time.perf_counter()
    S = D.Sector(spec)
    torch.cuda.synchronize()
    enum_s = time.perf_counter() - t0
    P = D.Program(prog)
    n = S.dim
    e_bar = emitted_per_row(S.reps()[0], prog)
    hbm, _ = peaks()
    rng = np.random.default_rng(1)
    x64 = torch.from_numpy(rng.normal(size=n) + 1j * rng.normal(size=n)).cuda()
    x32 = x64.to(torch.complex64)
    y32, y64 = torch.empty_like(x32), torch.empty_like(x64)
    walk32 = time_applies(lambda: D.matvec(S, S, P, [x32], [y32], dtype="c64", stream=stream), 10, 3, stream, 1)
    t = time.perf_counter()
    r_plain = D.eigs_lowest(S, P, dtype="c128")
    t_plain = time.perf_counter() - t
    t = time.perf_counter()
    A = D.Csr(S, S, P)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t
    A.attach(P)
    cinfo = A.info()
    per32 = time_applies(lambda: D.matvec(S, S, P, [x32], [y32], dtype="c64", stream=stream), 200, 5, stream, 1)
    per64 = time_applies(lambda: D.matvec(S, S, P, [x64], [y64], dtype="c128", stream=stream), 100, 3, stream, 1)
    b_alg = n * (8 + 8 + 8) + n * e_bar * 8
    v0 = x64.cpu().numpy()
    D.lanczos(S, P, v0, 8, dtype="c64")
    torch.cuda.synchronize()
    t = time.perf_counter()
    D.lanczos(S, P, v0, 20, dtype="c64")
    e2e_s = time.perf_counter() - t
    D.memory_trim(0)   # each solve from an empty block cache, as on the 6x6 sector
    t = time.perf_counter()
    r64 = D.eigs_lowest(S, P, dtype="c128")
    t64 = time.perf_counter() - t
    D.memory_trim(0)
    t = time.perf_counter()
    r32 = D.eigs_lowest(S, P, dtype="c64", refine=True)
    t32 = time.perf_counter() - t
    D.memory_trim(0)
    t = time.perf_counter()
    r2 = D.eigs(S, P, 2)
    k2_s = time.perf_counter() - t
    out = {"workload": CHAIN32, "dim": n, "enumeration_s": enum_s, "csr_build_s": build_s, "nnz": cinfo["nnz"],
           "csr_bytes": cinfo["bytes"], "emitted_per_row": e_bar,
           "csr_ms_per_hv_fp32": per32, "hv_per_s_fp32": 1e3 / per32, "frac_fp32": b_alg / (per32 * 1e-3) / 1e9 / hbm,
           "csr_ms_per_hv_fp64": per64, "walk_ms_per_hv_fp32": walk32,
           "e2e_hv_per_s_20_steps": 20 / e2e_s,
           "time_to_e0": {"plain_fp64_walk_s": t_plain, "csr_fp64_s": t64, "csr_fp32_refined_s": t32,
                          "rel_err_fp32_refined": abs(r32["e0"] - r64["e0"]) / abs(r64["e0"]),
                          "e0": r64["e0"], "plain_e0": r_plain["e0"]},
           "k2": {"s": k2_s, "values": list(map(float, r2["values"])), "converged": r2["converged"],
                  "matvecs": r2["matvecs"], "lane": "thick-restart Lanczos on the CSR"}}
    A.close()
    S.close()
    if not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = reference_chain32(os.cpu_count() or 1)
        except Exception as e:
            out["cpu_baseline"] = {"unavailable": str(e)}
    return out


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
    """The reference engine's sampled thermal blocks on the host cores, on a bounded stratified sample of the same
    workload: one block of every S^z sector (momentum k = n_up mod 24), with the workload's 40 samples at depth 100.
    A block's cost grows with its dimension, so the whole workload's time is estimated as the sample's time times
    (states in all 554 blocks) / (states in the sample), and samples/s = 554 x 40 / that estimate."""
    from oracle import ref as R
    _, prods, _, betas = ftlm_workload()
    R.set_threads(threads)
    from qed_spin_b200 import lattice as lat
    blocks = [lat.chain_sector(FTLM_N, n_up, n_up % FTLM_N) for n_up in range(FTLM_N + 1)]
    rs = [R.Sector(s.n_sites, s.n_up, s.perms, s.chars, flips=s.flips, slc_mode=-1) for s in blocks]
    rs = [r for r in rs if r.dim > 0]
    rp = R.Operator(FTLM_N, prods).row_program()
    dims = [r.dim for r in rs]
    t = time.perf_counter()
    R.ftlm_blocks(rs, rp, FTLM_SAMPLES, FTLM_DEPTH, FTLM_SEED, betas)
    dt = time.perf_counter() - t
    total_states, total_blocks = 2 ** FTLM_N, 554
    est = dt * total_states / sum(dims)
    return {"value": total_blocks * FTLM_SAMPLES / est, "unit": "samples/s", "cores": threads, "kind": "reference",
            "sample": f"one block per S^z sector (momentum n_up mod 24; {len(rs)} blocks, dims {min(dims)}..{max(dims)}, "
                      f"{sum(dims)} states), {FTLM_SAMPLES} samples each, depth {FTLM_DEPTH}, its CSR lane and block "
                      f"scheduling, {dt:.1f} s; scaled to the 554 blocks ({total_states} states) by states"}


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


def levels_measure(args):
    """Config 1: the Heisenberg chain N = 20, Sz = 0, k = 0, lowest four levels (the k > 1 lane) on the device
    against the reference engine's krylov_schur_kernel on the host cores; and the CUDA-graph comparison."""
    import torch

    from qed_spin_b200 import device as D
    from qed_spin_b200 import lattice as lat
    from qed_spin_b200 import operators as ops
    out = {}
    torch.cuda.synchronize()
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
        n_up = {"sq36n11": 11, "sq36n12": 12}.get(args.profile_case, 3 * Ly)
        nn, nnn = lat.square_j1j2_bonds(6, Ly)
        spec = lat.square_k0_sector(6, Ly, n_up)
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

"""Benchmark: molecule-pair energies per second of erdst's refs-mode frame.

One step = one engconst frame of the refs workload "refs-ring12-water4096":
4,096 rigid 3-site waters in a 49.6 A box, a 12-site benzene-like test
particle inserted 2,000 times (uniform position + orientation), PME 64^3
order 4, ecorr on.  Units = insertions x solvent molecules = 8.19e6 per step.

  value  device time of K steps (CUDA events on the engine's stream, inputs
         resident in HBM), L2 flushed (256 MiB write) before every step
  e2e    the same K steps through the host C-ABI (ermod_engconst with host
         coordinates, H2D inside) plus a D2H read of edens each step, host
         wall time of the synchronous calls
  --impl reference   the reference's algorithm on the host cores (the CPU
         restatement under oracle/: brute-force pairs, one PME solve per
         insertion, binary-search binning, per-insertion ecorr update)

Multi-GPU (torchrun): frames are independent, each rank runs its own
frames with no collective in the step (weak scaling); the max device time
over ranks is reported.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIG = 2
METRIC = "mol-pair energies/s"
UNIT = "mol-pairs/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--maxins", type=int, default=None)
    ap.add_argument("--spectrum-path", type=int, default=0, choices=[0, 1, 2, 3],
                    help="PME solute spectrum (configs 2 and 3): 0 automatic, 1 spread + cuFFT, 2 direct site "
                         "sums, 3 plane spreading")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-sample", type=int, default=500, help="insertions per CPU reference step")
    ap.add_argument("--config", type=int, default=2, choices=[2, 3, 4, 5],
                    help="2: the headline refs frame; 3: the precision workload (32,768 waters, PME 128^3, "
                         "60-site chain, 4,096 insertions); 4: 64 solutes batched into one graph per frame; "
                         "5: GPU time to delta-mu within 0.05 kcal/mol, learned vs uniform insertion")
    ap.add_argument("--solute-sites", type=int, default=200, help="config 5: sites of the ring-recipe solute")
    ap.add_argument("--ins-per-frame", type=int, default=100000, help="config 5: insertions per frame")
    ap.add_argument("--long-frames", type=int, default=100,
                    help="config 5: frames of the uniform yardstick run (x insertions per frame)")
    ap.add_argument("--max-frames", type=int, default=50, help="config 5: frames of each compared run")
    ap.add_argument("--train-frames", type=int, default=10, help="config 5: uniform frames of training samples")
    ap.add_argument("--replicas", type=int, default=2, help="config 5: independent runs per insertion mode")
    ap.add_argument("--mix-uniform", type=float, default=0.2, help="config 5: uniform share eps of the proposal")
    ap.add_argument("--label-quantile", type=float, default=0.05,
                    help="config 5: training label 1 for this lowest fraction of insertion energies")
    return ap.parse_args()


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled every 10 ms through NVML while running
    (read-only queries), falling back to nvidia-smi at 200 ms where NVML is not importable."""
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None
        self.thread = None

    def _nvml_loop(self, nv, h):
        bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop:
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((float(sm), float(mx), [n for n, b in zip(self.NAMES, bits) if r & b]))
            except Exception:
                break
            time.sleep(0.01)

    def __enter__(self):
        self.stop = False
        try:
            import threading
            import pynvml as nv
            nv.nvmlInit()
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = int(vis.split(",")[self.device]) if vis and vis.split(",")[0].isdigit() else self.device
            h = nv.nvmlDeviceGetHandleByIndex(idx)
            self.thread = threading.Thread(target=self._nvml_loop, args=(nv, h), daemon=True)
            self.thread.start()
        except Exception:
            self.thread = None
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            try:
                self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                              "--format=csv,noheader,nounits", "-lms", "200"],
                                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            except OSError:
                self.proc = None
        return self

    def __exit__(self, *exc):
        self.stop = True
        if self.thread is not None:
            self.thread.join(timeout=2)
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            for r in (r.split(", ") for r in out.strip().splitlines() if r.count(",") >= 8):
                if r[1].strip().isdigit():
                    self.rows.append((float(r[1]), float(r[2]) if r[2].strip().isdigit() else None,
                                      [self.NAMES[i] for i in range(4) if r[5 + i].strip().lower() == "active"]))

    def summary(self):
        if not self.rows:
            return None
        sm = [r[0] for r in self.rows]
        mx = [r[1] for r in self.rows if r[1]]
        reasons = sorted({n for r in self.rows for n in r[2]})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows), "source": "nvml" if self.proc is None else "nvidia-smi"}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def kernel_bytes(stage: str, w, chunk: int, natoms: int, slvmax: int, ermax: int, maxdst: int, nsite: int) -> float:
    """Algorithmic DRAM bytes of ONE launch of each of the engine's kernels: what the launch must read and
    write at least once (inputs in, outputs out), independent of how the kernel stages them."""
    K = w.params["ms1max"]
    n = w.params["splodr"]
    # k1 planes the fused solve transforms: every mode above k1max has a Gaussian weight below 1e-9
    a1 = float(np.linalg.norm(np.asarray(w.frame(0)[1], dtype=np.float64).reshape(3, 3)[0]))
    k1max = min(K // 2, int(np.floor(np.sqrt(-np.log(1e-9)) * w.params["screen"] * a1 / np.pi)) + 1)
    KK, KH = K ** 3, K * K * (k1max + 1)
    if stage == "gather":       # potential grid once + reciprocal energies out + per-atom and per-molecule records
        return chunk * KK * 4 + slvmax * chunk * 8 + natoms * (64 if n == 4 else 12 * n + 16) + slvmax * 16
    if stage == "bin":          # every target's reciprocal and real-space energy rows in, its count row out
        return min(maxdst, 4096) * (slvmax * 8 * 2 + ermax * 4)
    if stage == "influence":    # spectrum read + write, influence function read
        return chunk * KH * 8 * 2 + KH * 4
    if stage == "pme_plane":    # site tables in, transformed planes out once, influence function in
        return chunk * KH * 8 + KH * 4 + chunk * nsite * (K // 2 + 1 + 2 * K) * 8
    if stage == "site_tables":  # solute sites in, per-site stencil transforms out (one launch per batch)
        return min(maxdst, 4096) * nsite * (16 + (K // 2 + 1 + 2 * K) * 8)
    if stage == "pme_rows":     # transformed planes in, potential grids out (insertion-fastest)
        return chunk * KH * 8 + chunk * KK * 4
    if stage == "transpose":    # potential grids read once, written once
        return 2 * chunk * KK * 4
    if stage == "spread":       # zero + scatter of the charge grids
        return chunk * KK * 4
    if stage == "real":         # solvent coordinates + real-space energy matrix of the batch
        return natoms * 16 + slvmax * maxdst * 8
    if stage == "ecorr":        # counts read twice + ecorr read-modify-write
        return 2 * maxdst * ermax * 4 + 16 * ermax * ermax
    return 0.0


def path_bytes_per_unit(w, natoms: int, slvmax: int, ermax: int, maxdst: int, nsite: int, batch: int = 4096) -> float:
    """Algorithmic HBM bytes of the whole path per mol-pair, as the scope table defines them:
    B = 16 N_atoms + 16 M s + 16 M K^3 + 16 M N_mol + 16 ermax^2 ceil(M / batch), divided by
    the frame's M N_mol units (solvent read once, insertions, a spectrum and a potential grid
    written and read per insertion, the FP64 energy matrix written and read, ecorr updated
    once per batch)."""
    K = w.params["ms1max"]
    B = (16 * natoms + 16 * maxdst * nsite + 16 * maxdst * K ** 3 + 16 * maxdst * slvmax
         + 16 * ermax * ermax * -(-maxdst // batch))
    return B / (maxdst * slvmax)


def profile_table(name: str):
    """{kernel: {column: value}} from a whitespace table under profiles/ ('#' lines are comments,
    the first other line names the columns, '-' marks a value not captured); {} when the file
    is absent."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return {}
    rows, cols = {}, None
    for line in open(p):
        if line.startswith("#") or not line.strip():
            continue
        f = line.split()
        if cols is None:
            cols = f
            continue
        rows[f[0]] = {c: float(v) for c, v in zip(cols[1:], f[1:]) if v != "-"}
    return rows


def bound_from_counters(c: dict) -> str:
    """The resource that bounds a kernel, read from its ncu counters (fractions of peak, stalls
    per issued instruction): the tensor pipe, DRAM, SM issue, the shared-memory / LSU queue
    (MIO throttle), the L1 / shared-memory unit, or -- none of them near its limit -- memory latency."""
    if not c:
        return "unmeasured"
    if c.get("tensor_pipe", 0.0) >= 0.5:
        return "tensor"
    if c.get("dram_frac", 0.0) >= 0.6:
        return "hbm"
    if c.get("issue_active", 0.0) >= 0.6 or max(c.get("fma_pipe", 0.0), c.get("lsu_pipe", 0.0)) >= 0.6:
        return "sm-issue"
    if c.get("l1_frac", 0.0) >= 0.65:
        return "l1-smem"
    if c.get("stall_mio", 0.0) >= 2.0:
        return "mio-queue"
    return "latency"


def cpu_baseline(w, sample: int, threads: int):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # the reference's algorithm restated on the CPU (the checker)
    prm = dict(w.params, maxins=sample)
    orc = oracle.Oracle(prm, w.topo, w.hist, precision=4, nthreads=threads)
    pos, cell = w.frame(0)
    orc.engconst(1, pos, cell)     # warm
    t0 = time.perf_counter()
    orc.engconst(2, pos, cell)
    dt = time.perf_counter() - t0
    units = sample * (w.topo.nummol - 1)
    return units / dt, dt, units


def run_reference(args, w):
    ws, rank, _ = dist_init()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    prm = dict(w.params, maxins=args.ref_sample)
    orc = oracle.Oracle(prm, w.topo, w.hist, precision=4, nthreads=threads)
    frames = [w.frame(i) for i in range(args.warmup + args.steps)]
    for i in range(args.warmup):
        orc.engconst(i + 1, *frames[i])
    t = []
    for i in range(args.steps):
        t0 = time.perf_counter()
        orc.engconst(args.warmup + i + 1, *frames[args.warmup + i])
        t.append(time.perf_counter() - t0)
    units = args.ref_sample * (w.topo.nummol - 1)
    total = sum(t)
    val = units * args.steps / total
    line = {"metric": METRIC, "value": val, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": w.name, "waters": int(w.topo.nummol - 1), "pme_grid": w.params["ms1max"],
                       "insertions_per_step": args.ref_sample,
                       "insertions_per_frame_full": w.params["maxins"]},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{args.ref_sample} insertions x {w.topo.nummol - 1} waters per step, "
                                       f"{args.steps} steps, FP32 restatement of the reference algorithm"},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def stage_pass(args, w, local, dev_pos, cell, flush):
    """Per-stage device times (CUDA events between stages, direct launches) over a few frames:
    the same kernels as the timed graph frames, timed one stage at a time for the roofline."""
    import torch
    from ermod_openacc_b200 import Engine
    eng = Engine(dict(w.params, stage_timing=1), w.topo, w.hist, device=local)
    n = min(args.steps, 10)
    for i in range(args.warmup):
        eng.engconst_dev(i + 1, dev_pos[i].data_ptr(), cell)
    stage = {k: 0.0 for k in Engine.STAGES}
    for i in range(n):
        flush.zero_()
        torch.cuda.synchronize()
        eng.engconst_dev(args.warmup + i + 1, dev_pos[args.warmup + i].data_ptr(), cell)
        for k, v in eng.timings().items():
            stage[k] += v
    eng.close()
    return stage, n


def d2h_bytes_per_step(eng) -> int:
    """Device-to-host bytes of one e2e step: engconst's status word (and, for a solute in
    solution, its per-species energies flceng), then the accumulators that
    accum(ecorr=False) copies (edens, eself when selfcal, slnuv, minuv/maxuv and the eight
    scalars)."""
    n = 16 + (8 * eng.maxdst * eng.numslv if eng.params["slttype"] == 1 else 0)
    n += 8 * eng.ermax + (8 * eng.esmax if eng.params["selfcal"] else 0) + 8 * eng.numslv
    n += 4 * 2 * (eng.numslv + 1) + 8 * 8
    return int(n)


def main():
    args = parse()
    from ermod_openacc_b200 import systems as S
    if args.config == 4:
        return main_batch(args)
    if args.config == 5:
        return main_delta_mu(args)
    w = S.make_workload(args.config, maxins=args.maxins)
    if args.spectrum_path:
        w.params["spectrum_path"] = args.spectrum_path
    if args.impl == "reference":
        run_reference(args, w)
        return
    import torch
    ws, rank, local = dist_init()
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    import __graft_entry__ as ge
    if rank == 0:
        ge.build_engine()
    if ws > 1:
        dist.barrier()
    from ermod_openacc_b200 import Engine
    eng = Engine(w.params, w.topo, w.hist, device=local)    # frames run as captured CUDA graphs
    nfr = args.warmup + args.steps
    frames = [w.frame(rank * nfr + i) for i in range(nfr)]
    cell = frames[0][1]
    dev_pos = torch.from_numpy(np.stack([f[0] for f in frames])).to(f"cuda:{local}")
    host_pos = torch.from_numpy(np.stack([f[0] for f in frames])).pin_memory()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")
    units = eng.maxdst * eng.slvmax

    for i in range(args.warmup):
        eng.engconst_dev(i + 1, dev_pos[i].data_ptr(), cell)
    torch.cuda.synchronize()
    launches0 = eng.launch_count()
    dev_ms = 0.0
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            eng.engconst_dev(args.warmup + i + 1, dev_pos[args.warmup + i].data_ptr(), cell)
            dev_ms += eng.last_ms()
    torch.cuda.synchronize()
    launches = eng.launch_count() - launches0
    if ws > 1:
        tt = torch.tensor([dev_ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        dev_ms = float(tt.item())
        dist.barrier()
    # e2e: host coordinates in pinned memory -> C-ABI (H2D inside) -> D2H of edens
    e2e_s = 0.0
    edens = None
    for i in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.engconst(nfr + i + 1, host_pos[args.warmup + i].numpy(), cell)
        edens = eng.accum(ecorr=False)["edens"]
        e2e_s += time.perf_counter() - t0
    if ws > 1:
        tt = torch.tensor([e2e_s], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    assert edens is not None and edens.sum() > 0
    if ws > 1:
        # the division's exchange (engstore's reduction, after the timed region): sums over ranks
        from ermod_openacc_b200 import parallel
        red, _ = parallel.engstore_all(eng, device=f"cuda:{local}")
        assert abs(red["edens"].sum() - eng.slvmax) < 1e-6 * eng.slvmax
    value = ws * units * args.steps / (dev_ms * 1e-3)
    e2e = ws * units * args.steps / e2e_s
    paths = eng.paths()
    # per-kernel stage times from a stage-timed pass of the same frames (direct launches)
    stage, nst = stage_pass(args, w, local, dev_pos, cell, flush)
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        peak, peak_src = float(json.load(open(peaks_path))["hbm_gbs"]), "measured"
    chunk = 32
    nbatch = -(-eng.maxdst // 4096)
    per_batch = ("real", "bin", "ecorr", "site_tables")
    order4 = w.params["splodr"] == 4 and max(w.params["ms1max"], w.params["ms2max"], w.params["ms3max"]) < 1024
    # square 64 planes with direct site sums on the tensor cores run two planes per CTA
    pair = (w.params["ms2max"] == 64 and w.params["ms3max"] == 64 and paths["spectrum_path"] == 2
            and eng.nsite_slt <= 64)
    kname = {"gather": "k_gather_rec" if order4 else "k_gather", "bin": "k_bin", "real": "k_real",
             "spread": "k_spread_box", "transpose": "k_transpose_phi",
             "pme_plane": "k_pme_plane_pair" if pair else "k_pme_plane",
             "pme_rows": "k_pme_lines" if w.params["ms1max"] <= 64 else "k_pme_rows",
             "site_tables": "k_site_tables", "influence": "k_influence", "ecorr": "k_ecorr_tma"}
    counters = profile_table("kernel_counters.txt")
    kernels = {}
    for k, kn in kname.items():
        if stage[k] <= 0:
            continue
        n_launch = nbatch * nst if k in per_batch else stage["chunks"]
        ms = stage[k] / n_launch
        io = kernel_bytes(k, w, chunk, eng.natoms, eng.slvmax, eng.ermax, eng.maxdst, eng.nsite_slt)
        c = counters.get(kn, {})
        kernels[kn] = {"ms_per_frame": round(stage[k] / nst, 4), "launches_per_frame": n_launch / nst,
                       "launch_ms": ms, "io_bytes_per_launch": io, "io_gbs": io / (ms * 1e-3) / 1e9,
                       "io_frac": io / (ms * 1e-3) / 1e9 / peak, "bound": bound_from_counters(c),
                       "ncu": c or None}
    dom = max(kernels, key=lambda k: kernels[k]["ms_per_frame"])
    # the whole path against the scope table's algorithmic bytes per mol-pair
    b_unit = path_bytes_per_unit(w, eng.natoms, eng.slvmax, eng.ermax, eng.maxdst, eng.nsite_slt)
    traffic = profile_table("frame_traffic.txt").get(w.name, {}).get("dram_bytes_per_unit")
    stage_share = {k: round(stage[k] / max(stage["total"], 1e-9), 4) for k in Engine.STAGES
                   if k not in ("total", "chunks") and stage[k] > 0}
    if rank != 0:
        if ws > 1:
            dist.destroy_process_group()
        return
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": w.name, "waters": int(eng.slvmax), "insertions_per_frame": int(eng.maxdst),
                       "solute_sites": int(eng.nsite_slt), "pme_grid": w.params["ms1max"],
                       "pme_order": w.params["splodr"], "ermax": int(eng.ermax),
                       "pme_solve": {0: "none", 1: "spread + cuFFT", 2: "fused, direct site sums",
                                     3: "fused, plane spreading + FFT"}[paths["spectrum_path"]],
                       "launch": "one CUDA graph per frame",
                       "l2": "flushed before every step (256 MiB write)",
                       "parallelism": f"frames sharded over {ws} rank(s), no collective in the step"},
            "stage_ms_per_frame": {k: round(stage[k] / nst, 4) for k in stage_share},
            "stage_share": stage_share,
            # headline: the whole frame against the HBM roofline of the scope table's algorithmic bytes
            # (a spectrum and a potential grid written and read per insertion, the FP64 energy matrix,
            # ecorr once per batch); the fused solve keeps most of those bytes in L2, so the kernels
            # themselves are bound by SM issue or latency: see roofline.kernels[*].bound
            "roofline": {"kernel": "engconst frame (all kernels)", "bound": "hbm",
                         "achieved": value * b_unit / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": value * b_unit / 1e9 / peak, "peak_source": peak_src,
                         "traffic": None if traffic is None else traffic * units,
                         "algorithmic_bytes_per_frame": b_unit * units, "bytes_per_unit": b_unit,
                         "dominant_kernel": dom, "kernels": kernels},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(4 * 3 * eng.natoms + 4 * eng.maxdst),
                    "d2h_bytes_per_step": d2h_bytes_per_step(eng)},
            "gpu_launches": int(launches)}
    parity = profile_table("parity_error_table.txt").get(w.name)
    if parity:
        line["parity_vs_fp64"] = parity
    clk_s = clk.summary()
    if clk_s:
        line["clocks"] = clk_s
    if ws == 1 and not args.no_cpu_baseline:
        sample = 2000 if args.config == 2 else 128      # 10-30 s of host work at most
        v, dt, u = cpu_baseline(w, sample, os.cpu_count() or 1)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
                                "sample": f"one frame of {sample} insertions x {u // sample} waters ({dt:.1f} s), "
                                          "FP32 restatement of the reference algorithm on all host threads"}
    print(json.dumps(line))
    if ws > 1:
        dist.destroy_process_group()


def main_batch(args):
    """Configuration 4: 64 solutes of 10..300 sites, 500 insertions each, in the shared water box,
    one CUDA-graph launch per frame for all of them (ermod_batch_engconst)."""
    import torch
    from ermod_openacc_b200 import Batch, Engine, systems as S
    import __graft_entry__ as ge
    ge.build_engine()
    ws = S.make_batch_workloads(64, maxins=args.maxins)
    torch.cuda.set_device(0)
    members = [Engine(w.params, w.topo, w.hist) for w in ws]
    batch = Batch(members)
    nfr = args.warmup + args.steps
    frames = [ws[0].frame(i) for i in range(nfr)]
    cell = frames[0][1]
    dev_pos = torch.from_numpy(np.stack([f[0] for f in frames])).to("cuda:0")
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda:0")
    units = sum(m.maxdst * m.slvmax for m in members)
    for i in range(args.warmup):
        batch.engconst_dev(i + 1, dev_pos[i].data_ptr(), cell)
    dev_ms = 0.0
    with ClockSampler(0) as clk:
        for i in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            batch.engconst_dev(args.warmup + i + 1, dev_pos[args.warmup + i].data_ptr(), cell)
            dev_ms += batch.last_ms()
    sizes = [int(m.nsite_slt) for m in members]
    # each member alone, its own one-graph frame, one after another: the batch graph's time against
    # the sum of these says how much running the members as branches of one graph already overlaps,
    # and bounds what a persistent frame kernel could still remove (launch and dependency gaps)
    alone_ms = 0.0
    for j, m in enumerate(members):
        for i in range(2):
            m.engconst_dev(nfr + 10 * j + i + 1, dev_pos[i % nfr].data_ptr(), cell)
        flush.zero_()
        torch.cuda.synchronize()
        m.engconst_dev(nfr + 10 * j + 3, dev_pos[0].data_ptr(), cell)
        alone_ms += m.last_ms()
    line = {"metric": METRIC, "value": units * args.steps / (dev_ms * 1e-3), "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "batch-64-solutes-water4096", "solutes": len(members),
                       "solute_sites": [min(sizes), max(sizes), sum(sizes) / len(sizes)],
                       "insertions_per_solute": int(members[0].maxdst), "waters": int(members[0].slvmax),
                       "launch": "one CUDA graph per frame for all solutes",
                       "l2": "flushed before every step (256 MiB write)"},
            "members_alone_ms_sum": alone_ms,
            "batch_over_alone": (dev_ms / args.steps) / alone_ms if alone_ms > 0 else None}
    clk_s = clk.summary()
    if clk_s:
        line["clocks"] = clk_s
    print(json.dumps(line))


def main_delta_mu(args):
    """Configuration 5: GPU time until the energy-representation solvation free energy is within
    0.05 kcal/mol of a long uniform-insertion run, for uniform and for learned insertion.

    Defaults follow the configuration: a 200-site ring-recipe solute in 4096 waters (49.6 A box,
    PME 64^3), 100,000 insertions per frame, a network (64-128-128-128-1, BF16 weights, FP32
    accumulation, over the 4x4x4 solvent-density features) trained on 1e6 uniform-insertion energies,
    and a 1e7-insertion uniform run (100 frames) as the yardstick.  The water is a disordered packing
    (the lattice has no cavities for a proposal to find); in the solution frames the waters keep 3 A
    from every solute site.  rho and aveuv come from soln frames with the solute at the box centre,
    rho0 / chi0 from refs insertions; delta-mu from the py-hnc functional on the GPU with slvfe's bin
    middles and pickgr = 3 grouping.  Each mode runs `replicas` independent insertion streams over the
    same solvent frames; its error after n frames is the RMS over replicas of the difference to the
    yardstick.  Times are CUDA-event device times of the frames (the learned mode's training is
    reported beside them)."""
    import torch
    import __graft_entry__ as ge
    ge.build_engine()
    from ermod_openacc_b200 import Engine, _capi as A, proposal as P, slvfe, systems as S
    torch.cuda.set_device(0)
    nins, gv, eps, npool = args.ins_per_frame, 32, args.mix_uniform, 16
    base = S.make_workload(2, seed=11)
    slt = S.lj_site() if args.solute_sites == 1 else S.ring_recipe_solute(args.solute_sites, 5)
    box, nside = base.box, base.nside
    # solution: the solute fixed at the centre, waters kept 3 A from every solute site
    sln_topo = S.Topology([slt, S.water()], [1, nside ** 3], [A.PT_SOLUTE, A.PT_SOLVENT])
    sln_prm = S.default_params(slttype=A.SLT_SOLN, ms1max=64, maxins=1, corrcal=0, wgtslf=0)
    sln_w = S.Workload("soln", sln_prm, sln_topo, {}, box, nside, npool, 11,
                       solute_center=np.array([box / 2] * 3), packing="random", avoid_sites=True, avoid_r=3.0)
    eng = Engine(sln_prm, sln_topo, {})
    for i in range(8):
        eng.engconst(i + 1, *sln_w.frame(i))
    sln, _ = eng.engstore()
    rho, aveuv = sln["edens"], [float(sln["slnuv"][0])]
    # slvfe reads engsln's bin middles (slvfe.F90:385) and reports bins merged by pickgr = 3
    _, middle, _, spec = slvfe.representative_bins(eng.uvcrd, eng.uvmax, eng.uvsoft)
    eng.close()
    # reference solvent: pure disordered water, insertions of the same solute
    ref_topo = S.Topology([S.water(), slt], [nside ** 3, 1], [A.PT_SOLVENT, A.PT_TEST_RIGID])
    ref_prm = S.default_params(ms1max=64, maxins=nins, corrcal=1)
    ref_w = S.Workload("refs", ref_prm, ref_topo, {}, box, nside, npool, 12, packing="random")
    frames = [ref_w.frame(i) for i in range(npool)]
    temp_K = ref_prm["temp"] / S.KB_KCAL

    def dmu(e):
        acc, _ = e.engstore()
        return slvfe.delta_mu_gpu(rho, acc["edens"], acc["ecorr"], middle, spec, temp_K, aveuv, group=3)[1]

    def run(mode, iseed, nfr, params=None, checkpoints=()):
        e = Engine(dict(ref_prm, proposal=mode, iseed=iseed), ref_topo, {})
        e.proposal_config(gv, eps, params, feature_cells=gv)
        out, ms = {}, 0.0
        for i in range(nfr):
            e.engconst(i + 1, *frames[i % npool])
            ms += e.last_ms()
            if (i + 1) in checkpoints:
                out[i + 1] = (dmu(e), ms)
        res = out if checkpoints else dmu(e)
        e.close()
        return res, ms

    long_dmu, long_ms = run(A.PROPOSAL_UNIFORM, 999, args.long_frames)
    # training samples: uniform insertions (train_frames x nins energies), then the device trainer
    e = Engine(dict(ref_prm, corrcal=0), ref_topo, {})
    e.proposal_config(gv, eps, feature_cells=gv)
    sample_ms = 0.0
    fs, es = [], []
    for i in range(args.train_frames):
        e.engconst(i + 1, *frames[(npool - 1 - i) % npool])
        sample_ms += e.last_ms()
        f, en, _ = e.insertion_samples()
        fs.append(f)
        es.append(en)
    e.close()
    feats, etot = np.concatenate(fs), np.concatenate(es)
    y, _ = P.labels_from_energies(etot, quantile=args.label_quantile)
    tr = P.Trainer(P.init_params(7), max_batch=4096)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    tr.fit(feats, y, epochs=4, batch=4096, lr=1e-3)
    ev1.record()
    torch.cuda.synchronize()
    train_ms = ev0.elapsed_time(ev1)
    params = tr.params()
    tr.close()
    cps = tuple(c for c in (1, 2, 4, 8, 16, 32, 50, 64) if c <= args.max_frames)
    curves = {}
    for mode in (A.PROPOSAL_UNIFORM, A.PROPOSAL_LEARNED):
        errs = {c: [] for c in cps}
        mspf = []
        for r in range(args.replicas):
            out, ms = run(mode, 100 + r, max(cps), params if mode == A.PROPOSAL_LEARNED else None, cps)
            for c in cps:
                errs[c].append(out[c][0] - long_dmu)
            mspf.append(ms / max(cps))
        rms = {c: float(np.sqrt(np.mean(np.square(errs[c])))) for c in cps}
        m = float(np.mean(mspf))
        hit = next((c for c in cps if rms[c] <= 0.05), None)
        curves["uniform" if mode == A.PROPOSAL_UNIFORM else "learned"] = {
            "rms_error_kcal": rms, "ms_per_frame": m, "frames_to_0.05": hit,
            "gpu_s_to_0.05": None if hit is None else hit * m / 1e3}
    tu, tl = curves["uniform"]["gpu_s_to_0.05"], curves["learned"]["gpu_s_to_0.05"]
    name = "ljsite" if args.solute_sites == 1 else f"ring{args.solute_sites}"
    line = {"metric": "s to delta-mu +/-0.05 kcal/mol", "value": tl, "unit": "s", "n_gpus": 1,
            "higher_is_better": False, "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"learned-{name}-water4096-disordered", "insertions_per_frame": nins,
                       "solute_sites": args.solute_sites, "frames_compared": max(cps),
                       "voxels_per_side": gv, "mix_uniform": eps, "label_quantile": args.label_quantile,
                       "training_samples": int(len(etot)), "replicas": args.replicas,
                       "slvfe": {"bin_coordinates": "engsln bin_middle", "group": 3, "path": "GPU FP64"},
                       "long_uniform_run": {"frames": args.long_frames, "insertions": args.long_frames * nins,
                                            "delta_mu_kcal": long_dmu, "gpu_s": long_ms / 1e3}},
            "uniform": curves["uniform"], "learned": curves["learned"],
            "training_gpu_s": (sample_ms + train_ms) / 1e3,
            "speedup_uniform_over_learned": None if (tu is None or tl is None) else tu / tl}
    print(json.dumps(line))


if __name__ == "__main__":
    main()

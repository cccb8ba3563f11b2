#!/usr/bin/env python
"""Throughput of msim's nonbonded force path on B200.

Workload (one "step" = one energy-and-force evaluation, i.e. one pass of
ElecLJ::add_to_energy_and_forces): 32,768 rigid 3-site waters (98,304 sites)
in a 99.437 A cubic box at 0.997 g/cm^3, seeded lattice + random orientations;
real-space Ewald + LJ with a 9 A group cutoff and 1 A switch, a 1.5 A
neighbour-list skin with the list rebuilt every 10 evaluations, eta 0.35 1/A,
P3M on a 96^3 mesh with order-5 assignment.

Default run: the mixed-precision form (FP32 pair and spline math, 64-bit
fixed-point accumulation) is the headline; the FP64 form is timed beside it
and the mixed form's force error against it is reported.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision mixed|fp64]
  python bench.py --impl reference ...   # the reference's own CPU code, all host cores

Timing: inputs resident in HBM; L2 (126 MB) flushed by a 256 MB write before
every timed evaluation; each evaluation bracketed by CUDA events on the stream
the library launches on; the per-rank sum is max-reduced over ranks.  e2e goes
through the public host-buffer call (mmnb_compute): H2D of positions from
pinned memory, D2H of forces and energy, timed by the wall clock per call.
"""
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

METRIC = "steps/s & pair evals/s, 98k-atom PPPM water: mixed vs FP64 GPU @1e-5 rel F"
NSIDE = 32
MESH = 96
DT_FS = 2.0
L2_FLUSH_BYTES = 256 << 20


def workload_cfg(box):
    return dict(rspace_cutoff=9.0, smoothing_width=1.0, neighbor_list_width=1.5, ewald_screening=0.35,
                use_p3m=True, p3m_grid_spacing=box / MESH, p3m_assignment_order=5, p3m_alias_sum_limit=2)


WORKLOAD = ("32768 rigid waters (98,304 sites), L=99.437 A, PPPM 96^3 order 5, eta 0.35/A, rc 9 A "
            "(1 A switch), skin 1.5 A, list rebuilt every 10 evaluations")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the FP64 comparison leg")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default launch choices instead of timing them (for launch-list captures)")
    return ap.parse_args()


# --------------------------------------------------------------------------- helpers
def dist_env():
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    return rank, world, local


def count_pair_work(p, wb):
    """Unique group pairs listed / within rc, and charged site pairs within the
    group cutoff, from the current list (what RSpaceEwald evaluates)."""
    pairs = p.pairlist()
    A = wb.positions[0::3]
    d = A[pairs[:, 0]] - A[pairs[:, 1]]
    d -= wb.box * np.floor(d / wb.box + 0.5)
    r2 = (d * d).sum(1)
    within = int((r2 <= 81.0).sum())
    return dict(listed=len(pairs), within=within, beyond=len(pairs) - within,
                coulomb_site_pairs=9 * within, lj_pairs=within)


def algorithmic_flops(work):
    # per unit costs fixed in the design notes: 40 flop per Coulomb site pair,
    # 20 per LJ pair, +30 per group pair within rc, +12 per listed pair beyond it
    return (40 * work["coulomb_site_pairs"] + 20 * work["lj_pairs"] + 30 * work["within"] +
            12 * work["beyond"])


class ClockSampler:
    """SM clock, power and clock-event (throttle) reasons of one GPU, polled
    through NVML (the library nvidia-smi reads) every millisecond while the
    timed region runs."""
    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown", 0x4: "sw_power_cap"}

    def __init__(self, bus_id):
        self.bus_id = bus_id
        self.samples = []
        self.max_mhz = None
        self._stop = None

    def __enter__(self):
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            self.nv = nv
            self.h = nv.nvmlDeviceGetHandleByPciBusId(self.bus_id.encode()) if self.bus_id else \
                nv.nvmlDeviceGetHandleByIndex(0)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
            reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
        except Exception as e:  # no NVML: report that, do not guess
            self.error = str(e)
            return self
        self._stop = threading.Event()

        def poll():
            while not self._stop.is_set():
                try:
                    self.samples.append((nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM), reasons(self.h)))
                except Exception:
                    pass
                time.sleep(0.001)
        self.thread = threading.Thread(target=poll, daemon=True)
        self.thread.start()
        time.sleep(0.005)
        return self

    def __exit__(self, *exc):
        if self._stop is not None:
            self._stop.set()
            self.thread.join()
        return False

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz,
                    "reasons": ["no samples: " + getattr(self, "error", "none taken")]}
        reasons = sorted({name for _, r in self.samples for bit, name in self.REASONS.items() if r & bit})
        return {"sm_mhz": statistics.median(c for c, _ in self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples), "source": "NVML, 1 ms polling"}


# --------------------------------------------------------------------------- our arm
def run_ours(args):
    import torch
    import molmodel_b200
    from molmodel_b200 import ElecLJ, water_box

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = torch.device("cuda", local)
    # a dedicated stream: the library launches on it, the events and the L2
    # flush are recorded on it (torch's default stream has handle 0)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)

    # each rank evaluates its own replica (different seed): no data-path collective
    wb = water_box(NSIDE, seed=args.seed + rank)
    cfg = workload_cfg(wb.box)

    def make(precision):
        p = ElecLJ(precision=precision, rebuild_interval=10, device=local, **cfg).init(wb)
        p.set_stream(stream.cuda_stream)
        return p

    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    d_r = torch.from_numpy(wb.positions.reshape(-1)).to(dev)
    d_f = torch.zeros(3 * wb.nsite, dtype=torch.float64, device=dev)
    d_e = torch.zeros(8, dtype=torch.float64, device=dev)

    def timed_loop(p, steps, warmup, graph=True):
        """K evaluations on HBM-resident positions, each bracketed by CUDA
        events after an L2 flush; graph=True replays a CUDA graph of one
        evaluation (the production path), graph=False launches kernel by kernel."""
        p.compute(wb.positions)  # first evaluation: host set-up and list build
        if graph:
            p.graph_capture(d_r.data_ptr(), d_f.data_ptr(), d_e.data_ptr())
            run = p.graph_launch
        else:
            def run():
                p.compute_device(d_r.data_ptr(), d_f.data_ptr(), d_e.data_ptr())
        for _ in range(warmup):
            flush.fill_(1.0)
            run()
        torch.cuda.synchronize(dev)
        l0 = p.launches()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)
        for a, b in evs:
            flush.fill_(1.0)
            a.record(stream)
            run()
            b.record(stream)
        torch.cuda.synchronize(dev)
        if world > 1:
            torch.distributed.barrier()
        # every timed evaluation ran on complete neighbour rows with finite
        # coordinates (mmnb_check raises otherwise)
        p.check()
        return sum(a.elapsed_time(b) for a, b in evs), p.launches() - l0

    def stage_times(p, steps):
        """Per-stage device times (CUDA events between stages) over `steps`
        kernel-by-kernel evaluations, each after an L2 flush."""
        p.set_timing(True)
        for _ in range(steps):
            flush.fill_(1.0)
            p.compute_device(d_r.data_ptr(), d_f.data_ptr(), d_e.data_ptr())
        st = p.timing()
        p.set_timing(False)
        return st

    bus = None
    try:
        pr = torch.cuda.get_device_properties(dev)
        bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
    except Exception:
        pass

    main = make(args.precision)
    # launch choices that change no result, timed on this GPU (mmnb_autotune)
    tuning = main.tuning if args.no_tune else main.autotune(wb.positions, iters=10)
    with ClockSampler(bus) as clk:
        total_ms, launches = timed_loop(main, args.steps, args.warmup, graph=True)
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    steps_per_s = world * args.steps / (total_ms / 1e3)
    nograph_ms, _ = timed_loop(main, args.steps, args.warmup, graph=False)
    stages = stage_times(main, args.steps)

    work = count_pair_work(main, wb)
    flops = algorithmic_flops(work)
    pair_ms = stages.get("rspace_pair")
    clocks = clk.summary()
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    nominal = 148 * (128 if args.precision == "mixed" else 64) * 2 * sm_mhz * 1e6 / 1e12
    if args.precision == "mixed":
        # the FP32 pipe bounds the mixed pair kernel; MEASURED_PEAKS.json holds
        # no FP32 figure, so it is measured here (FMA chains over the device)
        peak = molmodel_b200.potential.measure_fp32_peak(local)
        bound, peak_src = "fp32", "measured in this run: independent FFMA chains over all SMs, best of 4 launches"
    else:
        peak = nominal
        bound, peak_src = "fp64", "148 SMs x 64 FP64 lanes x 2 flop x median SM clock sampled in the run"
    achieved = flops / (pair_ms * 1e-3) / 1e12 if pair_ms else None
    traffic = read_profile_traffic(args.precision)
    roofline = {"bound": bound, "kernel": "rspace_pair", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "flop_per_launch": flops, "launch_ms": pair_ms, "peak_source": peak_src,
                "peak_nominal_at_sampled_clock": nominal,
                "stage_ms": stages, "stage_timing": f"{args.steps} kernel-by-kernel evaluations after the timed "
                "graph replays, events between stages on the library's stream"}
    # the memory/atomic-bound stages against algorithmic bytes (L2-resident working sets)
    nsite = wb.nsite
    mesh_pts = MESH ** 3
    alg = {"p3m_spread": nsite * 125 * 8 + nsite * 32,          # 64-bit reductions + positions, charges
           "p3m_gather": nsite * 125 * 4 + nsite * (24 + 32),   # potential reads + positions, outputs
           "p3m_fft": 2 * (mesh_pts * 4 + MESH * MESH * (MESH // 2 + 1) * 8)}  # one read + write per transform
    roofline["stage_bandwidth_GBs"] = {k: alg[k] / (stages[k] * 1e-3) / 1e9 for k in alg if stages.get(k)}
    roofline["stage_bytes"] = alg

    out = {"metric": METRIC, "value": steps_per_s, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "fp32+fixed64" if args.precision == "mixed" else "f64",
           "data": "synthetic: seeded water lattice, random orientations (one replica per GPU)",
           "config": {"workload": WORKLOAD, "precision": args.precision, "l2": "flushed (256 MB write) before every "
                      "timed step", "parallelism": f"replicas x{world}", "dt_fs_for_ns_per_day": DT_FS,
                      "launch": "CUDA graph of one evaluation, replayed per step",
                      "tuning": {"water_kernel_registers": 128 if tuning[0] == 4 else 96, "spread_layout":
                                 ("thread per site", "thread per site and x-plane",
                                  "lane per site and z-offset")[tuning[1]], "p3m_side_stream": bool(tuning[2]),
                                 "fp64_water_warps_per_block": tuning[3]}},
           "ms_per_step_without_graph": nograph_ms / args.steps,
           "pair_evals_per_s": work["coulomb_site_pairs"] * steps_per_s,
           "ns_per_day": steps_per_s / world * DT_FS * 86400 / 1e6,
           "pair_work_per_step": work, "roofline": roofline, "gpu_launches": launches, "clocks": clocks}

    # e2e through the public host-buffer call
    import ctypes
    pinned_r = torch.from_numpy(wb.positions.copy()).pin_memory()
    host_r = pinned_r.numpy()
    host_f = np.zeros_like(host_r)
    main.compute(host_r)
    e2e_times = []
    for _ in range(max(3, args.steps // 2)):
        flush.fill_(1.0)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        main.add_to_energy_and_forces(0.0, host_f, host_r)
        e2e_times.append(time.perf_counter() - t0)
    e2e_rate = world / statistics.mean(e2e_times)
    out["e2e"] = {"value": e2e_rate, "unit": "steps/s", "h2d_bytes_per_step": 8 * 3 * wb.nsite,
                  "d2h_bytes_per_step": 8 * 3 * wb.nsite + 8 * 4 + 4 * 8,
                  "timing": "wall clock per mmnb_compute call, L2 flushed before each"}

    # the FP64 form beside the mixed one, and the mixed form's error against it
    if args.precision == "mixed" and not args.no_compare:
        ref = make("fp64")
        fp64_ms, _ = timed_loop(ref, args.steps, args.warmup, graph=True)
        fp64_stages = stage_times(ref, args.steps)
        g64 = ref.compute(wb.positions)
        g32 = main.compute(wb.positions)
        df = g32["f"] - g64["f"]
        rms_f = float(np.sqrt((g64["f"] ** 2).sum(1).mean()))
        out["fp64"] = {"steps_per_s": world * args.steps / (fp64_ms / 1e3), "ms_per_step": fp64_ms / args.steps,
                       "stage_ms": fp64_stages}
        out["mixed_over_fp64"] = out["value"] / out["fp64"]["steps_per_s"]
        out["accuracy_vs_fp64"] = {
            "rms_rel_force": float(np.sqrt((df ** 2).sum() / (g64["f"] ** 2).sum())),
            "max_rel_force": float(np.sqrt((df ** 2).sum(1)).max() / rms_f),
            "rel_energy": abs(g32["total"] - g64["total"]) / abs(g64["total"])}
        ref.close()

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(wb, cfg)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    main.close()
    if rank == 0:
        print(json.dumps(out))


def read_profile_traffic(precision):
    """DRAM bytes per launch of the pair kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "rspace_pair_c3.txt")
    if not os.path.exists(path):
        return None
    key = f"dram_bytes_per_launch_{precision}:"
    for line in open(path):
        if line.startswith(key):
            try:
                return float(line.split(":", 1)[1])
            except ValueError:
                return None
    return None


# --------------------------------------------------------------------------- CPU legs
def _ref_worker(conn, seed, n_warm, n_eval):
    """One process: build the reference's ElecLJ path on the workload, run
    n_warm untimed evaluations (the first builds the neighbour list), then,
    on the coordinator's signals, time n_eval evaluations and then one
    neighbour-list rebuild (the reference's NeighborList::rebuild_periodic over
    the same anchors, on a list whose cells and stencil were set up untimed)."""
    sys.path.insert(0, ROOT)
    from molmodel_b200.water import water_box
    from oracle.oracle import reference, port, make_config
    lib = reference() or port()
    wb = water_box(NSIDE, seed=seed)
    wcfg = workload_cfg(wb.box)
    c = make_config(wb.box, **wcfg)
    o = lib.eleclj(c, wb.nsite, wb.groups, wb.exclusions, wb.site_mask, wb.q, wb.sigma, wb.epsilon, wb.rscreen)
    for _ in range(n_warm):
        o.eval(wb.positions)
    anchors = np.ascontiguousarray(wb.positions[0::3])
    conn.send(("ready", lib is reference()))
    conn.recv()
    times = []
    for _ in range(n_eval):
        t0 = time.perf_counter()
        o.eval(wb.positions)
        times.append(time.perf_counter() - t0)
    conn.send(("done", times))
    nl = lib.nbrlist(wb.nwater, wcfg["rspace_cutoff"], wcfg["neighbor_list_width"], wb.box)
    conn.recv()
    t0 = time.perf_counter()
    nl.update(anchors)  # a list that has never been built rebuilds (rebuild_periodic)
    conn.send(("built", time.perf_counter() - t0))


def cpu_baseline(wb, cfg, n_eval=3):
    """The reference's own code (oracle/_ref) on 1 host core: 3 evaluations
    and one list build, the build amortised over 10 steps."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    a, b = ctx.Pipe()
    pr = ctx.Process(target=_ref_worker, args=(b, wb.seed, 1, n_eval))
    pr.start()
    try:
        os.sched_setaffinity(pr.pid, {sorted(os.sched_getaffinity(0))[0]})
    except (AttributeError, OSError):
        pass
    _, is_ref = a.recv()
    a.send("go")
    _, times = a.recv()
    a.send("build")
    _, build = a.recv()
    pr.join()
    steady = min(times)
    per_step = steady + build / 10
    return {"value": 1.0 / per_step, "unit": "steps/s", "cores": 1, "kind": "reference" if is_ref else "port",
            "sample": f"{n_eval} evaluations of the same 98,304-site box on one pinned core (best taken) and "
                      f"one list build amortised over 10 steps: evaluation {steady:.2f} s, build {build:.2f} s"}


def run_reference(args):
    """The reference's CPU code on every host core: P = min(cores, steps)
    independent processes, each timing the same number of evaluations
    m = ceil(steps / P) (so no process waits on a straggler's extra one), then
    one list build each, all concurrently.  value = P / (t_eval + t_build / 10)
    with t_eval the wall time of the evaluation phase / m and t_build that of
    the build phase: the GPU arm's workload, whose list is rebuilt every 10
    evaluations."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    ncores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    steps = max(1, args.steps)
    nproc = min(ncores, steps)
    m = -(-steps // nproc)
    procs, pipes = [], []
    for i in range(nproc):
        a, b = ctx.Pipe()
        pr = ctx.Process(target=_ref_worker, args=(b, args.seed, 1 if args.warmup > 0 else 0, m))
        pr.start()
        procs.append(pr)
        pipes.append(a)
    is_ref = True
    for a in pipes:
        _, r = a.recv()
        is_ref = is_ref and r
    t0 = time.perf_counter()
    for a in pipes:
        a.send("go")
    for a in pipes:
        a.recv()
    wall_eval = time.perf_counter() - t0
    t0 = time.perf_counter()
    for a in pipes:
        a.send("build")
    for a in pipes:
        a.recv()
    wall_build = time.perf_counter() - t0
    for pr in procs:
        pr.join()
    per_step = wall_eval / m + wall_build / 10
    value = nproc / per_step
    out = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": steps,
           "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic: seeded water lattice, random orientations",
           "config": {"workload": WORKLOAD, "precision": "fp64 (reference CPU code)",
                      "parallelism": f"{nproc} independent processes, {m} timed evaluations each "
                                     f"({nproc * m} in all), then one list build each",
                      "list": "rebuilt every 10 evaluations: one timed reference list build per process, "
                              "amortised over 10 steps",
                      "phases_s": {"evaluations": wall_eval, "list_builds": wall_build}},
           "impl": "reference",
           "cpu_baseline": {"value": value, "unit": "steps/s", "cores": nproc,
                            "kind": "reference" if is_ref else "port",
                            "sample": f"{nproc * m} evaluations of the 98,304-site box over {nproc} processes "
                                      f"({m} each) and {nproc} list builds"},
           "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

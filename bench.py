#!/usr/bin/env python3
"""Throughput of HARM's per-step update on B200: zone-cycles/s on the 512^2
Fishbone-Moncrief torus (FP64, PPM reconstruction, HLL flux, flux-CT, 2D
Newton con-to-prim, midpoint RK2).  One zone-cycle = one active zone advanced
by one full RK2 step (the reference's nstep convention, main.c:54,88).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

The b200 arm runs the CUDA step (device-resident state, CUDA graph per step);
under torchrun each rank advances its own torus (replicas only: the path has
no exchange step on one GPU) and the value is the aggregate over ranks timed
as the maximum over ranks.  The reference arm times the reference's own CPU
step (compiled from its sources into oracle/_ref) on the host cores, one
process per core, each on its own torus.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "zone-cycles/s, 512² torus"
UNIT = "zone-cycles/s"
# algorithmic FP64 bytes per zone-cycle of the whole step, each value moved
# once: the state read and written (p in, pk out; pk and p in, p out: 5 x 64
# B), per substep the geometry (CENT, FACE1, FACE2 metric and sqrt(-g), CORN
# sqrt(-g), the 40 connection coefficients: 832 B), the floors (16 B) and
# the pflag read and write (8 B)
BYTES_PER_ZONE_CYCLE = 2032


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--lim", default="para", choices=["para", "mc"])
    ap.add_argument("--flux", default="hll", choices=["hll", "laxf"])
    ap.add_argument("--fluxadjust", type=int, default=3, choices=[0, 1, 2, 3],
                    help="FLUXADJUST: 0 every face uses --flux; 1-3 the per-zone HLL/LAXF switch of the 512^2 and "
                         "1024^2 configuration (FLUXBSQORHOANDU is 3)")
    ap.add_argument("--window-steps", type=int, default=20,
                    help="steps of the same-window comparison: steps 3.. from init, the window the reference arm "
                         "times, with the diagnostic currents on as the reference's step_ch() computes them")
    ap.add_argument("--e2e-steps", type=int, default=50)
    ap.add_argument("--evolve", type=int, default=400,
                    help="untimed steps from init before warm-up, so that the timed steps see a developed flow")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision measurement")
    ap.add_argument("--accuracy-t", type=float, default=100.0,
                    help="time (GM/c^3) to which FP64 and mixed runs go from init for the L1 comparison")
    ap.add_argument("--ensemble", type=int, default=64, help="tori in the batched-ensemble leg (0: skip it)")
    ap.add_argument("--ensemble-steps", type=int, default=200)
    ap.add_argument("--ensemble-steps-per-launch", type=int, default=10)
    ap.add_argument("--adjoint-n", type=int, default=256, help="grid of the adjoint leg (0: skip it)")
    ap.add_argument("--adjoint-t", type=float, default=100.0,
                    help="the adjoint leg runs as many steps as the forward run from init takes to this time")
    ap.add_argument("--adjoint-ckpt", type=int, default=16)
    ap.add_argument("--adjoint-steps", type=int, default=0,
                    help="if > 0, the adjoint leg runs this many steps instead of running to --adjoint-t")
    ap.add_argument("--ffde-t", type=float, default=5.0,
                    help="force-free leg (config C2, 512x256 dipole): both precisions run from init to this time "
                         "(0: skip the leg)")
    ap.add_argument("--ffde-steps", type=int, default=200, help="timed steps of the force-free leg")
    ap.add_argument("--sizes", default="512,1024",
                    help="grid sizes of the HLL/LAXF side measurements (empty: skip them)")
    ap.add_argument("--no-rows", action="store_true",
                    help="skip the measurements of the retry chain, the currents and the dump writer")
    ap.add_argument("--ref-budget", type=float, default=100.0,
                    help="reference arm: seconds of stepping per process after which it stops early")
    return ap.parse_args()


def workload(a, n):
    """The workload description shared by both arms."""
    sw = {0: "fixed " + a.flux.upper(), 1: "HLL/LAXF switch (FLUXBSQORHO)", 2: "HLL/LAXF switch (FLUXBSQOU)",
          3: "HLL/LAXF switch (FLUXBSQORHOANDU)"}[a.fluxadjust]
    return {"workload": f"{n}x{n} Fishbone-Moncrief torus, MKS a=0.9375, FP64, {a.lim.upper()} reconstruction, "
                        f"{a.flux.upper()} flux with per-zone {sw}, flux-CT, 2D Newton con-to-prim, RK2 midpoint, "
                        "courant 0.8", "n1": n, "n2": n, "fluxadjust": a.fluxadjust}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and throttle reasons sampled every few ms during the timed
    region (NVML; nvidia-smi's CSV query as the fallback)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}

    def __init__(self, gpu_index, period_s=0.002):
        self.gpu, self.period = gpu_index, period_s
        self.samples, self.reasons = [], set()
        self.smax = None
        self._stop = threading.Event()
        self._t = None

    def _run(self, nv, h):
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                for name, bit in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(self.period)

    def start(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(self.gpu)
            self.smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self._t = threading.Thread(target=self._run, args=(nv, h), daemon=True)
            self._t.start()
        except Exception:
            self._t = None

    def stop(self):
        if self._t is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        self._stop.set()
        self._t.join()
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.smax,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


# ------------------------------------------------------------------ reference
def _ref_lib(n, fluxadjust):
    """The reference's CPU step for the workload: its sources as the parity
    build patched them (FLUXADJUST FLUXBSQORHOANDU for the switch), compiled
    -O3 -march=native -ffp-contract=off for this host (oracle/build_ref.py
    --native, from the scratch tree the parity build left in oracle/_ref);
    the parity build itself (-O2) if that fails.  (path, flags) or None."""
    problem = "torusfa" if fluxadjust else "torus"
    parity = os.path.join(ROOT, "oracle", "_ref", f"libharmref_{problem}_{n}x{n}.so")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "oracle", "build_ref.py"), "--native", "--problem", problem,
                        "--sizes", f"{n}x{n}"], capture_output=True, text=True)
    lines = r.stdout.strip().splitlines()
    if r.returncode == 0 and lines and os.path.exists(lines[-1]):
        return lines[-1], "-O3 -march=native -ffp-contract=off"
    if os.path.exists(parity):
        return parity, "-O2 -ffp-contract=off (native build failed: %s)" % (r.stderr.strip().splitlines() or ["?"])[-1]
    return None


REF_WORKER = r"""
import ctypes, os, sys, time, tempfile
lib = ctypes.CDLL(sys.argv[1])
lim, nsteps, budget = int(sys.argv[2]), int(sys.argv[3]), float(sys.argv[5])
lib.hr_configure.argtypes = [ctypes.c_int]*3 + [ctypes.c_double, ctypes.c_int, ctypes.c_double]
lib.hr_configure(lim, int(sys.argv[4]), 2, 0.8, 0, 1e30)
w = tempfile.mkdtemp(prefix="harmref_")
fd = os.open(os.devnull, os.O_WRONLY); sv = os.dup(1); os.dup2(fd, 1); os.dup2(fd, 2)
lib.hr_init(w.encode())
ts = []
tstart = time.perf_counter()
for k in range(nsteps):
    t0 = time.perf_counter(); rc = lib.hr_step(1); ts.append(time.perf_counter() - t0)
    if rc: break
    if k >= 1 and time.perf_counter() - tstart > budget: break
os.write(sv, (" ".join("%.6f" % t for t in ts) + "\n").encode())
"""


def run_reference_procs(lib, lim, flux, nsteps, nprocs, budget_s=1e9):
    """nprocs independent reference processes (one torus each, library
    `lib`); per-step wall times of each (a process stops early once budget_s
    of stepping is spent).  Returns a list of lists."""
    procs = [subprocess.Popen([sys.executable, "-c", REF_WORKER, lib, str(lim), str(nsteps), str(flux), str(budget_s)],
                              stdout=subprocess.PIPE, stderr=subprocess.DEVNULL) for _ in range(nprocs)]
    out = []
    for p in procs:
        so, _ = p.communicate()
        line = so.decode().strip().splitlines()
        out.append([float(x) for x in line[-1].split()] if line else [])
    return out


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# the step window both arms time for the same-window comparison: steps
# WINDOW_FIRST.. from init (the reference's step_ch() from its own init())
WINDOW_FIRST = 3


def reference_arm(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    n = a.n
    lim = 4 if a.lim == "para" else 3
    flux = 1 if a.flux == "hll" else 0
    cfg = workload(a, n)
    cfg["parallelism"] = "one process per host core, independent tori"
    lib = _ref_lib(n, a.fluxadjust)
    if lib is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/libharmref_*_%dx%d.so "
                                                              "not present (built from the reference sources by "
                                                              "__graft_entry__.build())" % (n, n)}))
        return 0
    lib, cflags = lib
    nprocs = max(1, min(cpu_cores(), 16))
    t0 = time.time()
    # a reference step of this torus takes seconds per core: the timed steps
    # are the same-window steps (WINDOW_FIRST.. from init), bounded by a wall
    # budget so the run ends in minutes
    warm = WINDOW_FIRST - 1
    per = run_reference_procs(lib, lim, flux, warm + min(a.steps, a.window_steps), nprocs, budget_s=a.ref_budget)
    per = [p for p in per if len(p) > warm]
    if not per:
        print(json.dumps({"impl": "reference", "unavailable": "reference step failed"}))
        return 0
    ktimed = min(len(p) for p in per) - warm
    # aggregate: all processes advance concurrently; a timed step is the
    # slowest process's step
    step_times = [max(p[warm + k] for p in per) for k in range(ktimed)]
    tstep = sum(step_times) / len(step_times)
    value = len(per) * n * n / tstep
    window = f"steps {WINDOW_FIRST}-{WINDOW_FIRST + ktimed - 1} from init"
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": ktimed, "warmup": warm,
            "steps_requested": a.steps, "warmup_requested": a.warmup,
            "ms_per_step": tstep * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded torus of the reference's own init)", "config": cfg,
            "impl": "reference", "window": window,
            "work": "the reference's step_ch(), which computes the diagnostic currents every step "
                    "(WHICHCURRENTCALC 1, step_ch.c:143-156)",
            "build": cflags, "host_cpu": _host_cpu(),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": len(per), "kind": "reference",
                             "sample": f"{len(per)} processes x ({warm} warm-up + {ktimed} timed) reference "
                                       f"steps of a {n}x{n} torus ({window}), built {cflags}; wall "
                                       f"{time.time() - t0:.0f}s"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def _host_cpu():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ------------------------------------------------------------------ b200 arm
def max_over_ranks(x, dist=None, device="cpu"):
    """The job's time for a per-rank quantity: its maximum over ranks."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world, zones_per_rank, seconds_per_step):
    """Whole-job zone-cycles/s: every rank advances its own torus each step."""
    return world * zones_per_rank / seconds_per_step


def b200_arm(a):
    import torch
    import harm_ramt_b200 as hb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    stream = torch.cuda.current_stream()
    n = a.n
    lim = hb.LIM_PARA if a.lim == "para" else hb.LIM_MC
    flux = hb.FLUX_HLL if a.flux == "hll" else hb.FLUX_LAXF
    fa = a.fluxadjust
    h, geom, p0 = hb.torus_context(n, n, lim=lim, fluxmethod=flux, stream=stream.cuda_stream, fluxadjust=fa)

    def barrier():
        if dist is not None:
            dist.barrier()

    # advance past the start-up transient (the first steps from init run a
    # few hundred inversions to the 200-iteration Newton limit)
    if a.evolve:
        h.step_ch(a.evolve)
        h.sync()
    t_evolved = h.sync()["t"]
    # warm-up (also instantiates the CUDA graph of one step)
    h.step_ch(a.warmup)
    h.sync()
    # per-kernel device times of one step, events after every launch
    prof = h.profile_step()
    h.sync()

    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    h.step_ch(a.steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    st = h.sync()
    ms = max_over_ranks(ms, dist, "cuda")
    ms_step = ms / a.steps
    value = aggregate_rate(world, n * n, ms_step * 1e-3)

    # end to end through the C ABI with host buffers: each step uploads the
    # state from host memory, advances it and reads it back
    # (page-locked host buffers; the state of step k+1 is the output of k)
    bufs = [(hb.pinned_empty((n + 6, n + 6, 8)), hb.pinned_empty((n + 6, n + 6, 5), np.int32)) for _ in range(2)]
    h.get_prims(out=bufs[0])
    h2d = bufs[0][0].nbytes
    d2h = bufs[0][0].nbytes + bufs[0][1].nbytes
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(a.e2e_steps):
        src, dst = bufs[k % 2], bufs[(k + 1) % 2]
        h.set_prims(src[0], reset_gammacheck=False)
        h.step_ch(1)
        h.get_prims(out=dst)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / a.e2e_steps, dist, "cuda")
    e2e = aggregate_rate(world, n * n, e2e_s)

    # the device's FP64 instruction rate (own microbenchmark, CUDA events):
    # the step's FP64 kernels run without multiply-add contraction, so their
    # ceiling is the DADD/DMUL rate
    fp64_rates = hb.measure_fp64_peak()
    # roofline of the dominant kernel (largest share of the step's device time)
    peak, peak_kind = peaks()
    dom = max(prof, key=lambda k: prof[k][0])
    dom_ms, dom_launches = prof[dom]
    per_launch_ms = dom_ms / max(dom_launches, 1)
    kbytes = {**KERNEL_BYTES, **(KERNEL_BYTES_SWITCH if a.fluxadjust else {})}
    alg_bytes = kbytes.get(dom, 0) * n * n
    achieved = alg_bytes / (per_launch_ms * 1e-3) / 1e9 if per_launch_ms > 0 else 0.0
    step_alg = BYTES_PER_ZONE_CYCLE * n * n / (ms_step * 1e-3) / 1e9
    total_prof = sum(v[0] for v in prof.values())
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": (TRAFFIC_512[dom] * (n * n) / (512 * 512)) if dom in TRAFFIC_512 else None,
                "bytes_per_zone": kbytes.get(dom, 0), "launch_ms": per_launch_ms,
                "share_of_step": dom_ms / total_prof if total_prof else None,
                "whole_step": {"achieved": step_alg, "frac": step_alg / peak,
                               "bytes_per_zone_cycle": BYTES_PER_ZONE_CYCLE},
                "kernels_ms_per_step": {k: round(v[0], 4) for k, v in prof.items()}}
    # the second ceiling: FP64 instructions the kernel issues per zone (ncu,
    # FP64_INSTR_PER_ZONE) over its event-timed launch, against the measured
    # DADD rate
    fp64 = {"peak_dadd_per_s": fp64_rates["dadd"], "peak_dmul_per_s": fp64_rates["dmul"],
            "peak_dfma_per_s": fp64_rates["dfma"], "how": "harm_measure_fp64_peak: independent DADD/DMUL/DFMA chains "
                                                          "on every SM, CUDA events"}
    for kname, per_zone in FP64_INSTR_PER_ZONE.items():
        if kname in prof and prof[kname][1]:
            # the k_update class times k_update with k_update_tail after it
            # (two launches a substep): its per-launch time is per substep
            nl = prof[kname][1] // 2 if kname == "k_update" else prof[kname][1]
            ms_l = prof[kname][0] / nl
            rate = per_zone * n * n / (ms_l * 1e-3)
            fp64[kname] = {"fp64_instr_per_zone": per_zone, "achieved_per_s": rate, "launch_ms": ms_l,
                           "frac_of_dadd_peak": rate / fp64_rates["dadd"]}
            if kname == "k_update":
                fp64[kname]["launch_ms_includes"] = "k_update_tail"
    roofline["fp64"] = fp64

    mixed = None
    if not a.no_mixed:
        mixed = mixed_precision_leg(a, hb, stream, lim, flux, value, barrier, dist)
    ens = None
    if a.ensemble > 0:
        ens = ensemble_leg(a, hb, stream, lim, flux, barrier, dist)
    adj = None
    if a.adjoint_n > 0:
        adj = adjoint_leg(a, hb, dist)
    rows = None
    if not a.no_rows:
        rows = rows_leg(a, hb, stream, lim, flux, ms_step, barrier, dist)
    sizes = None
    if a.sizes:
        sizes = sizes_leg(a, hb, stream, lim, barrier, dist)
    ffde = ffde_leg(a, hb, stream, barrier, dist) if a.ffde_t > 0 else None
    window = same_window_leg(a, hb, stream, lim, flux, barrier, dist) if a.window_steps > 0 else None
    launches = sum(v[1] for v in prof.values()) * a.steps
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        rl = _ref_lib(n, a.fluxadjust)
        per = run_reference_procs(rl[0], 4 if a.lim == "para" else 3, 1 if a.flux == "hll" else 0, WINDOW_FIRST, 1) \
            if rl else None
        if per and len(per[0]) == WINDOW_FIRST:
            t1 = per[0][-1]
            cpu = {"value": n * n / t1, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"reference step_ch() of the {n}x{n} torus on one host core, step {WINDOW_FIRST} from "
                             f"init ({t1:.2f} s), built {rl[1]}"}
    h.close()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Fishbone-Moncrief torus, init of "
                                                             "init.fishmon.c restated on the host)",
                "config": {**workload(a, n),
                           "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                           "l2": "working set per step (geometry 126 planes x %.1f MB) exceeds L2" %
                                 ((n + 6) * (n + 6) * 8 / 1e6),
                           "state": f"torus advanced {a.evolve} steps from init (t={t_evolved:.4g}) before warm-up"},
                "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
                "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu, "clocks": clk, "mixed": mixed,
                "ensemble": ens, "adjoint": adj, "rows": rows, "sizes": sizes, "ffde": ffde, "same_window": window,
                "newton_iters_per_zone_substep": st["newton_iters"] / max(1, (a.evolve + a.warmup + a.steps + 1) * 2 * n * n),
                "t_end": st["t"], "dt_end": st["dt"]}
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


def ffde_leg(a, hb, stream, barrier, dist):
    """Config C2: the force-free aligned rotator (EOMFFDE on flat space,
    defcoord 6 grid, r in [1, 100] stellar radii, dipole field, surface
    rotating at 0.2; MC + LAXF), 512 x 256, built by the library's own
    set-up.  FP64 and mixed each run from init to t = a.ffde_t (untimed),
    then a.ffde_steps steps are timed with CUDA events.  Reported beside the
    rates: the mixed state's relative L1 against FP64 at t = a.ffde_t (B and
    the velocity), and the fraction of zones whose drift Lorentz factor sits
    at the cap GAMMAMAX that enforces B^2 - E^2 > 0 (E.B = 0 holds by
    construction of the inversion)."""
    import torch
    n1, n2, ng = 512, 256, hb.NG
    world = int(os.environ.get("WORLD_SIZE", "1"))
    out = {"workload": f"{n1}x{n2} force-free aligned rotator (flat space, log-r grid, r in [1, 100], dipole, "
                       f"surface angular frequency 0.2), MC + LAXF, RK2, courant 0.8; state at t={a.ffde_t:g} "
                       f"from init, then {a.ffde_steps} timed steps",
           "data": "synthetic (init.ns.c dipole restated on the host: harm_dipole_geometry, harm_dipole_init)"}
    at_t = {}
    for name, prec in (("fp64", hb.PREC_FP64), ("mixed", hb.PREC_MIXED)):
        h, g, _ = hb.dipole_context(n1, n2, precision=prec, stream=stream.cuda_stream)
        st = h.run_to(a.ffde_t)
        p, _ = h.get_prims()
        at_t[name] = (p[ng:-ng, ng:-ng], st["realnstep"])
        gc = g["gcov"][ng:-ng, ng:-ng, 3, 1:4, 1:4]
        u = at_t[name][0][..., 2:5]
        gamma = np.sqrt(1.0 + np.einsum("...i,...ij,...j->...", u, gc, u))
        capped = float((gamma > 25.0 * (1 - 1e-9)).mean())
        h.set_end_time(1.0e30)  # run_to left the end time at a.ffde_t: steps past it would have dt = 0
        h.step_ch(a.warmup)
        h.sync()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        h.step_ch(a.ffde_steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda") / a.ffde_steps
        prof = h.profile_step()
        h.sync()
        h.close()
        out[name] = {"value": aggregate_rate(world, n1 * n2, ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
                     "steps_to_t": int(at_t[name][1]), "zones_at_gamma_cap": capped,
                     "max_drift_gamma": float(gamma.max()),
                     "kernels_ms_per_step": {k: round(v[0], 4) for k, v in prof.items() if v[1]}}
    out["mixed"]["speedup_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    pd, pm = at_t["fp64"][0], at_t["mixed"][0]
    l1 = lambda x, y: float(np.abs(x - y).sum() / np.abs(y).sum())
    out["mixed"]["l1_vs_fp64_at_t"] = {"B": l1(pm[..., 5:8], pd[..., 5:8]), "u": l1(pm[..., 2:5], pd[..., 2:5])}
    return out


def sizes_leg(a, hb, stream, lim, barrier, dist):
    """The configuration at the other grid sizes of --sizes (the per-zone
    switch as in the headline), and at the headline size each fixed Riemann
    solver (fluxadjust 0, HLL and LAXF): whole-job zone-cycles/s after 100
    untimed steps, device time of 100 steps (max over ranks)."""
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    flux = hb.FLUX_HLL if a.flux == "hll" else hb.FLUX_LAXF
    runs = [(n, flux, a.fluxadjust, f"{a.flux}_switch{a.fluxadjust}") for n in [int(x) for x in a.sizes.split(",") if x]
            if n != a.n]
    runs += [(a.n, hb.FLUX_HLL, 0, "hll_fixed"), (a.n, hb.FLUX_LAXF, 0, "laxf_fixed")]
    out = {}
    for n, fl, fa, name in runs:
        h, _, _ = hb.torus_context(n, n, lim=lim, fluxmethod=fl, stream=stream.cuda_stream, fluxadjust=fa)
        h.step_ch(100)
        h.sync()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        h.step_ch(100)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda") / 100
        h.sync()
        h.close()
        out[f"{n}_{name}"] = {"value": aggregate_rate(world, n * n, ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
                              "workload": f"{n}x{n} torus, FP64, {a.lim.upper()} + "
                                          f"{['LAXF', 'HLL'][fl]}, fluxadjust {fa}, steps 101-200 from init"}
    return out


def same_window_leg(a, hb, stream, lim, flux, barrier, dist):
    """The reference arm's window and work on the device: a fresh torus from
    init, steps WINDOW_FIRST.. (a.window_steps of them), the diagnostic
    currents on as in the reference's step_ch().  (1) device-resident state,
    CUDA events; (2) end to end through the C ABI from host buffers: each
    step uploads the state, steps and reads state and flags back."""
    import torch
    n = a.n
    world = int(os.environ.get("WORLD_SIZE", "1"))
    K = a.window_steps
    out = {"window": f"steps {WINDOW_FIRST}-{WINDOW_FIRST + K - 1} from init",
           "work": "step_ch() with the diagnostic currents (J^mu, Faraday slots) every step"}
    h, _, _ = hb.torus_context(n, n, lim=lim, fluxmethod=flux, stream=stream.cuda_stream, currents=True,
                               fluxadjust=a.fluxadjust)
    h.step_ch(WINDOW_FIRST - 1)
    h.sync()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    h.step_ch(K)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda") / K
    h.close()
    out["value"] = aggregate_rate(world, n * n, ms * 1e-3)
    out["unit"] = UNIT
    out["ms_per_step"] = ms
    h, _, _ = hb.torus_context(n, n, lim=lim, fluxmethod=flux, stream=stream.cuda_stream, currents=True,
                               fluxadjust=a.fluxadjust)
    h.step_ch(WINDOW_FIRST - 1)
    bufs = [(hb.pinned_empty((n + 6, n + 6, 8)), hb.pinned_empty((n + 6, n + 6, 5), np.int32)) for _ in range(2)]
    h.get_prims(out=bufs[0])
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(K):
        src, dst = bufs[k % 2], bufs[(k + 1) % 2]
        h.set_prims(src[0], reset_gammacheck=False)
        h.step_ch(1)
        h.get_prims(out=dst)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / K, dist, "cuda")
    h.close()
    out["e2e"] = {"value": aggregate_rate(world, n * n, e2e_s), "unit": UNIT, "ms_per_step": e2e_s * 1e3,
                  "h2d_bytes_per_step": bufs[0][0].nbytes, "d2h_bytes_per_step": bufs[0][0].nbytes + bufs[0][1].nbytes}
    return out


def rows_leg(a, hb, stream, lim, flux, ms_step, barrier, dist):
    """The step's optional parts on the benchmark torus (device time, CUDA
    events, max over ranks): (1) the diagnostic currents every step
    (currents = 1) against the plain step (ms_step) in the developed flow;
    (2) the UTOPRIMTRYAGAIN retry chain (tryagain = 1) against the 2D
    inversion alone over the first steps from init, where the start-up
    transient fails inversions; (3) the reference-layout dump file written
    from the device state."""
    import tempfile

    import torch
    n = a.n

    def timed(h, k):
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        h.step_ch(k)
        e1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1), dist, "cuda") / k

    out = {}
    # (1) currents, developed flow
    h, geom, _ = hb.torus_context(n, n, lim=lim, fluxmethod=flux, stream=stream.cuda_stream, currents=True,
                                  fluxadjust=a.fluxadjust)
    h.step_ch(a.evolve + a.warmup)
    h.sync()
    k = max(20, min(a.steps, 200))
    ms_cur = timed(h, k)
    h.sync()
    out["currents"] = {"ms_per_step": ms_cur, "ms_per_step_without": ms_step, "overhead": ms_cur / ms_step - 1.0,
                       "steps": k, "what": "Faraday slots and J^mu after every step (step_ch.c:143-156)"}
    # (3) dump file of that state (needs the currents)
    header, coords = hb.torus_dump_coords(hb.torus_params(n, n))
    fd, path = tempfile.mkstemp(prefix="harm_dump_")
    os.close(fd)
    try:
        h.write_dump(path, header, coords)  # first call: buffers
        t0 = time.perf_counter()
        h.write_dump(path, header, coords)
        dt_dump = time.perf_counter() - t0
        size = os.path.getsize(path)
    finally:
        os.unlink(path)
    h.close()
    out["dump"] = {"seconds": max_over_ranks(dt_dump, dist, "cuda"), "bytes": size,
                   "MB_per_s": size / 1e6 / dt_dump,
                   "what": "reference dump file (dump.c layout, text) of the 512^2 state from the device"}
    # (2) retry chain over the start-up transient
    ks = 40
    res = {}
    for name, ta in (("with_chain", True), ("without_chain", False)):
        h, _, _ = hb.torus_context(n, n, lim=lim, fluxmethod=flux, stream=stream.cuda_stream, tryagain=ta,
                                   fluxadjust=a.fluxadjust)
        h.step_ch(1)  # the graph
        h.sync()
        res[name] = timed(h, ks)
        st = h.sync()
        res[name + "_fixups"] = st["fixups"]
        h.close()
    out["tryagain"] = {"ms_per_step": res["with_chain"], "ms_per_step_without": res["without_chain"],
                       "steps": ks, "state": "steps 2-41 from init",
                       "repaired_zones": {"with_chain": res["with_chain_fixups"],
                                          "without_chain": res["without_chain_fixups"]},
                       "what": "failed 2D inversions retried by 5D1, 2D, 1D, 1D_OPT, 1D_FINAL, 2D_FINAL, 5D2_FINAL "
                               "(step_ch.c:608-626) before fixup_utoprim repairs the rest"}
    return out


def adjoint_leg(a, hb, dist):
    """The differentiated form on its configuration: the adjoint_n^2 torus
    from init (MC + HLL, the seeded 4% u perturbation), as many steps as a
    run from init takes to t = adjoint_t (so that the torus and the horizon
    are causally connected), a checkpoint every adjoint_ckpt steps, then
    the adjoint back to the initial state (harm_adjoint_run) for J = sum_n
    dt_n (horizon mass flux + horizon EM energy flux).  Reports device times
    of the forward and the backward pass (max over ranks) and the gradient's
    size with respect to the initial A_phi and u.  One untimed short call
    first loads the kernels."""
    n, C = a.adjoint_n, a.adjoint_ckpt
    par = hb.torus_params(n, n)
    geom = hb.torus_geometry(par)
    p0, A, norm = hb.torus_init_vpot(par, geom)

    def ctx():
        h = hb.HarmGPU(n, n, geom["dx1"], geom["dx2"], lim=hb.LIM_MC, fluxmethod=hb.FLUX_HLL, gam=par.gam,
                       gammamax=par.gammamax)
        h.upload_geometry(geom["gcov"], geom["gcon"], geom["gdet"], geom["conn"], geom["floors"])
        h.set_prims(p0)
        h.set_time(0.0, 1e-5, 0)
        return h

    if a.adjoint_steps > 0:
        K = a.adjoint_steps
    else:
        h = ctx()
        K = int(h.run_to(a.adjoint_t)["realnstep"])
        h.close()
    h = ctx()
    h.adjoint(C, C, 1.0, 1.0, None)
    h.close()
    h = ctx()
    J, grad, dts, ms = h.adjoint(K, C, 1.0, 1.0, None)
    h.close()
    fwd, bwd = max_over_ranks(ms[0], dist, "cuda"), max_over_ranks(ms[1], dist, "cuda")
    gA = hb.vpot_adjoint(par, geom, grad, norm)
    return {"workload": f"{n}x{n} Fishbone-Moncrief torus from init (seeded 4% u perturbation), MC + HLL, FP64",
            "steps": K, "checkpoint_every": C, "t_end": float(dts.sum()),
            "grad_A_phi_l2": float((gA ** 2).sum() ** 0.5), "grad_u_l2": float((grad[..., 1] ** 2).sum() ** 0.5),
            "objective": "sum_n dt_n (horizon mass flux + horizon EM energy flux)", "J": J,
            "forward_ms": fwd, "backward_ms": bwd, "forward_ms_per_step": fwd / K, "backward_ms_per_step": bwd / K,
            "backward_over_forward": bwd / fwd,
            "grad_A_phi_max": float(abs(gA).max()), "grad_u_max": float(abs(grad[..., 1]).max()),
            "dJ_dlnu_max": float(abs(grad[..., 1] * p0[..., 1]).max()),
            "dJ_dA_phi_times_A_max": float(abs(gA).max() * abs(A).max()),
            "note": "backward = segment replays with recording + adjoint kernels, per-slot graphs captured in the call"}


def ensemble_leg(a, hb, stream, lim, flux, barrier, dist):
    """The batched form: a.ensemble tori of uneven size and parameters
    (harm_ramt_b200.ensemble.sample_tori), tile shapes autotuned per torus,
    a.ensemble_steps steps of all of them (1) as one CUDA graph launch per
    a.ensemble_steps_per_launch steps holding every torus as a branch, and
    (2) torus after torus, each with its own per-step graph launches, from
    the same initial states.  Aggregate zone-cycles/s of both, FP64 and
    mixed; max over ranks."""
    import torch
    from harm_ramt_b200 import autotune
    from harm_ramt_b200 import ensemble as ens
    specs = ens.sample_tori(a.ensemble, seed=7)
    zones = sum(s["n1"] * s["n2"] for s in specs)
    K, S = a.ensemble_steps, a.ensemble_steps_per_launch
    K -= K % S
    world = int(os.environ.get("WORLD_SIZE", "1"))
    out = {"tori": a.ensemble, "zones_per_step": zones, "steps": K, "steps_per_launch": S,
           "sizes": "N1, N2 uniform in {64, 96, ..., 384}; a ~ U[0, 0.99]; beta log-uniform [10, 1000]; "
                    "rmax ~ U[10, 16]; seed 7"}

    def timed(fn):
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1), dist, "cuda")

    for name, prec in (("fp64", hb.PREC_FP64), ("mixed", hb.PREC_MIXED)):
        members = ens.build(hb, specs, lim=lim, fluxmethod=flux, precision=prec, stream=stream.cuda_stream,
                            fluxadjust=a.fluxadjust)
        tiles = {}
        for (h, p0), s in zip(members, specs):
            up, sm, _ = autotune.tune(h, reps=2, key=(s["n1"], s["n2"], prec, lim, flux))
            tiles[f"{up[0]}x{up[1]}/{sm[0]}x{sm[1]}"] = tiles.get(f"{up[0]}x{up[1]}/{sm[0]}x{sm[1]}", 0) + 1
            ens.reset(h, p0)
        hs = [h for h, _ in members]
        for h in hs:  # capture each member's own step graph outside the timed region
            h.step_ch(1)
        for (h, p0) in members:
            ens.reset(h, p0)
        ms_seq = timed(lambda: [h.step_ch(K) for h in hs])
        failed_seq = [k for k, h in enumerate(hs) if h.sync(raise_on_fail=False)["fail_code"]]
        for (h, p0) in members:
            ens.reset(h, p0)
        e = hb.Ensemble(hs, steps_per_launch=S, stream=stream.cuda_stream)
        ms_ens = timed(lambda: e.step(K))
        st = e.sync(raise_on_fail=False)
        failed = [k for k, s in enumerate(st) if s["fail_code"]]
        e.close()
        for h in hs:
            h.close()
        v_ens = aggregate_rate(world, zones, ms_ens * 1e-3 / K)
        v_seq = aggregate_rate(world, zones, ms_seq * 1e-3 / K)
        out[name] = {"graph_batched": v_ens, "sequential_per_torus": v_seq, "speedup": v_ens / v_seq,
                     "ms_per_step_batched": ms_ens / K, "ms_per_step_sequential": ms_seq / K,
                     "tiles_chosen": tiles, "failed_members": failed, "failed_members_sequential": failed_seq}
    return out


# diagnostic times of the accuracy curve (GM/c^3); the last one is --accuracy-t
ACC_TIMES = (1.0, 3.0, 10.0, 30.0)


def accuracy_curve(a, hb, stream, lim, flux):
    """Relative L1 differences against the FP64 run from the same initial
    torus, at a ladder of times up to accuracy_t, for (1) the mixed form and
    (2) the FP64 path started from a copy of the initial state whose u was
    perturbed by a seeded relative 1e-15 (a few ulps).  (2) is the floor set
    by the flow's own sensitivity: no arithmetic change can be compared
    against FP64 more closely than round-off-level noise grows."""
    n = a.n
    times = [t for t in ACC_TIMES if t < a.accuracy_t] + [a.accuracy_t]
    runs = {}
    for name in ("fp64", "mixed", "fp64_perturbed"):
        prec = hb.PREC_MIXED if name == "mixed" else hb.PREC_FP64
        h, _, p0 = hb.torus_context(n, n, lim=lim, fluxmethod=flux, precision=prec, tf=times[0], fluxadjust=a.fluxadjust,
                                    stream=stream.cuda_stream)
        if name == "fp64_perturbed":
            rng = np.random.default_rng(20240607)
            pp = p0.copy()
            pp[3:-3, 3:-3, 1] *= 1.0 + 1e-15 * (2.0 * rng.random(pp[3:-3, 3:-3, 1].shape) - 1.0)
            h.set_prims(pp)
            h.bound_prims()
        snaps = []
        try:
            for T in times:
                st = h.run_to(T)
                p, _ = h.get_prims(with_flags=False)
                snaps.append((p[3:-3, 3:-3].copy(), h.get_horizon()["pcum_rho"], st["realnstep"]))
        except hb.HarmError as e:
            st = h.sync(raise_on_fail=False)
            h.close()
            return {"error": f"{name} run stopped at t={st['t']:.4g}: {e}"}
        h.close()
        runs[name] = snaps
    l1 = lambda x, y: float(np.abs(x - y).sum() / np.abs(y).sum())

    def diff(name, k):
        p, m, _ = runs[name][k]
        q, mq, _ = runs["fp64"][k]
        return {"rho": l1(p[..., 0], q[..., 0]), "u": l1(p[..., 1], q[..., 1]), "B": l1(p[..., 5:8], q[..., 5:8]),
                "horizon_mass_flux_integrated": abs(m - mq) / abs(mq)}
    return {"t": times, "steps_fp64": [r[2] for r in runs["fp64"]],
            "mixed_vs_fp64": [diff("mixed", k) for k in range(len(times))],
            "fp64_perturbed_1e-15_vs_fp64": [diff("fp64_perturbed", k) for k in range(len(times))]}


def mixed_precision_leg(a, hb, stream, lim, flux, value_fp64, barrier, dist):
    """The mixed form: throughput on the same developed torus, and relative
    L1 errors against FP64 for runs from init to t = accuracy_t."""
    import torch
    n = a.n
    hm, _, _ = hb.torus_context(n, n, lim=lim, fluxmethod=flux, precision=hb.PREC_MIXED, stream=stream.cuda_stream,
                                fluxadjust=a.fluxadjust)
    if a.evolve:
        hm.step_ch(a.evolve)
    hm.step_ch(a.warmup)
    hm.sync()
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    hm.step_ch(a.steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1), dist, "cuda") / a.steps
    world = int(os.environ.get("WORLD_SIZE", "1"))
    vm = aggregate_rate(world, n * n, ms * 1e-3)
    prof = hm.profile_step()
    hm.close()
    out = {"value": vm, "unit": UNIT, "ms_per_step": ms, "speedup_vs_fp64": vm / value_fp64,
           "kernels_ms_per_step": {k: round(v[0], 4) for k, v in prof.items()}}
    if a.accuracy_t > 0:
        out["l1_vs_fp64"] = accuracy_curve(a, hb, stream, lim, flux)
    return out


# algorithmic bytes per active zone of one launch (FP64): every plane each
# kernel must read or write once, 8 bytes a value
KERNEL_BYTES = {
    "k_flux": 8 * (8 + 2 * 21 + 2 * 8),       # prims once, FACE1+FACE2 geometry, F1+F2 out
    "k_update": 8 * (8 + 8 + 21 + 40 + 2 + 2 * 8 + 1 + 8) + 4,  # pi, pb, CENT geo, conn, floors, 2 faces x2, emf, pf, pflag
    "k_emf": 8 * (2 + 3 + 1),
    "k_bsqflags": 8 * (8 + 21) + 1,
}
# with the per-zone HLL/LAXF switch the first substep's k_flux also reads the
# CENT geometry (21 values) and writes the two flag bytes, the second reads
# the flux choice: averaged over the two launches of a step
KERNEL_BYTES_SWITCH = {"k_flux": KERNEL_BYTES["k_flux"] + (8 * 21 + 2 + 1) / 2}
# FP64-pipe instructions (thread slots: adds, multiplies, comparisons and the
# FMAs of division and square root) per active zone of one launch, from one
# ncu capture of each kernel at 512^2 in the developed flow
# (sm__inst_executed_pipe_fp64.sum x 32 / zones; profiles/k_flux_*, k_update_*;
# the k_flux launch captured is a first substep, which also forms the flags)
FP64_INSTR_PER_ZONE = {"k_flux": 3940, "k_update": 1983}
# dram__bytes_read.sum + dram__bytes_write.sum per launch from the same
# captures, scaled by zone count
TRAFFIC_512 = {"k_flux": 145.9e6, "k_update": 196.6e6}


def main():
    a = parse()
    if a.impl == "reference":
        return reference_arm(a)
    return b200_arm(a)


if __name__ == "__main__":
    sys.exit(main())

"""Benchmark: seconds per EZmock mock on B200 (create_dens_field + populate).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One step = one mock of the single-mock workload (Ngrid 512^3, box 2500 Mpc/h,
n = 2e-4 (h/Mpc)^3, rho_c 0.8, rho_exp 20, pdf_base 0.3, sigma_v 400 km/s,
synthetic BBKS P(k) with sigma_8 = 0.81, z = 0.8, MT19937) through the C-ABI
library: the initial field, three Zel'dovich displacement FFTs, the CIC
density and the tracer population.  With N > 1 (torchrun, one process per
GPU) every rank produces its own mocks (independent seeds; replicas, weak
scaling) and the slowest rank's device time defines the job time.

The JSON line reports
  value      : s/mock with inputs resident on the GPU (catalogue left on the
               GPU), from CUDA events on the library's stream, max over ranks;
  e2e        : s/mock through the public EZmock_* calls with host buffers
               (P(k) upload, catalogue copied into malloc'd host arrays);
  roofline   : the dominant kernel's algorithmic bytes / launch time against
               the measured HBM copy bandwidth;
  cpu_baseline (rank 0, N = 1): the reference's own libEZmock sources
               (oracle/_ref, OpenMP, all host cores) on the same workload.
`--impl reference` runs only that CPU path and prints its line.
"""
import argparse
import ctypes
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

from ezmock_b200.replicas import job_seconds_per_mock  # noqa: E402

METRIC = "s/mock at 512^3 (FP32 production mode)"
STAGES = ["rng", "ic", "fft_i", "fft_j", "fft_k", "cic", "bias", "select", "emit", "vel",
          "d2h"]


def workload_desc(cfg):
    pops = cfg.population_list()
    desc = "; ".join(f"n={n:g}, rho_c={a:g}, rho_exp={e:g}, pdf_base={pb:g}, sigma_v={sv:g}"
                     for n, a, e, pb, sv in pops)
    return (f"{cfg.name}: 1 mock {cfg.Ng}^3, box {cfg.Lbox:g} Mpc/h, "
            f"{len(pops)} population{'s' if len(pops) > 1 else ''} ({desc}), "
            f"{'MT19937' if cfg.rng else 'MRG32k3a'}, z={cfg.z:g}")


def pk_trim_len(k, Ng, Lbox):
    """Number of P(k) bins the library keeps (linear_pk.c:114-126)."""
    kmin = 2 * math.pi / Lbox
    kmax = math.pi * Ng / Lbox * math.sqrt(3)
    imin = int(np.searchsorted(k, kmin, side="right"))
    imax = int(np.searchsorted(k, kmax, side="right"))
    imin = max(imin - 3, 0)
    imax = min(imax + 3, len(k))
    return imax - imin


def algorithmic_bytes(Ng, b):
    """Compulsory HBM bytes per launch of each stage (FP32: b = 4)."""
    N = Ng ** 3
    Nk = Ng * Ng * (Ng // 2 + 1)
    H = Nk * 2 * b                               # one half-complex spectrum
    return {
        "ic": 2 * Nk * 4 + H,                    # draws read, spectrum written
        "fft_i": 3 * H,                          # read S, write 2 spectra
        "fft_j": 5 * H,                          # read 2, write 3
        "fft_k": 3 * H + 3 * N * b,              # read 3 spectra, write 3 psi
        "cic": 3 * N * b + 4 * N * b,            # read psi, write rho + 3 momenta
    }


def read_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def read_traffic(workload):
    """Per-launch DRAM bytes of each stage's kernel for `workload`, from the
    committed ncu summary (profiles/traffic.json)."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(workload, {})
    except Exception:
        return {}


class ClockSampler:
    """SM clock and throttle-reason samples, every 200 ms, while the timed
    region runs: read in this process through NVML (three calls per sample),
    or, where NVML cannot be loaded, from an `nvidia-smi -lms 200` process."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.nvml = None
        self.samples = []               # (host time, sm MHz, max MHz, reason names)
        self.window = None
        self.done = threading.Event()

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.idx)
            self.nvml = (pynvml, h)
            self.bits = [pynvml.nvmlClocksEventReasonHwSlowdown,
                         pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                         pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                         pynvml.nvmlClocksEventReasonSwPowerCap]
            self.th = threading.Thread(target=self._poll, daemon=True)
            self.th.start()
        except Exception:
            self.nvml = None
            self._start_smi()
        # the first sample before the warm-up: start-up stays out of the timed
        # region
        t_end = time.perf_counter() + 10.0
        while not self.samples and time.perf_counter() < t_end and \
                (self.nvml is not None or (self.proc and self.proc.poll() is None)):
            time.sleep(0.01)

    def _poll(self):
        nv, h = self.nvml
        while not self.done.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((time.perf_counter(), float(sm), float(mx),
                                     [n for n, b in zip(self.NAMES, self.bits) if r & b]))
            except Exception:
                pass
            self.done.wait(0.2)

    def _start_smi(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-i", str(self.idx), "-lms", "200"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read_smi, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read_smi(self):
        for line in self.proc.stdout:
            p = [x.strip() for x in line.strip().split(",")]
            if len(p) < 9:
                continue
            try:
                self.samples.append((time.perf_counter(), float(p[1]), float(p[2]),
                                     [n for n, v in zip(self.NAMES, p[5:9])
                                      if v.lower() == "active"]))
            except ValueError:
                continue

    def mark(self, t0, t1):
        """Keep only samples taken between host times t0 and t1 (the timed
        region)."""
        self.window = (t0, t1)

    def stop(self):
        self.done.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.nvml is None and not self.proc:
            return None
        self.th.join(timeout=2)
        if self.nvml is not None:
            try:
                self.nvml[0].nvmlShutdown()
            except Exception:
                pass
        sel = [x for x in self.samples
               if self.window is None or self.window[0] <= x[0] <= self.window[1]]
        if not sel and self.samples:     # timed region shorter than one period
            t_mid = 0.5 * (self.window[0] + self.window[1])
            sel = [min(self.samples, key=lambda x: abs(x[0] - t_mid))]
        if not sel:
            return None
        reasons = sorted({n for x in sel for n in x[3]})
        return {"sm_mhz": statistics.median(x[1] for x in sel), "sm_max_mhz": sel[-1][2],
                "reasons": reasons, "samples": len(sel),
                "source": "nvml" if self.nvml is not None else "nvidia-smi"}


def cpu_reference(cfg, k, P, steps, warmup, allow_scale=True, budget_s=240.0):
    """The reference's libEZmock (oracle/_ref, OpenMP, all host threads) on the
    workload.  Returns a dict: s/mock (median), its create_dens_field and
    populate_tracer parts (medians), the wall time of the three c2r FFTs of
    one field through the same FFTW interface (the project CPU FFT, FFTW3
    being absent), the sample description and the thread count."""
    from oracle.pyoracle import RefLib
    R = RefLib(32, nthread=0)
    nthreads = os.cpu_count()
    R.lib.ezref_fft_c2r_seconds.restype = ctypes.c_double
    R.lib.ezref_fft_c2r_seconds.argtypes = [ctypes.c_int, ctypes.c_int]

    def one(Ng, Lbox, seed):
        m = R.new(Lbox, Ng, cfg.rng, seed)
        m.eval_growth(cfg.z, cfg.omega_m)
        m.setup_pk(k, P)
        t0 = time.perf_counter()
        m.create()
        t1 = time.perf_counter()
        for n_t, *par in cfg.population_list():
            m.populate(par, int(round(n_t * Lbox ** 3)))
        t2 = time.perf_counter()
        return t2 - t0, t1 - t0, t2 - t1

    def run(Ng, Lbox, scale, what):
        for w in range(min(warmup, 1)):
            one(Ng, Lbox, 1000 + w)
        ts = [one(Ng, Lbox, 1 + s) for s in range(steps)]
        med = [statistics.median(t[i] for t in ts) * scale for i in range(3)]
        fft = R.lib.ezref_fft_c2r_seconds(Ng, 0) * scale
        return {"value": med[0], "create_s": med[1], "populate_s": med[2], "fft_s": fft,
                "sample": f"{what}, {nthreads} OpenMP threads; 1 warm-up, median of {steps}; "
                          "FFT: project CPU FFT (FFTW3 not installed), "
                          f"3 c2r FFTs {fft:.2f} s of the create_dens_field part",
                "cores": nthreads}

    # a half-size probe decides whether full-size steps fit in the budget
    ng_s = cfg.Ng // 2
    scale = 8 * math.log(cfg.Ng ** 3) / math.log(ng_s ** 3)
    t_small = one(ng_s, cfg.Lbox / 2, 1)[0]
    if t_small * scale * (steps + min(warmup, 1)) < budget_s or not allow_scale:
        return run(cfg.Ng, cfg.Lbox, 1.0, f"{steps} full {cfg.Ng}^3 mocks")
    return run(ng_s, cfg.Lbox / 2, scale,
               f"{steps} mocks at {ng_s}^3, box {cfg.Lbox / 2:g} (the same cell size and "
               f"tracer densities) x {scale:.2f} (N log N scaling to {cfg.Ng}^3)")


def config_of(cfg, n_gpus, b):
    """The workload description both arms print (identical dicts)."""
    pops = [int(round(n_t * cfg.Lbox ** 3)) for n_t, *_ in cfg.population_list()]
    return {"workload": workload_desc(cfg), "Ngrid": cfg.Ng, "Lbox": cfg.Lbox,
            "nexp": pops[0] if len(pops) == 1 else pops,
            "parallelism": f"replicas x{n_gpus}",
            "l2": f"inputs larger than L2 (psi {3 * cfg.Ng ** 3 * b / 1e9:.1f} GB, "
                  f"spectra {3 * cfg.Ng ** 2 * (cfg.Ng // 2 + 1) * 2 * b / 1e9:.1f} GB per mock)"}


def survey_bytes(cfg, b, ntr):
    """Compulsory HBM bytes of one whole mock (three c2r FFTs as two sweeps
    each with the spectrum generated on-chip, CIC, bias/select and emission
    per population, velocity painting, catalogue)."""
    N = cfg.Ng ** 3
    H = cfg.Ng ** 2 * (cfg.Ng // 2 + 1) * 2 * b
    npop = len(cfg.population_list())
    return 3 * (2 * H + N * b) + 4 * N * b + npop * (4 * N * b + 2 * N + 4 * N) + 6 * N * b + 6 * b * ntr


def measure(cfg, args, m, L, k, P, rep, local, n_gpus, seed0, clk):
    """Device-timed steps, a stage-timing pass and end-to-end steps of one
    workload on instance m; returns the line's measured keys."""
    pops = [(int(round(n_t * cfg.Lbox ** 3)), par) for n_t, *par in cfg.population_list()]
    b = 4 if args.prec == 32 else 8
    seed = [seed0]

    def device_step(timing):
        seed[0] += 1
        m.set_option(4, seed[0])
        m.create_dens_field_from_ic()
        stage_c = m.stage_times() if timing else {}
        n, stage_p = 0, {}
        for nexp_i, par in pops:
            n += m.populate_device(*par, nexp_i)
            if timing:
                for s_, v_ in m.stage_times().items():
                    if v_ >= 0:
                        stage_p[s_] = stage_p.get(s_, 0.0) + v_
        return n, stage_c, stage_p

    m.set_option(2, 0)                       # no per-stage events in the timed region
    for _ in range(args.warmup):
        device_step(False)
    m.sync()
    rep.barrier()
    l0 = L.EZmockB200_launch_count()
    L.EZmockB200_mark(m._ez, 0)
    t0 = time.perf_counter()
    ntr = 0
    for _ in range(args.steps):
        ntr = device_step(False)[0]
    L.EZmockB200_mark(m._ez, 1)
    ms = ctypes.c_double()
    L.EZmockB200_elapsed(m._ez, 0, 1, ctypes.byref(ms))
    wall = time.perf_counter() - t0
    launches = L.EZmockB200_launch_count() - l0
    if clk is not None:
        clk.mark(t0, t0 + wall)
    rep.barrier()
    t_dev = rep.reduce_max(ms.value / 1e3, f"cuda:{local}")
    value = job_seconds_per_mock(t_dev, n_gpus, args.steps)

    # stage times: a separate pass with CUDA events around every stage
    m.set_option(2, 1)
    stage_acc = {s: [] for s in STAGES}
    for _ in range(min(args.steps, 5)):
        _, st_c, st_p = device_step(True)
        for s in STAGES:
            v = st_c.get(s, -1) if s in ("rng", "ic", "fft_i", "fft_j", "fft_k", "cic") \
                else st_p.get(s, -1)
            if v >= 0:
                stage_acc[s].append(v)
    m.set_option(2, 0)

    # end to end through the public API with host buffers
    def e2e_step():
        seed[0] += 1
        m.set_option(4, seed[0])
        m.setup_linear_pk(k, P)               # P(k) table uploaded by the next call
        m.create_dens_field_from_ic()
        n = 0
        for nexp_i, par in pops:
            cat = m.populate_tracer(*par, nexp_i)
            n += len(cat[0])
        return n

    for _ in range(args.warmup):
        e2e_step()
    m.sync()
    rep.barrier()
    L.EZmockB200_mark(m._ez, 2)
    te0 = time.perf_counter()
    n_out = 0
    for s in range(args.steps):
        n_out = e2e_step()
    L.EZmockB200_mark(m._ez, 3)
    e2e_wall = time.perf_counter() - te0
    ems = ctypes.c_double()
    L.EZmockB200_elapsed(m._ez, 2, 3, ctypes.byref(ems))
    e2e = job_seconds_per_mock(rep.reduce_max(max(ems.value / 1e3, e2e_wall), f"cuda:{local}"),
                               n_gpus, args.steps)
    h2d = 3 * pk_trim_len(k, cfg.Ng, cfg.Lbox) * 8
    d2h = 6 * n_out * b

    peak, peak_kind = read_peak()
    algo = algorithmic_bytes(cfg.Ng, b)
    med = {s: statistics.median(v) for s, v in stage_acc.items() if v}
    stages = {s: {"ms": round(med[s], 4),
                  "GB/s": round(algo[s] / (med[s] * 1e-3) / 1e9, 1) if s in algo else None}
              for s in med}
    dom = max((s for s in algo if s in med), key=lambda s: med[s])
    achieved = algo[dom] / (med[dom] * 1e-3) / 1e9
    traffic = read_traffic(cfg.name).get(dom)
    roof = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "traffic": traffic, "algorithmic_bytes": algo[dom]}
    whole = survey_bytes(cfg, b, ntr)
    mock_roof = {"bytes": whole, "achieved_GBs": round(whole / value / 1e9, 1),
                 "frac": round(whole / value / 1e9 / peak, 4)}
    return {"value": value, "ms_per_step": t_dev * 1e3 / args.steps, "ntracer": ntr,
            "e2e": {"value": e2e, "unit": "s/mock", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches, "roofline": roof, "mock_roofline": mock_roof,
            "stages": stages, "wall_s_per_mock": wall / args.steps}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="single512")
    ap.add_argument("--rng", type=int, default=None, help="0 MRG32k3a, 1 MT19937")
    ap.add_argument("--prec", type=int, default=32)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-multi1024", action="store_true",
                    help="skip the 1024^3 three-population sub-measurement")
    args = ap.parse_args()

    from ezmock_b200.workloads import CONFIGS, bbks_pk
    cfg = CONFIGS[args.workload]
    if args.rng is not None:
        cfg.rng = args.rng
    k, P = bbks_pk()
    from ezmock_b200.replicas import Replicas, rank_env, rank_seed
    rank, world, local = rank_env()
    n_gpus = max(world, 1)
    b = 4 if args.prec == 32 else 8
    config = config_of(cfg, n_gpus, b)

    if args.impl == "reference":
        if rank != 0:
            return 0
        try:
            cb = cpu_reference(cfg, k, P, args.steps, args.warmup)
        except Exception as e:             # the reference build is missing
            print(json.dumps({"impl": "reference", "unavailable": f"reference build: {e}"}))
            return 0
        v = cb["value"]
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": "s/mock",
            "n_gpus": n_gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.prec == 32 else "f64",
            "data": "synthetic (BBKS P(k), sigma_8 = 0.81)", "config": config,
            "cpu_baseline": dict(cb, unit="s/mock", kind="reference"),
            "e2e": {"value": v, "unit": "s/mock", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}))
        return 0

    if world > 1:
        import torch
        torch.cuda.set_device(local)
    rep = Replicas(world, "nccl")

    from ezmock_b200 import EZmock
    m = EZmock(Lbox=cfg.Lbox, Ngrid=cfg.Ng, rng=cfg.rng, seed=rank_seed(rank), prec=args.prec)
    L = m._L
    m.set_option(3, local)            # device
    m.eval_growth_params(cfg.z, cfg.omega_m)
    m.setup_linear_pk(k, P)
    clk = ClockSampler(local)
    clk.start()
    res = measure(cfg, args, m, L, k, P, rep, local, n_gpus, rank_seed(rank), clk)
    del m

    sub = None
    if args.workload == "single512" and not args.no_multi1024 and args.prec == 32:
        # the 1024^3 mock with three populations of one field, measured the
        # same way (fewer steps), as a sub-object of the same line
        c2 = CONFIGS["multi1024"]
        a2 = argparse.Namespace(**vars(args))
        a2.steps, a2.warmup = min(args.steps, 5), min(args.warmup, 3)
        m2 = EZmock(Lbox=c2.Lbox, Ngrid=c2.Ng, rng=c2.rng, seed=rank_seed(rank) + 7919,
                    prec=args.prec)
        m2.set_option(3, local)
        m2.eval_growth_params(c2.z, c2.omega_m)
        m2.setup_linear_pk(k, P)
        r2 = measure(c2, a2, m2, m2._L, k, P, rep, local, n_gpus, rank_seed(rank) + 7919, None)
        del m2
        sub = dict(r2, metric="s/mock at 1024^3 (FP32, three populations of one field)",
                   unit="s/mock", steps=a2.steps, warmup=a2.warmup,
                   config=config_of(c2, n_gpus, b))
        if rank == 0 and n_gpus == 1 and not args.no_cpu_baseline:
            try:
                cb2 = cpu_reference(c2, k, P, 3, 1, budget_s=30.0)
                sub["cpu_baseline"] = dict(cb2, unit="s/mock", kind="reference")
            except Exception as e:
                sub["cpu_baseline"] = {"value": None, "sample": f"unavailable: {e}"}
    # the sampler stops after every timed region
    clocks = clk.stop()

    line = {
        "metric": METRIC, "value": res["value"], "unit": "s/mock", "n_gpus": n_gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if args.prec == 32 else "f64",
        "data": "synthetic (BBKS P(k), sigma_8 = 0.81)", "config": config,
        "ntracer": res["ntracer"], "e2e": res["e2e"], "gpu_launches": res["gpu_launches"],
        "roofline": res["roofline"], "mock_roofline": res["mock_roofline"],
        "stages": res["stages"], "clocks": clocks, "wall_s_per_mock": res["wall_s_per_mock"],
    }
    if sub is not None:
        line["multi1024"] = sub
    if rank == 0 and n_gpus == 1 and not args.no_cpu_baseline:
        try:
            cb = cpu_reference(cfg, k, P, 3, 1, budget_s=60.0)
            line["cpu_baseline"] = dict(cb, unit="s/mock", kind="reference")
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unit": "s/mock", "cores": None,
                                    "kind": "reference", "sample": f"unavailable: {e}"}
    if rank == 0:
        print(json.dumps(line))
    rep.barrier()
    rep.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())

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


def cpu_reference(cfg, k, P, steps, warmup, allow_scale=True):
    """The reference's libEZmock (oracle/_ref, OpenMP, all host threads) on the
    workload; returns (s/mock, sample description, threads)."""
    from oracle.pyoracle import RefLib
    R = RefLib(32, nthread=0)
    nthreads = os.cpu_count()

    def one(Ng, Lbox, seed):
        m = R.new(Lbox, Ng, cfg.rng, seed)
        m.eval_growth(cfg.z, cfg.omega_m)
        m.setup_pk(k, P)
        t0 = time.perf_counter()
        m.create()
        for n_t, *par in cfg.population_list():
            m.populate(par, int(round(n_t * Lbox ** 3)))
        return time.perf_counter() - t0

    # a 256^3 probe decides whether full-size steps fit in a few minutes
    ng_s = cfg.Ng // 2
    t_small = one(ng_s, cfg.Lbox / 2, 1)
    est = t_small * 8 * math.log(cfg.Ng ** 3) / math.log(ng_s ** 3)
    if est * (steps + min(warmup, 1)) < 240 or not allow_scale:
        for w in range(min(warmup, 1)):
            one(cfg.Ng, cfg.Lbox, 1000 + w)
        ts = [one(cfg.Ng, cfg.Lbox, 1 + s) for s in range(steps)]
        return (statistics.median(ts), f"{steps} full {cfg.Ng}^3 mocks (median), "
                f"{nthreads} OpenMP threads", nthreads)
    ts = [one(ng_s, cfg.Lbox / 2, 1 + s) for s in range(steps)]
    scale = 8 * math.log(cfg.Ng ** 3) / math.log(ng_s ** 3)
    return (statistics.median(ts) * scale,
            f"{steps} mocks at {ng_s}^3 (median) x {scale:.2f} (N log N scaling to "
            f"{cfg.Ng}^3), {nthreads} OpenMP threads", nthreads)


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
    args = ap.parse_args()

    from ezmock_b200.workloads import CONFIGS, bbks_pk
    cfg = CONFIGS[args.workload]
    if args.rng is not None:
        cfg.rng = args.rng
    k, P = bbks_pk()
    from ezmock_b200.replicas import Replicas, job_seconds_per_mock, rank_env, rank_seed
    rank, world, local = rank_env()
    n_gpus = max(world, 1)

    if args.impl == "reference":
        if rank != 0:
            return 0
        try:
            v, sample, cores = cpu_reference(cfg, k, P, args.steps, args.warmup)
        except Exception as e:             # the reference build is missing
            print(json.dumps({"impl": "reference", "unavailable": f"reference build: {e}"}))
            return 0
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": "s/mock",
            "n_gpus": n_gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic BBKS P(k)",
            "config": {"workload": workload_desc(cfg), "Ngrid": cfg.Ng, "Lbox": cfg.Lbox},
            "cpu_baseline": {"value": v, "unit": "s/mock", "cores": cores, "kind": "reference",
                             "sample": sample + "; FFT: project CPU FFT (FFTW3 not installed)"},
            "e2e": {"value": v, "unit": "s/mock", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}))
        return 0

    if world > 1:
        import torch
        torch.cuda.set_device(local)
    rep = Replicas(world, "nccl")

    from ezmock_b200 import EZmock
    m = EZmock(Lbox=cfg.Lbox, Ngrid=cfg.Ng, rng=cfg.rng, seed=rank_seed(rank),
               prec=args.prec)
    L = m._L
    m.set_option(3, local)            # device
    m.set_option(2, 1)                # stage timings
    m.eval_growth_params(cfg.z, cfg.omega_m)
    m.setup_linear_pk(k, P)
    # one or more populations of the same field: (nexp, [rho_c, rho_exp, pdf_base, sigma_v])
    pops = [(int(round(n_t * cfg.Lbox ** 3)), par) for n_t, *par in cfg.population_list()]
    b = 4 if args.prec == 32 else 8

    def barrier():
        rep.barrier()

    def reduce_max(x):
        return rep.reduce_max(x, f"cuda:{local}")

    seed = [rank_seed(rank)]

    def device_step():
        seed[0] += 1
        m.set_option(4, seed[0])
        m.create_dens_field_from_ic()
        stage_c = m.stage_times()
        n, stage_p = 0, {}
        for nexp_i, par in pops:
            n += m.populate_device(*par, nexp_i)
            for s_, v_ in m.stage_times().items():
                if v_ >= 0:
                    stage_p[s_] = stage_p.get(s_, 0.0) + v_
        return n, stage_c, stage_p

    clk = ClockSampler(local)
    clk.start()
    for _ in range(args.warmup):
        device_step()
    m.sync()
    barrier()
    l0 = L.EZmockB200_launch_count()
    L.EZmockB200_mark(m._ez, 0)
    t0 = time.perf_counter()
    stage_acc = {s: [] for s in STAGES}
    ntr = 0
    for _ in range(args.steps):
        ntr, st_c, st_p = device_step()
        for s in STAGES:
            v = st_p.get(s, -1) if s not in ("rng", "ic", "fft_i", "fft_j", "fft_k", "cic") else st_c[s]
            if v >= 0:
                stage_acc[s].append(v)
    L.EZmockB200_mark(m._ez, 1)
    ms = ctypes.c_double()
    L.EZmockB200_elapsed(m._ez, 0, 1, ctypes.byref(ms))
    wall = time.perf_counter() - t0
    launches = L.EZmockB200_launch_count() - l0
    clk.mark(t0, t0 + wall)
    barrier()
    t_dev = reduce_max(ms.value / 1e3)
    value = job_seconds_per_mock(t_dev, n_gpus, args.steps)

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

    # untimed warm-up of the host path (the catalogue's host blocks are
    # prepared after each copy-out; the device steps above used none)
    for _ in range(args.warmup):
        e2e_step()
    m.sync()
    barrier()
    L.EZmockB200_mark(m._ez, 2)
    te0 = time.perf_counter()
    n_out = 0
    for s in range(args.steps):
        n_out = e2e_step()
    L.EZmockB200_mark(m._ez, 3)
    e2e_wall = time.perf_counter() - te0
    ems = ctypes.c_double()
    L.EZmockB200_elapsed(m._ez, 2, 3, ctypes.byref(ems))
    e2e = job_seconds_per_mock(reduce_max(max(ems.value / 1e3, e2e_wall)), n_gpus, args.steps)
    # the sampler stops after every timed region
    clocks = clk.stop()
    h2d = 3 * pk_trim_len(k, cfg.Ng, cfg.Lbox) * 8
    d2h = 6 * n_out * b

    # roofline of the dominant kernel
    peak, peak_kind = read_peak()
    algo = algorithmic_bytes(cfg.Ng, b)
    med = {s: statistics.median(v) for s, v in stage_acc.items() if v}
    stages_gbs = {s: {"ms": round(med[s], 4),
                      "GB/s": round(algo[s] / (med[s] * 1e-3) / 1e9, 1) if s in algo else None}
                  for s in med}
    dom = max((s for s in algo if s in med), key=lambda s: med[s])
    achieved = algo[dom] / (med[dom] * 1e-3) / 1e9
    traffic = read_traffic(cfg.name).get(dom)
    roof = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "traffic": traffic, "algorithmic_bytes": algo[dom]}

    line = {
        "metric": METRIC, "value": value, "unit": "s/mock", "n_gpus": n_gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_dev * 1e3 / args.steps,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if args.prec == 32 else "f64",
        "data": "synthetic (BBKS P(k), sigma_8 = 0.81)",
        "config": {"workload": workload_desc(cfg), "Ngrid": cfg.Ng, "Lbox": cfg.Lbox,
                   "nexp": pops[0][0] if len(pops) == 1 else [p_[0] for p_ in pops],
                   "ntracer": ntr, "parallelism": f"replicas x{n_gpus}",
                   "l2": f"inputs larger than L2 (psi {3 * cfg.Ng ** 3 * b / 1e9:.1f} GB, "
                         f"spectra {3 * cfg.Ng ** 2 * (cfg.Ng // 2 + 1) * 2 * b / 1e9:.1f} GB "
                         "per mock)"},
        "e2e": {"value": e2e, "unit": "s/mock", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches, "roofline": roof, "stages": stages_gbs,
        "clocks": clocks, "wall_s_per_mock": wall / args.steps,
    }
    if rank == 0 and n_gpus == 1 and not args.no_cpu_baseline:
        try:
            v, sample, cores = cpu_reference(cfg, k, P, 1, 0)
            line["cpu_baseline"] = {"value": v, "unit": "s/mock", "cores": cores,
                                    "kind": "reference",
                                    "sample": sample + "; FFT: project CPU FFT "
                                    "(FFTW3 not installed)"}
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

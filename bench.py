"""Benchmark of the batched Cahn-Hilliard stepper (one JSON line on rank 0).

Workload: the batched ensemble -- 512 independent particles, grid sizes drawn
uniformly from {128, 192, 256, 384, 512}^2, R ~ U(0.25, 0.42) n, w = 2,
P ~ U(0.5, 2) x 5, chi ~ U(0.5, 1.5) x 0.5, kappa ~ U(0.5, 2) x 2, M0 = 1,
c0 = 0.5 + mean-free U(-0.01, 0.01) inside the particle (seed 0 + i), dt = 0.01,
mixed precision (FP64 state and reductions, FP32 flux transforms).  A "step"
is one time step of every particle (history row + stabilised update).

  value   pt-steps/s with the fields resident in HBM (esc_batch_run_device)
  e2e     the same through esc_batch_run with pinned host buffers: the H2D copy
          of c0 and the D2H copy of c and of the history are inside the timing
  fp64    the plain FP64 drop-in on the same workload (the 5x target's denominator)
  adjoint gradient of 1/2|c_T - c_target|^2 + 1e-3 F[c_T] w.r.t. c0 and (P, chi, kappa, M0)
          through 2000 mixed-precision steps at 256^2 and 512^2 (checkpoints every 45):
          the reverse sweep (recompute + adjoint) per step over the forward step
  batched_gradients  64 particles at 512^2, dL/d(P, chi, kappa, M0) through 1000 steps in
          one esc_batch_adjoint call: gradient throughput and cost against a forward run
  large_grids  the single-grid configurations (1024^2 and 4096^2, 10,000 steps): FP64
          drop-in and mixed rates side by side and the mixed error against FP64
  accuracy  after 2000 steps of the ensemble: mixed precision against the FP64
          drop-in per instance (max and L2 error of c, energy, mass drift), beside
          the FP64 drop-in restarted from c0 perturbed by 1e-8 relative, which
          measures how strongly the dynamics amplify any perturbation
  coupled  the coupled c-phi model of the reference's 3-D program at its own input
          (256^3, FP64): pt-steps/s, per-kernel times and HBM fractions, and the CPU
          oracle on a 64^3 sample (--coupled-only runs this leg alone)

The working set (1.7 GB mixed, 2.6 GB FP64) is far larger than the 126 MB L2,
so no flush is needed between steps.  Under torchrun every rank runs its own
ensemble (weak scaling, no collective on the data path); timings are the max
over ranks.  `--impl reference` times the CPU oracle (the reference's Julia
path is not runnable here) on a bounded sample of the same workload.
"""
from __future__ import annotations

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
PKG = os.path.join(ROOT, "embedded-spinodal-core-shell-julia_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "pt-steps/s batched FP32 vs plain FP64 (1 B200, <=1e-5 err); adjoint/forward time"
UNIT = "pt-steps/s"
SIZES = (128, 192, 256, 384, 512)
COUNT = 512
DT = 0.01
B_ALG_PER_PASS = 16.0   # bytes per grid point per pass: 8 B read + 8 B write of a complex FP32 field
B_ALG_PER_STEP = 64.0   # four passes per step


def ensemble(count=COUNT, seed_base=0, sizes=SIZES, rng_seed=0):
    """Seeded synthetic ensemble: returns (n list, phi list, c0 list, params list)."""
    import esc
    from esc import fields
    rng = np.random.default_rng(rng_seed)
    ns, phis, c0s, ps = [], [], [], []
    for i in range(count):
        n = int(rng.choice(sizes))
        R = rng.uniform(0.25, 0.42) * n
        phi = fields.particle_disc(n, spacing=1.0, radius=R, width=2.0)
        ns.append(n)
        phis.append(phi)
        c0s.append(fields.interior_noise(phi, seed_base + i))
        ps.append(esc.Parameters(P=5.0 * rng.uniform(0.5, 2.0), chi=0.5 * rng.uniform(0.5, 1.5),
                                 kappa=2.0 * rng.uniform(0.5, 2.0)))
    return ns, phis, c0s, ps


def read_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clock, power and throttle-reason sampling during the timed region.

    Reads NVML in a thread of this process (the counters `nvidia-smi --query-gpu` prints). A
    separate nvidia-smi process was measured to stall the GPU's work now and then (one timed
    region in four 9-45 % slow, SM clock at its maximum), the in-process sampler never did; the
    nvidia-smi process remains the fallback when NVML cannot be loaded."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
               ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4))

    def __init__(self, index: int, period_s: float = 0.025):
        self.index = index
        self.period_s = period_s
        self.proc = None
        self.path = None
        self.thread = None
        self.samples = []
        self.source = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            if not uuid.startswith("GPU-"):
                uuid = "GPU-" + uuid
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _nvml_sample(self):
        nv, h = self._nv, self._h
        try:
            reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        except Exception:
            reasons = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
        self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                             float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)),
                             nv.nvmlDeviceGetPowerUsage(h) / 1000.0, int(reasons)))

    def _nvml_loop(self):
        while not self._stop.wait(self.period_s):
            try:
                self._nvml_sample()
            except Exception:
                return

    def __enter__(self):
        try:
            self._nv, self._h = self._nvml_handle()
            self._nvml_sample()
            self._stop = threading.Event()
            self.thread = threading.Thread(target=self._nvml_loop, daemon=True)
            self.thread.start()
            self.source = "nvml"
            return self
        except Exception:
            self.thread = None
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            # nvidia-smi's start-up (driver initialisation over every GPU of the node) can
            # stall work on this GPU: wait for its first sample before anything is timed
            t_end = time.time() + 10.0
            while time.time() < t_end and self.proc.poll() is None:
                with open(self.path) as f:
                    if f.readline():
                        break
                time.sleep(0.02)
            time.sleep(0.3)
            self.source = "nvidia-smi"
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.thread is not None:
            self._stop.set()
            self.thread.join()
            try:
                self._nvml_sample()
                self._nv.nvmlShutdown()
            except Exception:
                pass
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def _read_smi(self):
        if not self.path or not os.path.exists(self.path):
            return
        names = [nm for nm, _ in self.REASONS]
        bits = dict(self.REASONS)
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm, mx = float(parts[0]), float(parts[1])
            except ValueError:
                continue
            try:
                pw = float(parts[2])
            except ValueError:
                pw = None
            mask = 0
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    mask |= bits[nm]
            self.samples.append((sm, mx, pw, mask))
        os.unlink(self.path)
        self.path = None

    def summary(self):
        self._read_smi()
        if not self.samples:
            return None
        sm = [s[0] for s in self.samples]
        pw = [s[2] for s in self.samples if s[2] is not None]
        reasons = sorted(nm for nm, bit in self.REASONS if any(s[3] & bit for s in self.samples))
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(s[1] for s in self.samples),
                "reasons": reasons, "power_w": statistics.median(pw) if pw else None,
                "samples": len(sm), "source": self.source}


def cpu_oracle_rate(ns, phis, c0s, ps, steps, workers):
    """pt-steps/s of the CPU oracle (literal 17-FFT restatement) on the given sample."""
    from oracle import core_shell_oracle as orc
    orc.set_workers(workers)
    t0 = time.perf_counter()
    pts = 0
    for n, phi, c0, p in zip(ns, phis, c0s, ps):
        op = orc.Parameters(A=p.A, B=p.B, chi=p.chi, P=p.P, ca=p.ca, cb=p.cb, cc=p.cc, kappa=p.kappa,
                            mobility=p.mobility, Q=p.Q)
        grid = orc.make_grid(n, 1.0)
        shape = orc.geometry(phi, op)
        c = c0.copy()
        for _ in range(steps):   # one step of run_simulation: transport_rate + energy + step
            orc.transport_rate(c, shape, grid, op)
            orc.energy(c, shape, grid, op)
            c = orc.step(c, shape, grid, op, DT)
        pts += n * n * steps
    return pts / (time.perf_counter() - t0)


def sample_subset(ns, k_per_size=1):
    out, seen = [], {}
    for i, n in enumerate(ns):
        if seen.get(n, 0) < k_per_size:
            out.append(i)
            seen[n] = seen.get(n, 0) + 1
    return out


def ensemble_config(count, sizes, pts, world):
    """The `config` both arms print for the batched-ensemble workload."""
    return {"workload": f"batched ensemble: {count} particles per GPU, n in {list(sizes)}, "
                        f"{pts} points, dt=0.01, mixed precision",
            "global_batch": count * world, "l2": "working set 1.7 GB >> 126 MB L2; no flush"}


def run_reference(args, world, rank):
    """CPU oracle on a bounded sample of the ensemble; rank 0 only.  The line carries the
    ensemble's own config (the rate is per point-step, so a sample of the workload measures it);
    `cpu_baseline.sample` names the sample."""
    if rank != 0:
        return 0
    sizes = [int(x) for x in args.sizes.split(",")]
    ns, phis, c0s, ps = ensemble(count=args.count, seed_base=0, rng_seed=0, sizes=sizes)
    full_pts = sum(n * n for n in ns)
    idx = sample_subset(ns)          # one particle of each grid size
    sub = [ns[i] for i in idx], [phis[i] for i in idx], [c0s[i] for i in idx], [ps[i] for i in idx]
    workers = os.cpu_count() or 1
    pts = sum(n * n for n in sub[0])
    cpu_oracle_rate(*[x[:1] for x in sub], steps=max(1, args.warmup // 3), workers=workers)
    t0 = time.perf_counter()
    rate = cpu_oracle_rate(*sub, steps=args.steps, workers=workers)
    wall = time.perf_counter() - t0
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * wall / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": ensemble_config(args.count, sizes, full_pts, world),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": workers, "kind": "port",
                         "sample": f"{len(idx)} particles of the ensemble, one of each size "
                                   f"{sorted(set(sub[0]))} ({pts} points) x {args.steps} steps; "
                                   "NumPy/scipy.fft restatement of core_shell.jl (Julia absent)"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def error_stats(cs, hs, ref_cs, ref_hs):
    """Per-instance errors of fields cs / histories hs against the reference run."""
    e_max = np.array([np.max(np.abs(a - b)) / np.max(np.abs(b)) for a, b in zip(cs, ref_cs)])
    e_l2 = np.array([np.linalg.norm(a - b) / np.linalg.norm(b) for a, b in zip(cs, ref_cs)])
    e_F = np.array([np.max(np.abs(h[2] - r[2]) / np.abs(r[2])) for h, r in zip(hs, ref_hs)])
    mass = np.array([np.max(np.abs(h[1] - h[1][0])) for h in hs])
    return {"max_rel_err_c": float(e_max.max()), "p50_max_rel_err_c": float(np.median(e_max)),
            "p90_max_rel_err_c": float(np.quantile(e_max, 0.9)),
            "frac_instances_le_1e-5": float(np.mean(e_max <= 1e-5)),
            "l2_rel_err_c_max": float(e_l2.max()), "energy_rel_err_max": float(e_F.max()),
            "mass_drift_max": float(mass.max())}


def accuracy_block(phis, ps, c0s, steps):
    """Mixed precision against the FP64 drop-in over the whole ensemble after
    `steps` steps (the configuration's 2000), next to the FP64 drop-in started
    from c0 perturbed by 1e-8 relative: spinodal decomposition amplifies any
    perturbation, and the second row shows how far a 1e-8 change of the input
    alone moves c (the conditioning of the problem, not an arithmetic error)."""
    import torch
    import esc

    def run(prec, cs0):
        b = esc.Batch(phis, params=ps, precision=prec)
        work = [torch.from_numpy(c).cuda() for c in cs0]
        hist = torch.zeros(len(cs0) * (steps + 1) * 6, dtype=torch.float64, device="cuda")
        b.run_device([w.data_ptr() for w in work], steps, DT, hist.data_ptr())
        torch.cuda.synchronize()
        out = [w.cpu().numpy() for w in work]
        h = hist.cpu().numpy().reshape(len(cs0), 6, steps + 1)
        b.close()
        return out, h

    ref_c, ref_h = run("fp64", c0s)
    mix_c, mix_h = run("mixed", c0s)
    rng = np.random.default_rng(12345)
    pert = [c * (1.0 + 1e-8 * (2.0 * rng.random(c.shape) - 1.0)) for c in c0s]
    per_c, per_h = run("fp64", pert)
    return {"steps": steps, "instances": len(c0s),
            "mixed_vs_fp64": error_stats(mix_c, mix_h, ref_c, ref_h),
            "fp64_from_c0_perturbed_1e-8_vs_fp64": error_stats(per_c, per_h, ref_c, ref_h),
            "fp64_mass_drift_max": float(max(np.max(np.abs(h[1] - h[1][0])) for h in ref_h))}


def single_grid_block(name, phi, c0, steps, peak_gbs):
    """One large grid through the single-particle context: the FP64 drop-in and
    the mixed precision side by side (device-resident, CUDA-event timed), with
    the mixed result's error against the FP64 one (c, energy, mass drift)."""
    import torch
    import esc
    n = phi.shape[0]
    # a dedicated stream: the queued run and the events bracketing it share it
    # (a null handle would leave the context on its own stream, outside the events)
    stream = torch.cuda.Stream()
    rates, out = {}, {}
    for prec in ("fp64", "mixed"):
        with esc.Context(phi, precision=prec) as ctx:
            ctx.set_stream(stream.cuda_stream)
            d = torch.from_numpy(c0).cuda()
            h = torch.zeros(6 * (steps + 1), dtype=torch.float64, device="cuda")
            ctx.run_device(d.data_ptr(), 3, DT)
            d.copy_(torch.from_numpy(c0))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.run_device_async(d.data_ptr(), steps, DT, h.data_ptr())
            e1.record(stream)
            ctx.wait()
            torch.cuda.synchronize()
            rates[prec] = n * n * steps / (e0.elapsed_time(e1) / 1000.0)
            out[prec] = (d.cpu().numpy(), h.cpu().numpy().reshape(6, steps + 1))
    err = error_stats([out["mixed"][0]], [out["mixed"][1]], [out["fp64"][0]], [out["fp64"][1]])
    err.pop("p50_max_rel_err_c")
    err.pop("p90_max_rel_err_c")
    return {"config": name, "n": n, "steps": steps, "fp64_pt_steps_per_s": rates["fp64"],
            "mixed_pt_steps_per_s": rates["mixed"], "mixed_over_fp64": rates["mixed"] / rates["fp64"],
            "mixed_step_frac_of_hbm_roofline": rates["mixed"] * B_ALG_PER_STEP / (peak_gbs * 1e9),
            "mixed_vs_fp64": err,
            "fp64_mass_drift": float(np.max(np.abs(out["fp64"][1][1] - out["fp64"][1][1][0])))}


def large_grid_configs(peak_gbs):
    """The single-grid configurations: the default example of core_shell.jl (256^2, disc R = 70,
    w = 4, interior noise, 1000 steps), the 1024^2 disc (R = 400, w = 2, c0 = 0.5 +
    U(-0.01, 0.01) over the whole field, seed 1) and the 4096^2 ellipse (semi-axes
    1600 along x and 1200 along y, w = 2, c0 = 0.5 + mean-free U(-0.01, 0.01)
    inside the particle, seed 5), 10,000 steps each, dt = 0.01."""
    from esc import fields
    phi2 = fields.particle_disc(1024, radius=400.0, width=2.0)
    c02 = fields.whole_field_noise(1024, seed=1)
    phi5 = fields.particle_ellipse(4096, a=1600.0, b=1200.0, width=2.0)
    c05 = fields.interior_noise(phi5, 5)
    phi0 = fields.particle_disc(256, radius=70.0, width=4.0)
    c00 = fields.interior_noise(phi0, 5749)
    return [single_grid_block("256^2 default example (disc R=70, w=4), 1000 steps", phi0, c00, 1000, peak_gbs),
            single_grid_block("1024^2 disc R=400, 10000 steps", phi2, c02, 10000, peak_gbs),
            single_grid_block("4096^2 ellipse 1600x1200, 10000 steps", phi5, c05, 10000, peak_gbs)]


def coupled_kernel_bytes(nx, ny, nz):
    """Bytes each of the twelve stages of a coupled step must move (FP64: real fields 8 B
    per point, half spectra 16 B per mode, nx*ny*(nz/2+1) modes), in launch order."""
    n3 = nx * ny * nz
    nk = nx * ny * (nz // 2 + 1)
    return [16 * n3 + 32 * nk, 64 * nk, 96 * nk, 32 * nk, 16 * nk + 24 * n3, 32 * n3, 32 * n3,
            8 * n3 + 16 * nk, 32 * nk, 96 * nk, 64 * nk, 32 * nk + 24 * n3]


def coupled_block(peak_gbs, steps=20, warmup=3, cpu=True):
    """The coupled c-phi model of the reference's 3-D program at its own input size
    (original/2023-3d/InputParams: 256^3, dx = 1, dt = 0.01, R = 70, c_0 = 0.5, noise 0.05,
    the InputParams constants), FP64, fields resident in HBM (esc_cphi_run_device), CUDA
    events around `steps` steps on the context's stream; per-kernel times of one step
    (esc_cphi_profile) with each kernel's bytes and fraction of the HBM peak; and the
    CPU oracle (NumPy/scipy.fft restatement) on a 64^3 sample."""
    import torch
    from esc import coupled
    shape = (256, 256, 256)
    c0, phi0 = coupled.initial_fields(*shape, 70.0)
    n3 = int(np.prod(shape))
    stream = torch.cuda.Stream()
    with coupled.Coupled(shape) as ctx:
        ctx.set_stream(stream.cuda_stream)
        dc, dp = torch.from_numpy(c0).cuda(), torch.from_numpy(phi0).cuda()
        torch.cuda.synchronize()
        ctx.run_device(dc.data_ptr(), dp.data_ptr(), warmup, DT)
        dc.copy_(torch.from_numpy(c0))
        dp.copy_(torch.from_numpy(phi0))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        done, reason = ctx.run_device(dc.data_ptr(), dp.data_ptr(), steps, DT)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        prof = ctx.profile(steps=3)
    rate = n3 * steps / (ms / 1000.0)
    nbytes = coupled_kernel_bytes(*shape)
    kernels = []
    for (name, kms), b in zip(prof.items(), nbytes):
        kernels.append({"kernel": name, "ms": round(kms, 4), "bytes": b,
                        "frac_of_hbm_peak": b / (kms / 1000.0) / (peak_gbs * 1e9)})
    dom = max(kernels, key=lambda k: k["ms"])
    step_bytes = sum(nbytes) / n3
    out = {"workload": "coupled c-phi 256^3 (original/2023-3d InputParams), FP64, dt=0.01",
           "steps": steps, "steps_done": done, "stop_reason": reason, "pt_steps_per_s": rate,
           "ms_per_step": ms / steps, "bytes_per_pt_step": step_bytes,
           "step_frac_of_hbm_peak": rate * step_bytes / (peak_gbs * 1e9),
           "dominant_kernel": dom, "kernels": kernels}
    if cpu:
        from oracle import coupled_oracle as cpl
        import scipy.fft as sfft
        cs, ps_ = cpl.initial_fields(64, 64, 64, 17.5)
        workers = os.cpu_count() or 1
        with sfft.set_workers(workers):
            cpl.run(cs, ps_, cpl.CoupledParameters(), DT, 1)
            t0 = time.perf_counter()
            cpl.run(cs, ps_, cpl.CoupledParameters(), DT, 5)
            tc = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": 64 ** 3 * 5 / tc, "unit": UNIT, "cores": workers, "kind": "port",
                               "sample": "64^3 x 5 steps of the NumPy/scipy.fft restatement of the 3-D loop"}
    return out


def batched_gradient_block(count=64, n=512, steps=1000):
    """Batched parameter-fit gradients: `count` particles at n^2 (disc R ~ U(0.25, 0.42) n,
    w = 2, sampled P, chi, kappa as in the ensemble), loss 1/2 |c_T - c_target|^2 + 1e-3 F[c_T]
    with c_target a forward run at (1.1 P, 0.9 chi), gradients w.r.t. (P, chi, kappa, M0)
    through `steps` steps for all particles in one esc_batch_adjoint call (mixed-precision
    forward and recompute, FP64 adjoint).  Reports the gradient throughput (and as a fraction
    of the 64 B per pt-step roofline), its cost against a forward run of the same batch, and
    the error of the gradients against the same call with an FP64 forward pass."""
    import esc
    ns, phis, c0s, ps = ensemble(count=count, seed_base=1000, sizes=(n,), rng_seed=7)
    pts = [esc.Parameters(A=p.A, B=p.B, chi=p.chi * 0.9, P=p.P * 1.1, ca=p.ca, cb=p.cb, cc=p.cc,
                          kappa=p.kappa, mobility=p.mobility, Q=p.Q) for p in ps]
    with esc.Batch(phis, params=pts, precision="mixed") as bt:
        targets, _, _ = bt.run(c0s, dt=DT, steps=steps, with_history=False)
    with esc.Batch(phis, params=ps, precision="mixed") as b:
        # warm-up with the timed shapes: the step graphs of a gradient call are built once per
        # (segment length, buffer) and reused, as in the repeated calls of a parameter fit
        b.run(c0s, dt=DT, steps=steps, with_history=False)
        b.adjoint(c0s, targets, dt=DT, steps=steps, lambda_F=1e-3, with_field_gradients=False)
        t0 = time.perf_counter()
        b.run(c0s, dt=DT, steps=steps, with_history=False)
        t_fwd = time.perf_counter() - t0
        t0 = time.perf_counter()
        L, _, th = b.adjoint(c0s, targets, dt=DT, steps=steps, lambda_F=1e-3, with_field_gradients=False)
        t_adj = time.perf_counter() - t0
    # the same gradients with an FP64 forward pass and recompute (the FP64 drop-in's arithmetic)
    with esc.Batch(phis, params=ps, precision="fp64") as b64:
        L64, _, th64 = b64.adjoint(c0s, targets, dt=DT, steps=steps, lambda_F=1e-3, with_field_gradients=False)
    th, th64 = np.asarray(th), np.asarray(th64)
    rel_th = np.max(np.abs(th - th64), axis=1) / np.max(np.abs(th64), axis=1)
    rel_L = np.abs(np.asarray(L) - np.asarray(L64)) / np.abs(np.asarray(L64))
    rate = count * n * n * steps / t_adj
    return {"particles": count, "n": n, "steps": steps, "gradient_call_s": t_adj, "forward_call_s": t_fwd,
            "gradient_pt_steps_per_s": rate,
            "gradient_step_frac_of_hbm_roofline": rate * B_ALG_PER_STEP / (read_peaks()[0] * 1e9),
            "gradient_call_over_forward_call": t_adj / t_fwd,
            "vs_fp64_forward": {"dL_dtheta_rel_err_max": float(rel_th.max()),
                                "dL_dtheta_rel_err_median": float(np.median(rel_th)),
                                "L_rel_err_max": float(rel_L.max())},
            "dL_dtheta_particle0": [float(x) for x in th[0]], "L_particle0": float(L[0])}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--count", type=int, default=COUNT)
    ap.add_argument("--sizes", default=",".join(str(n) for n in SIZES),
                    help="grid sizes the particles are drawn from (a single size gives a uniform batch, "
                         "e.g. a small case for profiling)")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--accuracy-steps", type=int, default=2000)
    ap.add_argument("--no-large", action="store_true", help="skip the 1024^2 and 4096^2 single-grid runs")
    ap.add_argument("--no-coupled", action="store_true", help="skip the coupled c-phi 256^3 leg")
    ap.add_argument("--gradients-only", action="store_true",
                    help="run only the batched-gradient leg (64 x 512^2) and print its JSON object")
    ap.add_argument("--gradient-steps", type=int, default=1000)
    ap.add_argument("--default-example-only", action="store_true",
                    help="run only the 256^2 default example of core_shell.jl (1000 steps, FP64 and mixed)")
    ap.add_argument("--coupled-only", action="store_true",
                    help="run only the coupled c-phi 256^3 leg and print its JSON object")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, world, rank)

    import torch
    import esc
    torch.cuda.set_device(local)
    if args.coupled_only:
        print(json.dumps(coupled_block(read_peaks()[0], steps=args.steps, warmup=args.warmup,
                                       cpu=not args.no_cpu)), flush=True)
        return 0
    if args.default_example_only:
        from esc import fields
        phi0 = fields.particle_disc(256, radius=70.0, width=4.0)
        c00 = fields.interior_noise(phi0, 5749)
        print(json.dumps(single_grid_block("256^2 default example (disc R=70, w=4), 1000 steps", phi0, c00, 1000,
                                           read_peaks()[0])), flush=True)
        return 0
    if args.gradients_only:
        print(json.dumps(batched_gradient_block(steps=args.gradient_steps)), flush=True)
        return 0
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    sizes = tuple(int(x) for x in args.sizes.split(","))
    ns, phis, c0s, ps = ensemble(count=args.count, seed_base=rank * args.count, rng_seed=rank, sizes=sizes)
    pts = sum(n * n for n in ns)
    dc0 = [torch.from_numpy(c).cuda() for c in c0s]

    def timed_device_run(precision, steps, warmup):
        b = esc.Batch(phis, params=ps, precision=precision)
        # a dedicated (non-default) stream: the library forks its size groups from it and joins
        # them back, and the CUDA events bracketing the K steps are recorded on it
        stream = torch.cuda.Stream()
        b.set_stream(stream.cuda_stream)
        work = [c.clone() for c in dc0]
        torch.cuda.synchronize()  # the clones ran on the default stream
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        # the sampler starts before the warm-up, so that its start-up pause does not
        # leave the GPU idle between the warm-up and the timed steps
        with ClockSampler(local) as clk:
            b.run_device([w.data_ptr() for w in work], warmup, DT)
            for w, c in zip(work, dc0):
                w.copy_(c)
            torch.cuda.synchronize()
            barrier()
            torch.cuda.synchronize()
            ev0.record(stream)
            # queued without waiting: ev1 follows the join of every size group in stream
            # order, so the interval is the device's time for exactly K steps
            b.run_device_async([w.data_ptr() for w in work], steps, DT)
            ev1.record(stream)
            bads = b.wait()
            torch.cuda.synchronize()
        barrier()
        ms = ev0.elapsed_time(ev1)
        return b, work, ms, clk.summary(), bads

    # ---- mixed precision (the product path) ----
    bm, cm, ms_mixed, clocks, bads = timed_device_run("mixed", args.steps, args.warmup)
    ms_mixed = max_over_ranks(ms_mixed)
    value = world * pts * args.steps / (ms_mixed / 1000.0)
    n_groups = len(set(ns))
    # per size group: init, 4 phases per step, the final history row (3), fin, and one step-counter
    # advance per captured 32-step chunk and per remainder
    gpu_launches = n_groups * (1 + 4 * args.steps + 3 + 1 + args.steps // 32 + (1 if args.steps % 32 else 0))

    # roofline of the dominant kernel: per-phase CUDA-event timing on the same batch
    prof = bm.profile_phases(steps=5)
    best = None
    counts = {}
    for n in ns:
        counts[n] = counts.get(n, 0) + 1
    for n, cnt, msl in prof:
        for ph, m in enumerate(msl):
            if best is None or m > best[3]:
                best = (n, cnt, ph, m)
    names = ["row_a", "col_a", "row_b", "col_b"]
    peak, peak_kind = read_peaks()
    dn, dcnt, dph, dms = best
    achieved = B_ALG_PER_PASS * dn * dn * dcnt / (dms / 1000.0) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(f"{names[dph]}_{dn}")
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": f"k_{names[dph]} n={dn} x{dcnt} (mixed)",
                "peak_kind": peak_kind,
                "step_frac": value / world * B_ALG_PER_STEP / (peak * 1e9),
                "phase_ms": {f"{n}x{cnt}": [round(x, 4) for x in msl] for n, cnt, msl in prof}}
    bm_final = [w.cpu().numpy() for w in cm]
    tuned = [{k: g[k] for k in ("n", "instances", "rows", "cols")} for g in bm.describe()]
    bm.close()

    # ---- plain FP64 drop-in on the same workload ----
    fp64 = None
    max_err = None
    if not args.no_fp64:
        bf, cf, ms64, clocks64, _ = timed_device_run("fp64", args.steps, args.warmup)
        ms64 = max_over_ranks(ms64)
        v64 = world * pts * args.steps / (ms64 / 1000.0)
        f_final = [w.cpu().numpy() for w in cf]
        max_err = max(float(np.max(np.abs(a - b))) for a, b in zip(bm_final, f_final))
        fp64 = {"value": v64, "unit": UNIT, "ms_per_step": ms64 / args.steps, "speedup_mixed_over_fp64": value / v64,
                "clocks": clocks64,
                "kernel_families": [{k: g[k] for k in ("n", "rows", "cols")} for g in bf.describe()]}
        bf.close()

    # ---- end to end through esc_batch_run with pinned host buffers ----
    b = esc.Batch(phis, params=ps, precision="mixed")
    host = [torch.from_numpy(c).pin_memory() for c in c0s]
    hist = [torch.zeros(6 * (args.steps + 1), dtype=torch.float64).pin_memory() for _ in c0s]
    import ctypes
    lib = esc.load_library()
    dp = ctypes.POINTER(ctypes.c_double)
    carr = (dp * len(host))(*[ctypes.cast(h.data_ptr(), dp) for h in host])
    harr = (dp * len(hist))(*[ctypes.cast(h.data_ptr(), dp) for h in hist])
    bad = (ctypes.c_int64 * len(host))()
    lib.esc_batch_run(b._h, carr, args.warmup, DT, harr, bad)
    for h, c in zip(host, c0s):
        h.copy_(torch.from_numpy(c))
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    st = lib.esc_batch_run(b._h, carr, args.steps, DT, harr, bad)
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    b.close()
    if st not in (0, 3):
        raise RuntimeError(f"esc_batch_run failed with status {st}")
    h2d = 8 * pts
    d2h = 8 * pts + 8 * 6 * (args.steps + 1) * len(ns)
    e2e = {"value": world * pts * args.steps / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
           "note": "one esc_batch_run call of K steps: c0 H2D once, c and history D2H once (per-step share shown)"}

    # ---- adjoint / forward time (calibration workload: 256^2 and 512^2, 2000 steps) ----
    adjoint = None
    if not args.no_adjoint:
        from esc import fields
        adjoint = []
        for n in (256, 512):
            phi = fields.particle_disc(n, radius=0.35 * n, width=2.0)
            c0 = fields.interior_noise(phi, 1)
            base_p = esc.Parameters()
            pt = esc.Parameters(P=base_p.P * 1.1, chi=base_p.chi * 0.9)
            ct, _ = esc.run_simulation(c0, phi, dt=DT, steps=2000, p=pt, precision="mixed")
            with esc.Context(phi, precision="mixed") as ctx:
                ctx.run(c0, dt=DT, steps=20, with_history=False)
                ctx.adjoint(c0, ct, dt=DT, steps=2000, lambda_F=1e-3, ckpt_every=45)  # builds the step graphs
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                ctx.run(c0, dt=DT, steps=2000, with_history=False)
                tf = time.perf_counter() - t0
                t0 = time.perf_counter()
                L, g, th = ctx.adjoint(c0, ct, dt=DT, steps=2000, lambda_F=1e-3, ckpt_every=45)
                ta = time.perf_counter() - t0
            adjoint.append({"n": n, "steps": 2000, "ckpt_every": 45, "forward_s": tf, "adjoint_call_s": ta,
                            "reverse_step_over_forward_step": (ta - tf) / tf,
                            "adjoint_call_over_forward": ta / tf,
                            "dL_dtheta": [float(x) for x in th]})

    accuracy = None
    if not args.no_accuracy:
        accuracy = accuracy_block(phis, ps, c0s, args.accuracy_steps)
    large = None
    if not args.no_large:
        large = large_grid_configs(peak)
    batched_grad = None
    if not args.no_adjoint:
        batched_grad = batched_gradient_block()
    coupled_leg = None
    if not args.no_coupled:
        coupled_leg = coupled_block(peak, cpu=(rank == 0 and world == 1 and not args.no_cpu))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        idx = sample_subset(ns)
        sub = ([ns[i] for i in idx], [phis[i] for i in idx], [c0s[i] for i in idx], [ps[i] for i in idx])
        workers = os.cpu_count() or 1
        csteps = 3
        rate = cpu_oracle_rate(*sub, steps=csteps, workers=workers)
        cpu = {"value": rate, "unit": UNIT, "cores": workers, "kind": "port",
               "sample": f"{len(idx)} particles (one per size, {sum(ns[i] ** 2 for i in idx)} points) x {csteps} "
                         "steps of the NumPy/scipy.fft restatement of core_shell.jl (Julia absent)"}

    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    mix_acc = (accuracy or {}).get("mixed_vs_fp64") or {}
    targets = {  # the north-star targets next to what this run measured
        "step_frac_of_hbm_roofline": roofline["step_frac"], "step_frac_target": 0.60,
        "mixed_over_fp64": (value / fp64["value"]) if fp64 else None, "mixed_over_fp64_target": 5.0,
        "frac_instances_within_1e-5": mix_acc.get("frac_instances_le_1e-5"), "within_1e-5_target": 1.0,
    }
    line = {
        "metric": METRIC, "value": value, "unit": UNIT,
        "fp64_dropin_value": fp64["value"] if fp64 else None, "targets": targets,
        "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_mixed / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 state / f32 flux transforms",
        "data": "synthetic",
        "config": ensemble_config(args.count, sizes, pts, world),
        "e2e": e2e, "gpu_launches": gpu_launches, "roofline": roofline, "cpu_baseline": cpu,
        "fp64_dropin": fp64, "max_abs_err_vs_fp64": max_err, "accuracy": accuracy, "large_grids": large,
        "clocks": clocks,
        "adjoint": adjoint, "batched_gradients": batched_grad, "coupled": coupled_leg,
        "nonfinite_instances": int(sum(1 for x in bads if x >= 0)),
        "kernel_families": tuned,
    }
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())

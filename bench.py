#!/usr/bin/env python3
"""Benchmark of the D3Q19 moving-boundary step (GLUPS and fraction of the HBM roofline).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--storage S] [--impl ours|reference]

One JSON line on rank 0.  A "step" is one lattice-Boltzmann time step of the
whole workload (geometry, links, bounce-back, loads, fused stream+collide,
body update).  The default is the workload the metric is quoted on: the
flapping wing pair at 512x256x256 with FP16-deviation population storage.
``value`` is device-timed (CUDA events on the library's stream) with the
populations resident in HBM; ``e2e`` runs the same steps through the C ABI one
call at a time with the body state written from pinned host memory and the
step's loads read back every step.  ``roofline`` uses the fused
stream+collide kernel's own CUDA-event launch times and its algorithmic
traffic of 38 * s bytes per fluid cell (19 reads + 19 writes of s-byte
populations); ``roofline.step_frac`` divides the same bytes by the whole step.

Workloads (lattice units):
  flapping_plates    512x256x256, two 64x12x2 plates as 2x8192 triangles,
                     stroke 60 sin, pitch 45 cos, T = 4000, nu 0.004, TRT,
                     ray-root links rebuilt every step (default)
  ellipsoid_channel  256x128x128, ellipsoid (24,12,12) at x=64, inflow 0.05,
                     nu 0.005, RR3, interpolated links, velocity inlet /
                     zero-gradient outlet / periodic y,z
  articulated_bird   768x384x384, ellipsoid body + tail + two 3-segment wings
                     (~145k triangles), free flight, RR3
  shear_wave         64^3 periodic, nu 0.01, magic 1/4 (L2-resident)
Multi-GPU: the step does not shard here (one GPU per lattice), so N GPUs run N
independent replicas; ``value`` is the aggregate and ``scaling`` is weak.

On one GPU the line also carries
  ``variants``  FP32 / FP16-deviation / BF16-deviation storage on the flapping
                plates (512x256x256, TRT): GLUPS, the kernel's and the whole
                step's roofline fractions, and the force averaged over the
                third stroke period of a three-period run against FP64;
  ``precision_form``  the metric's own figures from ``variants``: FP16 step
                speed-up over FP32, roofline fractions, force error vs FP64;
  ``articulated``  the articulated bird at 768x384x384 in FP16-deviation
                storage: GLUPS and the share of the step outside the fused kernel;
  ``ellipsoid_channel``  the RR3 channel at 256x128x128 in FP32;
  ``adjoint``   the discrete adjoint on the plates of the precision workload
                scaled to 256x128x128 over one period: lift and power
                gradients, cost against a forward pass, central differences
                (h = 1e-3 rad) of the full objective and at the unperturbed
                run's topology, the least-squares slope over +-2e-2 rad, and
                FP32 vs FP64 gradients at 96x48x48.
(--no-variants / --no-adjoint / --no-cpu skip the extras.)
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "numi-gpu-physics_b200"))

FALLBACK_HBM_GBS = 6650.0
WORKLOAD_DEFAULT = "flapping_plates"
STORAGE_DEFAULT = "f16dev"
METRIC = "D3Q19 GLUPS & %HBM peak, FP16-store vs FP32 at stated force error; adjoint/fwd"


LATTICE_OVERRIDE = None  # (nx, ny, nz) for small profiling cases; geometry scales with it


def build_case(name: str, storage: int, collision: str | None = None):
    import bfx._lib as L
    import bfx.cases as cases
    coll_id = {"trt": L.COLLISION_TRT, "rr3": L.COLLISION_RR3, "reg": L.COLLISION_REGULARIZED,
               "limiter": L.COLLISION_TRT_LIMITER}
    if name == "ellipsoid_channel":
        kw = {}
        if LATTICE_OVERRIDE:
            nx, ny, nz = LATTICE_OVERRIDE
            kw = dict(nx=nx, ny=ny, nz=nz, radii=(24.0 * nx / 256, 12.0 * ny / 128, 12.0 * nz / 128))
        if collision:
            kw["collision"] = coll_id[collision]
        cfg, rows, body, mesh = cases.ellipsoid_channel(storage=storage, **kw)
        desc = (f"ellipsoid_channel {cfg.nx}x{cfg.ny}x{cfg.nz} semi-axes {tuple(rows[0][:3])} at x={cfg.nx // 4}, "
                f"inflow u_x=0.05 velocity inlet, zero-gradient outflow, periodic y/z, nu=0.005, "
                f"{collision or 'rr3'}, interpolated bounce-back")
        collision = collision or "rr3"
    elif name == "flapping_plates":
        kw = {}
        if LATTICE_OVERRIDE:
            kw = dict(zip(("nx", "ny", "nz"), LATTICE_OVERRIDE))
        if collision:
            kw["collision"] = coll_id[collision]
        cfg, rows, body, mesh = cases.flapping_plates(storage=storage, **kw)
        desc = (f"flapping_plates {cfg.nx}x{cfg.ny}x{cfg.nz} two 64x12x2 flat plates (2x8192 triangles), "
                f"stroke 60deg sin, pitch 45deg cos, T=4000, nu=0.004, {collision or 'trt'}, ray-root links "
                f"rebuilt each step")
        collision = collision or "trt"
    elif name == "articulated_bird":
        kw = {}
        if LATTICE_OVERRIDE:
            nx, ny, nz = LATTICE_OVERRIDE
            f = nx / 768.0
            kw = dict(nx=nx, ny=ny, nz=nz, body_radii=(60.0 * f, 18.0 * f, 18.0 * f),
                      wing_spans=(50.0 * f, 48.0 * f, 42.0 * f), chords=(36.0 * f, 28.0 * f, 20.0 * f, 12.0 * f),
                      resolution=max(f, 0.25), sponge_width=32.0 * f)
        if collision:
            kw["collision"] = coll_id[collision]
        cfg, rows, body, mesh = cases.articulated_bird(storage=storage, **kw)
        desc = (f"articulated_bird {cfg.nx}x{cfg.ny}x{cfg.nz} ellipsoid body + tail + two 3-segment wings "
                f"(shoulder/elbow/wrist, {mesh['tris'].shape[0]} triangles), free 6-DOF flight, inflow 0.04, "
                f"nu=0.002, {collision or 'rr3'}, sponge 32, linear links rebuilt each step")
        collision = collision or "rr3"
    elif name == "shear_wave":
        n = LATTICE_OVERRIDE[0] if LATTICE_OVERRIDE else 64
        cfg, rows, body, mesh = cases.shear_wave(n=n, viscosity=0.01, magic=0.25, axis="z", storage=storage,
                                                 collision=coll_id[collision] if collision else L.COLLISION_TRT)
        desc = f"shear_wave {n}^3 periodic, u_x=0.01 sin(2 pi z/{n}), nu=0.01, magic 1/4, {collision or 'trt'}"
        collision = collision or "trt"
    else:
        raise SystemExit(f"unknown workload {name}")
    return cfg, rows, body, mesh, desc, collision


COLLISION_OVERRIDE = None


def make_lattice(name, storage, device):
    import bfx._lib as L
    from bfx.simulation import Lattice, bird_struct
    cfg, rows, body, mesh, desc, coll = build_case(name, storage, COLLISION_OVERRIDE)
    cfg.device = device
    bs = None
    if body is not None:
        bs = L.BodyState()
        bs.position[:] = list(body[0])
        bs.orientation[:] = list(body[1])
        bs.velocity[:] = list(body[2])
        bs.omega_body[:] = list(body[3])
    lat = Lattice(cfg, bird_struct(rows) if rows is not None else None, bs, mesh)
    return lat, cfg, desc, coll


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons of this process's GPU,
    polled read-only through NVML every ~2 ms on a background thread (a
    100 ms nvidia-smi loop cannot see a timed region of a few milliseconds).
    `region()` brackets the timed region; the summary reports the samples
    inside it, or, when the region was shorter than one poll, every sample
    taken while the bench's GPU work ran.  Falls back to nvidia-smi when NVML
    is unavailable."""

    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.samples = []  # (host time, sm MHz, set of reason names)
        self.max_mhz = None
        self.windows = []
        self._stop = threading.Event()
        self._thread = None
        self._proc = None
        self.source = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def _poll_nvml(self, nv, h):
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        while not self._stop.is_set():
            try:
                mhz = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                r = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
                self.samples.append((time.perf_counter(), mhz, {k for k, b in bits.items() if r & b}))
            except Exception:
                return
            self._stop.wait(0.002)

    def _read_smi(self):
        for ln in self._proc.stdout:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                mhz, self.max_mhz = float(parts[1]), float(parts[2])
            except ValueError:
                continue
            self.samples.append((time.perf_counter(), mhz,
                                 {nm for nm, v in zip(self.NAMES, parts[5:9]) if v.lower() == "active"}))

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self._thread = threading.Thread(target=self._poll_nvml, args=(nv, h), daemon=True)
            self.source = "nvml 2 ms"
        except Exception:
            try:
                self._proc = subprocess.Popen(
                    ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                     "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self._thread = threading.Thread(target=self._read_smi, daemon=True)
                self.source = "nvidia-smi 100 ms"
            except OSError:
                return self
        self._thread.start()
        return self

    def region(self):
        sampler = self

        class _Region:
            def __enter__(self):
                self.t0 = time.perf_counter()

            def __exit__(self, *exc):
                sampler.windows.append((self.t0, time.perf_counter()))
        return _Region()

    def __exit__(self, *exc):
        self._stop.set()
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()
        if self._thread is not None:
            self._thread.join(timeout=5)

    def summary(self):
        inside = [s for s in self.samples if any(a <= s[0] <= b for a, b in self.windows)]
        use = inside or self.samples
        sm = [s[1] for s in use]
        reasons = sorted(set().union(*[s[2] for s in use])) if use else []
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(use), "samples_in_timed_region": len(inside), "source": self.source}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(workload: str, storage_name: str):
    """Per-launch DRAM bytes of the fused kernel from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    try:
        for ln in open(path):
            parts = ln.split()
            if len(parts) >= 3 and not ln.startswith("#") and parts[0] == workload and parts[1] == storage_name:
                return float(parts[2])
    except OSError:
        pass
    return None


def time_steps(lat, steps, warmup, clocks=None):
    """Device time of `steps` steps (CUDA events on the library stream), then the
    fused interior kernel's own per-launch CUDA-event times over a second run of
    the same steps (per-launch events disable the step graphs, so they are kept
    out of the whole-step timing).  `clocks` (a ClockSampler) marks the timed
    region."""
    lat.advance(warmup, batch_size=max(warmup, 1))
    l0 = lat.launch_count()
    if clocks is not None:
        with clocks.region():
            lat.timer_begin()
            lat.advance(steps, batch_size=steps)
            ms = lat.timer_end()
    else:
        lat.timer_begin()
        lat.advance(steps, batch_size=steps)
        ms = lat.timer_end()
    l1 = lat.launch_count()
    lat.set_kernel_timing(True)
    lat.advance(min(steps, 400), batch_size=min(steps, 400))
    kms, klaunch = lat.kernel_timing()
    lat.set_kernel_timing(False)
    return ms, l1 - l0, kms, klaunch


def e2e_steps(lat, steps):
    """Per-step C-ABI calls with host buffers: body state in (pinned), loads out."""
    import ctypes as ct
    import bfx._lib as L
    try:
        import torch
        pinned_in = torch.empty(ct.sizeof(L.BodyState), dtype=torch.uint8).pin_memory()
        pinned_out = torch.empty(ct.sizeof(L.Loads), dtype=torch.uint8).pin_memory()
        body = L.BodyState.from_address(pinned_in.data_ptr())
        loads = L.Loads.from_address(pinned_out.data_ptr())
    except Exception:  # pinned memory unavailable: plain host structs
        body, loads = L.BodyState(), L.Loads()
    cur = lat.body()
    ct.memmove(ct.addressof(body), ct.addressof(cur), ct.sizeof(L.BodyState))
    lib = lat.lib
    lat.timer_begin()
    for _ in range(steps):
        rc = lib.bfx_set_body(lat.handle, ct.byref(body))
        rc |= lib.bfx_advance(lat.handle, 1, 1, 0, None, 0, None)
        rc |= lib.bfx_last_loads(lat.handle, ct.byref(loads))
        if rc:
            raise RuntimeError(L.last_error(lat.handle))
    ms = lat.timer_end()
    return ms, ct.sizeof(L.BodyState), ct.sizeof(L.Loads)


def force_history(name, storage, steps, device):
    """Per-step force (N) of `steps` steps from the start, recorded on the device."""
    lat, cfg, _, _ = make_lattice(name, storage, device)
    _, samples = lat.advance(steps, batch_size=steps, record_samples=True)
    f = np.array([[samples[i].force[0], samples[i].force[1], samples[i].force[2]] for i in range(steps)])
    lat.close()
    return f


def storage_forms(device, steps=200, warmup=5, periods=3):
    """FP32 / FP16-deviation / BF16-deviation on the flapping-plate workload
    (512x256x256, TRT, links rebuilt every step): whole-step throughput, the
    fused kernel's and the whole step's fractions of the HBM roofline, and the
    force averaged over the last stroke period of a `periods`-period run
    (steps 8001-12000 for three periods of T = 4000) against an FP64 run of
    the same kernels."""
    import bfx._lib as L
    peak, _ = measured_peak()
    period = 4000
    total = periods * period
    window = (total - period, total)  # 0-based slice: steps total-period+1 ... total
    ref_hist = force_history("flapping_plates", L.STORAGE_F64, total, device)
    ref = ref_hist[window[0]:window[1]].mean(axis=0)
    out = {"workload": "flapping_plates 512x256x256 TRT, stroke 60 deg, pitch 45 deg, T=4000",
           "force_window_steps": [window[0] + 1, window[1]], "periods_run": periods,
           "force_reference": "FP64 storage, same kernels", "force_reference_value_N": ref.tolist()}
    base = None
    for st in (L.STORAGE_F32, L.STORAGE_F16_DEVIATION, L.STORAGE_BF16_DEVIATION):
        nm = L.STORAGE_NAMES[st]
        vlat, cfg, _, _ = make_lattice("flapping_plates", st, device)
        cells = cfg.nx * cfg.ny * cfg.nz
        vms, _, vkms, vkl = time_steps(vlat, steps, warmup)
        fluid = cells - int(np.count_nonzero(vlat.mask()))
        vlat.close()
        rate = cells * steps / (vms / 1000.0) / 1e9
        kernel_s = vkms / max(vkl, 1) / 1000.0
        ach = fluid * 38 * L.STORAGE_BYTES[st] / kernel_s / 1e9
        step_s = vms / steps / 1000.0
        hist = force_history("flapping_plates", st, total, device)
        f = hist[window[0]:window[1]].mean(axis=0)
        err = float(np.linalg.norm(f - ref) / max(np.linalg.norm(ref), 1e-30))
        base = rate if base is None else base
        out[nm] = {"value": rate, "unit": "GLUPS", "ms_per_step": step_s * 1000.0, "kernel_ms": kernel_s * 1000.0,
                   "achieved_gbs": ach, "roofline_frac": ach / peak,
                   "step_roofline_frac": fluid * 38 * L.STORAGE_BYTES[st] / step_s / 1e9 / peak,
                   "speedup_vs_f32": rate / base, "cycle_mean_force_error_vs_f64": err,
                   "cycle_mean_force_N": f.tolist()}
    return out


def workload_measure(name, storage, device, steps=100, warmup=5):
    """Whole-step GLUPS of one workload in one storage form, the fused
    kernel's roofline fraction and the share of the step spent outside it
    (geometry, links, loads, body)."""
    import bfx._lib as L
    peak, _ = measured_peak()
    lat, cfg, desc, coll = make_lattice(name, storage, device)
    cells = cfg.nx * cfg.ny * cfg.nz
    ms, launches, kms, kl = time_steps(lat, steps, warmup)
    fluid = cells - int(np.count_nonzero(lat.mask()))
    body = lat.body()
    lat.close()
    kernel_s = kms / max(kl, 1) / 1000.0
    ach = fluid * 38 * L.STORAGE_BYTES[storage] / kernel_s / 1e9
    step_ms = ms / steps
    return {"workload": desc, "collision": coll, "storage": L.STORAGE_NAMES[storage], "steps": steps,
            "value": cells * steps / (ms / 1e3) / 1e9, "unit": "GLUPS", "ms_per_step": step_ms,
            "kernel_ms": kernel_s * 1e3, "achieved_gbs": ach, "roofline_frac": ach / peak,
            "step_roofline_frac": fluid * 38 * L.STORAGE_BYTES[storage] / (step_ms / 1e3) / 1e9 / peak,
            "outside_kernel_share": max(0.0, 1.0 - kernel_s * 1e3 / step_ms), "gpu_launches": launches,
            "body_position_after": [float(x) for x in body.position]}


def articulated_measure(device, steps=100, warmup=5):
    """The articulated bird (768x384x384, RR3, FP16-deviation storage, free
    6-DOF flight, ~145k triangles on shoulder / elbow / wrist segments)."""
    import bfx._lib as L
    return workload_measure("articulated_bird", L.STORAGE_F16_DEVIATION, device, steps, warmup)


def adjoint_measure(device, scan_points=11, scan_half_width=2e-2, fd_h=1e-3):
    """Discrete adjoint on the flapping-plate pair of the precision workload
    scaled to 256x128x128 (span 32, chord 6, thickness 2, 2 x 8,192
    triangles; T = 2000, one period, FP32, TRT, linear links): gradient of the
    cycle-mean lift and aerodynamic power with respect to (stroke amplitude,
    pitch amplitude, pitch phase, deviation amplitude) and its cost against a
    plain forward pass.  Checked against (a) central differences with
    h = 1e-3 rad and (b) the least-squares slope of J over `scan_points`
    offsets in +-2e-2 rad, with the slope's standard error (the scatter of J
    about the line: cover / uncover events make J piecewise smooth); and the
    FP32 against the FP64 gradient at 96x48x48."""
    import bfx._lib as L
    import bfx.cases as cases
    from bfx.simulation import Lattice, bird_struct

    def plates(storage, theta=None, n=(256, 128, 128), span=32.0, chord=6.0):
        cfg, rows, body, mesh = cases.flapping_plates(
            nx=n[0], ny=n[1], nz=n[2], span=span, chord=chord, thickness=2.0, n_chord=32, n_span=128, period=2000.0,
            stroke_deg=60.0, pitch_deg=45.0, deviation_deg=5.0, viscosity=0.004, storage=storage,
            link_rule=L.LINK_LINEAR, sponge_width=12.0)
        if theta is not None:
            rows = cases.with_kinematic_parameters(rows, theta)
        cfg.device = device
        bs = L.BodyState()
        bs.position[:] = list(body[0])
        bs.orientation[:] = list(body[1])
        return Lattice(cfg, bird_struct(rows), bs, mesh), rows

    steps = 2000
    lat, rows = plates(L.STORAGE_F32)
    theta0 = np.array(cases.kinematic_parameters(rows), dtype=np.float64)
    lat.advance(1)  # warm the code paths, then time a plain forward pass on a fresh handle
    lat.close()
    lat, _ = plates(L.STORAGE_F32)
    lat.timer_begin()
    lat.advance(steps, batch_size=steps)
    fwd_ms = lat.timer_end()
    lat.close()
    out = {"case": "flapping_plates 256x128x128, span 32, chord 6, thickness 2, 2x8192 triangles, T=2000, "
                   "nu=0.004, TRT, linear links, FP32", "steps": steps,
           "parameters": ["stroke amplitude", "pitch amplitude", "pitch phase", "deviation amplitude"],
           "theta": theta0.tolist(), "forward_ms": fwd_ms}
    for name, fw, pw in (("lift", (0.0, 0.0, 1.0), 0.0), ("power", (0.0, 0.0, 0.0), 1.0)):
        lat, _ = plates(L.STORAGE_F32)
        r = lat.adjoint(steps, fw, pw)
        lat.close()
        out[name] = {"objective": r.objective, "gradient": list(r.gradient), "adjoint_forward_ms": r.forward_ms,
                     "adjoint_reverse_ms": r.reverse_ms, "checkpoint_interval": r.checkpoint_interval,
                     "snapshots": r.snapshots, "work_bytes": r.work_bytes,
                     "cost_vs_forward": (r.forward_ms + r.reverse_ms) / fwd_ms}

    def objectives(theta, replay=None, mode=0, storage=L.STORAGE_F32):
        lat, _ = plates(storage, theta)
        if replay is not None:
            lat.replay_topology(mode, replay.data_ptr(), steps)
        lift, power = 0.0, 0.0
        for _ in range(steps):
            lat.advance(1)
            ld = lat.loads()
            lift += ld.force[2]
            power += ld.power
        lat.close()
        return lift / steps, power / steps

    offsets = np.linspace(-scan_half_width, scan_half_width, scan_points)
    fd = {"lift": [], "power": []}
    scan = {"lift": [], "power": []}
    for k in range(4):
        vals = []
        for o in offsets:
            th = theta0.copy()
            th[k] += o
            vals.append(objectives(th))
        tp, tm = theta0.copy(), theta0.copy()
        tp[k] += fd_h
        tm[k] -= fd_h
        (lp, pp), (lm, pm) = objectives(tp), objectives(tm)
        fd["lift"].append((lp - lm) / (2 * fd_h))
        fd["power"].append((pp - pm) / (2 * fd_h))
        vals = np.array(vals)
        A = np.vstack([np.ones_like(offsets), offsets]).T
        for j, name in enumerate(("lift", "power")):
            coef, *_ = np.linalg.lstsq(A, vals[:, j], rcond=None)
            resid = vals[:, j] - A @ coef
            sigma = float(np.sqrt(np.sum(resid ** 2) / max(len(offsets) - 2, 1)))
            stderr = sigma / float(np.sqrt(np.sum((offsets - offsets.mean()) ** 2)))
            scan[name].append({"slope": float(coef[1]), "slope_stderr": stderr, "residual_std": sigma,
                               "J": vals[:, j].tolist()})
    # Central differences at the topology of the unperturbed run (its
    # occupancy recorded step by step and replayed in the perturbed runs), in
    # FP64 with h = 1e-4 rad: the derivative of the smooth piece of J, which
    # the adjoint computes (a larger h moves fluid cells next to the wall
    # across the link rule's clamps, a smaller one reaches the FP32
    # resolution of the geometry).
    import torch
    rec = torch.empty((steps, 256 * 128 * 128), dtype=torch.uint8, device=f"cuda:{device}")
    objectives(theta0, rec, 1, L.STORAGE_F64)
    fd_frozen = {"lift": [], "power": []}
    hf = 1e-4
    for k in range(4):
        tp, tm = theta0.copy(), theta0.copy()
        tp[k] += hf
        tm[k] -= hf
        (lp, pp), (lm, pm) = objectives(tp, rec, 2, L.STORAGE_F64), objectives(tm, rec, 2, L.STORAGE_F64)
        fd_frozen["lift"].append((lp - lm) / (2 * hf))
        fd_frozen["power"].append((pp - pm) / (2 * hf))
    del rec
    out["frozen_topology_h"] = hf
    for name in ("lift", "power"):
        g = np.array(out[name]["gradient"])
        ff = np.array(fd_frozen[name])
        out[name]["central_difference_frozen_topology"] = ff.tolist()
        out[name]["relative_difference_vs_frozen_topology_fd"] = float(np.max(np.abs(g - ff)) /
                                                                       max(np.max(np.abs(ff)), 1e-30))
    for name in ("lift", "power"):
        g = np.array(out[name]["gradient"])
        f = np.array(fd[name])
        sl = np.array([d["slope"] for d in scan[name]])
        se = np.array([d["slope_stderr"] for d in scan[name]])
        out[name]["central_difference"] = f.tolist()
        out[name]["relative_difference_vs_fd"] = float(np.max(np.abs(g - f)) / max(np.max(np.abs(f)), 1e-30))
        out[name]["regression"] = scan[name]
        out[name]["relative_difference_vs_regression"] = float(np.max(np.abs(g - sl)) /
                                                                max(np.max(np.abs(sl)), 1e-30))
        out[name]["regression_noise_relative"] = float(np.max(se) / max(np.max(np.abs(sl)), 1e-30))
    out["central_difference_h"] = fd_h
    out["regression_offsets"] = offsets.tolist()
    # FP64 reference gradient on a 96x48x48 lattice (the same case scaled)
    small = dict(n=(96, 48, 48), span=12.0, chord=2.25)
    grads = {}
    for st in (L.STORAGE_F32, L.STORAGE_F64):
        lat, _ = plates(st, **small)
        grads[st] = np.array(list(lat.adjoint(steps, (0.0, 0.0, 1.0), 0.0).gradient))
        lat.close()
    out["fp64_reference_96x48x48"] = {
        "gradient_fp64": grads[L.STORAGE_F64].tolist(), "gradient_fp32": grads[L.STORAGE_F32].tolist(),
        "relative_difference": float(np.max(np.abs(grads[L.STORAGE_F32] - grads[L.STORAGE_F64])) /
                                     max(np.max(np.abs(grads[L.STORAGE_F64])), 1e-30))}
    return out


def cpu_port_rate(name, seconds_budget=12.0, max_steps=64, warmup=1, warmup_budget=30.0):
    """The oracle (CPU restatement of the reference path) on the same workload:
    `warmup` untimed steps (fewer if they exceed `warmup_budget` seconds), then
    timed steps until `max_steps` or `seconds_budget`.  Returns the rate, the
    timed steps, the threads, the timed seconds and the warm-up steps run."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle as O  # noqa: F401  (the oracle, CPU baseline only)
    from helpers import oracle_twin
    cfg, rows, body, mesh, desc, _ = build_case(name, 0, COLLISION_OVERRIDE)
    osim = oracle_twin(cfg, rows, body, mesh)
    w0 = time.perf_counter()
    warm = 0
    while warm < max(warmup, 1):
        osim.step()
        warm += 1
        if time.perf_counter() - w0 > warmup_budget:
            break
    t0 = time.perf_counter()
    steps = 0
    while steps < max_steps:
        osim.step()
        steps += 1
        if time.perf_counter() - t0 > seconds_budget:
            break
    dt = time.perf_counter() - t0
    cells = cfg.nx * cfg.ny * cfg.nz
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return cells * steps / dt / 1e9, steps, threads, dt, warm


def bench_config(desc, cfg, coll, world):
    """The `config` object both arms print (the same workload, so the same keys)."""
    cells = cfg.nx * cfg.ny * cfg.nz
    return {"workload": desc, "lattice": [cfg.nx, cfg.ny, cfg.nz], "collision": coll,
            "l2": (f"inputs larger than L2 ({19 * cells * 2 / 1e6:.0f} MB of populations at 2 B, "
                   f"{19 * cells * 4 / 1e6:.0f} MB at 4 B; no flush needed)") if 19 * cells * 2 > 126e6
            else "L2-resident working set",
            "parallelism": f"replicas{world}"}


def run_reference_arm(args, rank, world):
    name = args.workload
    if rank != 0:
        return 0
    cfg, rows, body, mesh, desc, coll = build_case(name, 0, COLLISION_OVERRIDE)
    budget = 150.0
    per_step_budget = budget / max(args.steps + args.warmup, 1)
    rate, steps, cores, dt, warm = cpu_port_rate(name, seconds_budget=min(60.0, per_step_budget * args.steps),
                                                 max_steps=max(1, args.steps), warmup=args.warmup)
    cells = cfg.nx * cfg.ny * cfg.nz
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "GLUPS", "n_gpus": world,
        "steps": steps, "warmup": warm, "ms_per_step": dt * 1000.0 / max(steps, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "storage": "f32", "data": "synthetic",
        "config": bench_config(desc, cfg, coll, world),
        "cpu_baseline": {"value": rate, "unit": "GLUPS", "cores": cores, "kind": "port",
                         "sample": f"{steps} full steps of the {name} workload ({cells} cells) on the CPU "
                                   f"restatement of the reference step (oracle/, C + OpenMP, FP32 populations: "
                                   f"the reference has no 16-bit storage)"},
        "e2e": {"value": rate, "unit": "GLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--workload", default=WORKLOAD_DEFAULT)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--lattice", type=int, nargs=3, default=None, help="profiling override of the lattice size")
    ap.add_argument("--collision", default=None, choices=["trt", "rr3", "reg", "limiter"])
    ap.add_argument("--storage", default=STORAGE_DEFAULT, choices=["f32", "f16dev", "bf16dev", "f64"])
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    global LATTICE_OVERRIDE, COLLISION_OVERRIDE
    LATTICE_OVERRIDE = tuple(args.lattice) if args.lattice else None
    COLLISION_OVERRIDE = args.collision

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    if args.impl == "reference":
        rc = run_reference_arm(args, rank, world)
        if dist is not None:
            dist.destroy_process_group()
        return rc

    import bfx._lib as L
    main_storage = {v: k for k, v in L.STORAGE_NAMES.items()}[args.storage]
    lat, cfg, desc, coll = make_lattice(args.workload, main_storage, local)
    cells = cfg.nx * cfg.ny * cfg.nz
    sbytes = L.STORAGE_BYTES[main_storage]

    def barrier():
        if dist is not None:
            import torch
            torch.cuda.synchronize()
            dist.barrier()

    barrier()
    with ClockSampler(local) as clocks:
        ms, launches, kms, klaunch = time_steps(lat, args.steps, args.warmup, clocks)
    barrier()
    if dist is not None:
        import torch
        t = torch.tensor([ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * cells * args.steps / (ms / 1000.0) / 1e9
    e2e_n = min(args.steps, 200)
    e2e_ms, h2d, d2h = e2e_steps(lat, e2e_n)
    solid_cells = int(np.count_nonzero(lat.mask()))
    if dist is not None:
        import torch
        t = torch.tensor([e2e_ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = world * cells * e2e_n / (e2e_ms / 1000.0) / 1e9
    lat.close()

    peak, peak_kind = measured_peak()
    fluid = cells - solid_cells
    bytes_per_launch = fluid * 38 * sbytes
    kernel_s = kms / max(klaunch, 1) / 1000.0
    achieved = bytes_per_launch / kernel_s / 1e9
    traffic = profiled_traffic(args.workload, args.storage)
    staged = coll in ("trt", "rr3", "reg") and args.storage in ("f16dev", "bf16dev")
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_kind": f"of {peak_kind}",
                "kernel": ("k_stream (TMA-staged fused AA stream+collide, 16-bit storage)" if staged
                           else "k_bulk (fused AA stream+collide over every fluid cell)"),
                "bytes_per_launch": bytes_per_launch, "bytes_rule": "fluid cells x 19 x 2 x storage bytes",
                "kernel_ms": kernel_s * 1000.0,
                "step_frac": bytes_per_launch / (ms / args.steps / 1000.0) / 1e9 / peak}

    line = {
        "metric": METRIC, "value": value, "unit": "GLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if main_storage != L.STORAGE_F64 else "f64",
        "storage": args.storage, "data": "synthetic",
        "config": bench_config(desc, cfg, coll, world),
        "e2e": {"value": e2e_value, "unit": "GLUPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": e2e_n, "calls": "bfx_set_body + bfx_advance(1) + bfx_last_loads per step"},
        "roofline": roofline,
        "gpu_launches": launches,
        "clocks": clocks.summary(),
    }

    if rank == 0 and world == 1 and not args.no_variants:
        v = storage_forms(local)
        line["variants"] = v
        if args.workload == "flapping_plates":
            line["precision_form"] = {
                "f16dev_step_speedup_vs_f32": v["f16dev"]["speedup_vs_f32"],
                "bf16dev_step_speedup_vs_f32": v["bf16dev"]["speedup_vs_f32"],
                "f16dev_kernel_roofline_frac": v["f16dev"]["roofline_frac"],
                "f16dev_step_roofline_frac": v["f16dev"]["step_roofline_frac"],
                "f16dev_cycle_mean_force_error_vs_f64": v["f16dev"]["cycle_mean_force_error_vs_f64"],
                "bf16dev_cycle_mean_force_error_vs_f64": v["bf16dev"]["cycle_mean_force_error_vs_f64"],
                "force_window_steps": v["force_window_steps"]}
        line["articulated"] = articulated_measure(local)
        line["ellipsoid_channel"] = workload_measure("ellipsoid_channel", L.STORAGE_F32, local)
    if rank == 0 and world == 1 and not args.no_adjoint:
        line["adjoint"] = adjoint_measure(local)

    if rank == 0 and world == 1 and not args.no_cpu:
        rate, steps, cores, dt, _ = cpu_port_rate(args.workload)
        line["cpu_baseline"] = {"value": rate, "unit": "GLUPS", "cores": cores, "kind": "port",
                                "sample": f"{steps} full steps of the same workload on the CPU restatement "
                                          f"(oracle/, C + OpenMP, FP32 populations, {dt:.1f} s)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

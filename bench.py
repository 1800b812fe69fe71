#!/usr/bin/env python
"""Benchmark of the H.psi / Taylor path on B200.

Workload (one "step"): one full FP64 Hamiltonian application H.psi
(kinetic order-4 star + local potential + KB projectors) on the sphere system
R = 12 bohr, h = 0.2 (904,089 inner points), 32 atoms x 9 projectors, 128
complex128 states -- the configuration the headline metric is quoted on.
Inputs are seeded synthetic data (no data set exists for this path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl hpsi|reference]

value  = point-states per second of H.psi with psi resident in HBM (the batch,
         2.2 GB, is far larger than the 126 MB L2, so no flush is needed);
e2e    = the same metric through the C ABI with pinned host buffers (the
         host->device copy of psi's np inner rows and the device->host copy of
         H psi inside the timed region of every step, pipelined over state
         slabs by the library);
extra  = FP32-storage H.psi, the fused Taylor step (FP64 and FP32).
Multi-GPU: independent replicas (the path has no exchange step), weak scaling.
--impl reference times the reference CPU path (the reference's own compiled
stencil kernel plus the oracle's restatement of the rest) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "octopus-debian-package_b200")
sys.path.insert(0, PKG)
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "H·ψ Gpoint-states/s (FP64, full H with KB)"
UNIT = "Gpoint-states/s"
WORKLOAD = "sphere R=12 h=0.2 (np=904089), 32 KB atoms x 9 projectors, 128 complex128 states"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="hpsi", choices=["hpsi", "reference"])
    ap.add_argument("--small", action="store_true", help="small case (for profiler captures)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="headline H.psi and its roofline only (no e2e, FP32, Taylor, TD or other "
                         "configurations): a short process for profiler captures of the full-size pass")
    ap.add_argument("--configs", action="store_true",
                    help="instead of the headline line, one line per other configuration "
                         "(64^3 box, 2000-step TD, 64 grouped systems, adjoint gradient)")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(path="profiles/pass_blk_fp64_sphere64.md"):
    """dram bytes per launch of the pass kernel from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, path)) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_full_launch:"):
                    return float(line.split(":")[1].split()[0])
    except Exception:
        pass
    return None


class Clocks:
    """SM clock and throttle-reason sampler for the timed region (NVML every
    2 ms, read-only; nvidia-smi every 200 ms when NVML is unavailable)."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80}

    def __init__(self, gpu_index=0, period=0.002):
        self.idx = gpu_index
        self.period = period
        self.samples = []  # (sm_mhz, reasons bitmask)
        self.max_mhz = None
        self.proc = None
        self.nvml = None
        self._stop = threading.Event()

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(self.idx)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}",
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _poll(self):
        nv = self.nvml
        while not self._stop.is_set():
            try:
                mhz = float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
                self.samples.append((mhz, rs))
            except Exception:
                pass
            time.sleep(self.period)

    def _read(self):
        for line in self.proc.stdout:
            try:
                f = [x.strip() for x in line.split(",")]
                self.max_mhz = float(f[1])
                self.samples.append((float(f[0]), int(f[2], 16)))
            except Exception:
                continue

    def __exit__(self, *a):
        self._stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        elif self.nvml is not None:
            self.t.join(timeout=1)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0}
        reasons = set()
        for _, rs in self.samples:
            for n, bit in self.REASONS.items():
                if rs & bit:
                    reasons.add(n)
        return {"sm_mhz": statistics.median(m for m, _ in self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "samples": len(self.samples),
                "source": "nvml" if self.nvml is not None else "nvidia-smi"}


def build_system(small=False):
    from hpsi import fixtures
    if small:
        return fixtures.config1(radius=8.0, spacing=0.2, natoms=8, nst=64, place_radius=5.5)
    return fixtures.config1()


SAMPLE_STATES = [0, 17, 38, 63, 64, 90, 111, 127]  # spread over the 16 state chunks


def rel_maxnorm_per_state(got, ref):
    """max over states of max_ip |got - ref| / max_ip |ref| (the parity metric)."""
    num = np.max(np.abs(np.asarray(got) - np.asarray(ref)), axis=0)
    den = np.max(np.abs(np.asarray(ref)), axis=0)
    return float(np.max(num / np.where(den == 0, 1.0, den)))


def cpu_reference_rate(sysm, sample, min_seconds=10.0, max_reps=200):
    """Reference CPU H.psi rate (Gpoint-states/s) on a sample of the states,
    and the CPU H psi of that sample (the parity check of the timed run)."""
    from oracle import oracle as O
    from hpsi.stencil import laplacian_weights, star_points
    m = sysm.mesh
    P = O.Projectors(sysm.proj.maps, sysm.proj.mats, sysm.proj.scals) if sysm.proj else None
    H = O.Hamiltonian(m, laplacian_weights(m.spacing), star_points(), v=sysm.v, projectors=P)
    psi = np.ascontiguousarray(sysm.psi[:, sample])
    ref = H.apply(psi)  # warm, and the check values
    t0 = time.perf_counter()
    reps = 0
    while True:
        H.apply(psi)
        reps += 1
        el = time.perf_counter() - t0
        if el >= min_seconds or reps >= max_reps:
            break
    n = len(sample)
    rate = m.np * n * reps / el / 1e9
    kind = "reference" if H.used_reference_kernel else "port"
    sample_txt = (f"{reps} H.psi applications on {n} of the {sysm.psi.shape[1]} states "
                  f"({el:.1f} s; stencil = reference operate.c compiled from source)" if kind == "reference"
                  else f"{reps} H.psi applications on {n} states ({el:.1f} s)")
    return rate, H.nthreads, kind, sample_txt, ref


def run_reference(args, rank, world):
    """--impl reference: the reference CPU path on the box's host cores, each
    step one H.psi over the whole 128-state batch of the workload."""
    if rank != 0:
        return
    sysm = build_system(args.small)
    from oracle import oracle as O
    from hpsi.stencil import laplacian_weights, star_points
    m = sysm.mesh
    P = O.Projectors(sysm.proj.maps, sysm.proj.mats, sysm.proj.scals)
    H = O.Hamiltonian(m, laplacian_weights(m.spacing), star_points(), v=sysm.v, projectors=P)
    psi = np.ascontiguousarray(sysm.psi)
    nst = psi.shape[1]
    for _ in range(args.warmup):
        H.apply(psi)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        H.apply(psi)
    el = time.perf_counter() - t0
    rate = m.np * nst * args.steps / el / 1e9
    kind = "reference" if H.used_reference_kernel else "port"
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "config": {"workload": WORKLOAD + (" [small]" if args.small else ""),
                                                 "step": "one H.psi (kinetic + local + KB) over the whole batch"},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": H.nthreads, "kind": kind,
                         "sample": f"each step = one H.psi on all {nst} states (stencil = the reference's "
                                   "operate.c compiled from source; vpsi and KB restated)"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    gpu = reference_gpu_rate(sysm, args)
    if gpu is not None:
        line["extra"] = {"reference_gpu_kernels": gpu}
    print(json.dumps(line), flush=True)


def reference_gpu_rate(sysm, args):
    """The reference's own GPU H.psi on the same batch: its share/opencl
    kernels (operate_map, vpsi, dprojector_bra, dprojector_ket per matrix with
    a synchronisation each) compiled from source for sm_100a and launched as
    the reference launches them; CUDA events over the steps.  None without a
    GPU or without the compiled kernels."""
    try:
        import torch
        if not torch.cuda.is_available():
            return None
        from oracle import refgpu
        if not refgpu.available():
            return None
    except Exception:
        return None
    from hpsi.stencil import laplacian_weights, star_points
    dev = torch.device("cuda", 0)
    m = sysm.mesh
    R = refgpu.RefHamiltonian(m, laplacian_weights(m.spacing), star_points(), sysm.v, sysm.proj, dev)
    x = torch.from_numpy(sysm.psi).to(dev)
    y = torch.zeros((m.np, x.shape[1]), dtype=torch.complex128, device=dev)
    proj = R.projection_buffer(x)
    for _ in range(args.warmup):
        R.apply(x, y, proj)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        R.apply(x, y, proj)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    return {"value": m.np * x.shape[1] / ms / 1e6, "unit": UNIT, "ms_per_step": ms,
            "kernels": "reference share/opencl operate_map + vpsi + dprojector_bra + dprojector_ket "
                       "(one launch per matrix, synchronised), NVRTC-compiled for sm_100a with the "
                       "reference's flags"}


class Ranks:
    """One process per GPU: barrier and max over ranks (NCCL on the GPUs; the
    CPU tests drive the same code over gloo)."""

    def __init__(self, world, device):
        self.world = world
        self.device = device

    def barrier(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max(self, v):
        if self.world == 1:
            return v
        import torch
        import torch.distributed as dist
        t = torch.tensor([v], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())


def _cuda_ms(fn, reps, warm=2):
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def run_configs(args):
    """The configurations other than the headline, one JSON line each (1 GPU).

    Time steps: the order-4 star Laplacian has E_max = 9.75 / h^2 Ha (244 Ha at
    h = 0.2, 156 Ha at h = 0.25) and the 4th-order Taylor series is stable only
    for dt * E_max <= 2 sqrt(2), so the TD run on the h = 0.2 sphere uses
    dt = 0.005 and the adjoint run on the h = 0.25 box dt = 0.01 (dt = 0.02
    diverges on these grids in any implementation of the method).
    """
    import torch
    from hpsi import fixtures, lib
    from hpsi.mesh import index_box_mesh
    from hpsi.stencil import laplacian_weights, star_points
    dev = torch.device("cuda", 0)

    def emit(d):
        print(json.dumps(d), flush=True)

    # ---- 64^3 box, kinetic + local, 32 states ----------------------------------
    s0 = fixtures.config0()
    m = s0.mesh
    dm = lib.DeviceMesh(m)
    ham = lib.Hamiltonian(dm, laplacian_weights(m.spacing), star_points(), v=s0.v)
    x = torch.from_numpy(s0.psi).to(dev)
    y = torch.zeros((m.np, 32), dtype=torch.complex128, device=dev)
    ms64 = _cuda_ms(lambda: ham.apply(x, y), 20)
    x32, y32 = x.to(torch.complex64), y.to(torch.complex64)
    ms32 = _cuda_ms(lambda: ham.apply(x32, y32), 20)
    emit({"config": "box 64^3 h=0.25, 32 states, kinetic + local (no KB)", "unit": UNIT,
          "fp64": {"value": m.np * 32 / ms64 / 1e6, "ms": ms64}, "fp32": {"value": m.np * 32 / ms32 / 1e6, "ms": ms32},
          "alg_bytes_fp64_per_apply": m.np * 32 * 32 + m.np * 8})
    del ham, dm, x, y, x32, y32

    # ---- TD: config-1 system, laser, 2000 steps, FP32 graph vs FP64 plain --------
    s1 = build_system(args.small)
    m = s1.mesh
    dm = lib.DeviceMesh(m)
    ham = lib.Hamiltonian(dm, laplacian_weights(m.spacing), star_points(), v=s1.v, projectors=s1.proj)
    nsteps = 200 if args.small else 2000
    dt = 0.005
    laser = dict(E0=0.01, omega=0.057, T=nsteps * dt)
    res = {}
    for name, dtype, graph in (("fp64_plain", torch.complex128, False), ("fp32_graph", torch.complex64, True)):
        xs = torch.from_numpy(s1.psi).to(dev).to(dtype)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        E, D, N = ham.td_propagate(xs, nsteps, dt, graph=graph, **laser)
        el = time.perf_counter() - t0
        res[name] = (nsteps / el, E, D, N)
        del xs
    # ETRS (two half-step exponentials per step) and the density of the
    # propagated states, FP64, same system
    xs = torch.from_numpy(s1.psi).to(dev)
    ham.td_propagate(xs, 2, dt, graph=True, propagator="etrs", **laser)
    torch.cuda.synchronize()
    ns_e = 100 if args.small else 400
    t0 = time.perf_counter()
    ham.td_propagate(xs, ns_e, dt, graph=True, propagator="etrs", **laser)
    r_etrs = ns_e / (time.perf_counter() - t0)
    w = np.full(s1.psi.shape[1], 2.0)
    rho = dm.density(xs, w)
    ms_rho = _cuda_ms(lambda: dm.density(xs, w, rho=rho, accumulate=True), 20)
    # ghost rows of a two-slab partition of this mesh: device pack of the rows
    # partition 0 sends (hpsi_ghost_pack), compared with the H psi it feeds
    from hpsi.domain import partition_z
    doms = partition_z(m, 2)
    d0 = doms[0]
    smap, _ = d0.device_maps(dev)
    sbuf = torch.empty((smap.numel(), xs.shape[1]), dtype=xs.dtype, device=dev)
    lp = torch.zeros((d0.mesh.np_part, xs.shape[1]), dtype=xs.dtype, device=dev)
    lp[: d0.np_local + d0.np_ghost] = xs[torch.from_numpy(d0.global_rows[: d0.np_local + d0.np_ghost]).to(dev)]
    ms_pack = _cuda_ms(lambda: lib.ghost_pack(lp, smap, sbuf), 20)
    ghost_info = {"partitions": 2, "np_local": d0.np_local, "ghost_rows": d0.np_ghost,
                  "rows_sent": int(smap.numel()), "pack_ms": ms_pack,
                  "pack_GB_per_s": 2 * sbuf.numel() * sbuf.element_size() / ms_pack / 1e6,
                  "message_MB": sbuf.numel() * sbuf.element_size() / 1e6}
    del lp, sbuf
    # Lanczos step (TDLanczosTol = 1e-5, TDExpOrder 30) at dt = 0.05, ten times
    # the Taylor-4 limit on this grid; host-synchronised every Krylov iteration
    ham.lanczos_step(xs, 0.05, max_order=30, tol=1e-5)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lz_it, lz_res = ham.lanczos_step(xs, 0.05, max_order=30, tol=1e-5)
    torch.cuda.synchronize()
    ms_lz = (time.perf_counter() - t0) * 1e3
    del xs
    (r64, E64, D64, N64), (r32, E32, D32, N32) = res["fp64_plain"], res["fp32_graph"]
    emit({"config": f"TD exp_mid, sphere R=12 h=0.2, 128 states, KB, laser E0=0.01 w=0.057 sin^2, "
                    f"{nsteps} steps dt={dt}", "unit": "TD steps/s",
          "fp64_plain": r64, "fp32_graph": r32, "speedup_fp32_graph": r32 / r64,
          "energy_rel_err_max": float(np.max(np.abs(E32 - E64) / np.abs(E64))),
          "dipole_abs_err_max": float(np.max(np.abs(D32 - D64))),
          "dipole_rel_err_max": float(np.max(np.abs(D32 - D64)) / max(np.max(np.abs(D64)), 1e-300)),
          "norm_rel_err_max": float(np.max(np.abs(N32 - N64) / N64)),
          "etrs_fp64_graph_steps_per_s": r_etrs,
          "density_accumulate_fp64": {"ms": ms_rho, "GB_per_s": m.np * s1.psi.shape[1] * 16 / ms_rho / 1e6},
          "lanczos_fp64_dt0.05": {"ms": ms_lz, "krylov_dim": lz_it, "error_estimate": lz_res},
          "ghost_pack_fp64": ghost_info})
    del ham, dm

    # ---- 64 grouped systems of uneven size, 100 Taylor steps -----------------------
    systems = fixtures.config3(nsys=16 if args.small else 64)
    nsys = len(systems)
    hams, dms, xs64 = [], [], []
    pts = 0
    for sy in systems:
        d_ = lib.DeviceMesh(sy.mesh)
        h_ = lib.Hamiltonian(d_, laplacian_weights(sy.mesh.spacing), star_points(), v=sy.v, projectors=sy.proj)
        dms.append(d_)
        hams.append(h_)
        xs64.append(torch.from_numpy(sy.psi).to(dev))
        pts += sy.mesh.np * sy.nst
    sides = np.array([round(sy.mesh.np ** (1 / 3)) for sy in systems])
    nsts = np.array([sy.nst for sy in systems])
    grp = lib.Group(hams)
    out = {}
    steps = 100
    for name, dtype in (("fp64", torch.complex128), ("fp32", torch.complex64)):
        ys = [xx.to(dtype) for xx in xs64]
        grp.taylor_steps(ys, 2, 0.01)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        grp.taylor_steps(ys, steps, 0.01)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        out[name] = {"steps_per_s": steps / el, "Gpoint_states_per_s": pts * steps * 4 / el / 1e9}
        del ys
    emit({"config": f"{nsys} systems, cubic sides {int(sides.min())}..{int(sides.max())} (h=0.25), "
                    f"{int(nsts.min())}..{int(nsts.max())} states, 2..16 KB atoms; {steps} Taylor-4 steps dt=0.01, "
                    "persistent grouped launch + CUDA graph", "unit": "group steps/s (H.psi point-states/s: 4 per step)",
          "total_point_states": int(pts), **out})
    grp.close()
    del hams, dms, xs64

    # ---- adjoint gradient: 64^3, 16 states, 500 steps, checkpoint every 25 ----------
    s0 = fixtures.config0(nst=16)
    m = s0.mesh
    dm = lib.DeviceMesh(m)
    ham = lib.Hamiltonian(dm, laplacian_weights(m.spacing), star_points(), v=s0.v)
    nsteps = 100 if args.small else 500
    eps = np.random.default_rng(7).normal(0.0, 0.005, nsteps)
    psi0 = torch.from_numpy(s0.psi).to(dev)
    tg = torch.from_numpy(fixtures.random_states(m, 16, np.random.default_rng(8))).to(dev)
    # warm-up with the same call: the checkpoint workspace (3 GB at these sizes)
    # is allocated once per Hamiltonian, as in repeated optimiser iterations
    ham.adjoint_gradient(psi0, tg, eps, 0.01, ckpt=25)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    J, ge, gv, gc = ham.adjoint_gradient(psi0, tg, eps, 0.01, ckpt=25)
    el = time.perf_counter() - t0
    emit({"config": f"adjoint gradient, box 64^3 h=0.25, 16 states, {nsteps} steps dt=0.01, checkpoint 25",
          "unit": "s per gradient", "seconds": el, "forward_equiv_steps_per_s": nsteps / el, "J": J,
          "grad_eps_norm": float(np.linalg.norm(ge)), "grad_v_norm": float(np.linalg.norm(gv))})


def _adjoint_extra(dev, small):
    """Config 4 in the headline line: one adjoint gradient (64^3 box, 16 states,
    500 steps, checkpoints every 25), wall time around the call."""
    import torch
    from hpsi import fixtures, lib
    from hpsi.stencil import laplacian_weights, star_points
    s0 = fixtures.config0(nst=16)
    m = s0.mesh
    dm = lib.DeviceMesh(m)
    ham = lib.Hamiltonian(dm, laplacian_weights(m.spacing), star_points(), v=s0.v)
    nsteps = 100 if small else 500
    eps = np.random.default_rng(7).normal(0.0, 0.005, nsteps)
    psi0 = torch.from_numpy(s0.psi).to(dev)
    tg = torch.from_numpy(fixtures.random_states(m, 16, np.random.default_rng(8))).to(dev)
    # warm-up with the same call: the checkpoint workspace (3 GB at these sizes)
    # is allocated once per Hamiltonian, as in repeated optimiser iterations
    ham.adjoint_gradient(psi0, tg, eps, 0.01, ckpt=25)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    J, ge, gv, gc = ham.adjoint_gradient(psi0, tg, eps, 0.01, ckpt=25)
    el = time.perf_counter() - t0
    ham.close()
    dm.close()
    return {"workload": f"adjoint gradient, box 64^3 h=0.25, 16 states, {nsteps} steps dt=0.01, checkpoint 25",
            "seconds_per_gradient": el, "forward_equiv_steps_per_s": nsteps / el, "J": J,
            "grad_eps_norm": float(np.linalg.norm(ge))}


def _group_extra(dev, small, timed):
    """Config 3: uneven independent systems advanced together (one persistent
    stencil launch per Horner level, CUDA graph), FP64 and FP32 storage.
    Roofline: algorithmic bytes of a Taylor step, 14 S per point-state of the
    useful states (read psi once per level, write the level, update psi)."""
    import torch
    from hpsi import fixtures, lib
    from hpsi.stencil import laplacian_weights, star_points
    systems = fixtures.config3(nsys=16 if small else 64)
    hams, dms, xs = [], [], []
    pts = 0
    for sy in systems:
        d_ = lib.DeviceMesh(sy.mesh)
        h_ = lib.Hamiltonian(d_, laplacian_weights(sy.mesh.spacing), star_points(), v=sy.v, projectors=sy.proj)
        dms.append(d_)
        hams.append(h_)
        xs.append(torch.from_numpy(sy.psi).to(dev))
        pts += sy.mesh.np * sy.nst
    grp = lib.Group(hams)
    out = {"systems": len(systems), "point_states": int(pts), "steps": 10, "dt": 0.01}
    peak, _ = peaks()
    for name, dtype, S in (("fp64", torch.complex128, 16), ("fp32", torch.complex64, 8)):
        ys = [x.to(dtype) for x in xs]
        ms = timed(lambda: grp.taylor_steps(ys, 10, 0.01), 1, 1)
        alg = pts * 14 * S * 10
        out[name] = {"ms_per_taylor_step": ms / 10, "taylor_steps_per_s": 10 / (ms / 1e3),
                     "hpsi_Gpoint_states_per_s": 4 * pts * 10 / (ms / 1e3) / 1e9,
                     "roofline": {"achieved_GBs": alg / (ms / 1e3) / 1e9, "frac": alg / (ms / 1e3) / 1e9 / peak,
                                  "alg_bytes_per_step": alg / 10}}
        del ys
    grp.close()
    return out


def _box_extra(dev, timed, steps):
    """Config 0: 64^3 box, 32 states, kinetic + local H.psi, FP64 and FP32
    storage; roofline of the whole apply (2 S + 8/nst bytes per point-state)."""
    import torch
    from hpsi import fixtures, lib
    from hpsi.stencil import laplacian_weights, star_points
    s0 = fixtures.config0()
    m = s0.mesh
    dm = lib.DeviceMesh(m)
    ham = lib.Hamiltonian(dm, laplacian_weights(m.spacing), star_points(), v=s0.v)
    x = torch.from_numpy(s0.psi).to(dev)
    peak, _ = peaks()
    out = {"workload": "box 64^3 h=0.25 (np=262144), 32 states, kinetic + local"}
    for name, dtype, S in (("fp64", torch.complex128, 16), ("fp32", torch.complex64, 8)):
        xx = x.to(dtype)
        y = torch.zeros((m.np, 32), dtype=dtype, device=dev)
        ms = timed(lambda: ham.apply(xx, y), steps, 3)
        alg = m.np * 32 * 2 * S + m.np * 8
        out[name] = {"value": m.np * 32 * steps / (ms / 1e3) / 1e9, "unit": UNIT, "ms_per_step": ms / steps,
                     "roofline": {"achieved_GBs": alg / (ms / steps / 1e3) / 1e9,
                                  "frac": alg / (ms / steps / 1e3) / 1e9 / peak}}
    return out


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.configs:
        if rank == 0:
            run_configs(args)
        return

    import torch
    import torch.distributed as dist
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)

    sysm = build_system(args.small)
    m = sysm.mesh
    nst = sysm.psi.shape[1]
    dm = lib.DeviceMesh(m)
    ham = lib.Hamiltonian(dm, laplacian_weights(m.spacing), star_points(), v=sysm.v, projectors=sysm.proj)
    x = torch.from_numpy(sysm.psi).to(dev)
    y = torch.zeros((m.np, nst), dtype=torch.complex128, device=dev)
    st = torch.cuda.current_stream()

    ranks = Ranks(world, dev)
    barrier = ranks.barrier
    max_over_ranks = ranks.max

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1))

    # ---- headline: FP64 full H.psi, device resident ------------------------
    for _ in range(args.warmup):
        ham.apply(x, y)
    torch.cuda.synchronize()
    barrier()
    n0 = lib.launch_count()
    lib.profile_enable(True)
    with Clocks(local) as clk:
        ms = timed(lambda: ham.apply(x, y), args.steps, 0)
    launches = lib.launch_count() - n0
    npass, pass_ms = lib.profile_query("pass_fp64")
    nbra, bra_ms = lib.profile_query("bra_fp64")
    nket, ket_ms = lib.profile_query("ket_fp64")
    lib.profile_enable(False)
    ms_step = ms / args.steps
    value = world * m.np * nst * args.steps / (ms / 1e3) / 1e9
    sample = [i for i in SAMPLE_STATES if i < nst]
    y_sample = y[:, sample].cpu().numpy()

    # roofline of the dominant kernel (fused stencil pass).  Inside H.psi the
    # KB bra runs concurrently with the pass on a side stream, so the pass is
    # timed on its own as well (the same launches without the KB term: one
    # pass kernel per call) and the roofline uses that duration.
    S = 16
    alg_bytes = m.np * nst * 2 * S + m.np * 8.0  # read psi + write H psi, read v
    terms_kl = lib.TERM_KINETIC | lib.TERM_LOCAL_POTENTIAL
    pass_alone_ms = timed(lambda: ham.apply(x, y, terms=terms_kl), args.steps, 2) / args.steps
    pass_avg_ms = pass_alone_ms
    achieved = alg_bytes / (pass_avg_ms / 1e3) / 1e9
    peak, peak_kind = peaks()
    traffic = profile_traffic()

    extra = None
    e2e = None
    ke = 0
    if not args.no_extras:
        # ---- e2e through the C ABI with pinned host buffers (right after the timed
        # region, before the other workloads) --------------------------------------
        xh = torch.from_numpy(sysm.psi).pin_memory()
        yh = torch.zeros((m.np, nst), dtype=torch.complex128).pin_memory()
        ke = args.steps
        ham.apply(xh, yh)
        barrier()
        t0 = time.perf_counter()
        for _ in range(ke):
            ham.apply(xh, yh)
        torch.cuda.synchronize()
        el = max_over_ranks(time.perf_counter() - t0)
        e2e = world * m.np * nst * ke / el / 1e9

        # ---- extras: FP32 storage, Taylor steps ----------------------------------
        x32 = x.to(torch.complex64)
        y32 = y.to(torch.complex64)
        ms32 = timed(lambda: ham.apply(x32, y32), args.steps, 2)
        value32 = world * m.np * nst * args.steps / (ms32 / 1e3) / 1e9
        tk = max(2, args.steps // 4)
        xt = x.clone()
        ms_t64 = timed(lambda: ham.taylor_step(xt, 0.02), tk, 1)
        xt32 = x32.clone()
        ms_t32 = timed(lambda: ham.taylor_step(xt32, 0.02), tk, 1)
        # the Taylor step with the density of the propagated batch fused into its
        # last pass (the fuse_density_exp_apply of the reference's propagation)
        rho_t = torch.zeros(m.np, dtype=torch.float64, device=dev)
        wts = np.full(nst, 2.0)
        ms_td = timed(lambda: ham.taylor_step_density(xt, 0.02, wts, rho=rho_t), tk, 1)
        ms_rho = timed(lambda: dm.density(xt, wts, rho=rho_t), tk, 1)
        del xt, xt32

        # ---- TD steps (exp_mid + laser): FP64 plain launches vs FP32 graph replay --
        # dt = 0.005: at h = 0.2 the order-4 star Laplacian reaches E_max ~ 244 Ha, and
        # the 4th-order Taylor series is stable only for dt * E_max <= 2 sqrt(2); dt = 0.02
        # (dt * E_max = 4.9) diverges within a few steps in any implementation.  The
        # FP32-vs-FP64 observables are compared over the whole 200-step run.
        dt_td = 0.005
        ntd = 200
        laser = dict(E0=0.01, omega=0.057, T=ntd * dt_td)
        td = {}
        for name, xs, graph in (("td_fp64_plain", x.clone(), False), ("td_fp32_graph", x32.clone(), True)):
            xw = xs.clone()
            ham.td_propagate(xw, 1, dt_td, graph=graph, **laser)  # warm-up (workspaces, graph path)
            del xw
            torch.cuda.synchronize()
            barrier()
            t0 = time.perf_counter()
            E, D, N = ham.td_propagate(xs, ntd, dt_td, graph=graph, **laser)
            el = max_over_ranks(time.perf_counter() - t0)
            td[name] = {"steps_per_s": ntd / el, "ms_per_step": el / ntd * 1e3, "energy": E, "dipole": D, "norm": N}
            del xs
        e64, e32 = td["td_fp64_plain"].pop("energy"), td["td_fp32_graph"].pop("energy")
        d64, d32 = td["td_fp64_plain"].pop("dipole"), td["td_fp32_graph"].pop("dipole")
        nn64, nn32 = td["td_fp64_plain"].pop("norm"), td["td_fp32_graph"].pop("norm")
        td["fp32_vs_fp64"] = {"energy_rel_err_max": float(np.max(np.abs(e32 - e64) / np.abs(e64))),
                              "dipole_abs_err_max": float(np.max(np.abs(d32 - d64))),
                              "dipole_rel_err_max": float(np.max(np.abs(d32 - d64)) / max(np.max(np.abs(d64)), 1e-300)),
                              "norm_rel_err_max": float(np.max(np.abs(nn32 - nn64) / nn64)),
                              "steps": ntd, "dt": dt_td, "laser": "E0=0.01 w=0.057 sin^2 envelope over the run"}

        # ---- other configurations, measured in the same run --------------------------
        box = _box_extra(dev, timed, args.steps)
        group = _group_extra(dev, args.small, timed)
        adjoint = _adjoint_extra(dev, args.small)
        extra = {
            "fp32_storage_hpsi": {"value": value32, "unit": UNIT, "ms_per_step": ms32 / args.steps},
            "taylor4_fp64": {"steps_per_s": tk / (ms_t64 / 1e3), "ms_per_step": ms_t64 / tk},
            "taylor4_fp32": {"steps_per_s": tk / (ms_t32 / 1e3), "ms_per_step": ms_t32 / tk},
            "taylor4_fp64_with_density": {"ms_per_step": ms_td / tk, "ms_density_pass_alone": ms_rho / tk},
            **td,
            "config0_box64": box,
            "config3_group": group,
            "config4_adjoint": adjoint,
        }

    # ---- CPU baseline and the oracle check of the timed run (rank 0, N=1) -----
    cpu = None
    err = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, cores, kind, sample_txt, ref = cpu_reference_rate(sysm, sample)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample_txt}
        err = {"rel_maxnorm_per_state_max": rel_maxnorm_per_state(y_sample, ref), "states": sample,
               "tolerance": 1e-12, "of": "the FP64 H psi of the timed run vs the FP64 CPU oracle"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD + (" [small]" if args.small else ""),
                       "step": "one H.psi (kinetic + local + KB) over the whole batch",
                       "l2": "inputs (2.2 GB) larger than L2; no flush",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "traffic_kind": "ncu DRAM bytes (read + write) of one full-size launch of the same "
                                         "kernel (committed profile summary)",
                         "kernel": "pass_blk_kernel FP64 (fused stencil + local potential)",
                         "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": pass_avg_ms,
                         "timing": "pass alone (apply without the KB term), CUDA events over the launches"},
            "kernels": {"pass_fp64": {"launches": npass, "ms": pass_ms,
                                      "note": "inside H.psi, concurrent with the KB bra on a side stream"},
                        "bra_fp64": {"launches": nbra, "ms": bra_ms},
                        "ket_fp64": {"launches": nket, "ms": ket_ms}},
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        if e2e is not None:
            line["e2e"] = {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(m.np * nst * S),
                           "d2h_bytes_per_step": int(m.np * nst * S), "calls": ke}
        if extra is not None:
            line["extra"] = extra
        if err is not None:
            line["err_vs_oracle"] = err
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

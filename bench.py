#!/usr/bin/env python
"""Benchmark of the FDTD time-step loop on B200.

Workload (one GPU): the 256^3 gold nanorod dimer -- 40 nm rods, 10 nm
diameter, hemispherical caps, 2 nm gap along x -- with Drude + 2CP and the
hydrodynamic nonlocal current (beta = sqrt(3/5) v_F), 12-cell CPML, an
x-polarised TFSF plane wave along +z and the 6-face DFT flux boxes at 201
wavelengths (500-1200 nm), dx = 1 nm, S = 0.5.  Inputs are synthetic (the
geometry is rasterised on the host; fields start at zero).

A bench "step" is one block of 128 FDTD time steps: the launch period of the
stepper (32 DFT samples taken every 4 time steps and one FP64 phasor
contraction).  value = grid cells * time steps / seconds / 1e9, summed over
ranks (independent replicas, one per GPU: the reference is single-GPU and the
path is run as replicas only).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "fdtd-cuda_b200"))

METRIC = "Gcell-steps/s at 256^3 vs plain; adjoint/forward time ratio; batched sims/s"
BLOCK = 128  # time steps per bench step
WORKLOAD = ("256^3 Au rod dimer (40 nm rods, 10 nm diameter, 2 nm gap), Drude+2CP + "
            "hydrodynamic current, 12-cell CPML, TFSF x-polarised plane wave, "
            "201-wavelength DFT flux boxes, dx = 1 nm, S = 0.5")


def workload_params(mod, precision, grid=256, **over):
    """The 256^3 nonlocal rod-dimer configuration as fdtd_params (grid
    shrinks it for profiling captures)."""
    n_in = grid - 2 * 12 - 1
    kw = dict(
        Tend=20000, dx=1e-9, dy=1e-9, dz=1e-9, NCELLX=n_in, NCELLY=n_in, NCELLZ=n_in,
        NcpmlX=12, NcpmlY=12, NcpmlZ=12, material=3, first_medium=1, NUM_freq=201,
        WL_or_freq=1, lam_min=500e-9, lam_max=1200e-9, BandWidth=7e14, lam_0=705e-9,
        NONLOCAL=3, hydro_D=3.0, fermi_velocity=1.39e6, inc_phi_deg=90.0,
        geometry=1, axis=0, rod_length=40e-9, rod_diameter=10e-9, gap=2e-9,
        precision=precision,
    )
    kw.update(over)
    return mod.default_params(**kw)


def small_params(mod, precision, **over):
    """The small plain configuration: 64^3 total grid (43 + 2 * 10 + 1),
    dx = 2 nm, S = 0.5, a gold sphere of radius 10 nm at the centre
    (Drude + 2CP gold), 10-cell CPML with kappa_max = 1, the TFSF box 8
    cells inside the CPML, an x-polarised plane wave along +z whose pulse
    (centred at 600 nm, bandwidth 3e15) spans 400-900 nm, 2000 time steps
    and the 6-face DFT flux boxes at 101 wavelengths 400-900 nm."""
    kw = dict(
        Tend=1999, dx=2e-9, dy=2e-9, dz=2e-9, NCELLX=43, NCELLY=43, NCELLZ=43,
        NcpmlX=10, NcpmlY=10, NcpmlZ=10, cpml_kappa_max=1.0, tfsf_inset=8,
        nano_sphere=1, nano_sphere_radius=10e-9, material=3, first_medium=1,
        NUM_freq=101, WL_or_freq=1, lam_min=400e-9, lam_max=900e-9, lam_0=600e-9,
        BandWidth=3e15, inc_phi_deg=90.0, precision=precision,
    )
    kw.update(over)
    return mod.default_params(**kw)


# ----------------------------------------------------------------------
# helpers

class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.lines:
            return None
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profile_traffic(key):
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(key)
    except (OSError, ValueError):
        return None


def pass_bytes(dims, params, esize, which):
    """Algorithmic DRAM bytes of one E or H pass launch: each cell reads the
    three components it updates and the three of the other field and
    writes the three it updates (9 values per cell), and each psi value of
    the six CPML slabs is read and written once (E extent: Nc+1 cells per
    slab, H extent: Nc).  The material byte is read inside the dispersive
    bounding box only and is not counted."""
    nx, ny, nz = dims.nx, dims.ny, dims.nz
    n3 = (nx, ny, nz)
    total = nx * ny * nz * 9 * esize
    nc = (params.NcpmlX, params.NcpmlY, params.NcpmlZ)
    for ax in range(3):
        w = nc[ax] + 1 if which == "e" else nc[ax]
        # two slabs, two psi components each (the components other than ax)
        total += 2 * 2 * w * (nx * ny * nz // n3[ax]) * 2 * esize
    return total


# ----------------------------------------------------------------------
# the reference arm and the CPU baseline: the oracle port on host cores

def max_over_ranks(x, world, device):
    """The largest of a per-rank value over all ranks (the step time of the
    slowest replica), on the process group's device."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), or the platform string."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or platform.machine()


def cpu_sample(steps=200, grid=256, num_freq=201):
    """Times the FP64 CPU restatement (oracle) on the same workload over a
    fixed window of time steps after the first (which allocates the DFT
    accumulators); the window includes its DFT samples (every 4 steps)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cores = os.cpu_count() or 1
    O.lib().orc_set_threads(cores)
    p = workload_params(O, 1, grid=grid, NUM_freq=num_freq)
    s = O.OracleSim(p, threads=cores)
    s.step(1)
    t0 = time.perf_counter()
    s.step(steps)
    dt = time.perf_counter() - t0
    cells = s.shape[0] * s.shape[1] * s.shape[2]
    return {"value": cells * steps / dt / 1e9, "unit": "Gcell-steps/s", "cores": cores,
            "kind": "port", "cpu": cpu_model(),
            "sample": f"time steps 1-{steps} of the {grid}^3 workload (FP64, {steps // 4} DFT samples "
                      f"at {num_freq} wavelengths), {dt:.1f} s"}


def step_bytes(dims, params, st, esize):
    """Algorithmic DRAM bytes of one whole time step, by kernel family:
    the two Yee passes (pass_bytes), the TFSF table launch (per entry: the
    31-byte table row and a read-modify-write of one field value), the
    dispersive cells (per component and cell: 21 state and field values
    and the 16-byte cell entry; hydrodynamic cells add the density ring and
    the 48-byte neighbour list), the DFT sample (a field read and a ring
    write per row every dft_every steps) and the DFT contraction (per
    64 samples: the ring read and a read and write of the FP64 re/im
    accumulators of every row and frequency)."""
    out = {"e_pass": pass_bytes(dims, params, esize, "e"), "h_pass": pass_bytes(dims, params, esize, "h")}
    out["tfsf"] = (st.tfsf_entries_h + st.tfsf_entries_e) * (31 + 2 * esize)
    nd = sum(dims.n_metal_cells)
    out["dispersive"] = nd * ((21 + (3 if dims.hydro else 0)) * esize + 16 + (48 if dims.hydro else 0))
    every = max(params.dft_every, 1)
    out["dft_sample"] = st.dft_rows * 2 * esize / every
    out["dft_contract"] = st.dft_rows * (64 * esize + dims.num_freq * 32) / (64 * every)
    out["total"] = sum(out.values())
    return out


BATCH_SEED = 20261203


def batch_members(mod, n=64, steps=3000, seed=BATCH_SEED):
    """The batched workload: n independent gold-sphere simulations, cubic
    grids with total edges drawn uniformly from 48..128 cells, dx = 2 nm,
    Drude+2CP gold, 10-cell CPML, TFSF pulse centred at 600 nm, 51
    wavelengths 400-900 nm, FP32.  Sphere radii are drawn from 5-25 nm and
    clamped so that the sphere stays inside the absorption box of the grid
    (a TFSF inset of 4 and a box offset of 2 cells keep the smallest grids
    usable)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        edge = int(rng.integers(48, 129))
        r_nm = float(rng.uniform(5.0, 25.0))
        half_box = (edge - 2 * (10 + 4 + 2)) / 2.0  # cells from the centre to the abs box
        r_nm = min(r_nm, 2.0 * (half_box - 1.5))
        n_in = edge - 2 * 10 - 1
        out.append(mod.default_params(
            Tend=steps - 1, dx=2e-9, dy=2e-9, dz=2e-9, NCELLX=n_in, NCELLY=n_in, NCELLZ=n_in,
            NcpmlX=10, NcpmlY=10, NcpmlZ=10, nano_sphere=1, nano_sphere_radius=r_nm * 1e-9,
            material=3, first_medium=1, NUM_freq=51, WL_or_freq=1, lam_min=400e-9,
            lam_max=900e-9, lam_0=600e-9, BandWidth=3e15, tfsf_inset=4, box_offset=2,
            cpml_kappa_max=1.0, precision=mod.FDTD_FP32))
    return out


def batch_bench(mod, torch, stream, sp, dev, n, steps):
    """sims/s of the batched path (fdtd_batch_run: all members in one
    persistent pass kernel per half step) against the same members run one
    after another with fdtd_run, both timed with CUDA events on one stream;
    creation is outside both timed regions."""
    params = batch_members(mod, n, steps)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    b = mod.Batch(params, device=dev)
    torch.cuda.synchronize()
    ev[0].record(stream)
    b.run(sp)
    ev[1].record(stream)
    torch.cuda.synchronize()
    t_batch = ev[0].elapsed_time(ev[1]) / 1e3
    launches = b.stats()[0]
    tuning = b.tuning()
    for i in range(n):
        b.sim(i).check()
    cells = sum(p.NCELLX + 21 for p in params)
    b.close()
    t_seq = 0.0
    for p in params:
        s = mod.Sim(p, device=dev)
        torch.cuda.synchronize()
        ev[0].record(stream)
        s.run(sp)
        ev[1].record(stream)
        torch.cuda.synchronize()
        t_seq += ev[0].elapsed_time(ev[1]) / 1e3
        s.check()
        s.close()
    edges = [p.NCELLX + 21 for p in params]
    total = sum(e ** 3 for e in edges) * steps
    return {"sims_per_s": round(n / t_batch, 3), "sequential_sims_per_s": round(n / t_seq, 3),
            "speedup": round(t_seq / t_batch, 2), "members": n, "time_steps": steps,
            "batched_s": round(t_batch, 3), "sequential_s": round(t_seq, 3),
            "batched_gcell_steps_per_s": round(total / t_batch / 1e9, 2),
            "edges": [min(edges), max(edges)], "seed": BATCH_SEED, "gpu_launches": launches,
            "tuning": tuning}


def adjoint_params(mod, steps=4000, precision=None):
    """The adjoint workload: 96^3 grid (10-cell CPML), dx = 2 nm, FP32 fields,
    a 32 x 32 x 16-cell design region at the centre whose cells blend
    between vacuum and Drude+2CP gold, TFSF pulse centred at 600 nm and a
    wavelength grid of 1 nm steps from 550 to 785 nm so that 550, 633 and
    785 nm are DFT frequencies (indices 0, 83, 235)."""
    n_in = 96 - 2 * 10 - 1
    c = 48
    box = [c - 16, c + 16, c - 16, c + 16, c - 8, c + 8]
    return mod.default_params(
        Tend=steps - 1, dx=2e-9, dy=2e-9, dz=2e-9, NCELLX=n_in, NCELLY=n_in, NCELLZ=n_in,
        NcpmlX=10, NcpmlY=10, NcpmlZ=10, nano_sphere=0, material=3, first_medium=1,
        NUM_freq=236, WL_or_freq=1, lam_min=550e-9, lam_max=785e-9, lam_0=600e-9,
        BandWidth=3e15, design_box=box,
        precision=mod.FDTD_FP32 if precision is None else precision)


def large_params(mod, precision=None):
    """The large nonlocal workload: 384 x 384 x 256 grid, dx = 1 nm, 12-cell
    CPML, a 3 x 3 array of gold nanodisks (30 nm diameter, 10 nm high, 60 nm
    pitch) on a 20 nm dielectric slab (eps 2.25), hydrodynamic current,
    plane wave at normal incidence, 5 wavelengths 600-900 nm, FP32 fields."""
    return mod.default_params(
        Tend=11999, dx=1e-9, dy=1e-9, dz=1e-9, NCELLX=384 - 25, NCELLY=384 - 25, NCELLZ=256 - 25,
        NcpmlX=12, NcpmlY=12, NcpmlZ=12, material=3, first_medium=1, NUM_freq=5, WL_or_freq=1,
        lam_min=600e-9, lam_max=900e-9, lam_0=750e-9, BandWidth=7e14, NONLOCAL=3, hydro_D=3.0,
        fermi_velocity=1.39e6, geometry=2, disk_diameter=30e-9, disk_height=10e-9, pitch=60e-9,
        disk_nx=3, disk_ny=3, slab_eps=2.25, slab_thickness=20e-9,
        precision=mod.FDTD_FP32 if precision is None else precision)


def large_bench(mod, torch, stream, sp, dev, blocks=2, adjoint_steps=12000):
    """Forward throughput of the large nonlocal workload over a bounded
    number of 128-step blocks (the full run is 12000 steps), and the device
    memory the simulation holds (its adjoint: large_adjoint_bench)."""
    free0, _ = torch.cuda.mem_get_info(dev)
    s = mod.Sim(large_params(mod), device=dev)
    free1, _ = torch.cuda.mem_get_info(dev)
    s.step(2 * BLOCK, sp)  # warm-up: the two graphs of a DFT contraction period
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(stream)
    s.step(BLOCK * blocks, sp)
    ev[1].record(stream)
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1])
    s.check()
    d = s.dims
    cells = d.nx * d.ny * d.nz
    out = {"value": round(cells * BLOCK * blocks / (ms / 1e3) / 1e9, 3), "unit": "Gcell-steps/s",
           "grid": [d.nx, d.ny, d.nz], "time_steps": BLOCK * blocks,
           "dispersive_cells": list(d.n_metal_cells), "device_bytes": int(free0 - free1)}
    s.close()
    out["adjoint"] = large_adjoint_bench(mod, torch, dev, steps=adjoint_steps)
    return out


LARGE_DESIGN = [192 - 32, 192 + 32, 192 - 32, 192 + 32, 128, 138]  # 64 x 64 x 10 over the central disk
LARGE_FREQS = [0, 1, 2, 3, 4]


def large_adjoint_bench(mod, torch, dev, steps=12000, every=400):
    """The adjoint at the large geometry with the hydrodynamic model: a
    64 x 64 x 10 design region over the central disk (its cells blend
    between vacuum and the hydrodynamic metal), rho ~ U[0, 1] from the
    seed, objective = the absorption cross-section summed over the 5
    wavelengths, checkpoints every 400 steps, `steps` time steps (the whole
    12000-step run by default: the pulse, delayed by 4908 steps, has passed
    the disks); forward and backward throughput and the device memory the
    checkpoints and adjoint state take."""
    import numpy as np
    p = large_params(mod)
    p.Tend = steps - 1
    for a, v in enumerate(LARGE_DESIGN):
        p.design_box[a] = v
    b = LARGE_DESIGN
    free0, _ = torch.cuda.mem_get_info(dev)
    s = mod.Sim(p, device=dev)
    rng = np.random.default_rng(BATCH_SEED)
    s.set_design(rng.uniform(0, 1, (b[5] - b[4], b[3] - b[2], b[1] - b[0])))
    free1, _ = torch.cuda.mem_get_info(dev)
    s.forward(LARGE_FREQS, every)
    free2, _ = torch.cuda.mem_get_info(dev)
    s.backward()  # warm-up: buffers and the segment graphs
    free3, _ = torch.cuda.mem_get_info(dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    L = s.forward(LARGE_FREQS, every)
    t1 = time.perf_counter()
    g, gp = s.backward()
    t2 = time.perf_counter()
    s.check()
    st = s.stats()
    d = s.dims
    cs = d.nx * d.ny * d.nz * steps
    out = {"grid": [d.nx, d.ny, d.nz], "design": [64, 64, 10], "time_steps": steps,
           "full_run_steps": 12000, "checkpoint_every": every, "model": "hydrodynamic (Drude+2CP + nonlocal current)",
           "forward_s": round(t1 - t0, 3), "backward_s": round(t2 - t1, 3),
           "ratio": round((t2 - t1) / (t1 - t0), 3),
           "forward_gcell_steps_per_s": round(cs / (t1 - t0) / 1e9, 2),
           "backward_gcell_steps_per_s": round(cs / (t2 - t1) / 1e9, 2),
           "sim_bytes": int(free0 - free1),
           "forward_state_bytes": int(free1 - free2),
           "adjoint_state_bytes": int(free2 - free3),
           "recorded_steps": int(st.adj_record_steps), "record_bytes": int(st.adj_record_bytes),
           "checkpoints": int(st.adj_checkpoints),
           "memory_note": "forward_state_bytes: the adjoint state, the trajectory record of the recorded "
                          "steps and the checkpoints of the others, all allocated by the forward; the "
                          "backward recomputes only the steps that were not recorded",
           "objective": L, "grad_rho_max": float(np.abs(g).max()),
           "timing": "host wall clock around each blocking C-ABI call, after a warm-up pair"}
    s.close()
    return out


ADJOINT_FREQS = [0, 83, 235]


def adjoint_bench(mod, torch, stream, dev, steps=4000, every=200):
    """Forward (with checkpoints) and backward (segment recompute + reverse
    sweep) wall time of the adjoint workload; ratio = backward / forward."""
    import numpy as np
    p = adjoint_params(mod, steps)
    s = mod.Sim(p, device=dev)
    b = list(p.design_box)
    rng = np.random.default_rng(BATCH_SEED)
    s.set_design(rng.uniform(0, 1, (b[5] - b[4], b[3] - b[2], b[1] - b[0])))
    s.forward(ADJOINT_FREQS, every)  # warm-up: buffers, graphs
    s.backward()
    torch.cuda.synchronize()
    fw, bw = [], []
    for _ in range(3):  # median of three forward + backward pairs
        t0 = time.perf_counter()
        L = s.forward(ADJOINT_FREQS, every)
        t1 = time.perf_counter()
        g, gp = s.backward()
        t2 = time.perf_counter()
        fw.append(t1 - t0)
        bw.append(t2 - t1)
    s.check()
    st = s.stats()
    s.close()
    f_s, b_s = statistics.median(fw), statistics.median(bw)
    # a finite-difference check of one design cell: central differences
    # (h = 1e-3) of the FP64 forward objective against the FP32 adjoint
    q = adjoint_params(mod, steps, precision=mod.FDTD_FP64)
    s64 = mod.Sim(q, device=dev)
    rho = np.random.default_rng(BATCH_SEED).uniform(0, 1, (b[5] - b[4], b[3] - b[2], b[1] - b[0])).astype(np.float32)
    cell = (8, 16, 16)
    vals = []
    for d in (1e-3, -1e-3):
        r = rho.copy()
        r[cell] += d
        s64.set_design(r)
        vals.append(s64.forward(ADJOINT_FREQS, every))
    s64.close()
    fd = (vals[0] - vals[1]) / 2e-3
    cells = (96 ** 3) * steps
    out = {"forward_s": round(f_s, 4), "backward_s": round(b_s, 4),
           "ratio": round(b_s / f_s, 3), "objective": L,
           "objective_def": "absorption cross-section (m^2) summed over 550, 633, 785 nm",
           "grad_rho_max": float(np.abs(g).max()), "grad_params": [float(x) for x in gp],
           "fd_check": {"cell": list(cell), "adjoint": float(g[cell]), "fd_fp64": fd,
                        "rel": abs(float(g[cell]) - fd) / abs(fd)},
           "forward_gcell_steps_per_s": round(cells / f_s / 1e9, 2),
           "time_steps": steps, "checkpoint_every": every, "grid": 96, "design": [32, 32, 16],
           "recorded_steps": int(st.adj_record_steps), "record_bytes": int(st.adj_record_bytes),
           "checkpoints": int(st.adj_checkpoints),
           "timing": "host wall clock around each blocking C-ABI call, median of 3"}
    return out


def ref_deck_case(tend):
    """The reference-geometry deck used to time the reference's own CUDA
    build beside this one: the 256^3 grid of the workload (12-cell CPML,
    dx = 1 nm) with the reference's gold sphere (r = 10 nm) and its
    hydrodynamic model, 201 wavelengths."""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from ref_cases import BASE
    n_in = 256 - 2 * 12 - 1
    return dict(BASE, Tend=tend, dx=1e-9, dy=1e-9, dz=1e-9, NCELLX=n_in, NCELLY=n_in,
                NCELLZ=n_in, NcpmlX=12, NcpmlY=12, NcpmlZ=12, nano_sphere=1,
                nano_sphere_radius=10e-9, NUM_freq=201, NONLOCAL=3, BandWidth=7e14,
                lam_0=705e-9)


def ref_gpu_build(t1=40, t2=240):
    """Times the unmodified reference program (oracle/_ref/fdtd_ref, its own
    CUDA build for sm_100a) on the reference-geometry deck: wall time of two
    runs of t1 and t2 time steps, so that set-up and output cancel."""
    import shutil
    import tempfile
    binp = os.path.join(ROOT, "oracle", "_ref", "fdtd_ref")
    if not os.access(binp, os.X_OK):
        return {"unavailable": "oracle/_ref/fdtd_ref was not built"}
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from ref_cases import deck
    walls = []
    for tend in (t1, t2):
        d = tempfile.mkdtemp(prefix="fdtd_ref_")
        try:
            os.makedirs(os.path.join(d, "videofiles"), exist_ok=True)
            with open(os.path.join(d, "Input.txt"), "w") as f:
                f.write(deck(ref_deck_case(tend)))
            t0 = time.perf_counter()
            r = subprocess.run([binp], cwd=d, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE,
                               timeout=600)
            walls.append(time.perf_counter() - t0)
            if r.returncode != 0:
                return {"unavailable": f"reference exited {r.returncode}: "
                                       f"{r.stderr.decode(errors='replace')[-200:]}"}
        finally:
            shutil.rmtree(d, ignore_errors=True)
    cells = 256 ** 3
    rate = cells * (t2 - t1) / max(walls[1] - walls[0], 1e-9) / 1e9
    out = {"value": round(rate, 4), "unit": "Gcell-steps/s", "dtype": "f64",
           "deck": "256^3, Au sphere r = 10 nm, hydrodynamic model, 12-cell CPML, "
                   "201 wavelengths, dx = 1 nm",
           "method": f"wall time of {t2} minus {t1} time steps of the whole program",
           "wall_s": [round(w, 3) for w in walls]}
    # kernel time alone, from an ncu launch list of the same program on the
    # same deck (profiles/reference_cuda_kernels_256.md)
    try:
        with open(os.path.join(ROOT, "profiles", "reference_kernels.json")) as f:
            k = json.load(f)
        out["kernel_only"] = {"value": round(cells / (k["kernel_ms_per_step"] / 1e3) / 1e9, 4),
                              "unit": "Gcell-steps/s", "kernel_ms_per_step": k["kernel_ms_per_step"],
                              "source": "profiles/reference_cuda_kernels_256.md (ncu gpu__time_duration.sum, "
                                        f"{k['steps']} time steps)"}
    except (OSError, ValueError, KeyError):
        pass
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return
    cb = cpu_sample(grid=args.grid, num_freq=args.num_freq)
    line = {
        "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": cb["unit"],
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "note": "the reference has no CPU implementation; "
                   "this arm times the FP64 C restatement of its update equations (oracle/) "
                   "on all host cores"},
        "cpu_baseline": cb,
        "e2e": {"value": cb["value"], "unit": cb["unit"], "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if not args.no_ref_gpu:
        try:
            line["reference_cuda_build"] = ref_gpu_build()
        except Exception as e:  # reported, not fatal: the CPU arm stands
            line["reference_cuda_build"] = {"unavailable": f"{type(e).__name__}: {e}"[:200]}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------
# our arm

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    # a DFT contraction period is two bench steps (blocks): the defaults time
    # whole periods
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--grid", type=int, default=256, help="smaller grids for ncu captures")
    ap.add_argument("--num-freq", type=int, default=201)
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-large", action="store_true")
    ap.add_argument("--large-adjoint-steps", type=int, default=12000,
                    help="time steps of the large-geometry adjoint run (multiple of 400)")
    ap.add_argument("--batch-members", type=int, default=64)
    ap.add_argument("--batch-steps", type=int, default=3000)
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="reference arm: skip timing the reference's own CUDA build")
    ap.add_argument("--write-ref-deck", metavar="DIR",
                    help="write the reference-geometry deck (Input.txt, videofiles/) into DIR and exit: "
                         "the working directory for running or profiling the reference's own build")
    ap.add_argument("--ref-tend", type=int, default=40, help="Tend of the deck --write-ref-deck writes")
    args = ap.parse_args()
    if args.write_ref_deck:
        sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
        from ref_cases import deck
        os.makedirs(os.path.join(args.write_ref_deck, "videofiles"), exist_ok=True)
        with open(os.path.join(args.write_ref_deck, "Input.txt"), "w") as f:
            f.write(deck(ref_deck_case(args.ref_tend)))
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    import torch.distributed as dist
    if world > 1:
        # one process per GPU over NCCL; gloo where no GPU is present (the
        # CPU-only reference arm and the harness tests)
        timeout = __import__("datetime").timedelta(seconds=600)
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", device_id=torch.device("cuda", local), timeout=timeout)
        else:
            dist.init_process_group("gloo", timeout=timeout)

    if args.impl == "reference":
        run_reference(args, rank, world)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    import ctypes as C

    import numpy as np

    import fdtd_b200 as F
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks_(x):
        return max_over_ranks(x, world, "cuda")

    def timed_blocks(sim, k):
        st0 = sim.stats()
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            sim.step(BLOCK, sp)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = max_over_ranks_(e0.elapsed_time(e1))
        st1 = sim.stats()
        return ms, st1.kernels - st0.kernels

    # --- FP32 headline ----------------------------------------------------
    p32 = workload_params(F, F.FDTD_FP32, grid=args.grid, NUM_freq=args.num_freq)
    sim = F.Sim(p32, device=dev)
    d = sim.dims
    tune = sim.stats()
    cells = d.nx * d.ny * d.nz
    for _ in range(args.warmup):
        sim.step(BLOCK, sp)
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        ms, launches = timed_blocks(sim, args.steps)
    sim.check()
    value = world * cells * BLOCK * args.steps / (ms / 1e3) / 1e9

    # --- roofline of the dominant kernels ------------------------------------
    # each kernel alone, 20 launches back to back on this stream, timed with
    # CUDA events inside fdtd_time_kernel (the fields change; reset after)
    kms = {name: sim.time_kernel(which, 20, sp) for name, which in (
        ("e_pass", F.FDTD_KERNEL_E_PASS), ("h_pass", F.FDTD_KERNEL_H_PASS))}
    torch.cuda.synchronize()
    alg = pass_bytes(d, p32, 4, "e")
    alg_h = pass_bytes(d, p32, 4, "h")
    peak, peak_kind = measured_peak()
    achieved = alg / (kms["e_pass"] / 1e3) / 1e9
    sb = step_bytes(d, p32, tune, 4)
    step_ms = ms / args.steps / BLOCK
    step_gbs = sb["total"] / (step_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": "e_pass_s<float> (Yee + CPML E pass, whole grid)",
                "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4),
                "traffic": profile_traffic("e_pass_fp32_256"),
                "alg_bytes_per_launch": alg, "launch_ms": round(kms["e_pass"], 4),
                "peak_source": peak_kind,
                "h_pass": {"launch_ms": round(kms["h_pass"], 4),
                           "achieved": round(alg_h / (kms["h_pass"] / 1e3) / 1e9, 1),
                           "frac": round(alg_h / (kms["h_pass"] / 1e3) / 1e9 / peak, 4)},
                "step": {"alg_bytes": {k: int(v) for k, v in sb.items()},
                         "ms": round(step_ms, 5), "achieved": round(step_gbs, 1),
                         "frac": round(step_gbs / peak, 4),
                         "note": "all algorithmic bytes of one whole time step / (ms_per_step / 128)"}}

    # --- end to end through the public API with host buffers --------------
    # every bench step: pinned H2D of the block's source samples, the block,
    # pinned D2H of the block's probe rows (ex, ey, ez at the gap centre)
    sim.reset()
    src = torch.empty(BLOCK, dtype=torch.float64, pin_memory=True)
    src_np = src.numpy()
    pulse = F.coefficients(p32, 102)
    probe_host = torch.empty(BLOCK * 3, dtype=torch.float64, pin_memory=True)
    for _ in range(0 if args.no_e2e else args.warmup):
        t0 = sim.t
        src_np[:] = pulse[t0:t0 + BLOCK]
        sim.set_source(t0, BLOCK, src.data_ptr(), sp)
        sim.step(BLOCK, sp)
        sim.probe_range(t0, BLOCK, probe_host.data_ptr(), sp)
        stream.synchronize()
    barrier()
    w0 = time.perf_counter()
    for _ in range(0 if args.no_e2e else args.steps):
        t0 = sim.t
        src_np[:] = pulse[t0:t0 + BLOCK]
        sim.set_source(t0, BLOCK, src.data_ptr(), sp)
        sim.step(BLOCK, sp)
        sim.probe_range(t0, BLOCK, probe_host.data_ptr(), sp)
        stream.synchronize()
    w1 = time.perf_counter()
    barrier()
    e2e_s = max_over_ranks_(w1 - w0)
    e2e = None if args.no_e2e else {"value": round(world * cells * BLOCK * args.steps / e2e_s / 1e9, 3),
           "unit": "Gcell-steps/s", "h2d_bytes_per_step": BLOCK * 8,
           "d2h_bytes_per_step": BLOCK * 3 * 8,
           "note": "public C-ABI calls per step: fdtd_set_source (pinned H2D), fdtd_step, "
                   "fdtd_get_probe_range (pinned D2H), stream sync"}
    sim.close()

    # --- FP64 build of the same workload -----------------------------------
    fp64 = None
    if not args.no_fp64:
        sim64 = F.Sim(workload_params(F, F.FDTD_FP64, grid=args.grid, NUM_freq=args.num_freq),
                      device=dev)
        for _ in range(max(2, args.warmup)):  # both graphs of a DFT contraction period
            sim64.step(BLOCK, sp)
        torch.cuda.synchronize()
        ms64, _ = timed_blocks(sim64, args.steps)
        sim64.check()
        fp64 = {"value": round(world * cells * BLOCK * args.steps / (ms64 / 1e3) / 1e9, 3),
                "unit": "Gcell-steps/s", "ms_per_step": round(ms64 / args.steps, 3)}
        sim64.close()

    # --- the reference-geometry deck (Input.txt through fdtd_load_input_txt),
    # the one the reference's own CUDA build is timed on in the reference arm
    refdeck = None
    if not args.no_fp64 and args.grid == 256:
        import tempfile
        sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
        from ref_cases import deck
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "Input.txt")
            with open(path, "w") as f:
                f.write(deck(ref_deck_case(20000)))
            pr = F.load_input_txt(path)
        refdeck = {"deck": "256^3, Au sphere r = 10 nm, hydrodynamic model, 12-cell CPML, "
                           "201 wavelengths, dx = 1 nm (read from Input.txt)",
                   "unit": "Gcell-steps/s"}
        for prec, name in ((F.FDTD_FP64, "f64"), (F.FDTD_FP32, "f32")):
            pr.precision = prec
            sm = F.Sim(pr, device=dev)
            for _ in range(max(2, args.warmup)):  # both graphs of a DFT contraction period
                sm.step(BLOCK, sp)
            torch.cuda.synchronize()
            msr, _ = timed_blocks(sm, args.steps)
            sm.check()
            refdeck[name] = round(world * sm.dims.nx * sm.dims.ny * sm.dims.nz * BLOCK * args.steps
                                  / (msr / 1e3) / 1e9, 3)
            sm.close()

    large = None
    if not args.no_large and args.grid == 256:
        large = large_bench(F, torch, stream, sp, dev, adjoint_steps=args.large_adjoint_steps)

    adjoint = None
    if not args.no_adjoint and args.grid == 256:
        adjoint = adjoint_bench(F, torch, stream, dev)

    batched = None
    if not args.no_batch and args.grid == 256:
        batched = batch_bench(F, torch, stream, sp, dev, args.batch_members, args.batch_steps)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and args.grid == 256:
        cpu = cpu_sample()

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Gcell-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD if args.grid == 256 else f"{args.grid}^3 variant",
                       "grid": [d.nx, d.ny, d.nz],
                       "time_steps_per_step": BLOCK, "num_freq": d.num_freq,
                       "dispersive_cells": list(d.n_metal_cells),
                       "l2": "no flush: working set (403 MB of fields + 7 GB DFT) > 126 MB L2",
                       "dft_period": "one FP64 contraction of 64 samples per 2 steps (blocks), beside the "
                                     "steps; the timed steps " + ("cover whole periods" if args.steps % 2 == 0
                                                                  else "end half a period off (odd --steps)"),
                       "tuning": {k: getattr(tune, k) for k in ("h_stages", "h_minb", "h_ty", "h_kchunk", "h_eminb", "h_estages", "e_stages", "e_minb", "e_ty", "e_kchunk", "e_eminb", "e_estages", "h_pdl", "e_pdl", "h_tma", "h_etma", "e_tma", "e_etma", "h_ms", "e_ms")},
                       "parallelism": f"replicas x{world}"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "clocks": clk.summary(), "gpu_launches": launches, "fp64": fp64,
            "reference_deck": refdeck, "batched": batched, "adjoint": adjoint,
            "large_nonlocal": large,
        }
        if fp64 and cpu:
            # FP64 on the GPU against the FP64 CPU restatement (the headline
            # value is FP32)
            fp64["vs_cpu_baseline"] = round(fp64["value"] / cpu["value"], 1)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

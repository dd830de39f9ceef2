"""Benchmark of the B200 FDTD leapfrog step (one JSON line on rank 0).

Workload (N = 1): the 3-D dielectric-sphere case - 512^3 Yee grid, eps = 4
sphere of radius 0.3*N at the centre (stair-cased on cell centres), PML 16 on
every face, TF/SF plane wave theta = 30, phi = 45, psi = 0 (TF/SF box inset
32 cells), dx = 0.5 mm, lambda = 20 mm, Courant 0.5.  Synthetic input
(seeded, generated here).  One "step" is one leapfrog time step of the whole
grid.  Fields, PML auxiliaries and eps (~3.7 GB) are far larger than L2, so
no flush is needed between steps.

  value  : Gcell-updates/s of the chosen form (FP32 fused step), inputs
           resident in HBM, CUDA events on the library's stream, max over
           ranks.
  e2e    : the same metric through the C ABI with host buffers: each e2e
           step uploads eps from pinned host memory, advances a chunk of
           time steps and downloads Ez to pinned host memory, with the
           library's asynchronous copies (fdtd_upload_material_async /
           fdtd_download_field_async): a step's upload and the previous
           step's download run on the copy engines while the GPU computes.
  roofline: the field-update launches of one timed unit, timed together
           by CUDA events on the library's streams over the K steps that
           follow the timed region (those events cost about 1.5 % of a
           step, so `value` is measured without them): a pair of time steps on
           the two-step path (PML shell, two-step core, TF/SF pair passes),
           one time step on the single-step sweep (item classes, TF/SF post
           pass).  achieved = algorithmic bytes of the unit's cell-updates
           (cells * steps * B, B = 4*(12 + m + 12*f_PML) bytes per
           cell-update) over its measured time, against the measured HBM
           copy bandwidth.  A two-step pass reads and writes each value once
           for two steps, so its compulsory traffic is cells * B per pair:
           compulsory_frac (that over the time, against the same peak) is
           the fraction of the bandwidth the pass actually needs, and
           `traffic` (ncu DRAM bytes per unit, profiles/) shows what it moved.
  cpu_baseline: the reference fdtd3d CPU build (oracle/_ref/fdtd3d) on a
           bounded sample of the same physics (one process).

`--impl reference` runs only the reference CPU build on the host cores
(concurrent independent processes, one per core used) and prints its line.
Multi-GPU (--gpus N under torchrun): independent replicas, no collective
("scaling": "weak").
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gcell-updates/s"
N_DEFAULT = 512
PML = 16
TFSF = 32


def kernel_label(step_kernel: str) -> str:
    if step_kernel == "sweep2_tma":
        return ("sweep2_kernel (lean / z-edge core, two time steps per pass) + sweep3d_kernel (x/y PML shell, "
                "two single steps) + tfsf2_fused (TF/SF corrections of the pair): E and H of two time steps")
    if step_kernel == "sweep3d_tma":
        return ("sweep3d_kernel (lean / z-edge PML / PML / full item classes) + tfsf_post_kernel: "
                "E and H of one time step")
    return f"{step_kernel}: E and H of one time step"


def adjoint_extra(fd) -> dict:
    """Adjoint of the 2-D TMz objective at the benchmark size (512^2, PML 16,
    128^2 design of eps ~ U[1, 12] at the centre, Gaussian source 64 cells
    left of it, 16^2 probe 64 cells right of it, 4000 steps, checkpoint every
    200), FP32; wall time of the C-ABI calls, each after one warm-up call."""
    n, pml, steps, every = 512, 16, 4000, 200
    c = n // 2
    d0, d1 = c - 64, c + 64
    src = (d0 - 64, c)
    p0, p1 = (d1 + 64, c - 8), (d1 + 80, c + 8)
    rng = np.random.default_rng(2024)
    eps = np.ones((n, n))
    eps[d0:d1, d0:d1] = rng.uniform(1.0, 12.0, (128, 128)).astype(np.float32)
    kw = dict(mode=2, size=(n, n), use_pml=True, pml=pml, teta=90, phi=0, psi=90, point_source=(src[0], src[1], 0),
              point_source_mask=1 << 2, point_source_kind=1, point_source_bandwidth=0.5, precision=fd.PREC_FP32)
    with fd.Simulation(materials={"eps": eps}, **kw) as sim:
        sim.objective(steps, p0, p1, fd.PREC_FP32)
        t0 = time.perf_counter()
        j = sim.objective(steps, p0, p1, fd.PREC_FP32)
        tf = time.perf_counter() - t0
        sim.backward(steps, every, p0, p1, fd.PREC_FP32)
        t0 = time.perf_counter()
        _, g = sim.backward(steps, every, p0, p1, fd.PREC_FP32)
        tb = time.perf_counter() - t0
    return {"config": "TMz 512^2, PML 16, design 128^2, 4000 steps, checkpoint 200, FP32",
            "objective": j, "forward_s": tf, "backward_s": tb, "backward_over_forward": tb / tf,
            "design_grads_per_s": 128 * 128 / tb, "all_cell_grads_per_s": n * n / tb,
            "gradient_finite": bool(np.isfinite(g).all())}


def batch_extra(fd, steps: int = 1000) -> dict:
    """256 TMz instances, sides ~ U{64..1024} (seeded), eps of random 8x8-cell
    blocks ~ U[1, 12], PML 10, Gaussian point source at each centre, FP32:
    the tuned persistent batch launch (CUDA graph) against the same instances
    run one after another through fdtd_step."""
    rng = np.random.default_rng(4)
    sizes = [(int(a), int(b)) for a, b in rng.integers(64, 1025, (256, 2))]
    phys = dict(dx=0.0005, wavelength=0.02, courant=0.5, use_pml=True, pml=10, point_source_mask=1 << 2,
                point_source_kind=1, point_source_bandwidth=0.5, teta=90, phi=0, psi=90)
    eps = []
    for nx, ny in sizes:
        blocks = rng.uniform(1.0, 12.0, ((nx + 7) // 8, (ny + 7) // 8)).astype(np.float32)
        eps.append(np.kron(blocks, np.ones((8, 8)))[:nx, :ny].astype(np.float64))
    cells = sum(a * b for a, b in sizes)
    b = fd.Batch(sizes, **phys)
    for i, e in enumerate(eps):
        b.set_eps(i, e)
    shape = b.tune(8)
    b.step(3)
    b.sync()
    b.step(1, t_start=0)
    b.sync()
    t0 = time.perf_counter()
    b.step(steps, t_start=0)
    b.sync()
    tb = time.perf_counter() - t0
    del b
    t0 = time.perf_counter()
    for (nx, ny), e in zip(sizes, eps):
        with fd.Simulation(materials={"eps": e}, mode=2, size=(nx, ny), point_source=(nx // 2, ny // 2, 0),
                           precision=fd.PREC_FP32, **phys) as sim:
            sim.step(steps)
            sim.sync()
    ts = time.perf_counter() - t0
    return {"config": f"256 TMz instances, {cells} cells, {steps} steps, FP32", "tuned_shape": list(shape),
            "batch_value": cells * steps / tb / 1e9, "sequential_value": cells * steps / ts / 1e9,
            "unit": METRIC, "batch_s": tb, "sequential_s": ts, "speedup": ts / tb}


def precision_extra(fd, n: int, steps: int, every: int, eps: np.ndarray) -> dict:
    """The benchmark workload in the FP64 plain form, FP32 and FP16 storage
    side by side, every `every` steps (computed on the device): for each fast
    form the relative L2 of the E family (Ex, Ey, Ez together) and of the H
    family against FP64, the relative energy difference, and per field two
    figures: `raw` = the component's L2 error over its own FP64 norm, and
    `dominant` = that error over the largest FP64 norm among its family's
    three components.  With psi = 0 the incident wave has no Ez, so Ez holds
    only the scattered field and the TF/SF leakage and its own norm is far
    below Ex's; the dominant-field figure measures it against the field that
    sets the rounding scale."""
    import torch

    sims = {name: fd.Simulation(device=0, **workload_kw(n, prec))
            for name, prec in (("fp64", fd.PREC_FP64_PLAIN), ("fp32", fd.PREC_FP32), ("fp16s", fd.PREC_FP16S))}
    for sim in sims.values():
        sim.set_material("eps", eps)
    buf = {k: torch.empty(n ** 3, dtype=torch.float64, device="cuda:0") for k in ("ref", "cmp")}
    rows = []
    done = 0
    t0 = time.perf_counter()
    while done < steps:
        k = min(every, steps - done)
        for sim in sims.values():
            sim.step(k)
        done += k
        row = {"step": done}
        energy = {name: sim.reduce(fd.REDUCE_ENERGY)[0] for name, sim in sims.items()}
        ref_sq, err_sq = {}, {}
        for comp in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
            sims["fp64"].field_device(comp, buf["ref"].data_ptr())
            sims["fp64"].sync()
            ref_sq[comp] = float(torch.sum(buf["ref"] ** 2))
            for name in ("fp32", "fp16s"):
                sims[name].field_device(comp, buf["cmp"].data_ptr())
                sims[name].sync()
                err_sq[(name, comp)] = float(torch.sum((buf["cmp"] - buf["ref"]) ** 2))
        for name in ("fp32", "fp16s"):
            for fam, comps in (("E", ("Ex", "Ey", "Ez")), ("H", ("Hx", "Hy", "Hz"))):
                dom = max(ref_sq[c] for c in comps) ** 0.5
                row[f"{name}_{fam}_family"] = (sum(err_sq[(name, c)] for c in comps) /
                                               max(sum(ref_sq[c] for c in comps), 1e-300)) ** 0.5
                for c in comps:
                    e = err_sq[(name, c)] ** 0.5
                    row[f"{name}_{c}_raw"] = e / max(ref_sq[c] ** 0.5, 1e-300)
                    row[f"{name}_{c}_dominant"] = e / max(dom, 1e-300)
            row[f"{name}_energy"] = abs(energy[name] - energy["fp64"]) / max(abs(energy["fp64"]), 1e-300)
        rows.append(row)
    for sim in sims.values():
        sim.close()
    worst = {}
    for name in ("fp32", "fp16s"):
        keys = [k for k in rows[0] if k.startswith(name + "_") and not k.endswith("_raw")]
        worst[name] = max(max(r[k] for k in keys) for r in rows)
    return {"config": f"{n}^3 sphere workload, {steps} steps, relative to the FP64 plain form",
            "normalisation": "family = L2 error of Ex,Ey,Ez (or Hx,Hy,Hz) together over their FP64 norm; "
                             "<comp>_dominant = L2 error of the component over the largest FP64 component norm "
                             "of its family; <comp>_raw = over the component's own FP64 norm; energy = relative "
                             "difference of the total field energy",
            "worst_family_dominant_energy": worst, "seconds": time.perf_counter() - t0, "checkpoints": rows}


def drude_extra(fd, n: int = 384, steps: int = 3000) -> dict:
    """Drude slab 64 cells thick normal to z at the centre, eps_inf = 1,
    omega_p = 2 pi 30 GHz, gamma = 2 pi 1 GHz for eps and mu; plane wave at
    normal incidence (15 GHz, E along x), PML 16, TF/SF box 24 cells in,
    FP32; running DFT of Ex on the slab's back face every step.  The slab
    stops two cells inside the TF/SF box on the four side faces: a Drude
    medium that reaches into the PML grows without bound under the
    reference's update rules themselves."""
    z0 = n // 2 - 32
    z1 = z0 + 64
    tf = 24
    om = np.zeros((n, n, n), dtype=np.float32)
    ga = np.zeros((n, n, n), dtype=np.float32)
    side = slice(tf + 2, n - tf - 2)
    om[side, side, z0:z1] = np.float32(2 * np.pi * 30e9)
    ga[side, side, z0:z1] = np.float32(2 * np.pi * 1e9)
    kw = dict(mode=3, size=n, use_pml=True, pml=16, use_tfsf=True, tfsf_left=tf, tfsf_right=tf, teta=0.0,
              phi=0.0, psi=0.0, dx=0.0005, wavelength=0.02, courant=0.5, use_metamaterials=True,
              precision=fd.PREC_FP32)
    with fd.Simulation(**kw) as sim:
        for name in ("omegape", "omegapm"):
            sim.set_material(name, om)
        for name in ("gammae", "gammam"):
            sim.set_material(name, ga)
        del om, ga
        sim.dft_setup("Ex", 2, z1, [15e9])
        sim.step(3)
        sim.sync()
        t0 = time.perf_counter()
        sim.step(steps, t_start=3)
        sim.sync()
        t = time.perf_counter() - t0
        spec = sim.dft()
        kernel = sim.step_kernel
        ex_max = float(np.max(np.abs(sim.field("Ex"))))
    return {"config": f"{n}^3 Drude slab, {steps} steps, FP32, running DFT of Ex at z = {z1}",
            "value": n ** 3 * steps / t / 1e9, "unit": METRIC, "seconds": t, "kernel": kernel,
            "dft_max_abs": float(np.max(np.abs(spec))), "dft_finite": bool(np.isfinite(spec).all()),
            "ex_max_abs": ex_max}


def workload_kw(n: int, precision: int) -> dict:
    return dict(mode=3, size=n, use_pml=True, pml=PML, use_tfsf=True, tfsf_left=TFSF, tfsf_right=TFSF,
                teta=30.0, phi=45.0, psi=0.0, dx=0.0005, wavelength=0.02, courant=0.5, precision=precision)


def sphere_eps(n: int) -> np.ndarray:
    c = (np.arange(n, dtype=np.float64) + 0.5 - n / 2.0) ** 2
    r2 = (0.3 * n) ** 2
    eps = np.ones((n, n, n), dtype=np.float64)
    for i in range(n):
        inside = (c[i] + c[:, None] + c[None, :]) < r2
        eps[i][inside] = 4.0
    return eps


def algorithmic_bytes_per_cell(n: int, word: int) -> tuple[float, float]:
    """B per cell-update: word * (12 + m + 12 f_PML), m = 1 (eps)."""
    inner = n - 2 * PML
    f_pml = 1.0 - (inner / n) ** 3
    return word * (12 + 1 + 12 * f_pml), f_pml


def max_over_ranks(value: float, dist, device) -> float:
    """The largest of every rank's value (a timed region is as long as its
    slowest replica); the value itself without a process group."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world: int, cells: int, steps: int, ms: float) -> float:
    """Whole-job Gcell-updates/s: every replica advanced `cells` cells `steps`
    times within `ms` (the max over ranks)."""
    return world * cells * steps / (ms * 1e-3) / 1e9


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region
    (queries only, every 20 ms).  Entering starts the sampler and waits for
    its first line, so that samples cover even a short timed region; only
    the lines read after `mark()` count."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines: list[str] = []
        self.start = 0
        self._first = threading.Event()

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            self._first.wait(timeout=10.0)
        except OSError:
            self.proc = None
        return self

    def mark(self) -> None:
        """The timed region starts now."""
        self.start = len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())
            self._first.set()

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines[self.start:]:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def run_reference_sample(n: int, steps: int, procs: int = 1, timeout: int = 900) -> dict:
    """Times the reference CPU build on an n^3 sample with the workload's physics.

    Each process prints the reference's own 'Total time' (step loop only).
    The reference's time steps run from t = 0, which updates nothing (its
    t > 0 guard, Source/Scheme/Scheme.inc.h:1032), so `steps` time steps are
    steps - 1 cell-updates per cell.  Returns aggregate Gcell-updates/s over
    `procs` concurrent processes."""
    from oracle.oracle import REF_BIN, reference_args, write_material_txt

    if not os.path.exists(REF_BIN):
        raise FileNotFoundError(REF_BIN)
    kw = workload_kw(n, 0)
    kw.pop("precision")
    if n < 2 * TFSF + 16:
        raise ValueError("reference sample grid must keep the workload's PML 16 and TF/SF 32")
    if steps < 2:
        raise ValueError("the reference's first time step updates nothing: time at least two")
    updates = steps - 1
    with tempfile.TemporaryDirectory() as tmp:
        epath = os.path.join(tmp, "eps.txt")
        write_material_txt(epath, sphere_eps(n))
        args = [REF_BIN] + reference_args(steps=steps, **kw) + ["--load-eps-from-file", epath]
        ps = []
        for i in range(procs):
            d = os.path.join(tmp, f"p{i}")
            os.makedirs(d)
            ps.append(subprocess.Popen(args, cwd=d, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
        rates, times = [], []
        for p in ps:
            out, _ = p.communicate(timeout=timeout)
            if p.returncode != 0:
                raise RuntimeError(f"reference exited {p.returncode}: {out[-500:]}")
            t = None
            for line in out.splitlines():
                if line.startswith("Total time = "):
                    t = float(line.split("=")[1].split()[0])
            times.append(t)
            rates.append(n ** 3 * updates / t / 1e9)
    return {"value": sum(rates), "per_process": rates, "seconds": times, "grid": n, "steps": steps,
            "updates": updates, "pml": kw["pml"], "tfsf": kw["tfsf_left"]}


def reference_arm(args) -> None:
    """--impl reference: the reference CPU build on the host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    procs = max(1, min(os.cpu_count() or 1, args.ref_procs))
    n = args.ref_grid
    steps = max(2, min(args.steps + 1, args.ref_steps))
    try:
        r = run_reference_sample(n, steps, procs=procs)
    except Exception as e:  # the binary is built in-tree; report why if it is not there
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU build could not run: {e}"}))
        return
    sample = (f"{procs} concurrent reference processes, each {n}^3 x {steps} time steps ({r['updates']} "
              f"updates: the first time step updates nothing) of the sphere workload "
              f"(PML {r['pml']}, TF/SF {r['tfsf']}, theta 30, phi 45), --use-ca-cb --use-ca-cb-pml")
    line = {
        "impl": "reference", "metric": METRIC, "value": r["value"], "unit": "Gcell-updates/s",
        "n_gpus": args.gpus, "steps": r["updates"], "warmup": 0,
        "ms_per_step": max(r["seconds"]) * 1e3 / r["updates"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"3-D dielectric sphere (sample {n}^3 of the 512^3 case)", "grid": n,
                   "pml": r["pml"], "tfsf_inset": r["tfsf"], "parallelism": f"{procs} CPU processes"},
        "cpu_baseline": {"value": r["value"], "unit": "Gcell-updates/s", "cores": procs, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": r["value"], "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", type=int, default=N_DEFAULT)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp16s", "fp64"])
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--e2e-chunk", type=int, default=50)
    ap.add_argument("--plain-steps", type=int, default=10)
    ap.add_argument("--ref-grid", type=int, default=96)
    ap.add_argument("--ref-steps", type=int, default=30)
    ap.add_argument("--ref-procs", type=int, default=64)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the side measurements (plain FP64, FP16, "
                    "adjoint, batch, precision checkpoints)")
    ap.add_argument("--precision-steps", type=int, default=2000, help="steps of the FP64/FP32/FP16 comparison")
    ap.add_argument("--precision-every", type=int, default=200, help="checkpoint interval of that comparison")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        reference_arm(args)
        return

    import torch

    import fdtd3d_b200 as fd

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    prec = {"fp32": fd.PREC_FP32, "fp16s": fd.PREC_FP16S, "fp64": fd.PREC_FP64_PLAIN}[args.precision]
    word = {"fp32": 4, "fp16s": 2, "fp64": 8}[args.precision]
    n = args.grid
    cells = n ** 3
    eps = sphere_eps(n)

    sim = fd.Simulation(device=local, **workload_kw(n, prec))
    sim.set_material("eps", eps)
    stream = torch.cuda.ExternalStream(sim.stream, device=local)
    sim.step(args.warmup)
    sim.sync()

    # timed region: K time steps, events on the library's stream (the
    # library's per-unit kernel timing stays off here: its events cost about
    # 1.5 % of the step time; the roofline takes them over the next K steps)
    l0 = sim.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        clocks.mark()
        ev0.record(stream)
        sim.step(args.steps)
        ev1.record(stream)
        ev1.synchronize()
    sim.sync()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    sim_kernel = sim.step_kernel
    launches = sim.launch_count() - l0
    # roofline region: the next K steps with every timed unit bracketed by
    # CUDA events on the library's stream (fdtd_profile)
    sim.profile(True)
    ev2 = torch.cuda.Event(enable_timing=True)
    ev3 = torch.cuda.Event(enable_timing=True)
    ev2.record(stream)
    sim.step(args.steps)
    ev3.record(stream)
    ev3.synchronize()
    ms_prof = ev2.elapsed_time(ev3)
    kernel_ms, kernel_launches = sim.kernel_time()
    sim.profile(False)
    ms = max_over_ranks(ms, dist, f"cuda:{local}")
    value = job_rate(world, cells, args.steps, ms)

    # roofline of the field half-step kernel
    peaks = measured_peaks()
    b_cell, f_pml = algorithmic_bytes_per_cell(n, word)
    avg_launch_ms = kernel_ms / max(kernel_launches, 1)
    # one timed unit per time step on the single-step sweep path (the sweep
    # kernels of the three item classes plus the TF/SF post pass), one per
    # pair of time steps on the two-step path (shell, core and the TF/SF pair
    # passes); the per-cell kernels take two timed units (E, H) per step
    steps_per_launch = args.steps / max(kernel_launches, 1)
    bytes_per_launch = cells * b_cell * steps_per_launch
    achieved = bytes_per_launch / (avg_launch_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": None,
                "kernel": kernel_label(sim_kernel) if steps_per_launch > 0.75
                else "fast_half_kernel (E or H family)", "avg_launch_ms": avg_launch_ms,
                "time_steps_per_launch": round(steps_per_launch, 3),
                "bytes_per_launch": bytes_per_launch,
                "algorithmic_bytes_per_cell_update": b_cell, "f_pml": f_pml,
                "peak_source": peaks["source"], "kernel_share_of_step": kernel_ms / ms_prof,
                "measured_over": "the K time steps after the timed region, each timed unit bracketed by "
                                 "CUDA events on the library's stream (fdtd_profile)"}
    if steps_per_launch > 1.5:
        # a two-step pass needs each value read and written once for the
        # pair: its compulsory bytes are those of one single step
        compulsory = cells * b_cell
        roofline["compulsory_bytes_per_launch"] = compulsory
        roofline["compulsory_frac"] = compulsory / (avg_launch_ms * 1e-3) / 1e9 / peaks["hbm_gbs"]
    traffic_file = os.path.join(ROOT, "profiles", f"traffic_{args.precision}.json")
    if os.path.exists(traffic_file):
        entry = json.load(open(traffic_file)).get(sim_kernel)
        if entry and entry.get("grid") == n:
            if "bytes_per_launch" in entry:
                roofline["traffic"] = entry["bytes_per_launch"]
            else:   # a per-step figure (the FP64 form times half-steps)
                roofline["traffic"] = entry["bytes_per_step"] * steps_per_launch
            roofline["traffic_source"] = entry["source"]

    # e2e through the C ABI with pinned host buffers
    h_eps = torch.from_numpy(eps.reshape(-1)).pin_memory()
    h_out = torch.empty(cells, dtype=torch.float64).pin_memory()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    lib = fd.load_library()
    # one untimed e2e step: creates the copy streams and their staging grids
    sim._check(lib.fdtd_upload_material_async(sim._h, 0, h_eps.data_ptr()), "upload_material_async")
    sim.step(1)
    sim._check(lib.fdtd_download_field_async(sim._h, 2, h_out.data_ptr()), "download_field_async")
    sim.sync()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.e2e_steps):
        sim._check(lib.fdtd_upload_material_async(sim._h, 0, h_eps.data_ptr()), "upload_material_async")
        sim.step(args.e2e_chunk)
        sim._check(lib.fdtd_download_field_async(sim._h, 2, h_out.data_ptr()), "download_field_async")
    sim.sync()   # the copy streams too; e1 then marks the end of the last copy-out
    e1.record(stream)
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    e2e_ms = max_over_ranks(e2e_ms, dist, f"cuda:{local}")
    e2e_value = job_rate(world, cells, args.e2e_steps * args.e2e_chunk, e2e_ms)
    finite = bool(np.isfinite(h_out.numpy()).all())
    sim.close()

    extras = {}
    if not args.no_extras and rank == 0:
        for name, p2, w2 in (("plain_fp64", fd.PREC_FP64_PLAIN, 8), ("fp16_storage", fd.PREC_FP16S, 2)):
            if p2 == prec:
                continue
            s2 = fd.Simulation(device=local, **workload_kw(n, p2))
            s2.set_material("eps", eps)
            s2.step(3)
            s2.sync()
            st = torch.cuda.ExternalStream(s2.stream, device=local)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            s2.profile(True)
            a.record(st)
            s2.step(args.plain_steps)
            b.record(st)
            b.synchronize()
            kms, kl = s2.kernel_time()
            s2.close()
            t2 = a.elapsed_time(b)
            bc, _ = algorithmic_bytes_per_cell(n, w2)
            spl = args.plain_steps / max(kl, 1)
            extras[name] = {"value": cells * args.plain_steps / (t2 * 1e-3) / 1e9, "unit": METRIC,
                            "steps": args.plain_steps, "ms_per_step": t2 / args.plain_steps,
                            "hbm_frac": cells * bc * spl / (kms / max(kl, 1) * 1e-3) / 1e9 / peaks["hbm_gbs"]}
        if "plain_fp64" in extras:
            extras["speedup_vs_plain_fp64"] = value / world / extras["plain_fp64"]["value"]
            # the plain form moves D / B for every cell (the reference's
            # formulation): its own DRAM traffic per step, from an ncu capture
            tf64 = os.path.join(ROOT, "profiles", "traffic_fp64.json")
            entry = json.load(open(tf64)).get("plain_fp64") if os.path.exists(tf64) else None
            if entry and entry.get("grid") == n:
                pf = extras["plain_fp64"]
                pf["own_bytes_per_step"] = entry["bytes_per_step"]
                pf["own_traffic_frac"] = entry["bytes_per_step"] / (pf["ms_per_step"] * 1e-3) / 1e9 / peaks["hbm_gbs"]
                pf["own_traffic_source"] = entry["source"]
        # the reference's own CUDA FP64 path, measured on this GPU type by its
        # GPU test (tests/test_gpu_reference_cuda.py; not run by the bench)
        ref_cuda = os.path.join(ROOT, "profiles", "reference_cuda_fp64.json")
        if os.path.exists(ref_cuda):
            extras["reference_cuda_fp64"] = json.load(open(ref_cuda))
        for name, fn in (("adjoint_tmz", lambda: adjoint_extra(fd)), ("batch_tmz", lambda: batch_extra(fd)),
                         ("drude_slab", lambda: drude_extra(fd)),
                         ("precision", lambda: precision_extra(fd, n, args.precision_steps, args.precision_every,
                                                                eps))):
            try:
                extras[name] = fn()
            except Exception as e:  # reported, not hidden: the main line stays valid
                extras[name] = {"error": f"{type(e).__name__}: {e}"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            r = run_reference_sample(args.ref_grid, args.ref_steps, procs=1)
            cpu = {"value": r["value"], "unit": "Gcell-updates/s", "cores": 1, "kind": "reference",
                   "sample": f"reference CPU build, 1 process, {r['grid']}^3 x {r['steps']} time steps "
                             f"({r['updates']} updates) of the sphere workload (PML {r['pml']}, "
                             f"TF/SF {r['tfsf']}), --use-ca-cb --use-ca-cb-pml"}
        except Exception as e:
            cpu = {"value": None, "unit": "Gcell-updates/s", "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Gcell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": {"fp32": "f32", "fp16s": "f16-storage/f32-compute", "fp64": "f64"}[args.precision],
            "data": "synthetic",
            "config": {"workload": f"3-D dielectric sphere eps=4 r=0.3N, {n}^3, PML {PML}, TF/SF inset {TFSF}, "
                                   "theta=30 phi=45 psi=0, dx=0.5mm, lambda=20mm, Courant 0.5",
                       "grid": n, "form": args.precision, "l2": "inputs larger than L2 (no flush)",
                       "parallelism": f"{world} independent replicas" if world > 1 else "single GPU"},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "Gcell-updates/s", "h2d_bytes_per_step": cells * 8,
                    "d2h_bytes_per_step": cells * 8, "time_steps_per_e2e_step": args.e2e_chunk,
                    "result_finite": finite},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "extras": extras,
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

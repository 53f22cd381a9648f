"""Benchmark: Jacobian entries per second of the flat 2.5D ERT operator on B200.

Workload (one "step"): ``jacobian()`` of a fresh seeded model on the flat section (120 m x 40 m,
4961 nodes, 9600 P1 triangles, 48 electrodes, 1232 dipole-dipole rows, 17 wavenumbers):
assembly of 17 operators, their factorization, the secondary-field solve for 48 sources,
quadrature + ABMN measurement, and the 1232 x 9600 normal-quadrupole Jacobian.

* ``value``: D*C / step time with the models already in HBM and J left in HBM, timed per step
  with CUDA events on the launching stream; L2 is flushed (256 MiB write) between steps,
  outside the timed events.
* ``e2e``: the same metric through the public API, ``ERTForward2p5D.jacobian(sigma)`` with the
  model in pinned host memory and J returned to the host, wall-clock per call, in steady state:
  the untimed warm-up calls (at least the field cache's capacity + 2) fill the field cache and
  the page-locked result buffers, whose first allocation is a one-time cost.
* ``--impl reference``: the reference's CPU path (FP64 oracle fields + the C restatement of the
  reference kernel on all host threads), one model per step.
* ``--workload terrain``: the same metric on the 2.5D terrain section (200 m x 50 m, 40,000 P1
  triangles under a three-sinusoid surface with jittered interior columns, 96 electrodes at 1 m,
  2538 Wenner-Schlumberger + dipole-dipole rows, numerical geometric factors, 19 wavenumbers;
  fields on the H2-refined discretization of 160,000 triangles, 80,601 dofs); a step is one fresh
  correlated log-normal model's fields and the 2538 x 40,000 Jacobian summed from the refined
  cells. The line also carries the exact vjp and jvp times. No CPU baseline is run (the
  reference's set-up alone solves 19 x 96 systems of 321,201 dofs).
* ``--workload box3d``: the same metric for the 3D operator (``ERTForward3D.jacobian(sigma,
  batch_size=32)``, series_batch_steps=1): 60 m x 40 m x 20 m box of 244,800 P1 tetrahedra,
  12 x 8 surface electrodes, 4000 dipole-dipole rows (192 field columns with singularity
  removal); a step is one fresh model's factorization, current + receiver fields and the 4000 x
  244,800 Jacobian (3.9 GB, larger than L2, so no flush is needed). Its CPU baseline is the FP64
  oracle's fields for one model plus the reference contraction on a sample of rows.

Multi-GPU (torchrun): every rank runs its own models (time-lapse steps are independent), no
collective on the data path; value = all ranks' entries / max-over-ranks time ("weak").
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "ad-tlert_b200"))

L2_FLUSH_BYTES = 256 << 20


def parse_args():
    parser = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=20)
    parser.add_argument("--warmup", type=int, default=5)
    parser.add_argument("--impl", choices=("b200", "reference"), default="b200")
    parser.add_argument("--e2e-steps", type=int, default=None)
    parser.add_argument("--max-n", type=int, default=8, help="dipole-dipole n range (8: 1232 rows, 3: 612)")
    parser.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU baseline leg (profiling runs)")
    parser.add_argument("--tuning", choices=("auto", "default"), default="auto",
                        help="auto: launch shapes chosen by the library's autotuner before warm-up; default: the "
                             "library's built-in rules (fixed launch counts, for profiling captures)")
    parser.add_argument("--no-surrogate", action="store_true", help="timelapse workload: plain FEM pass only")
    parser.add_argument("--training-models", type=int, default=20_000, help="timelapse workload: surrogate training set")
    parser.add_argument("--windows", type=int, default=None,
                        help="timelapse workload: invert only the first K windows of this rank's share")
    parser.add_argument("--workload", choices=("flat", "terrain", "box3d", "box3d-small", "timelapse"), default="flat",
                        help="flat: the 2.5D headline section; terrain: the 2.5D terrain section (40,000 triangles, "
                             "96 electrodes, 2538 rows, numerical geometric factors); box3d: the 3D box (244,800 "
                             "tetrahedra, 96 electrodes, 4000 rows); box3d-small: the same survey on 36,000 "
                             "tetrahedra (profiling captures); timelapse: the 363-window Gauss-Newton inversion of "
                             "365 time steps on the flat section (windows/s)")
    return parser.parse_args()


def workload(max_n: int):
    from adtlert_b200 import synthetic

    nodes, cells, electrodes, rows = synthetic.flat_section(max_n)
    return nodes, cells, electrodes, rows


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group(backend, timeout=timedelta(seconds=120))
    return rank, world


def max_over_ranks(value: float, world: int) -> float:
    if world == 1:
        return value
    import torch.distributed as dist

    device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else torch.device("cpu")
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


class ClockSampler:
    """SM clock and throttle reasons sampled every `period_s` through NVML (read-only queries) while
    the GPU works: the sampler is started before the warm-up steps and stopped after the timed
    steps. The GPU is addressed by its PCI bus id, so the samples belong to the device torch
    uses whatever CUDA_VISIBLE_DEVICES or the CUDA device ordering is. Falls back to nvidia-smi
    (same PCI id, 100 ms) when NVML cannot be loaded."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, device_index: int, period_s: float = 0.010):
        props = torch.cuda.get_device_properties(device_index)
        self.pci = f"{props.pci_domain_id:08X}:{props.pci_bus_id:02X}:{props.pci_device_id:02X}.0"
        self.period_s = period_s
        self.samples: list[tuple[float, int, int]] = []  # (sm MHz, max MHz, reasons mask)
        self._stop = None
        self._thread = None
        self._proc = None
        self._path = None

    def _nvml_loop(self, handle, nvml):
        while not self._stop.is_set():
            try:
                self.samples.append((float(nvml.nvmlDeviceGetClockInfo(handle, nvml.NVML_CLOCK_SM)),
                                     int(nvml.nvmlDeviceGetMaxClockInfo(handle, nvml.NVML_CLOCK_SM)),
                                     int(nvml.nvmlDeviceGetCurrentClocksEventReasons(handle))))
            except Exception:  # noqa: BLE001 - a failed query only loses a sample
                pass
            self._stop.wait(self.period_s)

    def __enter__(self):
        import threading

        self._stop = threading.Event()
        try:
            import pynvml as nvml

            nvml.nvmlInit()
            handle = nvml.nvmlDeviceGetHandleByPciBusId(self.pci)
            self._thread = threading.Thread(target=self._nvml_loop, args=(handle, nvml), daemon=True)
            self._thread.start()
            return self
        except Exception:  # noqa: BLE001
            self._thread = None
        handle, self._path = tempfile.mkstemp(suffix=".csv")
        os.close(handle)
        fields = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                  "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(["nvidia-smi", f"--id={self.pci}", f"--query-gpu={fields}",
                                           "--format=csv,noheader,nounits", "-lms", "100"],
                                          stdout=open(self._path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self._proc = None
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread is not None:
            self._thread.join(timeout=5)
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()
            try:
                for line in Path(self._path).read_text().splitlines():
                    parts = [x.strip() for x in line.split(",")]
                    if len(parts) >= 6 and parts[0].replace(".", "").isdigit():
                        mask = sum(bit for (_, bit), flag in zip(self.REASONS, parts[2:6]) if flag.lower().startswith("active"))
                        self.samples.append((float(parts[0]), int(float(parts[1])), mask))
            finally:
                Path(self._path).unlink(missing_ok=True)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        reasons = sorted({name for _, _, mask in self.samples for name, bit in self.REASONS if mask & bit})
        return {"sm_mhz": statistics.median(s for s, _, _ in self.samples), "sm_max_mhz": float(self.samples[0][1]),
                "reasons": reasons, "samples": len(self.samples), "pci_bus_id": self.pci,
                "window": f"warm-up and timed steps, {1e3 * self.period_s:g} ms NVML samples"}


def measured_peaks() -> dict:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return {"hbm_gbs": data["hbm_gbs"], "bf16_tflops": data["bf16_tflops"], "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def ncu_traffic() -> dict:
    path = ROOT / "profiles" / "traffic.json"
    return json.loads(path.read_text()) if path.exists() else {}


def run_reference(args, rank: int, world: int) -> dict:
    """The reference's CPU path on the host cores, one full model per step (bounded sample)."""

    sys.path.insert(0, str(ROOT))
    from adtlert_b200 import synthetic
    from oracle import baseline
    from oracle.ert2p5d import Oracle2p5D

    if args.workload == "timelapse":
        return timelapse_reference(args, world)
    if args.workload == "terrain":
        return {"impl": "reference", "unavailable": "no CPU run of the terrain workload: the reference's set-up "
                                                    "alone solves 19 x 96 FP64 systems of 321,201 dofs"}
    if args.workload in BOX3D:
        nodes, cells, electrodes, rows = box3d_workload(args.workload)
        base = box3d_cpu_baseline(nodes, cells, electrodes, rows)
        value = base["value"]
        return {
            "metric": "jacobian_entries_per_second", "value": value, "unit": "entries/s", "n_gpus": world,
            "steps": 1, "warmup": 0, "ms_per_step": 1e3 * len(rows) * len(cells) / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": box3d_config(len(rows), len(cells), len(nodes), 192, world), "cpu_baseline": base,
            "e2e": {"value": value, "unit": "entries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
    nodes, cells, electrodes, rows = workload(args.max_n)
    oracle = Oracle2p5D(nodes, cells, electrodes, rows)
    D, C = len(rows), len(cells)
    threads = baseline.host_threads()
    baseline.build()
    for i in range(args.warmup):
        baseline.jacobian(oracle, synthetic.layered_model(nodes, cells, 10_000 + i), threads)
    times = []
    for i in range(args.steps):
        sigma = synthetic.layered_model(nodes, cells, i)
        start = time.perf_counter()
        baseline.jacobian(oracle, sigma, threads)
        times.append(time.perf_counter() - start)
    total = sum(times)
    value = D * C * args.steps / total
    sample = f"{args.steps} models x full jacobian ({D} x {C}): SuperLU fields + C contraction"
    return {
        "metric": "jacobian_entries_per_second",
        "value": value,
        "unit": "entries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "impl": "reference",
        "config": config(D, C, 17, 48, world),
        "cpu_baseline": {"value": value, "unit": "entries/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "entries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def timelapse_reference(args, world: int) -> dict:
    """The reference's driver restated by the FP64 oracle (SciPy SuperLU fields, dense
    Jacobians, CSR CGLS) on the host cores: one full window (window 100, up to 15 iterations)."""

    sys.path.insert(0, str(ROOT))
    from adtlert_b200 import synthetic
    from oracle.ert2p5d import Oracle2p5D
    from oracle.timelapse import OracleTimeLapse

    nodes, cells, electrodes, rows = synthetic.flat_section()
    rho = synthetic.infiltration_series(nodes, cells, TIMELAPSE_STEPS, seed=0)
    operator = Oracle2p5D(nodes, cells, electrodes, rows)
    clean = np.stack([operator.apparent_resistivity(1.0 / rho[t]) for t in range(100, 103)])
    noise = np.random.default_rng(1).standard_normal((TIMELAPSE_STEPS, len(rows)))[100:103]
    observed = clean * np.exp(TIMELAPSE_NOISE * noise)
    initial = np.tile(np.log(np.median(observed, axis=1))[:, None], (1, len(cells)))
    oracle = OracleTimeLapse(nodes, cells, electrodes, rows, data_std=float(np.log1p(TIMELAPSE_NOISE)))
    start = time.perf_counter()
    _, _, chi2, _ = oracle.invert_window(np.log(observed), initial)
    seconds = time.perf_counter() - start
    value = 1.0 / seconds
    sample = f"window 100 of 363: {len(chi2)} Gauss-Newton iterations of the FP64 oracle driver, {seconds:.1f} s"
    return {"metric": "windows_per_second", "value": value, "unit": "windows/s", "n_gpus": world, "steps": 1,
            "warmup": 0, "ms_per_step": 1e3 * seconds, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": timelapse_config(363, world, len(rows), len(cells)),
            "cpu_baseline": {"value": value, "unit": "windows/s", "cores": int(torch.get_num_threads()), "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "windows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def config(D, C, W, E, world) -> dict:
    return {
        "workload": f"2.5D flat jacobian(): {C} P1 triangles, 4961 nodes, {E} electrodes, {D} dipole-dipole rows, {W} wavenumbers; fresh model per step",
        "rows": D,
        "cells": C,
        "wavenumbers": W,
        "electrodes": E,
        "l2": "flushed between steps (256 MiB write, outside the timed events)",
        "parallelism": f"replicas x{world} (independent models per rank)",
    }


def terrain_config(D, C, N, W, E, world) -> dict:
    return {
        "workload": f"2.5D terrain jacobian(): {C} P1 triangles (H2-refined to {4 * C}, {N} dofs), {E} electrodes, "
                    f"{D} Wenner-Schlumberger + dipole-dipole rows, {W} wavenumbers, numerical geometric factors; "
                    f"fresh model per step",
        "rows": D,
        "cells": C,
        "dofs": N,
        "wavenumbers": W,
        "electrodes": E,
        "l2": "inputs larger than L2 (19 x 80,601 x 96 fields, the 406 MB Jacobian); no flush",
        "parallelism": f"replicas x{world} (independent models per rank)",
    }


def run_terrain(args, rank: int, world: int) -> dict | None:
    from adtlert_b200 import ERTForward2p5D, Mesh, Survey, _native, synthetic

    device = torch.device("cuda", torch.cuda.current_device())
    nodes, cells, surface, electrodes, rows = synthetic.terrain_section()
    forward = ERTForward2p5D.from_mesh_survey(Mesh.from_arrays(nodes, cells, surface_node_ids=surface),
                                              Survey.from_arrays(electrodes, rows),
                                              topographic_geometric_factor_mode="numerical")
    lib, plan = forward._lib, forward._plan
    W, N, E, D, C, Cd = forward.W, forward.N, forward.E, forward.D, forward.C, forward.Cd
    stream = torch.cuda.current_stream(device)
    handle = _native.stream_handle(device)
    models = torch.as_tensor(np.stack([synthetic.correlated_model(nodes, cells, 1000 * rank + i)
                                       for i in range(args.warmup + args.steps)]), device=device)
    fields = torch.empty((1, W, N, E), dtype=torch.float32, device=device)
    normal = torch.empty((1, D), dtype=torch.float64, device=device)
    recip = torch.empty_like(normal)
    Jd = torch.empty((D, Cd), dtype=torch.float32, device=device)
    columns = forward._columns(None, None, discretization=True)
    slot = 15
    tuned = (forward.autotune(torch.as_tensor(synthetic.correlated_model(nodes, cells, 99_999 + rank)), repeats=2)
             if args.tuning == "auto" else forward.tuning())

    def call(name, *a):
        _native.check(getattr(lib, name)(plan, *a), plan, name)

    def sensitivity(i):
        call("adt_normal_jacobian", _native.ptr(fields), 0, D, _native.ptr(Jd), handle)
        forward._aggregate(Jd, columns)

    stages = (
        ("factorize", lambda i: call("adt_factorize_fields", slot, _native.ptr(models[i]), 1, handle)),
        ("solve_fields", lambda i: call("adt_solve_fields", slot, _native.ptr(models[i]), 1, _native.ptr(fields), handle)),
        ("measure", lambda i: call("adt_measure", _native.ptr(fields), 1, _native.ptr(normal), _native.ptr(recip), None,
                                   handle)),
        ("normal_jacobian", sensitivity),
    )
    result = timed_stages(args, rank, world, forward, stages, device, stream)
    if result is None:
        return None
    value_s, stage_ms, stage_launches, clock, launches = result
    info = forward.plan_info
    K, R = 3, info["features"]
    algorithmic = {
        # J on the refined cells written, summed into model cells; fields, dofs, factors, ABMN read
        "normal_jacobian": 4 * D * Cd + 4 * D * Cd + 4 * D * C + 4 * W * N * E + 4 * K * Cd + 4 * R * K * Cd + 16 * D,
        "factorize": 8 * W * info["nnz"] + 8 * W * info["factor_doubles_per_system"] + 8 * W * N * E,
        "solve_fields": 8 * W * info["factor_doubles_per_system"] + 2 * 8 * W * N * E + 4 * W * N * E,
        "measure": 4 * W * E * E * 3 + 16 * D,
    }
    peaks = measured_peaks()

    def roofline(name):
        count = max(1, stage_launches[name])
        per_launch_s = stage_ms[name] / 1e3 / count
        achieved = algorithmic[name] / count / per_launch_s / 1e9
        return {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": None, "kernel": name,
                "algorithmic_bytes_per_launch": algorithmic[name] / count, "launch_ms": per_launch_s * 1e3,
                "peak_source": peaks["source"]}

    # exact derivatives of the resistances through the public API (factorization cached)
    sigma = models[args.warmup].cpu()
    g = torch.as_tensor(np.random.default_rng(5).standard_normal(D))
    delta = sigma * torch.as_tensor(np.random.default_rng(6).standard_normal(C) * 1e-2, dtype=torch.float32)
    forward.vjp(sigma, g), forward.jvp(sigma, delta)
    torch.cuda.synchronize(device)
    start = time.perf_counter()
    forward.vjp(sigma, g)
    torch.cuda.synchronize(device)
    vjp_ms = 1e3 * (time.perf_counter() - start)
    start = time.perf_counter()
    forward.jvp(sigma, delta)
    torch.cuda.synchronize(device)
    jvp_ms = 1e3 * (time.perf_counter() - start)

    e2e_steps = args.e2e_steps or 3
    e2e_warmup = max(args.warmup, forward.normal_field_cache_max_entries + 2)
    host_models = [torch.as_tensor(synthetic.correlated_model(nodes, cells, 50_000 + 1000 * rank + i)).pin_memory()
                   for i in range(e2e_steps + e2e_warmup)]
    for i in range(e2e_warmup):
        out = forward.jacobian(host_models[i])
    torch.cuda.synchronize(device)
    barrier(world)
    start = time.perf_counter()
    for i in range(e2e_steps):
        out = forward.jacobian(host_models[e2e_warmup + i])
    torch.cuda.synchronize(device)
    e2e_time = max_over_ranks(time.perf_counter() - start, world)
    assert out.shape == (D, C)
    if rank != 0:
        return None
    base = None
    if world == 1 and not args.no_cpu_baseline:
        base = terrain_cpu_baseline(forward, host_models[-1].numpy(), out.numpy())
    return {
        "metric": "jacobian_entries_per_second",
        "value": world * D * C * args.steps / value_s,
        "unit": "entries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * value_s / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 fields / f64 factorization",
        "data": "synthetic (seeded log-normal resistivity, 5 m correlation length)",
        "config": terrain_config(D, C, N, W, E, world),
        "roofline": roofline(max(stage_ms, key=stage_ms.get)),
        "sensitivity_roofline": roofline("normal_jacobian"),
        "stages_ms": stage_ms,
        "vjp_ms": vjp_ms,
        "jvp_ms": jvp_ms,
        "clocks": clock,
        "e2e": {"value": world * D * C * e2e_steps / e2e_time, "unit": "entries/s", "h2d_bytes_per_step": 4 * C,
                "d2h_bytes_per_step": forward.dtype.itemsize * D * C + 1, "ms_per_step": 1e3 * e2e_time / e2e_steps,
                "warmup_calls": e2e_warmup},
        "gpu_launches": int(launches),
        "autotune": tuned,
        "cpu_baseline": base,
    }


def terrain_cpu_baseline(forward, sigma, J, sample_rows: int = 128) -> dict:
    """The reference's CPU path for the terrain Jacobian on the host cores: FP64 SuperLU fields of
    all wavenumbers on the refined field discretization plus the C contraction over sampled rows
    (extrapolated to every row), checked against the GPU Jacobian on those rows."""

    sys.path.insert(0, str(ROOT))
    from adtlert_b200.discretization import exact_node_indices
    from oracle import baseline

    D, C = J.shape
    threads = baseline.host_threads()
    baseline.build()
    potential = forward.primary_potential_discretization
    selection = exact_node_indices(potential.dof_nodes, forward.discretization.dof_nodes)
    oracle = baseline.TerrainBaseline(forward._problem, forward._unit_potentials(potential)[..., selection])
    start = time.perf_counter()
    fields = oracle.fields(sigma)
    fields_s = time.perf_counter() - start
    rows = np.linspace(0, D - 1, sample_rows).astype(np.int64)
    start = time.perf_counter()
    expected = oracle.jacobian_rows(fields, rows, threads)
    rows_s = time.perf_counter() - start
    error = float((np.abs(J[rows] - expected).max(axis=1) / np.abs(expected).max(axis=1)).max())
    seconds = fields_s + rows_s * D / sample_rows
    return {"value": D * C / seconds, "unit": "entries/s", "cores": threads, "kind": "port",
            "sample": f"one model: FP64 SuperLU fields of all {forward.W} wavenumbers on the refined discretization "
                      f"({forward.N} dofs, {fields_s:.1f} s, one thread) + the C contraction on {sample_rows} of "
                      f"{D} rows ({rows_s:.1f} s, {threads} threads), extrapolated to {D} rows",
            "max_row_error_vs_gpu": error}


def timed_stages(args, rank, world, forward, stages, device, stream):
    """Warm-up, the timed steps (CUDA events per step, max over ranks) and a per-stage breakdown:
    (elapsed seconds, stage ms, stage launches, clock summary, launches in the timed region)."""

    def step(i):
        for _, fn in stages:
            fn(i)

    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(device.index) as clocks:
        for i in range(args.warmup):
            step(i)
        torch.cuda.synchronize(device)
        barrier(world)
        torch.cuda.synchronize(device)
        launches0 = forward.kernel_launches()
        for k in range(args.steps):
            events[k][0].record(stream)
            step(args.warmup + k)
            events[k][1].record(stream)
        torch.cuda.synchronize(device)
    launches = forward.kernel_launches() - launches0
    barrier(world)
    torch.cuda.synchronize(device)
    elapsed = max_over_ranks(sum(a.elapsed_time(b) for a, b in events) / 1e3, world)
    clock = clocks.summary()
    stage_ms, stage_launches = {}, {}
    for name, fn in stages:
        total = 0.0
        for k in range(3):
            i = args.warmup + (k % args.steps)
            for other_name, other in stages:
                if other_name == name:
                    break
                other(i)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            before = forward.kernel_launches()
            a.record(stream)
            fn(i)
            b.record(stream)
            stage_launches[name] = forward.kernel_launches() - before
            torch.cuda.synchronize(device)
            total += a.elapsed_time(b)
        stage_ms[name] = total / 3
    return elapsed, stage_ms, stage_launches, clock, launches


BOX3D = {"box3d": (60, 40, 17), "box3d-small": (30, 20, 10)}


def box3d_workload(name: str):
    from adtlert_b200 import synthetic

    nodes, cells = synthetic.box_section(*BOX3D[name])
    electrodes, rows = synthetic.grid_survey()
    return nodes, cells, electrodes, rows


def box3d_config(D, C, N, columns, world) -> dict:
    return {
        "workload": f"3D jacobian(batch_size=32): {C} P1 tetrahedra, {N} nodes, 96 electrodes (12 x 8 grid), "
                    f"{D} dipole-dipole rows, {columns} field columns; fresh model per step",
        "rows": D,
        "cells": C,
        "nodes": N,
        "field_columns": columns,
        "l2": "inputs larger than L2 (the 3.9 GB Jacobian); no flush",
        "parallelism": f"replicas x{world} (independent models per rank)",
    }


def run_box3d(args, rank: int, world: int) -> dict | None:
    from adtlert_b200 import ERTForward3D, Mesh3D, Survey, _native, synthetic

    device = torch.device("cuda", torch.cuda.current_device())
    nodes, cells, electrodes, rows = box3d_workload(args.workload)
    forward = ERTForward3D.from_mesh_survey(Mesh3D.from_arrays(nodes, cells), Survey.from_arrays(electrodes, rows),
                                            series_batch_steps=1)
    lib, plan = forward._lib, forward._plan
    N, D, C, cols = forward.N, forward.D, forward.C, forward.columns
    stream = torch.cuda.current_stream(device)
    handle = _native.stream_handle(device)
    models = torch.as_tensor(np.stack([synthetic.ellipsoid_model(nodes, cells, 1000 * rank + i)
                                       for i in range(args.warmup + args.steps)]), device=device)
    fields = torch.empty((1, 1, N, cols), dtype=torch.float32, device=device)
    normal = torch.empty((1, D), dtype=torch.float64, device=device)
    recip = torch.empty_like(normal)
    J = torch.empty((D, C), dtype=torch.float32, device=device)
    slot = 15
    tuned = (forward.autotune(torch.as_tensor(synthetic.ellipsoid_model(nodes, cells, 99_999 + rank)), repeats=2)
             if args.tuning == "auto" else forward.tuning())

    def call(name, *a):
        _native.check(getattr(lib, name)(plan, *a), plan, name)

    stages = (
        ("factorize", lambda i: call("adt_factorize", slot, _native.ptr(models[i]), 1, handle)),
        ("solve_fields", lambda i: call("adt_solve_fields", slot, _native.ptr(models[i]), 1, _native.ptr(fields), handle)),
        ("measure", lambda i: call("adt_measure", _native.ptr(fields), 1, _native.ptr(normal), _native.ptr(recip), None,
                                   handle)),
        ("normal_jacobian", lambda i: call("adt_normal_jacobian", _native.ptr(fields), 0, D, _native.ptr(J), handle)),
    )

    def step(i):
        for _, fn in stages:
            fn(i)

    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(device.index) as clocks:
        for i in range(args.warmup):
            step(i)
        torch.cuda.synchronize(device)
        barrier(world)
        torch.cuda.synchronize(device)
        launches0 = forward.kernel_launches()
        for k in range(args.steps):
            events[k][0].record(stream)
            step(args.warmup + k)
            events[k][1].record(stream)
        torch.cuda.synchronize(device)
    launches = forward.kernel_launches() - launches0
    barrier(world)
    torch.cuda.synchronize(device)
    elapsed_max = max_over_ranks(sum(a.elapsed_time(b) for a, b in events) / 1e3, world)
    value = world * D * C * args.steps / elapsed_max
    clock = clocks.summary()

    stage_ms, stage_launches = {}, {}
    for name, fn in stages:
        total = 0.0
        reps = 3
        for k in range(reps):
            i = args.warmup + (k % args.steps)
            for other_name, other in stages:
                if other_name == name:
                    break
                other(i)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            before = forward.kernel_launches()
            a.record(stream)
            fn(i)
            b.record(stream)
            stage_launches[name] = forward.kernel_launches() - before
            torch.cuda.synchronize(device)
            total += a.elapsed_time(b)
        stage_ms[name] = total / reps
    info = forward.plan_info
    K, R = cells.shape[1], info["features"]
    algorithmic = {
        # J write + current/receiver fields read + cell dofs + per-cell template factors + ABMN
        "normal_jacobian": 4 * D * C + 4 * N * cols + 4 * K * C + 4 * R * K * C + 16 * D,
        # CSR values read, dense factors written
        "factorize": 8 * info["nnz"] + 8 * info["factor_doubles_per_system"],
        # factors read by the forward and backward solves, right-hand side and fields
        "solve_fields": 2 * 8 * info["factor_doubles_per_system"] + 3 * 8 * N * cols,
        "measure": 4 * N * cols + 16 * D,
    }
    peaks = measured_peaks()

    def roofline(name):
        count = max(1, stage_launches[name])
        per_launch_s = stage_ms[name] / 1e3 / count
        achieved = algorithmic[name] / count / per_launch_s / 1e9
        return {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": None, "kernel": name,
                "algorithmic_bytes_per_launch": algorithmic[name] / count, "launch_ms": per_launch_s * 1e3,
                "peak_source": peaks["source"]}

    # end to end: pinned host model in, J (page-locked) out; the untimed calls fill the field cache
    # and allocate the page-locked result buffers
    e2e_steps = args.e2e_steps or 3
    e2e_warmup = max(3, min(args.warmup, forward.normal_field_cache_max_entries + 2))
    host_models = [torch.as_tensor(synthetic.ellipsoid_model(nodes, cells, 50_000 + 1000 * rank + i)).pin_memory()
                   for i in range(e2e_steps + e2e_warmup)]
    for i in range(e2e_warmup):
        out = forward.jacobian(host_models[i], batch_size=32)
        del out
    torch.cuda.synchronize(device)
    barrier(world)
    start = time.perf_counter()
    for i in range(e2e_steps):
        out = forward.jacobian(host_models[e2e_warmup + i], batch_size=32)
        del out
    torch.cuda.synchronize(device)
    e2e_time = max_over_ranks(time.perf_counter() - start, world)
    e2e = {"value": world * D * C * e2e_steps / e2e_time, "unit": "entries/s", "h2d_bytes_per_step": 4 * C,
           "d2h_bytes_per_step": 4 * D * C, "ms_per_step": 1e3 * e2e_time / e2e_steps, "warmup_calls": e2e_warmup}
    if rank != 0:
        return None
    result = {
        "metric": "jacobian_entries_per_second",
        "value": value,
        "unit": "entries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * elapsed_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 fields / f64 factorization",
        "data": "synthetic (seeded 100 ohm-m background with three ellipsoids)",
        "config": box3d_config(D, C, N, cols, world),
        "roofline": roofline(max(stage_ms, key=stage_ms.get)),
        "sensitivity_roofline": roofline("normal_jacobian"),
        "stages_ms": stage_ms,
        "clocks": clock,
        "e2e": e2e,
        "gpu_launches": int(launches),
        "autotune": tuned,
    }
    if world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = box3d_cpu_baseline(nodes, cells, electrodes, rows)
    return result


def box3d_cpu_baseline(nodes, cells, electrodes, rows, sample_rows: int = 256) -> dict:
    """The FP64 oracle's fields for one model (SciPy SuperLU: one factorization, 192 right-hand
    sides) plus the reference's per-entry contraction (the C restatement, all host threads) on a
    sample of rows, extrapolated to the full Jacobian. The contraction takes the current and the
    receiver fields stacked as the rows of one field array, with A, B pointing at current rows
    and M, N at receiver rows."""

    sys.path.insert(0, str(ROOT))
    from adtlert_b200 import synthetic
    from oracle import baseline
    from oracle.ert3d import Oracle3D

    sample = np.linspace(0, len(rows) - 1, sample_rows).astype(int)
    oracle = Oracle3D(nodes, cells, electrodes, rows)
    sigma = synthetic.ellipsoid_model(nodes, cells, 90_000).astype(float)
    start = time.perf_counter()
    current, receiver, _ = oracle.fields(sigma)
    fields_s = time.perf_counter() - start
    n_cur = current.shape[0]
    phi = np.vstack((current, receiver))[None]  # (1, S, N)
    S = phi.shape[1]
    a, b, m, n = (oracle.abmn[sample, i] for i in range(4))
    a = np.where(a >= n_cur, S, a)
    b = np.where(b >= n_cur, S, b)
    m = np.where(m >= receiver.shape[0], S, m + n_cur)
    n = np.where(n >= receiver.shape[0], S, n + n_cur)
    templates = np.where(oracle.pair_keep.reshape(-1, oracle.K, oracle.K), oracle.volume_templates, 0.0)[None]
    threads = baseline.host_threads()
    baseline.build()
    start = time.perf_counter()
    baseline.normal_sensitivity(phi, a, b, m, n, oracle.dofs, templates, threads)
    contraction_s = time.perf_counter() - start
    D, C = len(rows), len(cells)
    full = fields_s + contraction_s * D / sample_rows
    return {"value": D * C / full, "unit": "entries/s", "cores": threads, "kind": "port",
            "sample": f"one model: FP64 SuperLU fields {fields_s:.1f} s (SciPy, one thread) + the reference contraction "
                      f"of {sample_rows} of {D} rows on {threads} threads ({contraction_s:.2f} s), extrapolated to "
                      f"{D} x {C}"}


def run_b200(args, rank: int, world: int) -> dict | None:
    from adtlert_b200 import ERTForward2p5D, Mesh, Survey, synthetic
    from adtlert_b200 import _native

    device = torch.device("cuda", torch.cuda.current_device())
    nodes, cells, electrodes, rows = workload(args.max_n)
    forward = ERTForward2p5D.from_mesh_survey(Mesh.from_arrays(nodes, cells), Survey.from_arrays(electrodes, rows))
    lib, plan = forward._lib, forward._plan
    W, N, E, D, C = forward.W, forward.N, forward.E, forward.D, forward.C
    stream = torch.cuda.current_stream(device)
    handle = _native.stream_handle(device)
    total_models = args.warmup + args.steps
    models = torch.as_tensor(
        np.stack([synthetic.layered_model(nodes, cells, 1000 * rank + i) for i in range(total_models)]), device=device
    )
    fields = torch.empty((1, W, N, E), dtype=torch.float32, device=device)
    normal = torch.empty((1, D), dtype=torch.float64, device=device)
    recip = torch.empty_like(normal)
    J = torch.empty((D, C), dtype=torch.float32, device=device)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)
    slot = 15
    # launch shapes chosen by the library's autotuner on a model outside the timed set
    tuned = (forward.autotune(torch.as_tensor(synthetic.layered_model(nodes, cells, 99_999 + rank)), repeats=3)
             if args.tuning == "auto" else forward.tuning())

    def call(name, *a):
        _native.check(getattr(lib, name)(plan, *a), plan, name)

    def factorize(i):
        call("adt_factorize_fields", slot, _native.ptr(models[i]), 1, handle)

    def solve(i):
        call("adt_solve_fields", slot, _native.ptr(models[i]), 1, _native.ptr(fields), handle)

    def measure(i):
        call("adt_measure", _native.ptr(fields), 1, _native.ptr(normal), _native.ptr(recip), None, handle)

    def sensitivity(i):
        call("adt_normal_jacobian", _native.ptr(fields), 0, D, _native.ptr(J), handle)

    stages = (("factorize", factorize), ("solve_fields", solve), ("measure", measure), ("normal_jacobian", sensitivity))

    def step(i):
        for _, fn in stages:
            fn(i)

    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(device.index, period_s=0.002) as clocks:  # ~1 ms steps: sample densely
        for i in range(args.warmup):
            step(i)
        torch.cuda.synchronize(device)
        barrier(world)
        torch.cuda.synchronize(device)
        launches0 = forward.kernel_launches()
        for k in range(args.steps):
            flush.fill_(float(k))
            events[k][0].record(stream)
            step(args.warmup + k)
            events[k][1].record(stream)
        torch.cuda.synchronize(device)
    launches = forward.kernel_launches() - launches0
    barrier(world)
    torch.cuda.synchronize(device)
    elapsed = sum(a.elapsed_time(b) for a, b in events) / 1e3
    elapsed_max = max_over_ranks(elapsed, world)
    value = world * D * C * args.steps / elapsed_max
    clock = clocks.summary()

    # the same steps replayed from a captured CUDA graph of the chain (the model copied into the
    # graph's input buffer inside the timed events)
    graph = forward.jacobian_graph()
    for i in range(args.warmup):
        graph.sigma.copy_(models[i])
        graph.launch()
    torch.cuda.synchronize(device)
    barrier(world)
    graph_events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                    for _ in range(args.steps)]
    for k in range(args.steps):
        flush.fill_(float(k))
        graph_events[k][0].record(stream)
        graph.sigma.copy_(models[args.warmup + k])
        graph.launch()
        graph_events[k][1].record(stream)
    torch.cuda.synchronize(device)
    graph_s = max_over_ranks(sum(a.elapsed_time(b) for a, b in graph_events) / 1e3, world)
    graph_line = {"value": world * D * C * args.steps / graph_s, "unit": "entries/s",
                  "ms_per_step": 1e3 * graph_s / args.steps, "kernels_per_step": graph.kernels}
    graph.close()

    # per-stage breakdown (same workload, L2 flushed, after the timed region)
    stage_ms, stage_launches = {}, {}
    reps = max(3, min(args.steps, 10))
    for name, fn in stages:
        total = 0.0
        for k in range(reps):
            i = args.warmup + (k % args.steps)
            for other_name, other in stages:  # rebuild the inputs each stage needs
                if other_name == name:
                    break
                other(i)
            flush.fill_(1.0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            before = forward.kernel_launches()
            fn(i)
            stage_launches[name] = forward.kernel_launches() - before
            b.record(stream)
            torch.cuda.synchronize(device)
            total += a.elapsed_time(b)
        stage_ms[name] = total / reps
    info = forward.plan_info
    K, R = cells.shape[1], info["features"]
    algorithmic = {
        # J write + fields read + cell dofs + per-cell template factors + ABMN
        "normal_jacobian": 4 * D * C + 4 * W * N * E + 4 * K * C + 4 * R * K * C + 16 * D,
        # CSR values read, dense factors written, forward-reduced right-hand side written (float64)
        "factorize": 8 * W * info["nnz"] + 8 * W * info["factor_doubles_per_system"] + 8 * W * N * E,
        # factors read by the backward levels, right-hand side read, primary read, fields written
        "solve_fields": 8 * W * info["factor_doubles_per_system"] + 2 * 8 * W * N * E + 4 * W * N * E,
        "measure": 4 * W * E * E * 3 + 16 * D,
    }
    dominant = max(stage_ms, key=stage_ms.get)
    peaks = measured_peaks()
    def roofline(name):
        launches = max(1, stage_launches[name])
        per_launch_bytes = algorithmic[name] / launches
        per_launch_s = stage_ms[name] / 1e3 / launches
        achieved = per_launch_bytes / per_launch_s / 1e9
        measured = ncu_traffic().get(name)
        traffic = measured["dram_bytes_per_step"] / launches if measured else None
        return {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "kernel": name,
                "algorithmic_bytes_per_launch": per_launch_bytes, "launch_ms": per_launch_s * 1e3,
                "peak_source": peaks["source"]}

    # end to end through the public API: pinned host model in, J on the host out
    e2e_steps = args.e2e_steps or max(3, min(args.steps, 10))
    e2e_warmup = max(args.warmup, forward.normal_field_cache_max_entries + 2)
    host_models = [torch.as_tensor(synthetic.layered_model(nodes, cells, 50_000 + 1000 * rank + i)).pin_memory()
                   for i in range(e2e_steps + e2e_warmup)]
    for i in range(e2e_warmup):
        out = forward.jacobian(host_models[i])
    torch.cuda.synchronize(device)
    barrier(world)
    start = time.perf_counter()
    for i in range(e2e_steps):
        out = forward.jacobian(host_models[e2e_warmup + i])
    torch.cuda.synchronize(device)
    e2e_time = max_over_ranks(time.perf_counter() - start, world)
    e2e = {
        "value": world * D * C * e2e_steps / e2e_time,
        "unit": "entries/s",
        "h2d_bytes_per_step": 4 * C,
        "d2h_bytes_per_step": 4 * D * C + 1,  # J and the fields' finiteness flag
        "ms_per_step": 1e3 * e2e_time / e2e_steps,
        "warmup_calls": e2e_warmup,
    }
    assert out.shape == (D, C)

    if rank != 0:
        return None
    result = {
        "metric": "jacobian_entries_per_second",
        "value": value,
        "unit": "entries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * elapsed_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 fields / f64 factorization",
        "data": "synthetic (seeded layered models with Gaussian anomalies)",
        "config": config(D, C, W, E, world),
        "roofline": roofline(dominant),
        "sensitivity_roofline": roofline("normal_jacobian"),
        "stages_ms": stage_ms,
        "clocks": clock,
        "e2e": e2e,
        "gpu_launches": int(launches),
        "autotune": tuned,
        "graph": graph_line,
    }
    result["operations_ms"] = operation_timings(forward, nodes, cells, device)
    if world == 1 and not args.no_cpu_baseline:
        result["reference_kernel"] = reference_kernel(forward, fields, J, handle, flush, device, stream)
        result["cpu_baseline"] = cpu_baseline(args, nodes, cells, electrodes, rows)
        result["cpu_operations_ms"] = cpu_operation_timings(nodes, cells, electrodes, rows)
    return result


def operation_timings(forward, nodes, cells, device, reps: int = 5) -> dict:
    """Wall-clock ms (median of ``reps``) of the operator's other public calls on the workload,
    host tensors in and out (adtlert/forward/ert2p5d.py:697-943): solve of a fresh model (assembly,
    factorization, fields, measurement) and of a cached one, and the derivative products of a
    model whose fields are cached."""

    from adtlert_b200 import synthetic

    rng = np.random.default_rng(7)
    sigma = torch.as_tensor(synthetic.layered_model(nodes, cells, 70_000), dtype=torch.float32)
    g = torch.as_tensor(rng.standard_normal(forward.D), dtype=torch.float32)
    delta = sigma * torch.as_tensor(rng.standard_normal(forward.C) * 1e-2, dtype=torch.float32)
    fresh = [torch.as_tensor(synthetic.layered_model(nodes, cells, 71_000 + i), dtype=torch.float32)
             for i in range(reps + 2)]

    def timed(fn, count=reps):
        values = []
        for i in range(count + 2):
            torch.cuda.synchronize(device)
            start = time.perf_counter()
            fn(i)
            torch.cuda.synchronize(device)
            if i >= 2:
                values.append(1e3 * (time.perf_counter() - start))
        return statistics.median(values)

    forward.solve(sigma)
    return {
        "solve_fresh_model": timed(lambda i: forward.solve(fresh[i])),
        "solve_cached_fields": timed(lambda i: forward.solve(sigma)),
        "vjp": timed(lambda i: forward.vjp(sigma, g)),
        "jvp": timed(lambda i: forward.jvp(sigma, delta)),
        "normal_vjp": timed(lambda i: forward.normal_vjp(sigma, g)),
        "normal_jvp": timed(lambda i: forward.normal_jvp(sigma, delta)),
        "timing": f"wall clock, host tensors in and out, median of {reps} after 2 untimed calls",
    }


def cpu_operation_timings(nodes, cells, electrodes, rows) -> dict:
    """The same calls on the FP64 oracle (SciPy SuperLU per wavenumber), once each, ms; the
    oracle keeps no fields between calls, so every call solves its own fields as the reference's
    CPU path does without a cache."""

    sys.path.insert(0, str(ROOT))
    from adtlert_b200 import synthetic
    from oracle.ert2p5d import Oracle2p5D

    oracle = Oracle2p5D(nodes, cells, electrodes, rows)
    rng = np.random.default_rng(7)
    sigma = synthetic.layered_model(nodes, cells, 70_000).astype(float)
    g = rng.standard_normal(len(rows))
    delta = sigma * rng.standard_normal(len(cells)) * 1e-2
    out = {}
    for name, fn in (("solve_fresh_model", lambda: oracle.apparent_resistivity(sigma)),
                     ("vjp", lambda: oracle.vjp(sigma, g)), ("jvp", lambda: oracle.jvp(sigma, delta)),
                     ("normal_vjp", lambda: oracle.normal_vjp(sigma, g)),
                     ("normal_jvp", lambda: oracle.normal_jvp(sigma, delta))):
        oracle._fields_cache = {}
        start = time.perf_counter()
        fn()
        out[name] = 1e3 * (time.perf_counter() - start)
    out["cores"] = int(torch.get_num_threads())
    out["kind"] = "port"
    return out


def reference_kernel(forward, fields, J, handle, flush, device, stream, reps: int = 20) -> dict:
    """The reference's own GPU kernel (normal_sensitivity<float, 3>, adtlert/forward/kernels.py:132-178,
    built by nvcc for sm_100 from the reference's source into oracle/_ref) on the same fields,
    timed beside this library's Jacobian kernel in the same process (CUDA events, L2 flushed
    before every launch, median of ``reps``): once as one launch over all rows, once as the
    reference's jacobian() issues it (64-row launches and a torch.cat, ert2p5d.py:984-1010)."""

    sys.path.insert(0, str(ROOT))
    from adtlert_b200 import _native
    from oracle import reference_kernel as refk

    if not refk.available():
        return {"unavailable": "oracle/_ref not built (the reference tree is needed at build time)"}
    W, N, E, D, C = forward.W, forward.N, forward.E, forward.D, forward.C
    phi, a, b, m, n, cells, templates = refk.operator_inputs(forward, fields)
    out = torch.empty((D, C), dtype=torch.float32, device=device)
    chunk = min(D, 64) if C >= 4096 else D

    def one_launch():
        refk.normal_sensitivity(phi, a, b, m, n, cells, templates, out, stream)

    def reference_chunking():
        parts = []
        for start in range(0, D, chunk):
            part = torch.empty((min(chunk, D - start), C), dtype=torch.float32, device=device)
            sl = slice(start, start + part.shape[0])
            refk.normal_sensitivity(phi, a[sl], b[sl], m[sl], n[sl], cells, templates, part, stream)
            parts.append(part)
        return torch.cat(parts)

    def ours():
        _native.check(forward._lib.adt_normal_jacobian(forward._plan, _native.ptr(fields), 0, D, _native.ptr(J), handle),
                      forward._plan, "adt_normal_jacobian")

    times = {"one": [], "chunked": [], "ours": []}
    for rep in range(reps + 3):
        for name, fn in (("one", one_launch), ("chunked", reference_chunking), ("ours", ours)):
            flush.fill_(float(rep))
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            fn()
            end.record(stream)
            torch.cuda.synchronize(device)
            if rep >= 3:
                times[name].append(start.elapsed_time(end))
    chunked = reference_chunking()
    one_launch()
    torch.cuda.synchronize(device)
    scale = float(out.abs().max())
    parity = float((out - J).abs().max()) / scale
    parity_chunked = float((chunked - out).abs().max()) / scale
    ms = {name: statistics.median(v) for name, v in times.items()}
    algorithmic = 4 * D * C + 4 * W * N * E + 4 * 3 * C + 4 * 9 * W * C + 16 * D  # J, fields, dofs, templates, ABMN
    peak = measured_peaks()["hbm_gbs"]
    return {
        "kernel": "reference normal_sensitivity<float, 3> (its source, nvcc -gencode arch=compute_100,code=sm_100, "
                  "blocks of 32 cells x 4 rows)",
        "ms_one_launch": ms["one"],
        "ms_reference_chunking": ms["chunked"],
        "launches_reference_chunking": -(-D // chunk),
        "ms_ours": ms["ours"],
        "ratio_one_launch": ms["one"] / ms["ours"],
        "ratio_reference_chunking": ms["chunked"] / ms["ours"],
        "hbm_frac_reference_one_launch": algorithmic / (ms["one"] * 1e-3) / 1e9 / peak,
        "parity_max_rel_vs_ours": parity,
        "parity_chunked_vs_one_launch": parity_chunked,
        "timing": f"median of {reps} launches each, L2 flushed before every launch, CUDA events on the launching stream",
    }


def cpu_baseline(args, nodes, cells, electrodes, rows) -> dict:
    sys.path.insert(0, str(ROOT))
    from adtlert_b200 import synthetic
    from oracle import baseline
    from oracle.ert2p5d import Oracle2p5D

    oracle = Oracle2p5D(nodes, cells, electrodes, rows)
    threads = baseline.host_threads()
    baseline.build()
    count, total = 0, 0.0
    while count < 3 or (total < 10.0 and count < 10):
        sigma = synthetic.layered_model(nodes, cells, 90_000 + count)
        start = time.perf_counter()
        baseline.jacobian(oracle, sigma, threads)
        total += time.perf_counter() - start
        count += 1
    D, C = len(rows), len(cells)
    return {"value": D * C * count / total, "unit": "entries/s", "cores": threads, "kind": "port",
            "sample": f"{count} models x full jacobian ({D} x {C}): FP64 SuperLU fields + C contraction, {total:.1f} s"}


TIMELAPSE_STEPS = 365
TIMELAPSE_NOISE = 0.02


def timelapse_workload():
    """Flat section, 365-step infiltration series and its noisy observed apparent resistivities
    (FEM of every step by this library, times exp(0.02 N(0, 1)), seed 1)."""

    from adtlert_b200 import ERTForward2p5D, Mesh, Survey, synthetic

    nodes, cells, electrodes, rows = synthetic.flat_section()
    forward = ERTForward2p5D.from_mesh_survey(Mesh.from_arrays(nodes, cells), Survey.from_arrays(electrodes, rows))
    rho = synthetic.infiltration_series(nodes, cells, TIMELAPSE_STEPS, seed=0)
    clean = np.concatenate([forward.apparent_resistivity_series(torch.as_tensor(1.0 / rho[i:i + 8], dtype=torch.float32))
                            .numpy() for i in range(0, TIMELAPSE_STEPS, 8)]).astype(float)
    observed = clean * np.exp(TIMELAPSE_NOISE * np.random.default_rng(1).standard_normal(clean.shape))
    initial = np.tile(np.log(np.median(observed, axis=1))[:, None], (1, len(cells)))
    return forward, nodes, cells, electrodes, rows, rho, clean, observed, initial


def timelapse_config(windows, world, D, C) -> dict:
    return {
        "workload": f"time-lapse Gauss-Newton inversion: {TIMELAPSE_STEPS} steps on the 2.5D flat section ({C} cells, "
                    f"{D} rows, 17 wavenumbers), {windows} windows of 3 steps, first-order spatial (50) and temporal "
                    f"(10) smoothness, CGLS 60 iterations, line search, at most 15 iterations per window (the "
                    f"reference's settings; a window the surrogate screen starts warm adds the screen's stop rules "
                    f"and CGLS count, reported under screening.warm_start_stop_rules)",
        "windows": windows,
        "steps": TIMELAPSE_STEPS,
        "cells": C,
        "rows": D,
        "noise": "2 % multiplicative (data_std log1p(0.02))",
        "l2": "inputs larger than L2 (three 47 MB Jacobians per window, re-read by every CGLS iteration); no flush",
        "parallelism": f"windows split across {world} rank(s) (window_share), no collective on the data path",
    }


def timed_inversion(inversion, observed, initial, windows, screen, device, world):
    """One pass over ``windows``: CUDA-event time (max over ranks), wall time with host arrays in
    and host models out, the result, and the library launches."""

    stream = torch.cuda.current_stream(device)
    torch.cuda.synchronize(device)
    barrier(world)
    launches0 = inversion.forward.kernel_launches()
    begin, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    wall = time.perf_counter()
    begin.record(stream)
    result = inversion.run(np.log(observed), initial, windows=windows, screen=screen)  # host arrays in
    end.record(stream)
    host_models = result.final_log_models.cpu()  # host result out
    wall = time.perf_counter() - wall
    launches = inversion.forward.kernel_launches() - launches0
    return max_over_ranks(begin.elapsed_time(end) / 1e3, world), max_over_ranks(wall, world), result, launches, host_models


def inversion_misfit(inversion, result, observed, clean) -> dict:
    covered = result.covered.cpu().numpy()
    predicted, _ = inversion.linearize(result.final_log_models[result.covered], jacobian=False)
    predicted = np.exp(predicted.cpu().numpy())
    iterations = [w["iterations"] for w in result.windows]
    chi2 = [w["final_chi2"] for w in result.windows]
    return {"final_chi2_mean": float(np.mean(chi2)), "final_chi2_max": float(np.max(chi2)),
            "rhoa_rms_rel_error_vs_observed": float(np.sqrt(np.mean((predicted / observed[covered] - 1.0) ** 2))),
            "rhoa_rms_rel_error_vs_noise_free": float(np.sqrt(np.mean((predicted / clean[covered] - 1.0) ** 2))),
            "iterations_mean": float(np.mean(iterations)), "iterations_max": int(np.max(iterations)),
            "linearized_models": inversion.linearize.evaluations}, predicted


def train_surrogate(forward, count: int, device) -> tuple:
    """Training set from the FEM, the trained surrogate, and its report (times, held-out error,
    GEMM throughput of a training step measured with CUDA events)."""

    from adtlert_b200.surrogate import Surrogate, training_set

    torch.cuda.synchronize(device)
    start = time.perf_counter()
    models, data = training_set(forward, count + 1024, seed=11)
    torch.cuda.synchronize(device)
    data_s = time.perf_counter() - start
    surrogate = Surrogate(forward, seed=0)
    start = time.perf_counter()
    history = surrogate.fit(models[:count], data[:count], epochs=30)
    torch.cuda.synchronize(device)
    train_s = time.perf_counter() - start
    held_out = surrogate.predict_log10(models[count:])
    error = (10.0 ** (held_out - data[count:]) - 1.0).double()
    # one training step timed alone: FLOPs of its 11 GEMMs over the step's device time
    net = surrogate.mlp
    x16 = surrogate._inputs(models[:net.batch], net.batch)
    xt16 = x16.T.contiguous()
    target = surrogate._targets(data[:net.batch], net.batch)
    for _ in range(3):
        net.gradients(x16, xt16, target)
    stream = torch.cuda.current_stream(device)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 20
    a.record(stream)
    for _ in range(reps):
        net.gradients(x16, xt16, target)
    b.record(stream)
    torch.cuda.synchronize(device)
    step_ms = a.elapsed_time(b) / reps
    sizes = net.sizes
    # forward, weight gradient and input gradient GEMMs (no input gradient for the first layer)
    flops = sum(2.0 * net.batch * sizes[i] * sizes[i + 1] * (3 if i > 0 else 2) for i in range(len(sizes) - 1))
    peak = measured_peaks()["bf16_tflops"]
    achieved = flops / (step_ms * 1e-3) / 1e12
    net.check_error()
    report = {"training_models": count, "held_out_models": 1024, "epochs": len(history), "data_seconds": data_s,
              "train_seconds": train_s, "final_train_mse_standardized": history[-1],
              "held_out_rhoa_rms_rel_error": float(torch.sqrt((error ** 2).mean())),
              "held_out_rhoa_max_rel_error": float(error.abs().max()),
              "forward_backward_ms": step_ms, "forward_backward_gflop": flops / 1e9,
              "gemm_tflops": achieved, "tensor_frac_of_measured_bf16_peak": achieved / peak,
              "network": "6144-1024-1024-1024-1232 (padded 1280), GELU, BF16 weights/activations, FP32 accumulate, Adam"}
    return surrogate, report


def run_timelapse(args, rank: int, world: int) -> dict | None:
    from adtlert_b200.surrogate import SurrogateScreen
    from adtlert_b200.timelapse import WindowedInversion, WindowSettings, window_share, window_starts

    device = torch.device("cuda", torch.cuda.current_device())
    forward, nodes, cells, electrodes, rows, rho, clean, observed, initial = timelapse_workload()
    D, C = forward.D, forward.C
    settings = WindowSettings(data_std=float(np.log1p(TIMELAPSE_NOISE)))
    starts = window_starts(TIMELAPSE_STEPS, 3)
    mine = window_share(len(starts), rank, world)
    if args.windows is not None:
        mine = mine[:args.windows]
    total_windows = len(mine) * world if args.windows is not None else len(starts)
    with ClockSampler(device.index) as clocks:
        warm = WindowedInversion(forward, settings)  # untimed warm-up windows on a separate cache
        for index in starts[-2:]:
            warm.invert_window(torch.as_tensor(np.log(observed[index:index + 3])), torch.as_tensor(initial[index:index + 3]))
        plain = WindowedInversion(forward, settings)
        plain_s, plain_wall, plain_result, plain_launches, _ = timed_inversion(plain, observed, initial, mine, None,
                                                                               device, world)
        plain_misfit, plain_predicted = inversion_misfit(plain, plain_result, observed, clean)
        screened_line = None
        if not args.no_surrogate:
            surrogate, report = train_surrogate(forward, args.training_models, device)
            screened = WindowedInversion(forward, settings)
            screen = SurrogateScreen(surrogate)
            launches_before = surrogate.mlp.launches
            s_s, s_wall, s_result, s_launches, _ = timed_inversion(screened, observed, initial, mine, screen, device,
                                                                   world)
            s_misfit, s_predicted = inversion_misfit(screened, s_result, observed, clean)
            iterations = sum(w["iterations"] for w in s_result.windows)
            # the same window candidates judged by the FEM instead of the network
            fem_judged = WindowedInversion(forward, settings)
            f_s, _, f_result, _, _ = timed_inversion(fem_judged, observed, initial, mine, SurrogateScreen(None), device,
                                                     world)
            f_misfit, _ = inversion_misfit(fem_judged, f_result, observed, clean)
            held = torch.as_tensor(np.log10(rho), device=device, dtype=torch.float64)
            series_error = 10.0 ** (surrogate.predict_log10(held).cpu().numpy() - np.log10(clean)) - 1.0
            report["series_rhoa_rms_rel_error"] = float(np.sqrt(np.mean(series_error ** 2)))
            report["series_rhoa_max_rel_error"] = float(np.abs(series_error).max())
            fem_line = {"value": total_windows / f_s, "misfit": f_misfit}
            rules = {"warm_start_stop_rules": {"stall_tolerance": screen.stall_tolerance,
                                               "objective_tolerance": screen.objective_tolerance,
                                               "cgls_iterations": screen.cgls_iterations}}
            screened_line = (s_s, s_wall, s_launches + surrogate.mlp.launches - launches_before, s_misfit, report,
                             dict(screen.counts, **rules), iterations, s_predicted, fem_line)
    if rank != 0:
        return None
    line = {
        "metric": "windows_per_second",
        "value": total_windows / plain_s,
        "unit": "windows/s",
        "n_gpus": world,
        "steps": len(mine),
        "warmup": 2,
        "ms_per_step": 1e3 * plain_s / max(len(mine), 1),
        "higher_is_better": True,
        "scaling": "strong" if args.windows is None else "weak",
        "vs_baseline": None,
        "dtype": "f32 Jacobians and fields / f64 factorization and CGLS / bf16 surrogate",
        "data": "synthetic (seeded layered base model, infiltration front to 8 m, 2 % noise)",
        "config": timelapse_config(total_windows, world, D, C),
        "misfit": plain_misfit,
        "e2e": {"value": total_windows / plain_wall, "unit": "windows/s",
                "h2d_bytes_per_step": int((observed.nbytes + initial.nbytes) / max(len(mine), 1)),
                "d2h_bytes_per_step": int(initial.nbytes / max(len(mine), 1)),
                "note": "the same run, wall clock, observed data and initial models copied from host arrays and "
                        "the combined models read back"},
        "clocks": clocks.summary(),
        "gpu_launches": int(plain_launches),
    }
    if screened_line is not None:
        s_s, s_wall, s_launches, s_misfit, report, counts, iterations, s_predicted, fem_line = screened_line
        line["value"] = total_windows / s_s
        line["ms_per_step"] = 1e3 * s_s / max(len(mine), 1)
        line["misfit"] = s_misfit
        line["e2e"]["value"] = total_windows / s_wall
        line["gpu_launches"] = int(s_launches)
        line["plain_fem"] = {"value": total_windows / plain_s, "e2e": total_windows / plain_wall,
                             "misfit": plain_misfit, "gpu_launches": int(plain_launches)}
        line["speedup_vs_plain_fem"] = plain_s / s_s
        line["fem_judged_warm_start"] = dict(fem_line, note="window candidates judged by the FEM, no network")
        line["screened_vs_plain_rhoa_rms_rel_difference"] = float(
            np.sqrt(np.mean((s_predicted / plain_predicted - 1.0) ** 2)))
        line["surrogate"] = report
        line["screening"] = dict(counts, iterations=iterations,
                                 fallback_rate=(counts["line_search_fallbacks"] + counts["warm_start_fallbacks"])
                                 / max(1, counts["line_search_screened"] + counts["line_search_fallbacks"]
                                       + counts["warm_starts"]))
    line["roofline"] = cgls_roofline(plain, observed, initial, mine[len(mine) // 2], device)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = timelapse_cpu_baseline(nodes, cells, electrodes, rows, observed, initial,
                                                      plain_misfit["iterations_mean"])
    return line


def cgls_roofline(inversion, observed, initial, index: int, device, reps: int = 5) -> dict:
    """Roofline of the CGLS step (adt_gn_step) on window ``index``: CUDA-event time of ``reps``
    calls on the launching stream after one untimed call. Algorithmic bytes = the window's float32
    Jacobians read once by each data pass (A^T b, then one per CGLS iteration run); the reduce and
    update kernels between the passes are inside the time."""

    from adtlert_b200.timelapse import WindowedInversion

    cold = WindowedInversion(inversion.forward, inversion.settings)
    models = cold._clip(torch.as_tensor(initial[index:index + 3], dtype=torch.float64, device=device)).contiguous()
    predicted, J = cold.linearize(models)
    obs = torch.as_tensor(np.log(observed[index:index + 3]), dtype=torch.float64, device=device)
    weights = torch.full_like(predicted, 1.0 / cold.settings.data_std)
    rhs = (-(weights * (predicted - obs))).contiguous()
    with torch.cuda.nvtx.range("untimed_gn_step"):  # the step profiling captures select (ncu --nvtx)
        cold.gauss_newton_step(J, weights, rhs, models)
    iterations = cold.cgls_iterations()
    stream = torch.cuda.current_stream(device)
    begin, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(device)
    begin.record(stream)
    for _ in range(reps):
        cold.gauss_newton_step(J, weights, rhs, models)
    end.record(stream)
    torch.cuda.synchronize(device)
    step_s = begin.elapsed_time(end) / 1e3 / reps
    passes = iterations + 1
    algorithmic = passes * J.numel() * J.element_size()
    peaks = measured_peaks()
    achieved = algorithmic / step_s / 1e9
    traffic = None
    path = ROOT / "profiles" / "traffic_cgls.json"
    if path.exists():  # DRAM bytes of one captured adt_gn_step, scaled to this step's data passes
        captured = json.loads(path.read_text())["adt_gn_step"]
        traffic = captured["dram_bytes"] * passes / (captured["cgls_iterations"] + 1)
    return {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "kernel": "normal_data_kernel (CGLS step)",
            "algorithmic_bytes_per_launch": algorithmic, "launch_ms": step_s * 1e3, "cgls_iterations": iterations,
            "jacobian_bytes": J.numel() * J.element_size(), "peak_source": peaks["source"],
            "note": "one adt_gn_step = A^T b pass + one data pass per CGLS iteration (each reads the window's "
                    "Jacobians once) + the reduce and update kernels; the first two models' Jacobians are "
                    "loaded evict-last so they stay in the 126 MB L2 between passes, hence achieved can pass "
                    "the HBM copy peak; traffic = DRAM bytes of one step captured by ncu (profiles/"
                    "traffic_cgls.json; ncu empties the caches before each launch, so every pass reads all three "
                    "Jacobians there), scaled to this step's passes"}


def timelapse_cpu_baseline(nodes, cells, electrodes, rows, observed, initial, iterations_per_window: float) -> dict:
    """The FP64 oracle restatement of the reference's driver (SciPy SuperLU fields, dense
    Jacobians, SciPy/torch CSR CGLS on the host) timed on one window for 2 Gauss-Newton
    iterations, extrapolated to windows/s with the GPU run's mean iterations per window."""

    sys.path.insert(0, str(ROOT))
    from oracle.timelapse import OracleTimeLapse

    oracle = OracleTimeLapse(nodes, cells, electrodes, rows, max_iterations=2, data_std=float(np.log1p(TIMELAPSE_NOISE)),
                             step_tolerance=0.0)
    start = time.perf_counter()
    _, _, chi2, taus = oracle.invert_window(np.log(observed[100:103]), initial[100:103])
    seconds = time.perf_counter() - start
    per_iteration = seconds / len(chi2)
    per_window = per_iteration * max(iterations_per_window, 1.0)
    threads = int(torch.get_num_threads())
    return {"value": 1.0 / per_window, "unit": "windows/s", "cores": threads, "kind": "port",
            "sample": f"window 100, {len(chi2)} Gauss-Newton iterations of the FP64 oracle driver in {seconds:.1f} s "
                      f"({per_iteration:.1f} s per iteration incl. the first linearization), extrapolated to "
                      f"{iterations_per_window:.1f} iterations per window"}


def main():
    args = parse_args()
    if args.impl == "reference":
        # the reference's CPU path on rank 0 only; the other ranks exit at once (no process group,
        # so no collective waits on rank 0's minutes of host work)
        rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
        if rank == 0:
            print(json.dumps(run_reference(args, rank, world)), flush=True)
        return
    rank, world = dist_setup(args)
    if args.workload == "timelapse":
        result = run_timelapse(args, rank, world)
    elif args.workload in BOX3D:
        result = run_box3d(args, rank, world)
    elif args.workload == "terrain":
        result = run_terrain(args, rank, world)
    else:
        result = run_b200(args, rank, world)
    if result is not None:
        print(json.dumps(result), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Benchmark: SOAP power spectrum with forces on one B200 (FP64 drop-in).

Workload (one step): one periodic cubic box of 1000 atoms at number density
0.1 A^-3 (L = 21.544 A), uniform positions rejection-sampled to a minimum
pair distance of 0.9 A, 4 species (1, 6, 7, 8) drawn uniformly, seeded;
hypers rc 5.5 A, ShiftedCosine 0.5 A, Gaussian width 0.3 A, GTO max_radial 7,
max_angular 6, spline accuracy 1e-8.  Output: the power spectrum plus its
positions and strain gradients, FP64 -- neighbour list, spherical expansion,
contraction, every row materialised in featomic's TensorMap layout.

* ``value``  atom-environments/s with positions resident in HBM and the
  TensorMap left in HBM (featomic_b200_calculator_compute_device), CUDA
  events on the launching stream, L2 flushed between steps.
* ``e2e``    the same through featomic's C API (featomic_calculator_compute)
  with host systems: host->device positions and device->host TensorMap
  inside the timed region.
* ``adjoint_form`` the adjoint form beside it: dense power spectrum with
  FP32 arithmetic plus forces and virial of a linear energy through the CUDA
  adjoint, on a 20 000-atom strained box, with its error against FP64.
* ``batched_form`` 4096 molecules through one persistent launch replayed from
  a CUDA graph (FP32, autotuned), power spectrum + forces + energies.
* ``surrogate_form`` the learned radial surrogate (MLP trained on the GPU,
  tcgen05 inference) against the spline, on a 100 000-atom box, with errors
  against FP64.
* ``cg_form`` the equivariant power spectrum (lambda-SOAP) of the same box:
  every Clebsch-Gordan block product in one launch, FP64.
* ``cpu_baseline`` / ``--impl reference``: featomic itself is Rust and cannot
  be built here (no cargo / crates), so the CPU side is the FP64 C++
  restatement in oracle/ (OpenMP, featomic's decomposition: spherical
  expansion over systems, power spectrum over samples).

Multi-GPU: the path has no exchange step; ``--gpus N`` runs N independent
replicas (one process per GPU) and reports the aggregate rate.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SOAP power-spectrum atom-envs/s with forces, 1 B200, at stated error vs FP64"
WORKLOAD = "random_box_1000_rho0.1_rc5.5_nmax7_lmax6_ps+positions+strain_fp64"
GRADIENTS = ["positions", "strain"]
N_ATOMS = 1000


def workload():
    from rascaline_b200 import workloads
    system = workloads.random_box(N_ATOMS, density=0.1, min_distance=0.9, seed=2)
    return system, workloads.hypers(5.5, 7, 6)


def config(extra=None):
    c = {
        "workload": WORKLOAD,
        "n_atoms": N_ATOMS,
        "gradients": GRADIENTS,
        "hypers": {"cutoff": 5.5, "max_radial": 7, "max_angular": 6, "gaussian_width": 0.3,
                   "smoothing": "ShiftedCosine 0.5", "spline_accuracy": 1e-8},
        "l2": "flushed between steps (256 MiB write); each step also writes 3.5 GB of output",
        "parallelism": "replicas",
    }
    if extra:
        c.update(extra)
    return c


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fd:
            data = json.load(fd)
        return float(data["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(kernel):
    """DRAM bytes per launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", f"{kernel}.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_launch:"):
            return float(line.split(":", 1)[1].split()[0])
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    QUERY = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[4:8]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {
            "sm_mhz": float(np.median(sm)) if sm else None,
            "sm_max_mhz": float(max(smax)) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def cpu_baseline(system, hypers, seconds=20.0):
    """The oracle (C++ FP64 restatement of featomic's path) on the host cores."""
    from oracle import oracle
    oracle.build()
    threads = os.cpu_count() or 1
    envs, elapsed, runs = 0, 0.0, 0
    while elapsed < seconds or runs == 0:
        t0 = time.perf_counter()
        oracle.compute("soap_power_spectrum", hypers, [system], gradients=tuple(GRADIENTS), threads=threads)
        elapsed += time.perf_counter() - t0
        envs += N_ATOMS
        runs += 1
        if runs >= 3 and elapsed > seconds / 2:
            break
    return {
        "value": envs / elapsed, "unit": "atom-envs/s", "cores": threads, "kind": "port",
        "sample": f"{runs} full compute(s) of the {N_ATOMS}-atom box (PS + positions + strain gradients, FP64), "
                  f"{elapsed:.1f} s; spherical expansion serial per system, power spectrum OpenMP over samples",
    }


def dist_setup(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        # one process per GPU over NCCL; the host-only paths (the reference
        # arm, tests) use gloo when no GPU is visible
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        else:
            dist.init_process_group("gloo", timeout=timedelta(seconds=300))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allreduce_max(value, world):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args):
    rank, world, _ = dist_setup(args.gpus)
    if rank != 0:
        barrier(world)
        return
    system, hypers = workload()
    from oracle import oracle
    oracle.build()
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        oracle.compute("soap_power_spectrum", hypers, [system], gradients=tuple(GRADIENTS), threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.compute("soap_power_spectrum", hypers, [system], gradients=tuple(GRADIENTS), threads=threads)
        times.append(time.perf_counter() - t0)
    ms = 1000.0 * float(np.mean(times))
    value = N_ATOMS / (ms / 1000.0)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "atom-envs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": config({"reference": "featomic is Rust and cannot be built here (no cargo/rustc, no crates); "
                                       "timed: the C++ FP64 restatement in oracle/ with all host threads"}),
        "cpu_baseline": {"value": value, "unit": "atom-envs/s", "cores": threads, "kind": "port",
                         "sample": f"full {N_ATOMS}-atom compute per step"},
        "e2e": {"value": value, "unit": "atom-envs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    barrier(world)


DENSE_PHASES = ("pair_features", "expansion", "contraction", "dl_dc", "pair_adjoint", "reductions")


def dense_phase_times(calc):
    """Device times (ms) of the phases of the calculator's last dense forward
    and backward passes (featomic_b200_dense_timings)."""
    import ctypes
    from rascaline_b200 import _c_api as C
    t = (ctypes.c_double * 6)()
    C.check(C.lib().featomic_b200_dense_timings(calc._handle, t, 6))
    return dict(zip(DENSE_PHASES, [float(x) for x in t]))


def dense_rooflines(phases, n_atoms, S, K, n_keys, n_props, grad_rows, peak, peak_kind, word=4):
    """HBM rooflines of the two tensor-core contractions of an FP32 dense
    pass: the power spectrum (coefficients read, values written) and dL/dc
    (coefficients and dL/dP rows read, dL/dc written); `grad_rows` dL/dP rows
    are read (one per atom, or one per species for a linear model)."""
    out = {}
    contraction = word * n_atoms * (S * K + n_keys * n_props)
    grad = word * (2 * n_atoms * S * K + grad_rows * n_keys * n_props)
    for name, phase, bytes_ in (("contraction", "contraction", contraction), ("dl_dc", "dl_dc", grad)):
        ms = phases.get(phase, 0.0)
        achieved = bytes_ / (ms / 1e3) / 1e9 if ms > 0 else 0.0
        out[name] = {"kernel": "dense_contraction_mma" if name == "contraction" else "dense_grad_coef_mma",
                     "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind, "algorithmic_bytes_per_launch": bytes_,
                     "time_ms": ms}
    return out


def adjoint_form(steps, warmup, n=20000):
    """The adjoint form on the 20 000-atom strained box (``n`` atoms, for
    profiling smaller cases of the same workload): dense power spectrum
    in FP32 arithmetic, then forces and virial of a linear energy model through
    the CUDA adjoint (no gradient blocks materialised).  One step = forward +
    backward; errors are measured once against the same calculation in FP64."""
    import torch
    import rascaline_b200 as rb
    from rascaline_b200 import workloads
    from rascaline_b200.torch_api import dense_backward, dense_power_spectrum

    system = workloads.random_box(n, density=0.1, min_distance=0.9, seed=5, strain=0.02)
    calc = rb.SoapPowerSpectrum(**workloads.hypers(5.0, 7, 6))
    positions = torch.tensor(system["positions"], device="cuda")
    types = system["types"].astype(np.int32)
    cells = np.asarray(system["cell"]).reshape(1, 9)
    sizes = np.array([n])
    species = np.unique(types)
    S = len(species)
    n_keys, n_props = S * (S + 1) // 2, 7 * 8 * 8
    rng = np.random.default_rng(11)
    d = n_keys * n_props
    weights = rng.normal(0.0, 1.0 / np.sqrt(d), size=(S, n_keys, n_props))  # per centre species
    grad = torch.as_tensor(weights[np.searchsorted(species, types)], device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def run(precision, g):
        values, state = dense_power_spectrum(calc, positions, types, cells, sizes, precision)
        forces, virial, _ = dense_backward(state, g, 1, strain=True, cell=False)
        return values, forces, virial

    results = {}
    for precision in (32, 64):
        g = grad.float() if precision == 32 else grad
        for _ in range(max(3, warmup)):
            run(precision, g)
        torch.cuda.synchronize()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        mids = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        stream = torch.cuda.current_stream()
        for k in range(steps):
            flush.zero_()
            starts[k].record(stream)
            values, state = dense_power_spectrum(calc, positions, types, cells, sizes, precision)
            mids[k].record(stream)
            forces, virial, _ = dense_backward(state, g, 1, strain=True, cell=False)
            ends[k].record(stream)
        torch.cuda.synchronize()
        fwd = float(np.mean([s.elapsed_time(m) for s, m in zip(starts, mids)]))
        bwd = float(np.mean([m.elapsed_time(e) for m, e in zip(mids, ends)]))
        phases = dense_phase_times(calc)
        values, forces, virial = run(precision, g)
        energy = float((values.double() * grad).sum())
        results[precision] = dict(ms=fwd + bwd, forward_ms=fwd, backward_ms=bwd, energy=energy, phases=phases,
                                  values=values.double(), forces=forces.double(), virial=virial.double())
    r32, r64 = results[32], results[64]
    peak, peak_kind = measured_peaks()
    K = 49 * 8
    rooflines = dense_rooflines(r32["phases"], n, S, K, n_keys, n_props, n, peak, peak_kind)

    def rel(a, b):
        return float((a - b).abs().max() / b.abs().max())

    return {
        "workload": f"random_box_{n}_rho0.1_strain0.02_rc5_nmax7_lmax6_ps+forces+virial_adjoint",
        "metric": "atom-envs/s (power spectrum + forces + virial)",
        "value": n / (r32["ms"] / 1000.0),
        "ms_per_step": r32["ms"],
        "forward_ms": r32["forward_ms"],
        "backward_ms": r32["backward_ms"],
        "dtype": "f32",
        "phases_ms": r32["phases"],
        "roofline": rooflines["contraction"],
        "roofline_dl_dc": rooflines["dl_dc"],
        "fp64_value": n / (r64["ms"] / 1000.0),
        "fp64_ms_per_step": r64["ms"],
        "error_vs_fp64": {
            "values_max_abs_over_max": rel(r32["values"], r64["values"]),
            "forces_max_abs_over_max": rel(r32["forces"], r64["forces"]),
            "virial_max_abs_over_max": rel(r32["virial"], r64["virial"]),
            "energy_rel": abs(r32["energy"] - r64["energy"]) / abs(r64["energy"]),
        },
        "steps": steps,
        "l2": "flushed between steps (256 MiB write); the 358 MB FP32 output also exceeds L2",
        "energy_model": "E = sum over atoms of w[centre species] . P, w ~ N(0, 1/sqrt(d)) seeded",
    }


def batched_form(steps, warmup):
    """The batched form on 4096 seeded molecules (5 to 60 atoms, species 1/6/7/8
    with p = .5/.3/.1/.1, uniform in a sphere of radius 1.2 N^(1/3) A, minimum
    distance 1.0 A): power spectrum rows, dE/dpositions and energies of a
    linear model, FP32.  The autotuner times the persistent launch replayed
    from a CUDA graph (every launch configuration) and the dense pipeline of
    the adjoint form, and keeps the fastest; `config.pipeline` says which ran
    (0 persistent, 1 dense).  Errors against the dense FP64 path on the same
    molecules."""
    import torch
    import rascaline_b200 as rb
    from rascaline_b200 import workloads
    from rascaline_b200.torch_api import Batch, dense_backward, dense_power_spectrum

    mols = workloads.molecules(4096, seed=3)
    positions = np.concatenate([m["positions"] for m in mols])
    types = np.concatenate([m["types"] for m in mols]).astype(np.int32)
    sizes = np.array([len(m["types"]) for m in mols])
    species = [1, 6, 7, 8]
    calc = rb.SoapPowerSpectrum(**workloads.hypers(5.0, 7, 6))
    batch = Batch(calc, sizes, types, species)
    rng = np.random.default_rng(17)
    W = rng.normal(0.0, 1.0 / np.sqrt(batch.n_keys * batch.n_properties),
                   size=(len(species), batch.n_keys, batch.n_properties))
    weights = torch.as_tensor(W, dtype=torch.float32, device="cuda").contiguous()
    pos = torch.as_tensor(positions, device="cuda")
    out = batch.outputs()
    tuned_ms = batch.tune(pos, out, weights=weights)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    for _ in range(max(3, warmup)):
        batch.run(pos, out, weights=weights)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    for k in range(steps):
        flush.zero_()
        starts[k].record(stream)
        batch.run(pos, out, weights=weights)
        ends[k].record(stream)
    torch.cuda.synchronize()
    ms = float(np.mean([s.elapsed_time(e) for s, e in zip(starts, ends)]))
    if batch.status() != 0:
        raise RuntimeError("the batched form reported an error")
    phases = dense_phase_times(calc) if batch.config["pipeline"] == 1 else None

    # end to end: positions from pinned host memory, gradients and energies back
    host_pos = torch.as_tensor(positions).pin_memory()
    host_grad = torch.empty((batch.n_atoms, 3), dtype=torch.float32).pin_memory()
    host_energy = torch.empty(batch.n_systems, dtype=torch.float32).pin_memory()
    e2e = []
    for k in range(max(3, steps // 2) + 2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pos.copy_(host_pos, non_blocking=True)
        batch.run(pos, out, weights=weights)
        host_grad.copy_(out["gradients"], non_blocking=True)
        host_energy.copy_(out["energies"], non_blocking=True)
        torch.cuda.synchronize()
        if k >= 2:
            e2e.append(time.perf_counter() - t0)
    e2e_ms = 1000.0 * float(np.mean(e2e))

    # error against FP64
    values64, state = dense_power_spectrum(calc, pos, types, np.zeros((len(mols), 9)), sizes, 64, species)
    G = torch.as_tensor(W[np.searchsorted(species, types)], device="cuda")
    grad64, _, _ = dense_backward(state, G, len(mols), strain=False, cell=False)
    atom_energy = (values64 * G).sum(dim=(1, 2))
    system = torch.as_tensor(np.repeat(np.arange(len(mols)), sizes), device="cuda")
    energy64 = torch.zeros(len(mols), dtype=torch.float64, device="cuda").index_add_(0, system, atom_energy)

    def rel(a, b):
        return float((a.double() - b).abs().max() / b.abs().max())

    errors = {
        "values_max_abs_over_max": rel(out["values"], values64),
        "gradients_max_abs_over_max": rel(out["gradients"], grad64),
        "energies_max_abs_over_max": rel(out["energies"], energy64),
    }
    del values64, state, G
    n = batch.n_atoms
    chosen = batch.config
    # the persistent kernel alone, for comparison
    persistent = dict(chosen, pipeline=0) if chosen["pipeline"] == 1 else None
    persistent_ms = None
    if persistent is not None:
        batch.config = {"warps": 8, "chunk": 32, "layout": 1, "ctas_per_sm": 1, "pipeline": 0}
        for _ in range(2):
            batch.run(pos, out, weights=weights)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            batch.run(pos, out, weights=weights)
        e1.record()
        torch.cuda.synchronize()
        persistent_ms = e0.elapsed_time(e1) / 3
        batch.config = chosen
    return {
        "workload": "molecules_4096_sizes5-60_rc5_nmax7_lmax6_ps+gradients+energies",
        "metric": "atom-envs/s (power spectrum + forces)",
        "value": n / (ms / 1000.0),
        "ms_per_step": ms,
        "n_atoms": n,
        "dtype": "f32",
        "config": chosen,
        "tuned_ms": tuned_ms,
        "persistent_kernel_ms": persistent_ms,
        "e2e": {"value": n / (e2e_ms / 1000.0), "unit": "atom-envs/s", "h2d_bytes_per_step": n * 24,
                "d2h_bytes_per_step": n * 12 + batch.n_systems * 4},
        "error_vs_fp64": errors,
        "gpu_launches_per_step": 1 if chosen["pipeline"] == 0 else 24,
        "phases_ms": phases,
        "roofline": dense_rooflines(phases, n, len(species), 49 * 8, batch.n_keys, batch.n_properties,
                                    len(species), *measured_peaks())["contraction"] if phases else None,
        "steps": steps,
        "l2": "flushed between steps (256 MiB write); the 2.4 GB FP32 output also exceeds L2",
        "energy_model": "E = sum over atoms of w[centre species] . P, w ~ N(0, 1/sqrt(d)) seeded",
    }


def surrogate_form(steps, warmup, train_steps=20000):
    """The learned radial surrogate on a 100 000-atom box (density 0.1 A^-3,
    minimum distance 0.9 A, 4 species; rc 6 A, max_radial 11, max_angular 8):
    the MLP 1 -> 64 -> 64 -> 108 (SiLU, BF16 weights, FP32 accumulation) is
    trained on 2^20 exact radial integrals with r uniform in [0, 6] A, then the
    FP32 dense power spectrum is computed with the spline and with the MLP;
    both are compared with the FP64 power spectrum (spline accuracy 1e-8)."""
    import torch
    import rascaline_b200 as rb
    from rascaline_b200 import workloads
    from rascaline_b200.surrogate import RadialSurrogate
    from rascaline_b200.torch_api import dense_power_spectrum

    n = 100000
    system = workloads.random_box(n, density=0.1, min_distance=0.9, seed=6)
    calc = rb.SoapPowerSpectrum(**workloads.hypers(6.0, 11, 8))
    pos = torch.tensor(system["positions"], device="cuda")
    types = system["types"].astype(np.int32)
    cells = np.asarray(system["cell"]).reshape(1, 9)

    s = RadialSurrogate(calc, seed=3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.make_dataset(1 << 20, seed=7)
    loss = s.train(train_steps, 8192, 3e-3, derivative_weight=0.1)
    s.fit_output_layer(0.01)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    r = torch.linspace(0.9, 6.0, 20001, dtype=torch.float64, device="cuda")
    exact, dexact = s.evaluate(r, "analytic")
    mlp, dmlp = s.evaluate(r, "tensor_cores")
    fp32w, dfp32w = s.evaluate(r, "cuda_cores")
    bf1, dbf1 = s.evaluate(r, "bf16_single")
    spl, dspl = s.evaluate(r, "spline")
    scale, dscale = exact.abs().amax(dim=0), dexact.abs().amax(dim=0)

    def rms(a, b, sc):
        return float((((a - b) / sc) ** 2).mean().sqrt())

    def mx(a, b, sc):
        return float(((a - b).abs() / sc).max())

    radial = {
        "mlp_values_rms": rms(mlp, exact, scale), "mlp_values_max": mx(mlp, exact, scale),
        "mlp_derivatives_rms": rms(dmlp, dexact, dscale), "mlp_derivatives_max": mx(dmlp, dexact, dscale),
        # the same network with FP32 weights on the CUDA cores, and with one
        # BF16 per weight: what three-part BF16 operands buy
        "fp32_weights_control_values_max": mx(fp32w, exact, scale),
        "fp32_weights_control_derivatives_max": mx(dfp32w, dexact, dscale),
        "single_bf16_control_values_max": mx(bf1, exact, scale),
        "single_bf16_control_derivatives_max": mx(dbf1, dexact, dscale),
        "spline_values_max": mx(spl, exact, scale), "spline_derivatives_max": mx(dspl, dexact, dscale),
        "normalisation": "each output divided by its largest magnitude over r in [0.9, 6] A",
    }
    rates = {}
    rr = torch.rand(1 << 22, dtype=torch.float64, device="cuda") * 6.0
    for method in ("tensor_cores", "spline", "analytic"):
        s.evaluate(rr[:4096], method)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        s.evaluate(rr, method)
        e1.record()
        torch.cuda.synchronize()
        rates[method] = rr.numel() / (e0.elapsed_time(e1) / 1000.0)

    def timed(precision):
        for _ in range(max(3, warmup)):
            dense_power_spectrum(calc, pos, types, cells, [n], precision)
        torch.cuda.synchronize()
        times = []
        for _ in range(steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            values, _ = dense_power_spectrum(calc, pos, types, cells, [n], precision)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
            del values
        values, _ = dense_power_spectrum(calc, pos, types, cells, [n], precision)
        return float(np.mean(times)), values

    ms64, v64 = timed(64)
    v64_max = float(v64.abs().max())
    ms_spline, v32 = timed(32)
    spline_err = float((v32.double() - v64).abs().max()) / v64_max
    del v32
    s.attach()
    try:
        ms_mlp, vm = timed(32)
    finally:
        s.attach(False)
    mlp_err = float((vm.double() - v64).abs().max()) / v64_max
    mlp_rms = float(((vm.double() - v64) ** 2).mean().sqrt()) / float((v64 ** 2).mean().sqrt())
    del vm, v64
    # forces (adjoint of a seeded random dL/dP) on a 5000-atom box of the same
    # density and hypers: spline and MLP in FP32 against FP64
    from rascaline_b200.torch_api import dense_backward
    small = workloads.random_box(5000, density=0.1, min_distance=0.9, seed=16)
    spos = torch.tensor(small["positions"], device="cuda")
    scell = np.asarray(small["cell"]).reshape(1, 9)
    sv64, st64 = dense_power_spectrum(calc, spos, small["types"], scell, [5000], 64)
    G = torch.randn(sv64.shape, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(5))
    f64, _, _ = dense_backward(st64, G, 1, cell=False)
    _, st32 = dense_power_spectrum(calc, spos, small["types"], scell, [5000], 32)
    f32, _, _ = dense_backward(st32, G.float(), 1, cell=False)
    s.attach()
    try:
        _, stm = dense_power_spectrum(calc, spos, small["types"], scell, [5000], 32)
        fm, _, _ = dense_backward(stm, G.float(), 1, cell=False)
    finally:
        s.attach(False)
    forces = {"spline_fp32_max_abs_over_max": float((f32.double() - f64).abs().max() / f64.abs().max()),
              "mlp_fp32_max_abs_over_max": float((fm.double() - f64).abs().max() / f64.abs().max()),
              "workload": "random_box_5000_rho0.1_rc6_nmax11_lmax8, dL/dP ~ N(0, 1) seeded"}
    del sv64, st64, st32, stm, G
    return {
        "workload": "random_box_100000_rho0.1_rc6_nmax11_lmax8_ps_values_fp32_spline_vs_mlp",
        "training": {"samples": 1 << 20, "steps": train_steps, "batch": 8192, "seconds": train_s, "final_loss": loss,
                     "seconds_includes": "training set, Adam steps and the output-layer fit"},
        "radial_error_vs_exact": radial,
        "radial_evaluations_per_s": rates,
        "power_spectrum_error_vs_fp64": {
            "spline_fp32_max_abs_over_max": spline_err,
            "mlp_fp32_max_abs_over_max": mlp_err,
            "mlp_fp32_rms_over_rms": mlp_rms,
        },
        "forces_error_vs_fp64": forces,
        "training_recipe": "Adam on values + 0.1 x-derivatives, then least-squares output layer (lambda 0.01) on "
                           "the tensor-core features; W2, W3 and activations as three BF16 parts on the tensor cores",
        "ms_per_step": {"fp64_spline": ms64, "fp32_spline": ms_spline, "fp32_mlp": ms_mlp},
        "atom_envs_per_s": {"fp64_spline": n / ms64 * 1e3, "fp32_spline": n / ms_spline * 1e3,
                            "fp32_mlp": n / ms_mlp * 1e3},
        "steps": steps,
        "note": "power spectrum values only (no gradients); the MLP replaces the spline in the FP32 pair features",
    }


def combined_form(steps, warmup, train_steps=20000, dropin_value=None):
    """batched + surrogate + adjoint on the 4096 molecules of the batched
    form: the learned radial surrogate (trained for these hypers: rc 5 A,
    max_radial 7, max_angular 6, 56 outputs) replaces the spline in the
    batch's dense pipeline (FP32 forward with the tensor-core contraction,
    then the adjoint of a linear energy model and the energies), timed like
    the batched form; errors against the FP64 spline path.  `vs_dropin` is
    this value over the FP64 drop-in's atom-envs/s of the same run."""
    import torch
    import rascaline_b200 as rb
    from rascaline_b200 import workloads
    from rascaline_b200.surrogate import RadialSurrogate
    from rascaline_b200.torch_api import Batch, dense_backward, dense_power_spectrum

    mols = workloads.molecules(4096, seed=3)
    positions = np.concatenate([m["positions"] for m in mols])
    types = np.concatenate([m["types"] for m in mols]).astype(np.int32)
    sizes = np.array([len(m["types"]) for m in mols])
    species = [1, 6, 7, 8]
    calc = rb.SoapPowerSpectrum(**workloads.hypers(5.0, 7, 6))
    s = RadialSurrogate(calc, seed=3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.make_dataset(1 << 20, seed=7)
    s.train(train_steps, 8192, 3e-3, derivative_weight=0.1)
    s.fit_output_layer(0.01)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    batch = Batch(calc, sizes, types, species)
    rng = np.random.default_rng(17)
    W = rng.normal(0.0, 1.0 / np.sqrt(batch.n_keys * batch.n_properties),
                   size=(len(species), batch.n_keys, batch.n_properties))
    weights = torch.as_tensor(W, dtype=torch.float32, device="cuda").contiguous()
    pos = torch.as_tensor(positions, device="cuda")
    out = batch.outputs()
    batch.config = {"warps": 4, "chunk": 32, "layout": 1, "ctas_per_sm": 2, "pipeline": 1}
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    s.attach()
    try:
        for _ in range(max(3, warmup)):
            batch.run(pos, out, weights=weights)
        torch.cuda.synchronize()
        stream = torch.cuda.current_stream()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        for k in range(steps):
            flush.zero_()
            starts[k].record(stream)
            batch.run(pos, out, weights=weights)
            ends[k].record(stream)
        torch.cuda.synchronize()
        ms = float(np.mean([a.elapsed_time(b) for a, b in zip(starts, ends)]))
        phases = dense_phase_times(calc)
        host_pos = torch.as_tensor(positions).pin_memory()
        host_grad = torch.empty((batch.n_atoms, 3), dtype=torch.float32).pin_memory()
        host_energy = torch.empty(batch.n_systems, dtype=torch.float32).pin_memory()
        e2e = []
        for k in range(max(3, steps // 2) + 2):
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            pos.copy_(host_pos, non_blocking=True)
            batch.run(pos, out, weights=weights)
            host_grad.copy_(out["gradients"], non_blocking=True)
            host_energy.copy_(out["energies"], non_blocking=True)
            torch.cuda.synchronize()
            if k >= 2:
                e2e.append(time.perf_counter() - t1)
        e2e_ms = 1000.0 * float(np.mean(e2e))
    finally:
        s.attach(False)
    values64, state = dense_power_spectrum(calc, pos, types, np.zeros((len(mols), 9)), sizes, 64, species)
    G = torch.as_tensor(W[np.searchsorted(species, types)], device="cuda")
    grad64, _, _ = dense_backward(state, G, len(mols), strain=False, cell=False)
    atom_energy = (values64 * G).sum(dim=(1, 2))
    system = torch.as_tensor(np.repeat(np.arange(len(mols)), sizes), device="cuda")
    energy64 = torch.zeros(len(mols), dtype=torch.float64, device="cuda").index_add_(0, system, atom_energy)

    def rel(a, b):
        return float((a.double() - b).abs().max() / b.abs().max())

    errors = {
        "values_max_abs_over_max": rel(out["values"], values64),
        "gradients_max_abs_over_max": rel(out["gradients"], grad64),
        "energies_max_abs_over_max": rel(out["energies"], energy64),
    }
    n = batch.n_atoms
    value = n / (ms / 1000.0)
    return {
        "workload": "molecules_4096_sizes5-60_rc5_nmax7_lmax6_ps+gradients+energies_mlp_radial",
        "metric": "atom-envs/s (power spectrum + forces)",
        "value": value,
        "ms_per_step": ms,
        "vs_dropin": value / dropin_value if dropin_value else None,
        "n_atoms": n,
        "dtype": "f32 (radial integral: BF16 tensor-core MLP)",
        "phases_ms": phases,
        "e2e": {"value": n / (e2e_ms / 1000.0), "unit": "atom-envs/s", "h2d_bytes_per_step": n * 24,
                "d2h_bytes_per_step": n * 12 + batch.n_systems * 4},
        "error_vs_fp64": errors,
        "surrogate_training_seconds": train_s,
        "steps": steps,
        "l2": "flushed between steps (256 MiB write)",
    }


def cg_form(steps, warmup):
    """Equivariant power spectrum (lambda-SOAP) of the 1000-atom benchmark box
    (rc 5.5 A, max_radial 7, max_angular 6, 4 species, neighbour types in the
    properties): every Clebsch-Gordan block product with l_1 <= l_2, all
    lambda, in one launch.  Timed: the product step on densities already on
    the GPU (CUDA events, FP64); beside it the whole compute() (spherical
    expansion through the C ABI, host->device copy, product) and the oracle's
    numpy product on a 50-centre sample of every block."""
    import torch
    import rascaline_b200 as rb
    from oracle import clebsch_gordan as ocg
    from rascaline_b200 import clebsch_gordan as cg

    system, hypers = workload()
    se = rb.SphericalExpansion(**hypers)
    calc = cg.EquivariantPowerSpectrum(se)
    host = se.compute([system])
    d1 = cg.keys_to_properties(cg._to_device(host, 1, torch.float64), ["neighbor_1_type"])
    d2 = cg.keys_to_properties(cg._to_device(host, 2, torch.float64), ["neighbor_2_type"])
    product = calc._cg_product
    for _ in range(max(3, warmup)):
        out = product.compute(d1, d2, "l_1", "l_2")
    torch.cuda.synchronize()
    in_bytes = sum(b.values.numel() * 8 for b in d1.blocks()) + sum(b.values.numel() * 8 for b in d2.blocks())
    out_bytes = sum(b.values.numel() * 8 for b in out.blocks())
    n_blocks = len(out)
    centres = sum(len(b.samples) for k, b in zip(d1.keys.values, d1.blocks()) if k[0] == 0)
    del out
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    for k in range(steps):
        starts[k].record()
        out = product.compute(d1, d2, "l_1", "l_2")
        ends[k].record()
        del out
    torch.cuda.synchronize()
    step_ms = float(np.mean([s.elapsed_time(e) for s, e in zip(starts, ends)]))
    # the kernel alone: the same tasks, planned once
    out, tasks = product.plan(d1, d2, "l_1", "l_2")
    for k in range(steps):
        starts[k].record()
        cg.cg_tensor_products(tasks)
        ends[k].record()
    torch.cuda.synchronize()
    ms = float(np.mean([s.elapsed_time(e) for s, e in zip(starts, ends)]))
    del out, tasks
    t0 = time.perf_counter()
    for _ in range(3):
        full = calc.compute([system], neighbors_to_properties=True)
        torch.cuda.synchronize()
        del full
    e2e_ms = (time.perf_counter() - t0) / 3 * 1000.0
    # CPU: the oracle's numpy product of every block pair on the first 50 centres
    t0 = time.perf_counter()
    sample_centres = 0
    for i, key in enumerate(d1.keys.values):
        for j, key2 in enumerate(d2.keys.values):
            if key[2] != key2[2] or key[0] > key2[0]:
                continue
            a = d1.block_by_id(i).values[:50].cpu().numpy()
            b = d2.block_by_id(j).values[:50].cpu().numpy()
            for lam in range(abs(int(key[0]) - int(key2[0])), int(key[0]) + int(key2[0]) + 1):
                ocg.cg_tensor_product(a, b, lam)
        sample_centres += min(50, len(d1.block_by_id(i).samples)) if key[0] == 0 else 0
    cpu_s = time.perf_counter() - t0
    peak, peak_kind = measured_peaks()
    achieved = (in_bytes + out_bytes) / (ms / 1000.0) / 1e9
    return {
        "workload": "random_box_1000_rho0.1_rc5.5_nmax7_lmax6_lambda_soap_fp64_neighbors_to_properties",
        "blocks": n_blocks,
        "centres": centres,
        "output_GB": out_bytes / 1e9,
        "kernel_ms": ms,
        "centres_per_s": centres / ms * 1e3,
        "product_step_ms": step_ms,
        "product_step_note": "compute() of the Clebsch-Gordan product on densities in HBM: key and label "
                             "bookkeeping in Python plus the launch",
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "note": "input + output bytes of the product kernel per launch; 9.4 FMA per output value"},
        "compute_e2e_ms": e2e_ms,
        "cpu_baseline": {"value": sample_centres / cpu_s, "unit": "centres/s", "cores": 1, "kind": "port",
                         "sample": "numpy einsum of every block pair on the first 50 centres of each block"},
        "gpu_launches_per_step": 1,
        "steps": steps,
    }


def lode_form(steps, warmup):
    """LODE spherical expansion of the 1000-atom benchmark box (potential
    exponent 1, smearing 1 A, k_cutoff 1.2 pi / smearing, GTO radius 5.5 A,
    max_radial 7, max_angular 6, 4 species): values, positions in HBM, output
    left in HBM, CUDA events around each compute.  Beside it: positions
    gradients of a 64-atom box (their rows grow as atoms^2), and the oracle's
    numpy restatement on the 1000-atom box (one run)."""
    import torch
    import rascaline_b200 as rb
    from oracle import lode as oracle_lode
    from rascaline_b200 import workloads

    system, _ = workload()
    n = len(system["types"])
    hypers = {"density": {"type": "SmearedPowerLaw", "smearing": 1.0, "exponent": 1},
              "basis": {"type": "TensorProduct", "max_angular": 6,
                        "radial": {"type": "Gto", "max_radial": 7, "radius": 5.5}}}
    calc = rb.LodeSphericalExpansion(**hypers)
    pos = torch.tensor(system["positions"], device="cuda")
    cell = np.asarray(system["cell"]).reshape(1, 9)

    def run(p, types, c, sizes, gradients=()):
        return calc.compute_device(p, types, c, sizes, gradients=list(gradients))

    for _ in range(max(3, warmup)):
        tm = run(pos, system["types"], cell, [n])
    torch.cuda.synchronize()
    del tm
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    kernel_ms = []
    for k in range(steps):
        starts[k].record()
        tm = run(pos, system["types"], cell, [n])
        ends[k].record()
        kernel_ms.append(calc.timings()["expansion"])
        del tm
    torch.cuda.synchronize()
    ms = float(np.mean([s.elapsed_time(e) for s, e in zip(starts, ends)]))
    k_vectors = len(oracle_lode.k_vectors(system["cell"], 1.2 * np.pi)[0])
    flops = 2.0 * n * 4 * k_vectors * 49 * 8  # the values contraction over k
    # positions gradients of a small box
    small = workloads.random_box(64, density=0.1, min_distance=0.9, seed=9)
    spos = torch.tensor(small["positions"], device="cuda")
    scell = np.asarray(small["cell"]).reshape(1, 9)
    for _ in range(2):
        tm = run(spos, small["types"], scell, [64], ["positions"])
    torch.cuda.synchronize()
    del tm
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(steps):
        tm = run(spos, small["types"], scell, [64], ["positions"])
        del tm
    t1.record()
    torch.cuda.synchronize()
    grad_ms = t0.elapsed_time(t1) / steps
    # the oracle on the 1000-atom box
    start = time.perf_counter()
    oracle_lode.compute(dict(hypers, basis=dict(hypers["basis"], spline_accuracy=None)), [system])
    cpu_s = time.perf_counter() - start
    return {
        "workload": "random_box_1000_rho0.1_lode_p1_smearing1_nmax7_lmax6_values_fp64",
        "metric": "atom-envs/s (LODE spherical expansion values)",
        "value": n / (ms / 1000.0),
        "ms_per_step": ms,
        "kernel_ms": float(np.mean(kernel_ms)),
        "k_vectors": k_vectors,
        "fp64_tflops_values_contraction": flops / (float(np.mean(kernel_ms)) / 1000.0) / 1e12,
        "gradients_64_atoms_ms": grad_ms,
        "dtype": "f64",
        "cpu_baseline": {"value": n / cpu_s, "unit": "atom-envs/s", "cores": 1, "kind": "port",
                         "sample": "one oracle (numpy) run on the 1000-atom box, analytic radial integral"},
        "gpu_launches_per_step": 5,
        "steps": steps,
    }


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=20)
    parser.add_argument("--warmup", type=int, default=5)
    parser.add_argument("--impl", default="b200", choices=["b200", "reference"])
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--no-chosen-forms", action="store_true",
                        help="skip the FP32 adjoint form measured beside the drop-in")
    parser.add_argument("--atoms", type=int, default=1000,
                        help="atoms in the box (1000 is the benchmark; smaller boxes are for profiling)")
    parser.add_argument("--only", choices=["adjoint", "batched", "surrogate", "combined", "cg", "lode"],
                        help="run one chosen form alone and print its object (profiling)")
    parser.add_argument("--adjoint-atoms", type=int, default=20000,
                        help="atoms of the adjoint form's box with --only adjoint (20000 is the benchmark)")
    parser.add_argument("--train-steps", type=int, default=20000,
                        help="training steps of the learned radial surrogate (20000 is the benchmark)")
    args = parser.parse_args()
    if args.only:
        import torch
        torch.cuda.set_device(0)
        form = {"adjoint": lambda k, w: adjoint_form(k, w, args.adjoint_atoms), "batched": batched_form, "cg": cg_form,
                "lode": lode_form,
                "surrogate": lambda k, w: surrogate_form(k, w, args.train_steps),
                "combined": lambda k, w: combined_form(k, w, args.train_steps)}[args.only]
        print(json.dumps({args.only + "_form": form(args.steps, args.warmup)}), flush=True)
        return
    global N_ATOMS, WORKLOAD
    if args.atoms != N_ATOMS:
        N_ATOMS = args.atoms
        WORKLOAD = WORKLOAD.replace("random_box_1000", f"random_box_{N_ATOMS}")
    if args.impl == "reference":
        return run_reference(args)

    rank, world, local = dist_setup(args.gpus)
    import torch
    torch.cuda.set_device(local)
    import rascaline_b200 as rb

    system, hypers = workload()
    calc = rb.SoapPowerSpectrum(**hypers)
    stream = torch.cuda.current_stream()
    positions = torch.tensor(system["positions"], device="cuda")
    types = system["types"]
    cells = system["cell"].reshape(1, 9)
    sizes = [N_ATOMS]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step():
        tm = calc.compute_device(positions, types, cells, sizes, gradients=GRADIENTS, stream=stream.cuda_stream)
        return tm

    for _ in range(max(3, args.warmup)):
        tm = step()
    torch.cuda.synchronize()

    # output sizes, for the algorithmic byte counts
    n_props = (6 + 1) * 8 * 8
    grad_rows = sum(b.gradient("positions").shape[0] for b in tm.blocks())
    samples = sum(b.shape[0] for b in tm.blocks())
    del tm
    n_pairs = len(rb.neighbor_list(system["positions"], system["cell"], 5.5)["first"])
    K = 49 * 8
    S = 4
    out_bytes = 8 * (samples * n_props + grad_rows * 3 * n_props + samples * 9 * n_props)
    # ps_positions_staged_kernel: every gradient row but the centres' own
    # (one per sample, written by ps_centre_rows_kernel), the coefficients and
    # the pair gradients read once
    pos_kernel_bytes = 8 * ((grad_rows - samples) * 3 * n_props + N_ATOMS * S * K + n_pairs * 3 * K)

    sampler = ClockSampler(int(os.environ.get("CUDA_VISIBLE_DEVICES", str(local)).split(",")[0])
                           if os.environ.get("CUDA_VISIBLE_DEVICES", "").isdigit() else local)
    sampler.start()
    barrier(world)
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    kernel_ms = []
    for k in range(args.steps):
        flush.zero_()
        starts[k].record(stream)
        tm = step()
        ends[k].record(stream)
        kernel_ms.append(calc.timings())
        del tm
    torch.cuda.synchronize()
    barrier(world)
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    ms_local = float(np.mean(step_ms))
    ms = allreduce_max(ms_local, world)

    # end to end through the C API with host buffers
    host_system = rb.System.from_dict(system)
    for _ in range(2):
        calc.compute(host_system, gradients=GRADIENTS)
    e2e_times = []
    for _ in range(max(3, args.steps // 4)):
        t0 = time.perf_counter()
        out = calc.compute(host_system, gradients=GRADIENTS)
        e2e_times.append(time.perf_counter() - t0)
        del out
    e2e_ms = allreduce_max(1000.0 * float(np.mean(e2e_times)), world)
    clocks = sampler.stop()

    if rank != 0:
        return
    peak, peak_kind = measured_peaks()
    pos_ms = float(np.mean([t["ps_positions"] for t in kernel_ms]))
    achieved = pos_kernel_bytes / (pos_ms / 1000.0) / 1e9
    phases = {name: float(np.mean([t[name] for t in kernel_ms])) for name in kernel_ms[0]}
    line = {
        "metric": METRIC,
        "value": world * N_ATOMS / (ms / 1000.0),
        "unit": "atom-envs/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded random box, no dataset)",
        "config": config({"phase_ms": phases, "output_bytes_per_step": out_bytes, "pairs": n_pairs,
                          "gradient_rows": grad_rows}),
        "e2e": {
            "value": world * N_ATOMS / (e2e_ms / 1000.0),
            "unit": "atom-envs/s",
            "h2d_bytes_per_step": N_ATOMS * (3 * 8 + 4),
            "d2h_bytes_per_step": out_bytes + n_pairs * 8,
        },
        "roofline": {
            "kernel": "ps_positions_staged_kernel",
            "bound": "hbm",
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": achieved / peak,
            "peak_source": peak_kind,
            "algorithmic_bytes_per_launch": pos_kernel_bytes,
            "traffic": profile_traffic("ps_positions_staged_random_box_1000"),
        },
        "clocks": clocks,
        # per step, this library's own kernels: neighbour list (assign, fill,
        # count, write), direction keys and segments, neighbourhood tables
        # (count, fill), fused spherical expansion, power spectrum positions
        # rows (staged) and centre rows (values, own positions rows and
        # strain); beside them 11 CUB sort / scan kernels
        "gpu_launches": 11 * args.steps,
    }
    if not args.no_chosen_forms:
        line["adjoint_form"] = adjoint_form(args.steps, args.warmup)
        # 13 kernels of this library and 9 CUB sort / scan kernels it launches
        line["adjoint_form"]["gpu_launches_per_step"] = 22
        line["batched_form"] = batched_form(args.steps, args.warmup)
        line["surrogate_form"] = surrogate_form(min(args.steps, 5), args.warmup, args.train_steps)
        line["combined_form"] = combined_form(args.steps, args.warmup, args.train_steps, line["value"])
        line["cg_form"] = cg_form(min(args.steps, 10), args.warmup)
        line["lode_form"] = lode_form(min(args.steps, 10), args.warmup)
        # a compact summary of the chosen forms placed before the long objects
        forms = {}
        for name in ("adjoint_form", "batched_form", "combined_form"):
            f = line[name]
            forms[name] = {"value": f["value"], "ms_per_step": f["ms_per_step"],
                           "errors_vs_fp64": f["error_vs_fp64"],
                           "roofline_frac": (f.get("roofline") or {}).get("frac")}
        forms["combined_form"]["vs_dropin"] = line["combined_form"]["vs_dropin"]
        sf = line["surrogate_form"]
        forms["surrogate_form"] = {"power_spectrum_error_vs_fp64": sf["power_spectrum_error_vs_fp64"],
                                   "forces_error_vs_fp64": sf["forces_error_vs_fp64"],
                                   "radial_evaluations_per_s": sf["radial_evaluations_per_s"]}
        line["forms"] = forms
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(system, hypers)
    # the contract's keys and the forms' summary first, the long objects last
    head = {k: v for k, v in line.items() if not k.endswith("_form")}
    tail = {k: v for k, v in line.items() if k.endswith("_form")}
    print(json.dumps({**head, **tail}), flush=True)


if __name__ == "__main__":
    main()

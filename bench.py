"""Benchmark of the B200 VBD cloth step (one JSON line on rank 0).

Headline workload (``draped-cloth``, single GPU): 256 x 256 vertices (65,536), 130,050
triangles, 195,585 bending hinges, 2 m side, released 4 mm above a static sphere (r = 0.4 m)
that stands on the ground plane; stable Neo-Hookean membrane tri_ke = tri_ka = 1e4, tri_kd =
1e-3, bending edge_ke = 1e-2, density 0.1 kg/m^2, contact ke = 1e4 with a 5 mm soft-contact
margin, dt = 1/600 s.  A step is one simulation substep as a user runs it:
``CollisionPipeline.collide`` + ``SolverVBD.step``.  The cloth first drapes for ``SETTLE`` steps
of the reference's fixed 10-iteration loop (untimed, the same trajectory for every arm), so the
timed steps start from a state in contact.

The metric is steps/s to a force-residual tolerance: every step iterates until the residual
gate (``SolverVBD.set_residual_gate``) is met -- the mean over the vertices of the Gauss-Seidel
residual |f_i| / (m_i |g|) that the sweeps form must fall to ``GATE_RHO`` times the mean Jacobi
residual at the step's inertia target y (the plain start), at most ``GATE_CAP`` iterations.  The
spec's 1e-3 of the gravity load (max over the vertices) is unreachable for Gauss-Seidel VBD on
these cloths, in FP32 and in FP64 alike, so the tolerance is the residual level the reference's
default 10 iterations reach: on the settled states the mean residual after 10 plain iterations is
0.87 (draped cloth) and 0.94 (batched worlds) of the residual at y (medians over 40 steps),
rounded up to GATE_RHO.  ``fixed_iterations`` reports the reference's own loop (10 iterations per
step) beside it.

``value`` is steps/s with inputs resident on the device (L2 flushed between timed steps);
``e2e`` is the same loop through the public API with the step's inputs copied from pinned host
memory and the result read back every step.  With --gpus N each rank runs its own replica of
the cloth (a single cloth does not shard), so per-GPU work is fixed ("weak" scaling).

At N = 1 the line also carries ``workloads``: the batched-worlds workload (512 independent cloth
worlds, 1.89 M vertices, one launch per color for all worlds) and the cloth-on-boxes workload
(1024 x 1024 cloth, 1.05 M vertices, on 16 boxes with self-contact; the gate is not available
with self-contact, so it runs the reference's fixed 10 iterations), each with the same fields.
``learned`` (on the line and on the batched-worlds entry) is the learned warm start against
plain VBD at the same residual, one network per feature set ("corrections", the headline, and
"kinematic"), trained on plain-VBD trajectories of other seeds: two drapes of 300 steps, and
256 batched worlds for 800 steps (204,800 cloth steps).  "Same residual" is made exact by
stepping both arms from the same recorded plain-VBD states (the relative gate then fixes the
same absolute tolerance for both), the learned solver fed that trajectory's own previous
correction as its history feature; the learned solver on its own trajectory is reported beside
it, with the residual at y its states reach.

``--impl reference`` times the CPU oracle (the reference's VBD step restated in C++, OpenMP over
the vertices of a color) on the host cores, on the same workload, gate and trajectory; the scene
is built with the checker's own set-up restatement, so that arm loads no product library.  The
reference itself needs Warp, which is not installed here.
The timed steps run inside an NVTX range named ``bench_timed`` (for ncu --nvtx-include).
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

import numpy as np

METRIC = "cloth steps/sec to residual ≤1e-3: learned warm-start vs plain VBD, 1×B200"
DT = 1.0 / 600.0
ITERATIONS = 10
MARGIN = 5.0e-3
SETTLE = 150      # untimed steps before the warm-up: the cloth settles into contact
GATE_CAP = 100    # iteration cap of a gated step
# relative tolerance per workload: the mean Gauss-Seidel residual must fall to GATE_RHO x the mean
# Jacobi residual at y (plain VBD needs about 10 iterations for it on the settled states)
GATE_RHO = {"draped-cloth": 0.9, "batched-worlds": 0.95}
WORKLOADS = {
    "draped-cloth": ("draped cloth 256x256 (65,536 vertices, 130,050 triangles, 195,585 hinges) released 4 mm above "
                     "a static sphere on the ground, 150 settling steps, plain VBD to the residual gate, dt=1/600, "
                     "fp32"),
    "batched-worlds": ("512 cloth worlds, N ~ U{16..96} per side (1.89 M vertices), side ~ U[0.5, 2] m, tri_ke ~ "
                       "logU[1e3, 1e5], 0-4 pins, ground per world, 150 settling steps, plain VBD to the residual "
                       "gate, dt=1/600, fp32, worlds sharded over ranks"),
    "cloth-on-boxes": ("cloth 1024x1024 (1,048,576 vertices, 2,093,058 triangles, 3,141,633 hinges), 4 m side, on "
                       "16 static boxes + ground, self-contact radius 2 mm margin 3 mm, 150 settling steps, "
                       "10 iterations, dt=1/600, fp32"),
}


def gate_config(workload: str) -> dict | None:
    rho = GATE_RHO.get(workload)
    if rho is None:
        return None
    return {"tolerance": rho, "max_iterations": GATE_CAP, "check_every": 1, "relative": True, "norm": "mean",
            "residual": "sweep"}


def build_scene(workload: str, device, builder_cls=None, n: int = 0, rank: int = 0, world: int = 1):
    """(model, q0, solver keywords, extra config) of a workload."""
    from newton_b200 import scenes

    kw = {} if builder_cls is None else {"builder_cls": builder_cls}
    if workload == "draped-cloth":
        model, q0 = scenes.draped_cloth(n=n or 256, seed=rank, device=device, height=0.904, **kw)
        return model, q0, {}, {}
    if workload == "cloth-on-boxes":
        model, q0 = scenes.cloth_on_boxes(n=n or 1024, device=device, **kw)
        return model, q0, dict(particle_enable_self_contact=True, particle_self_contact_radius=0.002,
                               particle_self_contact_margin=0.003), {}
    from newton_b200.sharding import extract_worlds, partition_worlds, world_vertex_counts

    if world == 1:
        full, q_full = scenes.batched_worlds(512, seed=0, device=device, **kw)
        return full, q_full, {}, {"batch_vertices": full.particle_count, "worlds_on_rank0": 512}
    full, q_full = scenes.batched_worlds(512, seed=0, device="cpu", **kw)
    ids = partition_worlds(world_vertex_counts(full), world)[rank]
    model, pidx = extract_worlds(full, ids, device=device)
    return model, q_full[pidx], {}, {"batch_vertices": full.particle_count, "worlds_on_rank0": int(len(ids))}


def algorithmic_bytes_per_iteration(model) -> int:
    """Compulsory bytes of one full Gauss-Seidel iteration, each datum read once:
    60 B/vertex + 44 B/triangle + 32 B/hinge + 8 B per CSR record + 8 B per vertex offset."""
    adj = model.soft_mesh_adjacency
    n_csr = (len(adj.v_adj_tris) + len(adj.v_adj_edges)) // 2
    V, T, E = model.particle_count, model.tri_count, model.edge_count
    return 60 * V + 44 * T + 32 * E + 8 * n_csr + 8 * (V + 1)


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed region: through NVML
    every millisecond from a thread (a timed region of a few milliseconds still gets samples);
    where NVML is unavailable, nvidia-smi every 200 ms."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.path = None
        self.thread = None
        self.samples = []

    def _nvml_handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        try:  # the NVML device of this process's CUDA device, by PCI bus id
            props = torch.cuda.get_device_properties(self.gpu_index)
            bus = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.gpu_index)

    def start(self):
        import threading

        try:
            nv, h = self._nvml_handle()
            reasons_fn = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self.stop_flag = False

            def poll():
                while not self.stop_flag:
                    self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), reasons_fn(h)))
                    time.sleep(0.001)

            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu_index)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict | None:
        if self.thread is not None:
            self.stop_flag = True
            self.thread.join(timeout=5)
            if not self.samples:
                return None
            reasons = sorted({name for _, bits in self.samples for name, bit in self.REASONS if bits & bit})
            return {"sm_mhz": statistics.median(c for c, _ in self.samples), "sm_max_mhz": self.max_mhz,
                    "reasons": reasons, "samples": len(self.samples), "source": "nvml, 1 ms"}
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = [n for n, _ in self.REASONS]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "source": "nvidia-smi, 200 ms"}


def measured_peaks() -> dict:
    here = os.path.dirname(os.path.abspath(__file__))
    try:
        with open(os.path.join(here, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return {"hbm_gbs": float(p["hbm_gbs"]), "source": "measured"}
    except Exception:
        return {"hbm_gbs": 6650.0, "source": "fallback"}


# ------------------------------------------------------------------------------------------------
# CPU legs: the oracle (the reference's step restated in C++) on the host cores
# ------------------------------------------------------------------------------------------------
def _oracle_stepper(model, threads: int, self_contact: dict | None):
    import oracle

    orc = oracle.VBDOracle(model, "f32", threads=threads)
    if self_contact:
        orc.set_self_contact(self_contact["particle_self_contact_radius"], self_contact["particle_self_contact_margin"])
    return orc


def _oracle_step(orc, model, q, qd, gate):
    import oracle

    if model.shape_count:
        orc.set_contacts(*oracle.collide(model, q, MARGIN))
    if gate is None:
        _, q, qd = orc.step(q, qd, None, DT, ITERATIONS)
        return q, qd, ITERATIONS
    _, q, qd, k, _ = orc.gated_step(q, qd, None, DT, gate["tolerance"], gate["max_iterations"],
                                    gate["check_every"], gate["norm"], gate["relative"])
    return q, qd, k


def _parity_of_first_step(model, orc, q, qd, gate, gpu_first: dict) -> dict:
    """The checker's view of the GPU's first timed step: the FP32 oracle takes the same gated step
    from the same state, the FP64 oracle the same number of iterations; max |dx| against both and
    the force residual of the GPU's positions (evaluated by the FP64 oracle after its own step)."""
    import oracle

    threads = os.cpu_count() or 1
    q_o, _, k_o = _oracle_step(orc, model, q, qd, gate)
    k_g = int(gpu_first["iterations"])
    orc64 = oracle.VBDOracle(model, "f64", threads=threads)
    if model.shape_count:
        orc64.set_contacts(*oracle.collide(model, q, MARGIN))
    _, q_64, _ = orc64.step(q, qd, None, DT, k_g)
    q_g = gpu_first["q"]
    orc64.set_positions(q_g)
    r = orc64.residual(DT)
    solvable = ((np.asarray(model.particle_flags) & 1) != 0) & (np.asarray(model.particle_mass) != 0)
    return {"max_dx_vs_fp32_oracle_m": float(np.abs(q_g - q_o).max()),
            "max_dx_vs_fp64_oracle_m": float(np.abs(q_g - q_64).max()),
            "tolerance_m": 1.0e-5, "iterations_gpu": k_g, "iterations_fp32_oracle": int(k_o),
            "residual_max_mg": float(r.max()), "residual_mean_mg": float(r[solvable].mean()) if solvable.any() else 0.0,
            "note": "the first timed step; residual |f_i|/(m_i|g|) of the GPU's positions, Jacobi, FP64"}


def cpu_sample(model, q, qd, gate, self_contact=None, max_seconds: float = 12.0, max_steps: int = 50,
               gpu_first: dict | None = None) -> dict:
    """The oracle stepping the same workload from the given state, on all host cores, for a
    bounded number of steps; with ``gpu_first`` (the GPU's first step from that state), also the
    parity of that step (untimed, before the sample)."""
    threads = os.cpu_count() or 1
    orc = _oracle_stepper(model, threads, self_contact)
    q, qd = np.asarray(q, np.float32), np.asarray(qd, np.float32)
    parity = _parity_of_first_step(model, orc, q, qd, gate, gpu_first) if gpu_first is not None else None
    t0 = time.perf_counter()
    steps, iters = 0, 0
    while True:
        q, qd, k = _oracle_step(orc, model, q, qd, gate)
        steps += 1
        iters += k
        el = time.perf_counter() - t0
        if el >= max_seconds or steps >= max_steps:
            break
    out = {"value": steps / el, "unit": "steps/s", "cores": threads, "kind": "port",
            "vertex_iterations_per_s": model.particle_count * iters / el, "mean_iterations": iters / steps,
            "sample": f"{steps} steps of the same workload from the same state ({model.particle_count} vertices, "
                      f"collide + VBD step{' to the residual gate' if gate else ', 10 iterations'}), {el:.1f} s, "
                      f"oracle stand-in, not reference (Warp is not installed)"}
    if parity is not None:
        out["parity"] = parity
    return out


def run_reference(args) -> None:
    """The CPU oracle on the headline workload: the scene built by the checker's set-up
    restatement, the same settling trajectory and gate, then the timed steps."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.setup import OracleModelBuilder

    workload = args.workload
    model, q0, solver_kw, _ = build_scene(workload, "cpu", builder_cls=OracleModelBuilder, n=args.n)
    gate = gate_config(workload) if not solver_kw else None
    threads = os.cpu_count() or 1
    orc = _oracle_stepper(model, threads, solver_kw)
    q, qd = q0.astype(np.float32), np.zeros_like(q0, dtype=np.float32)
    W, K = max(args.warmup, 3), max(args.steps, 1)
    for _ in range(SETTLE):  # settling: the reference's fixed loop, as in the GPU arm
        q, qd, _ = _oracle_step(orc, model, q, qd, None)
    for _ in range(W):
        q, qd, _ = _oracle_step(orc, model, q, qd, gate)
    # the timed sample: up to K steps, bounded in time
    t0 = time.perf_counter()
    steps, iters = 0, 0
    while steps < K:
        q, qd, k = _oracle_step(orc, model, q, qd, gate)
        steps += 1
        iters += k
        if time.perf_counter() - t0 > 60.0:
            break
    el = time.perf_counter() - t0
    value = steps / el
    cb = {"value": value, "unit": "steps/s", "cores": threads, "kind": "port",
          "sample": f"{steps} steps after {SETTLE + W} settling/warm-up steps of the same trajectory, {el:.1f} s; "
                    f"oracle stand-in, not reference (Warp is not installed)"}
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "steps/s",
        "n_gpus": args.gpus,
        "steps": K,
        "warmup": W,
        "ms_per_step": 1e3 / value,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": dict(workload_config(workload, model, gate),
                       parallelism=_parallelism(workload, int(os.environ.get("WORLD_SIZE", "1")))),
        "mean_iterations": iters / steps,
        "cpu_baseline": cb,
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _parallelism(workload: str, world: int) -> str:
    return f"worlds sharded x{world}" if workload == "batched-worlds" else f"replicas x{world}"


def workload_config(workload: str, model, gate) -> dict:
    """The config object of a workload (identical for the GPU arm and the reference arm)."""
    return {"workload": WORKLOADS[workload], "vertices": int(model.particle_count), "triangles": int(model.tri_count),
            "hinges": int(model.edge_count), "iterations": ("gated" if gate else ITERATIONS), "dt": DT,
            "settle_steps": SETTLE, "settle": "fixed 10 iterations", "l2": "flushed between timed steps",
            "residual_gate": gate or "not available with self-contact: fixed 10 iterations"}


# ------------------------------------------------------------------------------------------------
# GPU arm
# ------------------------------------------------------------------------------------------------
def _launches_per_step(solver, gate_stats, steps: int, colors: int) -> float:
    """Kernels one step launched: the collide kernel + the step graph's top-level kernel nodes +
    (gated) the loop body's kernels per pass of the body (sweeps of a body pass that return at
    once after the gate's decision count as launches)."""
    top = solver.step_kernel_count()
    if gate_stats is None:
        return 1 + (top if top >= 0 else 3 + ITERATIONS * colors)
    passes = gate_stats["body_passes"] / max(gate_stats["steps"], 1)
    return 1 + top + passes * gate_stats["body_kernels"] if top >= 0 else -1


def measure_workload(workload: str, dev, W: int, K: int, world: int, rank: int, local: int, args, cpu: bool) -> dict:
    import torch
    import torch.distributed as dist

    from newton_b200 import CollisionPipeline
    from newton_b200.autotune import time_iterations, tune_sweep
    from newton_b200.solvers import SolverVBD

    model, q0, solver_kw, extra = build_scene(workload, dev, n=args.n, rank=rank, world=world)
    gate = gate_config(workload) if not solver_kw else None
    solver = SolverVBD(model, iterations=ITERATIONS, **solver_kw)
    if gate:
        solver.set_residual_gate(**gate)
    fixed = SolverVBD(model, iterations=ITERATIONS, **solver_kw)  # the reference's fixed loop
    pipe = CollisionPipeline(model, soft_contact_margin=MARGIN)
    contacts = pipe.contacts()
    s0, s1 = model.state(), model.state()
    s0.particle_q.copy_(torch.from_numpy(q0).to(dev))
    stream = torch.cuda.current_stream(dev)

    def substep(solver=solver):
        nonlocal s0, s1
        pipe.collide(s0, contacts)
        solver.step(s0, s1, None, contacts, DT)
        s0, s1 = s1, s0

    for _ in range(SETTLE):
        substep(fixed)
    tune = None
    if not args.no_autotune:
        pipe.collide(s0, contacts)
        tune = tune_sweep(solver, s0, contacts, DT)
        fixed.set_launch(tune["lanes_per_vertex"], tune["block_size"])
    for _ in range(W):
        substep()
    torch.cuda.synchronize()
    # the state the timed steps start from (also the CPU leg's and the fixed-count run's start)
    q_start, qd_start = s0.particle_q.clone(), s0.particle_qd.clone()
    if gate:
        solver.gate_stats(reset=True)

    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)  # > 126 MB L2
    sampler = ClockSampler(local)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    torch.cuda.nvtx.range_push("bench_timed")
    for k in range(K):
        flush.zero_()
        evs[k][0].record(stream)
        substep()
        evs[k][1].record(stream)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    ms = sum(a.elapsed_time(b) for a, b in evs) / K
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    batched = workload == "batched-worlds"
    value = (1e3 if batched else world * 1e3) / ms
    gstats = solver.gate_stats() if gate else None
    colors = len(model.particle_color_groups)
    launches = _launches_per_step(solver, gstats, K, colors)

    # ---- the reference's fixed 10-iteration loop from the same start ------------------------
    s0.particle_q.copy_(q_start)
    s0.particle_qd.copy_(qd_start)
    for _ in range(2):
        substep(fixed)
    s0.particle_q.copy_(q_start)
    s0.particle_qd.copy_(qd_start)
    torch.cuda.synchronize()
    fms = 0.0
    for k in range(K):
        flush.zero_()
        evs[k][0].record(stream)
        substep(fixed)
        evs[k][1].record(stream)
    torch.cuda.synchronize()
    fms = sum(a.elapsed_time(b) for a, b in evs) / K
    fixed_line = {"value": (1e3 if batched else world * 1e3) / fms, "unit": "steps/s", "ms_per_step": fms,
                  "iterations": ITERATIONS, "gpu_launches_per_step": _launches_per_step(fixed, None, K, colors)}

    # ---- roofline of the dominant kernel: the per-color sweep --------------------------------
    # one graph of 4 full iterations (every color once per iteration) replayed between CUDA events
    s0.particle_q.copy_(q_start)
    s0.particle_qd.copy_(qd_start)
    pipe.collide(s0, contacts)
    flush.zero_()
    per_launch_ms = time_iterations(solver, s0, contacts, DT, iterations=4, repeats=10) / colors
    b_iter = algorithmic_bytes_per_iteration(model)
    bytes_per_launch = b_iter / colors
    achieved = bytes_per_launch / (per_launch_ms * 1e-3) / 1e9
    peaks = measured_peaks()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"], "traffic": None,
                "kernel": "sweep_kernel (one color)", "algorithmic_bytes_per_launch": bytes_per_launch,
                "ms_per_launch": per_launch_ms,
                "traffic_note": "DRAM bytes per launch are measured by ncu on a separate capture (profiles/)"}
    if solver_kw:
        roofline["kernel"] = "one color: self-contact gather + sweep_kernel + truncation passes"

    # ---- end to end through the public API with host buffers --------------------------------
    # every step: H2D of the step's inputs (positions, velocities) from pinned host memory,
    # collide + step, D2H of the step's result (positions, velocities); positions and velocities
    # live in one [2, V, 3] block on each side (the states' arrays are views of it)
    V = model.particle_count
    h_state = torch.empty((2, V, 3), dtype=torch.float32, pin_memory=True)
    d_in = torch.empty((2, V, 3), dtype=torch.float32, device=dev)
    d_out = torch.empty((2, V, 3), dtype=torch.float32, device=dev)
    e_in, e_out = model.state(), model.state()
    e_in.particle_q, e_in.particle_qd = d_in[0], d_in[1]
    e_out.particle_q, e_out.particle_qd = d_out[0], d_out[1]
    h_state[0].copy_(q_start)
    h_state[1].copy_(qd_start)

    def e2e_step():
        d_in.copy_(h_state, non_blocking=True)
        pipe.collide(e_in, contacts)
        solver.step(e_in, e_out, None, contacts, DT)
        h_state.copy_(d_out, non_blocking=True)

    for _ in range(W):  # the solver captures its step graph for these buffers here, untimed
        e2e_step()
    h_state[0].copy_(q_start)
    h_state[1].copy_(qd_start)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_ms = 0.0
    for k in range(K):
        flush.zero_()
        e0.record(stream)
        e2e_step()
        e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
    e2e_ms /= K
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())

    out = {
        "metric": METRIC,
        "value": value,
        "unit": "steps/s",
        "ms_per_step": ms,
        "config": dict(workload_config(workload, model, gate), **extra),
        "colors": colors,
        "launch": solver.launch_info(),
        "mean_iterations": (gstats["mean_iterations"] if gstats else ITERATIONS),
        "gate_stats": gstats,
        "vertex_iterations_per_s": value * extra.get("batch_vertices", V) * (gstats["mean_iterations"] if gstats
                                                                            else ITERATIONS),
        "fixed_iterations": fixed_line,
        "roofline": roofline,
        "e2e": {"value": (1e3 if batched else world * 1e3) / e2e_ms, "unit": "steps/s",
                "h2d_bytes_per_step": 2 * V * 12, "d2h_bytes_per_step": 2 * V * 12},
        "gpu_launches": int(round(K * launches)) if launches >= 0 else None,
        "clocks": clocks,
        "autotune": tune,
        "status": solver.status(),
    }
    if cpu and rank == 0 and world == 1:
        if workload == "cloth-on-boxes":
            out["cpu_baseline"] = cpu_boxes_sample(dev, args)
        else:
            qs = q_start.cpu().numpy()
            qds = qd_start.cpu().numpy()
            out["cpu_baseline"] = cpu_sample(model, qs, qds, gate, max_steps=max(3, min(K, 50)),
                                             max_seconds=20.0 if batched else 12.0,
                                             gpu_first=_gpu_first_step(model, solver, pipe, q_start, qd_start, gate))
    out["_states"] = (model, q_start, qd_start)
    return out


def _gpu_first_step(model, solver, pipe, q_start, qd_start, gate) -> dict:
    """The gated step the timed loop began with, again from its start state (for the checker)."""
    import torch

    from newton_b200.solvers import SolverVBD

    check = SolverVBD(model, iterations=ITERATIONS)
    launch = solver.launch_info()
    check.set_launch(launch["lanes_per_vertex"], launch["block_size"])
    if gate:
        check.set_residual_gate(**gate)
    c = pipe.contacts()
    a, b = model.state(), model.state()
    a.particle_q.copy_(q_start)
    a.particle_qd.copy_(qd_start)
    pipe.collide(a, c)
    check.step(a, b, None, c, DT)
    torch.cuda.synchronize()
    k = check.gate_stats()["last_iterations"] if gate else ITERATIONS
    return {"q": a.particle_q.cpu().numpy(), "iterations": k}


def cpu_boxes_sample(dev, args) -> dict:
    """The oracle on a stated smaller cloth-on-boxes scene (the oracle's all-pairs self-contact
    detection is O(V T): 2e12 pair tests per detection at full size)."""
    import torch

    from newton_b200 import CollisionPipeline, scenes
    from newton_b200.solvers import SolverVBD

    kw = dict(particle_enable_self_contact=True, particle_self_contact_radius=0.002, particle_self_contact_margin=0.003)
    model, q0 = scenes.cloth_on_boxes(n=64, side=1.0, device=dev)
    solver = SolverVBD(model, iterations=ITERATIONS, **kw)
    pipe = CollisionPipeline(model, soft_contact_margin=MARGIN)
    c = pipe.contacts()
    a, b = model.state(), model.state()
    a.particle_q.copy_(torch.from_numpy(q0).to(dev))
    for _ in range(SETTLE):
        pipe.collide(a, c)
        solver.step(a, b, None, c, DT)
        a, b = b, a
    torch.cuda.synchronize()
    cb = cpu_sample(model, a.particle_q.cpu().numpy(), a.particle_qd.cpu().numpy(), None, self_contact=kw,
                    max_steps=20, max_seconds=10.0)
    cb["sample"] = "64x64 cloth (4,096 vertices, 1 m side) on 16 boxes with self-contact, " + cb["sample"]
    return cb


# training trajectories of the learned warm start (held out from the timed scenes: other seeds)
FEATURE_SETS = ("corrections", "kinematic")  # the first is the headline arm
TRAIN_EPOCHS = 60
LEARN_TRAIN = {
    # two 256x256 drapes (other seeds and sphere offsets), 300 plain-VBD steps each
    "draped-cloth": {"steps": 300, "samples_per_step": 8192},
    # 256 worlds of the batched distribution (seed 1) for 800 steps: 204,800 cloth steps
    "batched-worlds": {"steps": 800, "samples_per_step": 8192, "worlds": 256},
}


def learned_training_data(workload: str, dev):
    """Plain-VBD trajectories of the workload's distribution (other seeds than the timed scene):
    features of every feature set on the same samples, and the 20-iteration targets."""
    import torch

    from newton_b200 import CollisionPipeline, scenes
    from newton_b200 import learned as L
    from newton_b200.solvers import SolverVBD

    cfg = LEARN_TRAIN[workload]
    if workload == "draped-cloth":
        runs = [scenes.draped_cloth(n=256, seed=seed, device=dev, offset=off, height=0.904)
                for seed, off in ((1, (0.2, -0.1)), (4, (-0.15, 0.25)))]
    else:
        runs = [scenes.batched_worlds(cfg["worlds"], seed=1, device=dev)]
    Xs, Ts = {fs: [] for fs in FEATURE_SETS}, []
    cloth_steps = 0
    vertices = 0
    for i, (model, q0) in enumerate(runs):
        solver = SolverVBD(model, iterations=ITERATIONS)
        pipe = CollisionPipeline(model, soft_contact_margin=MARGIN)
        X, T = L.generate_dataset(model, q0, solver, pipe, steps=cfg["steps"], dt=DT, target_iterations=20,
                                  samples_per_step=cfg["samples_per_step"], seed=1 + i,
                                  trajectory_iterations=ITERATIONS, feature_set=FEATURE_SETS)
        for fs in FEATURE_SETS:
            Xs[fs].append(X[fs])
        Ts.append(T)
        cloth_steps += cfg["steps"] * (cfg.get("worlds", 1))
        vertices = model.particle_count
    X = {fs: torch.cat(Xs[fs]) for fs in FEATURE_SETS}
    T = torch.cat(Ts)
    info = {"cloth_steps": cloth_steps, "trajectory_steps": cfg["steps"] * len(runs),
            "samples": int(T.shape[0]), "samples_per_step": cfg["samples_per_step"],
            "sample_rate": cfg["samples_per_step"] / vertices,
            "target": "x after 20 plain iterations from y, minus y, over L; trajectories advance with 10"}
    return X, T, info


class _StepTimer:
    """CUDA events around each step, L2 flushed before each (the timed loops' protocol)."""

    def __init__(self, dev, flush):
        import torch

        self.torch, self.stream, self.flush, self.evs = torch, torch.cuda.current_stream(dev), flush, []

    def before(self):
        self.flush.zero_()
        e = self.torch.cuda.Event(enable_timing=True)
        e.record(self.stream)
        self.evs.append([e])

    def after(self):
        e = self.torch.cuda.Event(enable_timing=True)
        e.record(self.stream)
        self.evs[-1].append(e)

    def ms(self) -> float:
        self.torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in self.evs) / max(len(self.evs), 1)


def learned_ab(dev, workload: str, plain: dict, start_state, K: int) -> dict:
    """The learned warm start against plain VBD at the same residual tolerance (the BASELINE metric).

    One warm-start network per feature set is trained on plain-VBD trajectories of the workload's
    distribution (other seeds).  Then, from the plain arm's start state, the plain gated
    trajectory is recorded (3 + K steps), and every arm takes one gated step from each recorded
    state ("teacher forced"): both start each step from the same state, so the relative gate holds
    them to the same absolute force residual, and the iterations and times of the last K steps
    are compared.  The learned solver running its own trajectory ("free_running") is reported
    beside it with the residual at y its states end with (the relative gate refers to it)."""
    import torch

    from newton_b200 import CollisionPipeline
    from newton_b200 import learned as L
    from newton_b200.solvers import SolverVBD

    t0 = time.time()
    X, T, info = learned_training_data(workload, dev)
    info["data_s"] = time.time() - t0
    model, q_start, qd_start = start_state
    gate = gate_config(workload)
    launch = plain["launch"]
    batched = workload == "batched-worlds"
    pipe = CollisionPipeline(model, soft_contact_margin=MARGIN)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    W = 3
    states = L.record_plain_states(model, q_start, qd_start, pipe, gate, W + K, DT, launch)
    tp = _StepTimer(dev, flush)
    plain_tf = L.teacher_forced_steps(model, states, pipe, gate, DT, None, launch, warm=W, timer=tp)
    plain_ms = tp.ms()
    arms = {}
    nets = {}
    for fs in FEATURE_SETS:
        mlp = L.WarmStartMLP(dev, seed=0, feature_set=fs)
        nets[fs] = mlp
        mlp.set_standardization(X[fs])
        t1 = time.time()
        hist = mlp.train(mlp.standardize(X[fs]), T, epochs=TRAIN_EPOCHS, batch=16384, lr=2e-3)
        torch.cuda.synchronize()
        t_train = time.time() - t1
        tl = _StepTimer(dev, flush)
        tf = L.teacher_forced_steps(model, states, pipe, gate, DT, mlp, launch, warm=W, timer=tl)
        ms = tl.ms()
        # free running: the learned solver along its own trajectory from the same start
        solver = SolverVBD(model, iterations=ITERATIONS)
        solver.set_launch(launch["lanes_per_vertex"], launch["block_size"])
        solver.set_warm_start(mlp, ITERATIONS)
        solver.set_residual_gate(**gate)
        c = pipe.contacts()
        s0, s1 = model.state(), model.state()
        s0.particle_q.copy_(q_start)
        s0.particle_qd.copy_(qd_start)
        tfr = _StepTimer(dev, flush)
        for k in range(W + K):
            if k == W:
                solver.gate_stats(reset=True)
            if k >= W:
                tfr.before()
            pipe.collide(s0, c)
            solver.step(s0, s1, None, c, DT)
            if k >= W:
                tfr.after()
            s0, s1 = s1, s0
        fr_ms = tfr.ms()
        fr = solver.gate_stats()
        arms[fs] = {
            "steps_per_s": 1e3 / ms,
            "ms_per_step": ms,
            "mean_iterations": tf["mean_iterations"],
            "capped_steps": tf["capped_steps"],
            "speedup_at_equal_residual": plain_ms / ms,
            "iteration_ratio": tf["mean_iterations"] / plain_tf["mean_iterations"],
            "status": tf["status"],
            "free_running": {"steps_per_s": 1e3 / fr_ms, "mean_iterations": fr["mean_iterations"],
                             "capped_steps": fr["capped_steps"],
                             "last_reference_residual": fr["last_reference_residual"],
                             "status": solver.status()},
            "train": {"train_s": t_train, "epochs": TRAIN_EPOCHS, "mse_first_epoch": hist[0], "mse_last_epoch": hist[-1],
                      "target_variance": float(T.var(0).mean())},
        }
        del solver
    head = arms[FEATURE_SETS[0]]
    flops = 2 * (64 * 128 + 128 * 128 + 128 * 3) * model.particle_count
    plain0_us, learned0_us = _start_cost(model, q_start, pipe, nets[FEATURE_SETS[0]], 20)
    start_us = learned0_us - plain0_us
    return {
        "tolerance": gate,
        "protocol": "teacher forced: both arms step from the same recorded plain-VBD states (same y, same "
                    "absolute tolerance); last K of 3 + K steps, L2 flushed before each",
        "feature_set": FEATURE_SETS[0],
        "plain_steps_per_s": 1e3 / plain_ms,
        "plain_mean_iterations": plain_tf["mean_iterations"],
        "plain_capped_steps": plain_tf["capped_steps"],
        "plain_last_reference_residual": plain_tf["last_reference_residual"],
        "learned_steps_per_s": head["steps_per_s"],
        "learned_mean_iterations": head["mean_iterations"],
        "learned_capped_steps": head["capped_steps"],
        "speedup_at_equal_residual": head["speedup_at_equal_residual"],
        "learned_status": head["status"],
        "feature_sets": arms,
        "training_data": info,
        "mlp_flop_per_step": flops,
        "learned_start": {"us_per_step": start_us, "mlp_tflops": flops / (start_us * 1e-6) / 1e12,
                          "note": "features + tcgen05 inference + bounded start, one kernel: a learned step "
                                  "with 0 sweeps minus a plain one (CUDA events, 20 steps)"},
        "unit": "batch steps/s" if batched else "steps/s",
        "note": "the networks never saw the timed scene",
    }


def sweep_profile(workload: str, n: int, worlds: int, steps: int) -> dict:
    """The profile harness of the sweep: the workload's scene (``worlds`` batched worlds, or an
    ``n`` x ``n`` cloth), a few plain 10-iteration steps, then ``steps`` steps inside an NVTX range
    named ``sweep_profile`` (for ncu --nvtx-include); returns their mean device time."""
    import torch

    from newton_b200 import CollisionPipeline, scenes
    from newton_b200.solvers import SolverVBD

    dev = torch.device("cuda:0")
    if workload == "batched-worlds" and worlds:
        model, q0 = scenes.batched_worlds(worlds, seed=0, device=dev)
        kw = {}
    else:
        model, q0, kw, _ = build_scene(workload, dev, n=n)
    solver = SolverVBD(model, iterations=ITERATIONS, **kw)
    pipe = CollisionPipeline(model, soft_contact_margin=MARGIN)
    c = pipe.contacts()
    a, b = model.state(), model.state()
    a.particle_q.copy_(torch.from_numpy(q0).to(dev))
    for _ in range(3):
        pipe.collide(a, c)
        solver.step(a, b, None, c, DT)
        a, b = b, a
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("sweep_profile")
    e0.record()
    for _ in range(steps):
        pipe.collide(a, c)
        solver.step(a, b, None, c, DT)
        a, b = b, a
    e1.record()
    torch.cuda.nvtx.range_pop()
    e1.synchronize()
    return {"workload": workload, "vertices": model.particle_count, "colors": len(model.particle_color_groups),
            "launch": solver.launch_info(), "steps": steps, "ms_per_step": e0.elapsed_time(e1) / steps,
            "algorithmic_bytes_per_iteration": algorithmic_bytes_per_iteration(model)}


def _start_cost(model, q0, pipe, mlp, steps: int, nvtx: str | None = None) -> tuple:
    """Device time per step (us) of a plain and of a learned solver with 0 sweeps from q0 (their
    difference is the learned start: features + tcgen05 inference + start, one kernel); the
    learned steps run inside the NVTX range ``nvtx`` when given."""
    import torch

    from newton_b200.solvers import SolverVBD

    c = pipe.contacts()
    out = []
    for warm in (False, True):
        solver = SolverVBD(model, iterations=0)
        if warm:
            solver.set_warm_start(mlp, 0)
        a, b = model.state(), model.state()
        a.particle_q.copy_(q0)
        pipe.collide(a, c)
        for _ in range(3):
            solver.step(a, b, None, c, DT)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if warm and nvtx:
            torch.cuda.nvtx.range_push(nvtx)
        e0.record()
        for _ in range(steps):
            solver.step(a, b, None, c, DT)
        e1.record()
        if warm and nvtx:
            torch.cuda.nvtx.range_pop()
        e1.synchronize()
        out.append(e0.elapsed_time(e1) / steps * 1e3)
    return out[0], out[1]


def learned_start_profile(workload: str, n: int, worlds: int, steps: int) -> dict:
    """The profile harness of the learned start (the warm-start step mode's fused tcgen05 kernel):
    the workload's scene, an untrained corrections network, a learned solver and a plain one, both
    with 0 sweeps; three steps each, then ``steps`` steps of the learned solver inside an NVTX range
    named ``learned_start`` (for ncu --nvtx-include).  Returns the mean device time of a step of
    each and their difference, the learned start's cost."""
    import torch

    from newton_b200 import CollisionPipeline, scenes
    from newton_b200 import learned as L

    dev = torch.device("cuda:0")
    if workload == "batched-worlds" and worlds:
        model, q0 = scenes.batched_worlds(worlds, seed=0, device=dev)
    else:
        model, q0, _, _ = build_scene(workload, dev, n=n)
    pipe = CollisionPipeline(model, soft_contact_margin=MARGIN)
    mlp = L.WarmStartMLP(dev, seed=0, feature_set="corrections")
    plain_us, learned_us = _start_cost(model, torch.from_numpy(q0).to(dev), pipe, mlp, steps, nvtx="learned_start")
    return {"workload": workload, "vertices": model.particle_count, "steps": steps, "plain_step_us": plain_us,
            "learned_step_us": learned_us, "learned_start_us": learned_us - plain_us}


def mlp_kernels(rows: int, repeats: int) -> dict:
    """Device time of the warm-start MLP kernels on random rows (the profile harness): tcgen05
    inference, the mma.sync inference it replaced, and one training pass (forward + backward +
    weight-gradient GEMMs)."""
    import ctypes

    import torch

    from newton_b200 import _lib
    from newton_b200 import learned as L

    dev = torch.device("cuda:0")
    lib = _lib.load()
    mlp = L.WarmStartMLP(dev, seed=0)
    gen = torch.Generator(device=dev).manual_seed(0)
    X = torch.randn(rows, L.IN, device=dev, generator=gen)
    T = torch.randn(rows, L.OUT, device=dev, generator=gen)
    Y = torch.empty(rows, L.OUT, device=dev)
    flops = 2 * (L.IN * L.HID + L.HID * L.HID + L.HID * L.OUT) * rows
    stream = torch.cuda.current_stream(dev)

    def timed(fn) -> float:
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(repeats):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / repeats

    t_tc = timed(lambda: _lib.check(lib.vbd_mlp_forward(_lib.ptr(mlp.params), _lib.ptr(mlp.w16), _lib.ptr(X), rows,
                                                        _lib.ptr(Y), mlp._stream())))
    t_ms = timed(lambda: _lib.check(lib.vbd_mlp_forward_mma_sync(_lib.ptr(mlp.params), _lib.ptr(mlp.w16), _lib.ptr(X),
                                                                 rows, _lib.ptr(Y), mlp._stream())))
    t_tr = timed(lambda: mlp.gradients(X, T))
    peak = 1628.3
    try:
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")) as f:
            peak = float(json.load(f)["bf16_tflops"])
    except Exception:
        pass
    cnt = ctypes.c_uint32()
    _lib.check(lib.vbd_mlp_timeouts(ctypes.byref(cnt), 0))
    return {"rows": rows, "flop_per_row": flops // rows,
            "tcgen05_inference_ms": t_tc, "tcgen05_inference_tflops": flops / (t_tc * 1e-3) / 1e12,
            "tcgen05_frac_of_bf16_peak": flops / (t_tc * 1e-3) / 1e12 / peak,
            "mma_sync_inference_ms": t_ms, "mma_sync_inference_tflops": flops / (t_ms * 1e-3) / 1e12,
            "training_pass_ms": t_tr, "training_tflops": 3 * flops / (t_tr * 1e-3) / 1e12,
            "input_gbs_tcgen05": rows * L.IN * 4 / (t_tc * 1e-3) / 1e9, "timeouts": cnt.value}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned warm-start A/B")
    ap.add_argument("--no-workloads", action="store_true", help="skip the batched-worlds and cloth-on-boxes entries")
    ap.add_argument("--n", type=int, default=0, help="grid vertices per side (default: the workload's)")
    ap.add_argument("--workload", default="draped-cloth", choices=sorted(WORKLOADS))
    ap.add_argument("--sweep-profile", action="store_true",
                    help="only run the sweep profile harness (--workload, --n, --worlds, --steps) and print its JSON")
    ap.add_argument("--learned-start-profile", action="store_true",
                    help="only run the learned-start profile harness (--workload, --n, --worlds, --steps) and print "
                         "its JSON")
    ap.add_argument("--worlds", type=int, default=0,
                    help="batched worlds of --sweep-profile / --learned-start-profile (default 512)")
    ap.add_argument("--mlp-kernels", type=int, default=0, metavar="ROWS",
                    help="only time the warm-start MLP kernels on ROWS random rows and print their JSON")
    args = ap.parse_args()
    if args.sweep_profile:
        print(json.dumps(sweep_profile(args.workload, args.n, args.worlds, max(args.steps, 1))), flush=True)
        return
    if args.learned_start_profile:
        print(json.dumps(learned_start_profile(args.workload, args.n, args.worlds, max(args.steps, 1))), flush=True)
        return
    if args.mlp_kernels:
        print(json.dumps(mlp_kernels(args.mlp_kernels, max(args.steps, 5))), flush=True)
        return
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    W, K = max(args.warmup, 3), max(args.steps, 1)
    cpu = not args.no_cpu_baseline
    head = measure_workload(args.workload, dev, W, K, world, rank, local, args, cpu)
    start_state = head.pop("_states")
    scaling = "strong" if args.workload == "batched-worlds" else "weak"
    parallelism = _parallelism(args.workload, world)
    line = {
        "metric": METRIC,
        "value": head["value"],
        "unit": "steps/s",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": head["ms_per_step"],
        "higher_is_better": True,
        "scaling": scaling,
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": dict(head["config"], parallelism=parallelism),
    }
    line.update({k: v for k, v in head.items() if k not in ("metric", "value", "unit", "ms_per_step", "config")})
    if rank == 0 and world == 1 and not args.no_learned and args.workload in LEARN_TRAIN:
        # the learned arm starts where the plain arm's timed steps started
        line["learned"] = learned_ab(dev, args.workload, head, start_state, K)
    del start_state
    torch.cuda.empty_cache()
    if rank == 0 and world == 1 and not args.no_workloads:
        line["workloads"] = {}
        for wl in ("batched-worlds", "cloth-on-boxes"):
            if wl == args.workload:
                continue
            r = measure_workload(wl, dev, W, K, 1, 0, local, args, cpu)
            st = r.pop("_states")
            if not args.no_learned and wl in LEARN_TRAIN:
                r["learned"] = learned_ab(dev, wl, r, st, K)
            del st
            line["workloads"][wl] = r
            torch.cuda.empty_cache()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

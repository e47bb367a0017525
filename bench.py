"""Benchmark of the B200 VBD cloth step (one JSON line on rank 0).

Workload (single GPU): the draped-cloth scene -- 256 x 256 vertices (65,536), 130,050 triangles,
195,585 bending hinges, 2 m side, falling onto a static sphere (r = 0.4 m) and the ground plane,
stable Neo-Hookean membrane tri_ke = tri_ka = 1e4, tri_kd = 1e-3, bending edge_ke = 1e-2,
density 0.1 kg/m^2, contact ke = 1e4 with a 5 mm soft-contact margin, dt = 1/600 s, 10 VBD
iterations.  A step is one simulation substep as a user runs it: CollisionPipeline.collide +
SolverVBD.step.

``value`` is steps/s with inputs resident on the device (L2 flushed between timed steps);
``e2e`` is the same loop through the public API with the step's inputs copied from pinned host
memory and the result read back every step.  With --gpus N each rank runs its own replica of
the cloth (a single cloth does not shard), so per-GPU work is fixed ("weak" scaling).
``--impl reference`` times the CPU oracle (the reference's VBD step restated in C++, OpenMP over
the vertices of a color) on the host cores -- the reference itself needs Warp, which is not
installed here.

``--workload`` selects other cloth workloads (the default is the one above):
  * ``batched-worlds``: 512 independent cloth worlds (1.89 M vertices), the worlds sharded over
    the ranks by vertex count (no collective on the data path); ``value`` is whole-batch steps/s
    ("strong" scaling: the batch is fixed as N grows);
  * ``cloth-on-boxes``: 1024 x 1024 cloth (1.05 M vertices) on 16 static boxes with self-contact
    (radius 2 mm, margin 3 mm); replicas per rank.
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
WORKLOAD = ("draped cloth 256x256 (65,536 vertices, 130,050 triangles, 195,585 hinges) on a static sphere + "
            "ground, plain VBD, 10 iterations, dt=1/600, fp32")
WORKLOADS = {
    "draped-cloth": WORKLOAD,
    "batched-worlds": ("512 cloth worlds, N ~ U{16..96} per side (1.89 M vertices), side ~ U[0.5, 2] m, tri_ke ~ "
                       "logU[1e3, 1e5], 0-4 pins, ground per world, plain VBD, 10 iterations, dt=1/600, fp32, worlds "
                       "sharded over ranks"),
    "cloth-on-boxes": ("cloth 1024x1024 (1,048,576 vertices, 2,093,058 triangles, 3,141,633 hinges), 4 m side, on "
                       "16 static boxes + ground, self-contact radius 2 mm margin 3 mm, 10 iterations, dt=1/600, fp32"),
}


def algorithmic_bytes_per_iteration(model) -> int:
    """Compulsory bytes of one full Gauss-Seidel iteration, each datum read once:
    60 B/vertex + 44 B/triangle + 32 B/hinge + 8 B per CSR record + 8 B per vertex offset."""
    adj = model.soft_mesh_adjacency
    n_csr = (len(adj.v_adj_tris) + len(adj.v_adj_edges)) // 2
    V, T, E = model.particle_count, model.tri_count, model.edge_count
    return 60 * V + 44 * T + 32 * E + 8 * n_csr + 8 * (V + 1)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.path = None

    def start(self):
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
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks() -> dict:
    here = os.path.dirname(os.path.abspath(__file__))
    try:
        with open(os.path.join(here, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return {"hbm_gbs": float(p["hbm_gbs"]), "source": "measured"}
    except Exception:
        return {"hbm_gbs": 6650.0, "source": "fallback"}


def sweep_traffic_per_vertex_iteration() -> float | None:
    """DRAM bytes per vertex-iteration of the sweep kernel from the committed ncu summary, if any."""
    here = os.path.dirname(os.path.abspath(__file__))
    try:
        with open(os.path.join(here, "profiles", "sweep_traffic.json")) as f:
            return float(json.load(f)["dram_bytes_per_vertex_iteration"])
    except Exception:
        return None


def cpu_baseline(model, q0, max_seconds: float = 12.0) -> dict:
    import oracle

    threads = os.cpu_count() or 1
    orc = oracle.VBDOracle(model, "f32", threads=threads)
    q, qd = q0.astype(np.float32), np.zeros_like(q0, dtype=np.float32)
    t0 = time.perf_counter()
    steps = 0
    while True:
        if model.shape_count:
            orc.set_contacts(*oracle.collide(model, q, MARGIN))
        _, q, qd = orc.step(q, qd, None, DT, ITERATIONS)
        steps += 1
        el = time.perf_counter() - t0
        if el >= max_seconds or steps >= 50:
            break
    return {"value": steps / el, "unit": "steps/s", "cores": threads, "kind": "port",
            "sample": f"{steps} steps of the same workload (collide + 10-iteration VBD step), {el:.1f} s, "
                      f"oracle stand-in, not reference (Warp is not installed)"}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from newton_b200 import scenes

    model, q0 = scenes.draped_cloth(device="cpu")
    cb = cpu_baseline(model, q0, max_seconds=min(20.0, 4.0 * max(args.steps, 1)))
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": cb["value"],
        "unit": "steps/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 / cb["value"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "vertices": model.particle_count, "iterations": ITERATIONS},
        "cpu_baseline": cb,
        "e2e": {"value": cb["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def learned_ab(dev, n: int, plain_steps_per_s: float) -> dict:
    """Learned warm start against plain VBD on the draped-cloth distribution (bounded: ~30 s).

    Trains the warm-start network on two plain-VBD drapes (sphere offsets (0.2, -0.1) and
    (-0.15, 0.25); targets: 20-iteration corrections; 2048 sampled vertices per step), then on a
    held-out drape (offset (0.05, 0.1)) finds per checked step the fewest warm-started iterations
    whose mean residual matches plain VBD's 10-iteration one on the same state, and times
    ``SolverVBD.step`` in the learned mode at that count along its own trajectory."""
    import torch

    from newton_b200 import CollisionPipeline, _lib, scenes
    from newton_b200 import learned as L
    from newton_b200.solvers import SolverVBD

    t0 = time.time()
    Xs, Ts = [], []
    for seed, off in ((1, (0.2, -0.1)), (4, (-0.15, 0.25))):
        model, q0 = scenes.draped_cloth(n=n, seed=seed, device=dev, offset=off)
        solver = SolverVBD(model, iterations=ITERATIONS)
        pipe = CollisionPipeline(model, soft_contact_margin=MARGIN)
        X, T = L.generate_dataset(model, q0, solver, pipe, steps=300, dt=DT, target_iterations=20,
                                  samples_per_step=2048, seed=seed, trajectory_iterations=ITERATIONS)
        Xs.append(X)
        Ts.append(T)
    X, T = torch.cat(Xs), torch.cat(Ts)
    t_data = time.time() - t0
    mlp = L.WarmStartMLP(dev, seed=0)
    mlp.set_standardization(X)
    t1 = time.time()
    hist = mlp.train(mlp.standardize(X), T, epochs=20, batch=32768, lr=2e-3)
    torch.cuda.synchronize()
    t_train = time.time() - t1
    target_var = float(T.var(0).mean())

    model, q0 = scenes.draped_cloth(n=n, seed=2, device=dev, offset=(0.05, 0.1))
    solver = SolverVBD(model, iterations=ITERATIONS)
    pipe = CollisionPipeline(model, soft_contact_margin=MARGIN)
    k, records = L.calibrate_iterations(model, q0, solver, pipe, mlp, steps=300, dt=DT, check_every=30)
    solver_tf = SolverVBD(model, iterations=ITERATIONS)
    k_tf, records_tf = L.calibrate_iterations(model, q0, solver_tf, pipe, mlp, steps=300, dt=DT, check_every=30,
                                              advance="plain")

    # inference cost: features + MLP + start offset, after a forward pass
    c = pipe.contacts()
    s0 = model.state()
    s0.particle_q.copy_(torch.from_numpy(q0).to(dev))
    pipe.collide(s0, c)
    solver.forward(s0, c, DT)
    V = model.particle_count
    work = torch.empty(V * 70, dtype=torch.float32, device=dev)
    corr = torch.zeros((V, 3), dtype=torch.float32, device=dev)
    lib = _lib.load()
    stream = torch.cuda.current_stream(dev)

    def infer():
        _lib.check(lib.vbd_mlp_warm_start(solver._handle, _lib.ptr(mlp.params), _lib.ptr(mlp.w16), _lib.ptr(corr),
                                          _lib.ptr(mlp.mean), _lib.ptr(mlp.inv_std), _lib.ptr(work), work.numel(),
                                          solver._stream()))

    for _ in range(3):
        infer()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(20):
        infer()
    e1.record(stream)
    e1.synchronize()
    infer_ms = e0.elapsed_time(e1) / 20

    # the learned step mode at the calibrated iteration count, along its own trajectory
    k_run = min(k, 10)
    solver = SolverVBD(model, iterations=ITERATIONS)
    solver.set_warm_start(mlp, k_run)
    s0, s1 = model.state(), model.state()
    s0.particle_q.copy_(torch.from_numpy(q0).to(dev))

    def substep():
        nonlocal s0, s1
        pipe.collide(s0, c)
        solver.step(s0, s1, None, c, DT)
        s0, s1 = s1, s0

    for _ in range(200):
        substep()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(300):
        substep()
    e1.record(stream)
    e1.synchronize()
    learned_sps = 300 * 1e3 / e0.elapsed_time(e1)
    st = solver.status()
    flops = 2 * (64 * 128 + 128 * 128 + 128 * 3) * V
    return {
        "iterations_to_equal_residual": k,
        "not_reached_marker": 11,
        "plain_iterations": ITERATIONS,
        "plain_steps_per_s": plain_steps_per_s,
        "learned_steps_per_s_at_that_count": learned_sps,
        "speedup_at_equal_residual": (learned_sps / plain_steps_per_s) if k <= ITERATIONS else None,
        "learned_trajectory_status": st,
        "per_check": [{"step": r["step"], "plain_residual": r["plain"], "k_learned": r["k"],
                       "k_previous_correction": r["k_previous_correction"]} for r in records],
        "teacher_forced": {
            "iterations_to_equal_residual": k_tf,
            "note": "the state advances with plain VBD; at each checked step the learned start is scored on "
                    "that state",
            "per_check": [{"step": r["step"], "plain_residual": r["plain"], "k_learned": r["k"],
                           "k_previous_correction": r["k_previous_correction"],
                           "learned_residual_after_1_2_5_10": [r["warm"][i] for i in (0, 1, 4, 9)],
                           "plain_residual_after_1_2_5_10": [r["plain_curve"][i] for i in (0, 1, 4, 9)]}
                          for r in records_tf],
        },
        "train": {"samples": int(X.shape[0]), "data_s": t_data, "train_s": t_train, "epochs": 20,
                  "mse_first_epoch": hist[0], "mse_last_epoch": hist[-1], "target_variance": target_var},
        "inference_ms": infer_ms,
        "inference_tflops": flops / (infer_ms * 1e-3) / 1e12,
        "residual": "mean over solvable vertices of |f_i| / (m_i |g|) after the iterations",
    }


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned warm-start A/B")
    ap.add_argument("--n", type=int, default=0, help="grid vertices per side (default: the workload's)")
    ap.add_argument("--workload", default="draped-cloth", choices=sorted(WORKLOADS))
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist

    from newton_b200 import CollisionPipeline, scenes
    from newton_b200.autotune import time_iterations, tune_sweep
    from newton_b200.solvers import SolverVBD

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    W, K = max(args.warmup, 3), max(args.steps, 1)
    solver_kw = {}
    scaling, parallelism = "weak", f"replicas x{world}"
    if args.workload == "draped-cloth":
        model, q0 = scenes.draped_cloth(n=args.n or 256, seed=rank, device=dev)
    elif args.workload == "cloth-on-boxes":
        model, q0 = scenes.cloth_on_boxes(n=args.n or 1024, device=dev)
        solver_kw = dict(particle_enable_self_contact=True, particle_self_contact_radius=0.002,
                         particle_self_contact_margin=0.003)
    else:
        from newton_b200.sharding import extract_worlds, partition_worlds, world_vertex_counts

        full, q_full = scenes.batched_worlds(512, seed=0, device="cpu")
        ids = partition_worlds(world_vertex_counts(full), world)[rank]
        model, pidx = extract_worlds(full, ids, device=dev)
        q0 = q_full[pidx]
        job_vertices = full.particle_count
        scaling, parallelism = "strong", f"worlds sharded x{world}"
    solver = SolverVBD(model, iterations=ITERATIONS, **solver_kw)
    pipe = CollisionPipeline(model, soft_contact_margin=MARGIN)
    contacts = pipe.contacts()
    s0, s1 = model.state(), model.state()
    s0.particle_q.copy_(torch.from_numpy(q0).to(dev))
    stream = torch.cuda.current_stream(dev)

    def substep():
        nonlocal s0, s1
        pipe.collide(s0, contacts)
        solver.step(s0, s1, None, contacts, DT)
        s0, s1 = s1, s0

    # let the cloth reach the sphere so contacts are part of the measured steps
    for _ in range(W):
        substep()
    tune = None
    if not args.no_autotune:
        pipe.collide(s0, contacts)
        tune = tune_sweep(solver, s0, contacts, DT)
    for _ in range(W):
        substep()
    torch.cuda.synchronize()

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
    value = (1e3 if args.workload == "batched-worlds" else world * 1e3) / ms

    # ---- roofline of the dominant kernel: the per-color sweep --------------------------------
    # one graph of 4 full iterations (every color once per iteration) replayed between CUDA events
    colors = len(model.particle_color_groups)
    pipe.collide(s0, contacts)
    flush.zero_()
    per_launch_ms = time_iterations(solver, s0, contacts, DT, iterations=4, repeats=10) / colors
    # with self-contact an iteration also runs the contact gather and truncation passes
    b_iter = algorithmic_bytes_per_iteration(model)
    bytes_per_launch = b_iter / colors
    achieved = bytes_per_launch / (per_launch_ms * 1e-3) / 1e9
    peaks = measured_peaks()
    tpv = sweep_traffic_per_vertex_iteration()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
                "traffic": (tpv * model.particle_count / colors) if (tpv and args.workload == "draped-cloth") else None,
                "kernel": "sweep_kernel (one color)", "algorithmic_bytes_per_launch": bytes_per_launch,
                "ms_per_launch": per_launch_ms}
    if solver_kw:
        roofline["kernel"] = "one color: self-contact gather + sweep_kernel + truncation passes"

    # ---- residual reached by the plain 10-iteration step ------------------------------------
    pipe.collide(s0, contacts)
    solver.forward(s0, contacts, DT)
    solver.iterate(contacts, DT, ITERATIONS)
    resid = float(solver.residual(contacts, DT).item())

    # ---- end to end through the public API with host buffers --------------------------------
    # every step: H2D of the step's inputs (positions, velocities) from pinned host memory,
    # collide + step, D2H of the step's result (positions, velocities)
    # positions and velocities live in one [2, V, 3] block on each side (the states' arrays are
    # views of it), so each direction is one copy
    V = model.particle_count
    h_state = torch.empty((2, V, 3), dtype=torch.float32, pin_memory=True)
    d_in = torch.empty((2, V, 3), dtype=torch.float32, device=dev)
    d_out = torch.empty((2, V, 3), dtype=torch.float32, device=dev)
    e_in, e_out = model.state(), model.state()
    e_in.particle_q, e_in.particle_qd = d_in[0], d_in[1]
    e_out.particle_q, e_out.particle_qd = d_out[0], d_out[1]
    h_state[0].copy_(s0.particle_q)
    h_state[1].copy_(s0.particle_qd)

    def e2e_step():
        d_in.copy_(h_state, non_blocking=True)
        pipe.collide(e_in, contacts)
        solver.step(e_in, e_out, None, contacts, DT)
        h_state.copy_(d_out, non_blocking=True)

    for _ in range(W):  # the solver captures its step graph for these buffers here, untimed
        e2e_step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    Ke = max(K // 4, 10)
    e2e_ms = 0.0
    for k in range(Ke):
        flush.zero_()
        e0.record(stream)
        e2e_step()
        e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
    e2e_ms /= Ke
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())

    # kernels of one timed step: the collide kernel + the kernel nodes of the solver's step graph
    # (counted by the library when it captured the step)
    step_kernels = solver.step_kernel_count()
    launches_per_step = 1 + (step_kernels if step_kernels >= 0 else 3 + ITERATIONS * colors)
    st = solver.status()
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "steps/s",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": scaling,
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload], "vertices": V, "triangles": model.tri_count,
                   "hinges": model.edge_count,
                   "colors": colors, "iterations": ITERATIONS, "dt": DT, "l2": "flushed between timed steps",
                   "parallelism": parallelism, "launch": solver.launch_info(),
                   "step_kernel": solver.step_kernel_info(),
                   "residual_gate": "not applied: fixed 10 iterations (plain VBD)"},
        "vertex_iterations_per_s": value * V * ITERATIONS,
        "residual_after_step": resid,
        "roofline": roofline,
        "e2e": {"value": world * 1e3 / e2e_ms, "unit": "steps/s", "h2d_bytes_per_step": 2 * V * 12,
                "d2h_bytes_per_step": 2 * V * 12},
        "gpu_launches": K * launches_per_step,
        "clocks": clocks,
        "autotune": tune,
        "status": st,
    }
    if args.workload == "batched-worlds":
        line["config"]["worlds_on_rank0"] = int(len(np.unique(model.particle_world)))
        line["config"]["batch_vertices"] = job_vertices
        line["vertex_iterations_per_s"] = value * job_vertices * ITERATIONS
        line["e2e"]["value"] = 1e3 / e2e_ms
    if rank == 0 and world == 1 and not args.no_learned and args.workload == "draped-cloth":
        line["learned"] = learned_ab(dev, args.n or 256, value)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        if args.workload == "cloth-on-boxes":
            line["cpu_baseline"] = {"value": None, "unit": "steps/s", "cores": 0, "kind": "port",
                                    "sample": "not measured: the oracle's all-pairs self-contact detection is "
                                              "O(V*T) (2e12 pair tests per detection at this size)"}
        else:
            line["cpu_baseline"] = cpu_baseline(model, q0)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

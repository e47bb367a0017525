"""Launch-shape autotuner of the VBD sweep (lanes per vertex x threads per block).

For every candidate shape, ``iterations`` full Gauss-Seidel iterations (every color once) of the
staged API are captured into a CUDA graph and replayed with CUDA events around the replay, so
the timing is device time only (no host launch gaps).  Every block size computes the same
arithmetic; the lane count only changes the summation order of a vertex's element
contributions, so a tuned solver stays within the parity tolerance.
"""

from __future__ import annotations

import itertools

import torch

LANES = (0, 1, 2, 4, 8, 16)   # 0 = record-parallel sweep
BLOCKS = (64, 128, 256)


def time_iterations(solver, state, contacts, dt: float, iterations: int = 4, repeats: int = 5) -> float:
    """Device milliseconds of one full iteration (all colors), from graph replays."""
    dev = solver.model.device
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        solver.forward(state, contacts, dt)
        solver.iterate(contacts, dt, 1)  # warm the launch path outside capture
        with torch.cuda.graph(g, stream=side):
            solver.iterate(contacts, dt, iterations)
    torch.cuda.current_stream(dev).wait_stream(side)
    stream = torch.cuda.current_stream(dev)
    best = float("inf")
    for _ in range(repeats):
        solver.forward(state, contacts, dt)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.replay()
        e1.record(stream)
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / iterations)
    del g
    return best


def tune_sweep(solver, state, contacts, dt: float, iterations: int = 4, repeats: int = 5, lanes=LANES, blocks=BLOCKS,
               verbose: bool = False) -> dict:
    """Pick (lanes_per_vertex, block_size) for ``solver``; leaves the best shape set on it."""
    results = {}
    for L, B in itertools.product(lanes, blocks):
        solver.set_launch(L, B)
        results[(L, B)] = time_iterations(solver, state, contacts, dt, iterations, repeats)
        if verbose:
            print(f"lanes={L:2d} block={B:3d}: {results[(L, B)] * 1e3:8.1f} us/iteration")
    (L, B), t = min(results.items(), key=lambda kv: kv[1])
    solver.set_launch(L, B)
    return {"lanes_per_vertex": L, "block_size": B, "ms_per_iteration": t,
            "table": {f"{k[0]}x{k[1]}": round(v * 1e3, 2) for k, v in results.items()}, "table_unit": "us/iteration"}

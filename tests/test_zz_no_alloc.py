"""GPU test of vbd_step_static, the allocation-free step entry point.

vbd_step_static serves callers that cannot call cudaMalloc (code running during stream capture,
host callbacks or real-time loops where an allocation could block or synchronize the device,
embedders whose device memory belongs to a framework allocator): it runs the step with scratch
from a static device array instead of a VbdSolver's allocations.  This test calls it through the
C ABI twice in a row and compares each result with the solver entry point (vbd_step) on the same
inputs: within the parity tolerance, and bit for bit (both read the same packed contact table).
It also checks that the calls after the first leave the device memory in use unchanged.  The
file is named so that pytest collects it last.
"""

import ctypes

import numpy as np
import pytest
import torch

from newton_b200 import CollisionPipeline, _lib, scenes
from newton_b200.solvers import SolverVBD

pytestmark = pytest.mark.gpu

DT = 1.0 / 600.0
TOL = 1.0e-5  # m, the parity tolerance of the step tests


def _static_step(model, s_in, s_out, contacts, iterations):
    lib = _lib.load()
    dm = model.device_model()
    stream = ctypes.c_void_p(torch.cuda.current_stream(model.device).cuda_stream)
    c = ctypes.byref(contacts.c_struct()) if contacts is not None else None
    _lib.check(lib.vbd_step_static(dm.handle, _lib.ptr(s_in.particle_q), _lib.ptr(s_in.particle_qd),
                                   _lib.ptr(s_in.particle_f), _lib.ptr(s_out.particle_q), _lib.ptr(s_out.particle_qd),
                                   c, ctypes.c_float(DT), iterations, ctypes.c_float(1e-2), stream))


def test_static_step_matches_solver_step_twice():
    model, q0 = scenes.single_cloth(n=40, side=1.0, seed=11, pin_top_corners=True, ground=0.0,
                                    sphere=((0.0, 0.0, 0.5), 0.4), height=0.904)
    dev = model.device
    pipe = CollisionPipeline(model, soft_contact_margin=5e-3)
    solver = SolverVBD(model, iterations=10, lanes_per_vertex=4, block_size=128)

    # solver path
    a0, a1 = model.state(), model.state()
    a0.particle_q.copy_(torch.from_numpy(q0).to(dev))
    ca = pipe.contacts()
    ref = []
    for _ in range(2):
        pipe.collide(a0, ca)
        solver.step(a0, a1, None, ca, DT)
        torch.cuda.synchronize()
        ref.append((a1.particle_q.cpu().numpy(), a1.particle_qd.cpu().numpy(), a0.particle_q.cpu().numpy()))
        a0, a1 = a1, a0

    # allocation-free path, two calls in a row on the same static scratch
    b0, b1 = model.state(), model.state()
    b0.particle_q.copy_(torch.from_numpy(q0).to(dev))
    cb = pipe.contacts()
    # a warm-up call on scratch states: the first call on a device looks up the array's address
    w0, w1 = model.state(), model.state()
    pipe.collide(w0, cb)
    _static_step(model, w0, w1, cb, 1)
    torch.cuda.synchronize()
    reserved = torch.cuda.memory_reserved(dev)
    free0 = torch.cuda.mem_get_info(dev)[0]
    for k in range(2):
        pipe.collide(b0, cb)
        _static_step(model, b0, b1, cb, 10)
        torch.cuda.synchronize()
        q, qd, qin = b1.particle_q.cpu().numpy(), b1.particle_qd.cpu().numpy(), b0.particle_q.cpu().numpy()
        assert cb.count() > 0
        assert np.abs(q - ref[k][0]).max() <= TOL
        assert np.abs(qd - ref[k][1]).max() <= TOL / DT
        assert np.array_equal(q, ref[k][0]) and np.array_equal(qd, ref[k][1])
        assert np.array_equal(qin, q)  # state_in.particle_q holds the solved positions, as in vbd_step
        status = _lib.VbdStatus()
        _lib.check(_lib.load().vbd_step_static_status(ctypes.byref(status)))
        assert status.nonfinite_updates == 0 and status.singular_blocks == 0 and status.contact_overflow == 0
        b0, b1 = b1, b0
    # nothing was allocated by the two calls: torch's pool and the device's free memory are unchanged
    # (the free-memory check allows the driver's 2 MiB page granularity for unrelated bookkeeping)
    assert torch.cuda.memory_reserved(dev) == reserved
    assert torch.cuda.mem_get_info(dev)[0] >= free0 - (2 << 20)


def test_static_step_rejects_models_beyond_its_scratch():
    model, q0 = scenes.single_cloth(n=129, side=1.0, seed=12, ground=None)  # 16,641 > 16,384 particles
    s0, s1 = model.state(), model.state()
    with pytest.raises(_lib.VbdError, match="at most 16384"):
        _static_step(model, s0, s1, None, 1)

"""Particle-vs-static-shape contact generation (the soft branch of ``CollisionPipeline.collide``).

``CollisionPipeline.collide(state, contacts)`` fills ``contacts`` with one record per
(particle, shape) pair whose signed distance is below ``soft_contact_margin + shape margin +
particle radius`` -- ``newton/_src/sim/collide.py:1553-1590`` launching
``create_soft_contacts`` (``newton/_src/geometry/kernels.py:1020-1184``).  The work runs in the
CUDA library (``vbd_collide``).
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib
from .model import Contacts, Model, State


class CollisionPipeline:
    def __init__(self, model: Model, soft_contact_margin: float = 0.01, soft_contact_max: int | None = None):
        self.model = model
        self.soft_contact_margin = float(soft_contact_margin)
        self.soft_contact_max = model.particle_count * model.shape_count if soft_contact_max is None else soft_contact_max

    def contacts(self) -> Contacts:
        return Contacts(self.soft_contact_max, self.model.device)

    def collide(self, state: State, contacts: Contacts) -> None:
        lib = _lib.load()
        dm = self.model.device_model()
        stream = torch.cuda.current_stream(self.model.device).cuda_stream
        _lib.check(
            lib.vbd_collide(
                dm.handle,
                _lib.ptr(state.particle_q),
                ctypes.c_float(self.soft_contact_margin),
                ctypes.byref(contacts.c_struct()),
                ctypes.c_void_p(stream),
            )
        )

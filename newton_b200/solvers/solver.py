"""Solver plugin base class (``newton/_src/solvers/solver.py:187-431``)."""

from __future__ import annotations

from ..model import Contacts, Control, Model, State


class SolverBase:
    """Generic solver interface: ``step(state_in, state_out, control, contacts, dt)``."""

    def __init__(self, model: Model):
        self.model = model

    @property
    def device(self):
        return self.model.device

    def reset(self, state: State, world_mask=None, flags=None) -> None:
        """Reset solver-specific buffers (no-op by default, as in the reference)."""

    def step(self, state_in: State, state_out: State, control: Control | None, contacts: Contacts | None,
             dt: float) -> None:
        raise NotImplementedError()

    def notify_model_changed(self, flags: int) -> None:
        """Refresh internal copies of model data that changed after construction."""

    def update_contacts(self, contacts: Contacts, state: State | None = None) -> None:
        raise NotImplementedError()

    @classmethod
    def register_custom_attributes(cls, builder) -> None:
        pass

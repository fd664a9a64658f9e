"""Particle data for the Python mirror of the plugin: what HOOMD's
SystemDefinition, ParticleData and group provide to the reference's Stokes
class (positions, orientations in the acceleration slot, unwrapped positions
in the velocity slot, images, the box and the time step)."""
from __future__ import annotations

import numpy as np
import torch


class System:
    """N unit spheres in a periodic box (Lx, Ly, Lz, xy), state on one CUDA device."""

    def __init__(self, pos, box, dt, ori=None, device="cuda", timestep=0):
        pos = np.asarray(pos, np.float32)
        N = len(pos)
        if pos.shape[1] == 3:
            pos = np.concatenate([pos, np.zeros((N, 1), np.float32)], 1)
        self.N = N
        self.box = tuple(float(v) for v in box) if len(box) == 4 else (*map(float, box), 0.0)
        self.dt = float(dt)
        self.timestep = int(timestep)
        self.device = torch.device(device)
        t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=self.device).view(-1)
        self.pos = t(pos)
        self.pos_gb = t(pos)
        self.ori = t(np.tile([0.0, 0.0, 1.0], N) if ori is None else np.asarray(ori, np.float32))
        self.image = torch.zeros(3 * N, dtype=torch.int32, device=self.device)
        self.force = torch.zeros(6 * N, device=self.device)
        self.velocity = torch.zeros(11 * N, device=self.device)
        self.all = range(N)
        self.box_variant = None   # box_resize-style xy tilt (variant.shear_variant)
        self.methods = []

    def set_box_variant(self, variant):
        """Deform the box with a shear variant, as HOOMD's box_resize(xy=...) does."""
        self.box_variant = variant.cpp_variant if variant is not None else None

    def run(self, steps):
        """Advance every attached integration method by `steps` steps (hoomd.run)."""
        for _ in range(int(steps)):
            for m in self.methods:
                m.cpp_method.integrateStepOne(self.timestep)
            self.timestep += 1


_current: System | None = None


def set_current(system: System | None):
    """The system that 'now' offsets and new integrators refer to (hoomd.context.current)."""
    global _current
    _current = system


def current() -> System | None:
    return _current

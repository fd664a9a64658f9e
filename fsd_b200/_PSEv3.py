"""Mirror of the reference's compiled plugin module `_PSEv3` (module.cc:62-71).

Exports the same names: `Stokes` (Stokes.cc:1692-1710: setT, setShear,
setParams, OutputData, setResistanceTable, setSparseMath, AllocateWorkSpaces,
setFriction) and the shear-function classes of SpecificShearFunction.h,
VariantShearFunction.h and ShearFunction.h.  `Stokes` drives the CUDA path
through the C ABI (fsd_b200.core.FSD); the shear functions are host-side
arithmetic, restated with the reference's conventions: time steps are
unsigned 32-bit, so `timestep - offset` wraps for timesteps before the
offset, pi is the reference's 3.1415926536, and the chirp's log ratio is
single precision (logf).
"""
from __future__ import annotations

import math
import os
from pathlib import Path

import numpy as np

PI_REF = 3.1415926536


def _elapsed(timestep: int, offset: int) -> int:
    """(timestep - offset) as the reference's unsigned int arithmetic."""
    return (int(timestep) - int(offset)) & 0xFFFFFFFF


def _logf(x: float) -> float:
    return float(np.log(np.float32(x), dtype=np.float32))


class ShearFunction:
    """Base class (ShearFunction.h:19-36)."""

    def getShearRate(self, timestep: int) -> float:  # noqa: N802 (reference names)
        raise NotImplementedError

    def getStrain(self, timestep: int) -> float:  # noqa: N802
        raise NotImplementedError

    def getOffset(self) -> int:  # noqa: N802
        raise NotImplementedError


class SteadyShearFunction(ShearFunction):
    """SpecificShearFunction.h SteadyShearFunction."""

    def __init__(self, shear_rate: float, offset: int, dt: float):
        self.shear_rate, self.offset, self.dt = float(shear_rate), int(offset), float(dt)

    def getShearRate(self, timestep):  # noqa: N802
        return self.shear_rate

    def getStrain(self, timestep):  # noqa: N802
        return self.shear_rate * _elapsed(timestep, self.offset) * self.dt

    def getOffset(self):  # noqa: N802
        return self.offset


class SinShearFunction(ShearFunction):
    """Oscillatory shear, real (not angular) frequency."""

    def __init__(self, max_shear_rate: float, frequency: float, offset: int, dt: float):
        self.rate, self.freq, self.offset, self.dt = float(max_shear_rate), float(frequency), int(offset), float(dt)

    def getShearRate(self, timestep):  # noqa: N802
        return self.rate * math.cos(self.freq * 2 * PI_REF * (_elapsed(timestep, self.offset) * self.dt))

    def getStrain(self, timestep):  # noqa: N802
        return self.rate * math.sin(self.freq * 2 * PI_REF * (_elapsed(timestep, self.offset) * self.dt)) \
            / self.freq / 2 / PI_REF

    def getOffset(self):  # noqa: N802
        return self.offset


class ChirpShearFunction(ShearFunction):
    """Exponential chirp between angular frequencies omega_0 and omega_f over periodT."""

    def __init__(self, amp, omega_0, omega_f, periodT, offset, dt):  # noqa: N803
        self.amp, self.w0, self.wf = float(amp), float(omega_0), float(omega_f)
        self.T, self.offset, self.dt = float(periodT), int(offset), float(dt)

    def _omega(self, timestep):
        return self.w0 * math.exp(self.dt * _elapsed(timestep, self.offset) * _logf(self.wf / self.w0) / self.T)

    def _phase(self, timestep):
        lr = _logf(self.wf / self.w0)
        return self.T * self.w0 / lr * (math.exp(self.dt * _elapsed(timestep, self.offset) * lr / self.T) - 1)

    def getShearRate(self, timestep):  # noqa: N802
        return self.amp * self._omega(timestep) * math.cos(self._phase(timestep))

    def getStrain(self, timestep):  # noqa: N802
        return self.amp * math.sin(self._phase(timestep))

    def getOffset(self):  # noqa: N802
        return self.offset


class TukeyWindowFunction(ShearFunction):
    """Tukey window: strain is the window value, shear rate its time derivative."""

    def __init__(self, periodT, tukey_param, offset, dt):  # noqa: N803
        self.T, self.a, self.offset, self.dt = float(periodT), float(tukey_param), int(offset), float(dt)
        self.omega = 2 * PI_REF / self.a

    def _rel(self, timestep):
        return _elapsed(timestep, self.offset) * self.dt / self.T

    def getShearRate(self, timestep):  # noqa: N802
        t = self._rel(timestep)
        if t <= 0 or t >= 1 or (self.a / 2 <= t <= 1 - self.a / 2):
            return 0.0
        if t < 0.5:
            return -(math.sin(self.omega * (t - self.a / 2))) / 2 * self.omega / self.T
        return -(math.sin(self.omega * (t - 1 + self.a / 2))) / 2 * self.omega / self.T

    def getStrain(self, timestep):  # noqa: N802
        t = self._rel(timestep)
        if t <= 0 or t >= 1:
            return 0.0
        if self.a / 2 <= t <= 1 - self.a / 2:
            return 1.0
        if t < 0.5:
            return (1 + math.cos(self.omega * (t - self.a / 2))) / 2
        return (1 + math.cos(self.omega * (t - 1 + self.a / 2))) / 2

    def getOffset(self):  # noqa: N802
        return self.offset


class WindowedFunction(ShearFunction):
    """Strain = base strain x window; shear rate by the product rule."""

    def __init__(self, base: ShearFunction, window: ShearFunction):
        self.base, self.window = base, window

    def getShearRate(self, timestep):  # noqa: N802
        return self.base.getShearRate(timestep) * self.window.getStrain(timestep) + \
            self.base.getStrain(timestep) * self.window.getShearRate(timestep)

    def getStrain(self, timestep):  # noqa: N802
        return self.base.getStrain(timestep) * self.window.getStrain(timestep)

    def getOffset(self):  # noqa: N802
        return self.base.getOffset()


class VariantShearFunction:
    """Box tilt from a shear function, wrapped into [min_value, max_value)
    (VariantShearFunction.cc): 0 before the offset, the last value after
    offset + total_timestep."""

    def __init__(self, shear_func: ShearFunction, total_timestep: int, min_value: float, max_value: float):
        if int(total_timestep) <= 0:
            raise RuntimeError("Cannot create a shear_variant with 0 or negative points")
        self.f = shear_func
        self.total = int(total_timestep)
        self.lo, self.hi = float(min_value), float(max_value)
        self.range = self.hi - self.lo
        self.offset = shear_func.getOffset()
        self.end_value = self.wrapValue(shear_func.getStrain(self.offset + self.total))

    def wrapValue(self, v):  # noqa: N802
        return v - self.range * math.floor((v - self.lo) / self.range)

    def getValue(self, timestep):  # noqa: N802
        if timestep < self.offset:
            return 0.0
        if timestep >= self.offset + self.total:
            return self.end_value
        return self.wrapValue(self.f.getStrain(timestep))


class Stokes:
    """Mirror of the C++ integration method (Stokes.h / Stokes.cc).

    The constructor arguments follow Stokes.cc:47-83 with the HOOMD system
    definition, group and neighbour list replaced by a `fsd_b200.system.System`
    (which carries the particles and the box) and the neighbour-list kind
    (the neighbour list itself is built by the library each step)."""

    def __init__(self, system, group, T, seed, nlist_type, xi, error, fileprefix, period, ndsr, kappa, k_n,
                 beta_AF, epsq, sqm_B1, sqm_B2, N_mix, coef_B1_mask, coef_B2_mask, rot_diff, T_ext, omega_ext,
                 **solver):  # noqa: N803
        self.system = system
        self.group = group
        self.T = T
        self.seed = int(seed)
        self.nlist_type = nlist_type
        self.xi, self.error = float(xi), float(error)
        self.fileprefix, self.period = fileprefix, int(period)
        self.pair = dict(ndsr=ndsr, kappa=kappa, k_n=k_n, beta_AF=beta_AF, epsq=epsq)
        self.active = dict(sqm_B1=sqm_B1, sqm_B2=sqm_B2, N_mix=N_mix, coef_B1_mask=coef_B1_mask,
                           coef_B2_mask=coef_B2_mask, rot_diff=rot_diff, T_ext=T_ext, omega_ext=omega_ext)
        self.solver = solver
        self.shear_func: ShearFunction | None = None
        self.max_strain = 0.5
        self.fsd = None
        self._params_set = False
        self._table_set = False
        self.output_dir = Path(os.getcwd())

    def validateGroup(self):  # noqa: N802
        if self.group is not self.system.all and len(self.group) != self.system.N:
            raise RuntimeError("PSEv3 integrates every particle; groups other than all are not supported")

    def setT(self, T):  # noqa: N802
        self.T = T
        if self.fsd is not None:
            self.fsd.set_temperature(float(self.T(self.system.timestep)))

    def setShear(self, shear_func: ShearFunction, max_strain: float):  # noqa: N802
        if self.fsd is not None and float(max_strain) != self.max_strain:
            raise RuntimeError("max_strain fixes the spreading support; it cannot change after AllocateWorkSpaces")
        self.shear_func = shear_func
        self.max_strain = float(max_strain)

    def setParams(self):  # noqa: N802
        """Grid, support and splitting come from the library's set-up
        (Stokes.cc:118-696) when the workspaces are allocated."""
        self._params_set = True

    def setResistanceTable(self):  # noqa: N802
        """The Jeffrey-Onishi table ships with the library (fsd_b200/data)."""
        self._table_set = True

    def setFriction(self, friction_type, h0, alpha):  # noqa: N802
        """Frictional contact terms in the resistance table (Stokes.cc:1132-1191):
        "NONE" or "TYPE1" with the contact range h0 and the six strengths
        alpha (YA11, YA12, YB11, YB12, YC11, YC12); applied when the
        workspaces are allocated."""
        kind = str(friction_type).upper()
        if kind not in ("NONE", "TYPE1"):
            raise RuntimeError("Invalid Friction Type. Allowable types are: None, Type1")
        if self.fsd is not None:
            raise RuntimeError("setFriction must precede AllocateWorkSpaces")
        if kind == "TYPE1":
            alpha = [float(a) for a in alpha]
            if len(alpha) != 6:
                raise RuntimeError("TYPE1 friction takes six strengths")
            self.solver.update(friction_type=1, friction_h0=float(h0), friction_alpha=alpha)
        else:
            self.solver.update(friction_type=0)

    def setSparseMath(self):  # noqa: N802
        """Sparse storage is created with the workspaces (Stokes.cc:1066-1130)."""

    def AllocateWorkSpaces(self):  # noqa: N802
        from .core import FSD

        if not (self._params_set and self._table_set):
            raise RuntimeError("setParams and setResistanceTable must precede AllocateWorkSpaces")
        sysm = self.system
        Lx, Ly, Lz, xy = sysm.box
        kw = dict(self.pair, **self.active)
        kw.update(self.solver)
        self.fsd = FSD(sysm.N, (Lx, Ly, Lz, xy), device=sysm.device, xi=self.xi, error=self.error,
                       max_strain=self.max_strain, T=float(self.T(sysm.timestep)), dt=sysm.dt, seed=self.seed,
                       period=self.period, **kw)

    def integrateStepOne(self, timestep: int):  # noqa: N802
        """One step (Stokes.cc:1197-1683) through fsd_step."""
        sysm = self.system
        rate = self.shear_func.getShearRate(timestep) if self.shear_func else 0.0
        T = float(self.T(timestep))
        if self.fsd.params.T != T:
            self.fsd.set_temperature(T)
        if sysm.box_variant is not None:
            Lx, Ly, Lz, _ = sysm.box
            xy = float(sysm.box_variant.getValue(timestep))
            sysm.box = (Lx, Ly, Lz, xy)
            self.fsd.set_box(Lx, Ly, Lz, xy)
        self.fsd.step(timestep, rate, sysm.pos, sysm.ori, sysm.image, sysm.force, sysm.velocity, pos_gb=sysm.pos_gb)
        if self.period > 0 and timestep % self.period == 0:
            self.OutputData(timestep, sysm.box, rate)

    def OutputData(self, timestep, box, current_shear_rate):  # noqa: N802
        """Per-particle text output of Stokes::OutputData (Stokes.cc:703-931)."""
        from .output import write_output

        sysm = self.system
        write_output(self.output_dir, timestep, box, sysm.pos.cpu().numpy().reshape(-1, 4),
                     sysm.ori.cpu().numpy().reshape(-1, 3), sysm.pos_gb.cpu().numpy().reshape(-1, 4),
                     sysm.velocity.cpu().numpy(), self.pair, self.fsd.pse_info().ewald_cut + 0.4)

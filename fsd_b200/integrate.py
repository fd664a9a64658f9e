"""The integrator class of the plugin (integrate.py:17-154 of the reference),
same constructor arguments and defaults, over the CUDA path.

Without HOOMD, `group` is a fsd_b200.system.System (its `all`), and
stepping is `system.run(steps)`.  The neighbour list the reference asks HOOMD
for (cell, tree or stencil, r_cut + 0.4, rebuilt every step) is built by the
library each step; the three kinds give the same list."""
from __future__ import annotations

import math

from . import _PSEv3, shear_function
from . import system as _system
from .variant import setup_variant_input


class PSEv3:
    def __init__(self, group, T, seed=0, xi=0.5, error=0.001, function_form=None, max_strain=0.5,
                 fileprefix="stresslet", period=0, nlist_type="cell", friction_type="none", h0=0.0,
                 alpha=(0.0, 0.0, 0.0, 0.0, 0.0, 0.0), ndsr=1e-1, kappa=1 / 0.05, k_n=1e4, beta_AF=0., epsq=1e-5,
                 sqm_B1=0., sqm_B2=0., N_mix=1, coef_B1_mask=1.0, coef_B2_mask=1.0, rot_diff=0., T_ext=0.,
                 omega_ext=0., system=None, **solver):  # noqa: N803
        system = system or getattr(group, "system", None) or _system.current()
        if system is None:
            raise RuntimeError("no system: pass system= or call fsd_b200.system.set_current")
        T = setup_variant_input(T)
        period = int(period)
        self.rcut = math.sqrt(-math.log(error)) / xi
        if nlist_type.upper() not in ("CELL", "TREE", "STENCIL"):
            raise RuntimeError("Invalid neighborlist method specified. Valid options are: cell, tree, stencil.")
        self.system = system
        self.cpp_method = _PSEv3.Stokes(system, system.all, T, seed, nlist_type.upper(), xi, error, fileprefix,
                                        period, ndsr, kappa, k_n, beta_AF, epsq, sqm_B1, sqm_B2, N_mix,
                                        coef_B1_mask, coef_B2_mask, rot_diff, T_ext, omega_ext, **solver)
        self.cpp_method.validateGroup()
        if function_form is not None:
            self.cpp_method.setShear(function_form.cpp_function, max_strain)
        else:
            self.cpp_method.setShear(shear_function.steady(dt=0).cpp_function, max_strain)
        self.cpp_method.setParams()
        self.cpp_method.setResistanceTable()
        self.cpp_method.setFriction(friction_type.upper(), h0, alpha)
        self.cpp_method.setSparseMath()
        self.cpp_method.AllocateWorkSpaces()
        system.methods.append(self)

    def set_params(self, T=None, function_form=None, max_strain=0.5):
        if T is not None:
            self.cpp_method.setT(setup_variant_input(T))
        if function_form is not None:
            self.cpp_method.setShear(function_form.cpp_function, max_strain)

    def stop_shear(self, max_strain=0.5):
        self.cpp_method.setShear(shear_function.steady(dt=0).cpp_function, max_strain)

"""Box-deformation variant of the plugin (variant.py of the reference)."""
from __future__ import annotations

from . import _PSEv3


class shear_variant:  # noqa: N801 (reference name)
    """Wrapped strain of a shear function as the box tilt xy, for
    fsd_b200.system.System.set_box_variant (HOOMD's box_resize)."""

    def __init__(self, function_form, total_timestep, max_strain=0.5):
        if total_timestep <= 0:
            raise RuntimeError("Cannot create a shear_variant with 0 or negative points")
        self.cpp_variant = _PSEv3.VariantShearFunction(function_form.cpp_function, int(total_timestep),
                                                      -max_strain, max_strain)


class constant:  # noqa: N801
    """Constant value (hoomd.variant._setup_variant_input of a number)."""

    def __init__(self, value):
        self.value = float(value)

    def __call__(self, timestep):
        return self.value


class linear_interp:  # noqa: N801
    """Piecewise-linear value over (timestep, value) points (hoomd.variant.linear_interp)."""

    def __init__(self, points):
        self.points = sorted((int(t), float(v)) for t, v in points)

    def __call__(self, timestep):
        p = self.points
        if timestep <= p[0][0]:
            return p[0][1]
        for (t0, v0), (t1, v1) in zip(p, p[1:]):
            if timestep <= t1:
                return v0 + (v1 - v0) * (timestep - t0) / (t1 - t0)
        return p[-1][1]


def setup_variant_input(T):
    """A number or a variant, as hoomd.variant._setup_variant_input."""
    return T if callable(T) else constant(T)

"""Shear functions of the plugin (shear_function.py of the reference), over
the host-side classes of fsd_b200._PSEv3.  `zero='now'` takes the current
system's time step (fsd_b200.system.set_current), 0 when none is set."""
from __future__ import annotations

from . import _PSEv3
from . import system as _system


class _shear_function:  # noqa: N801 (reference name)
    def __init__(self, zero="now"):
        self.cpp_function = None
        now = _system.current().timestep if _system.current() is not None else 0
        if zero == "now":
            self._offset = now
        else:
            if zero < 0:
                raise RuntimeError("Cannot create a shear_function variant with a negative zero")
            if zero > now:
                raise RuntimeError("Cannot create a shear_function variant with a zero in the future")
            self._offset = int(zero)

    def get_shear_rate(self, timestep):
        return self.cpp_function.getShearRate(timestep)

    def get_strain(self, timestep):
        return self.cpp_function.getStrain(timestep)

    def get_offset(self):
        return self.cpp_function.getOffset()


class steady(_shear_function):  # noqa: N801
    def __init__(self, dt, shear_rate=0, zero="now"):
        _shear_function.__init__(self, zero)
        self.cpp_function = _PSEv3.SteadyShearFunction(shear_rate, self._offset, dt)


class sine(_shear_function):  # noqa: N801
    def __init__(self, dt, shear_rate, shear_freq, zero="now"):
        if shear_rate <= 0:
            raise RuntimeError("Shear rate must be positive (use steady class instead for zero shear)")
        if shear_freq <= 0:
            raise RuntimeError("Shear frequency must be positive (use steady class instead for steady shear)")
        _shear_function.__init__(self, zero)
        self.cpp_function = _PSEv3.SinShearFunction(shear_rate, shear_freq, self._offset, dt)


class chirp(_shear_function):  # noqa: N801
    def __init__(self, dt, amplitude, omega_0, omega_f, periodT, zero="now"):  # noqa: N803
        _shear_function.__init__(self, zero)
        self.cpp_function = _PSEv3.ChirpShearFunction(amplitude, omega_0, omega_f, periodT, self._offset, dt)


class tukey_window(_shear_function):  # noqa: N801
    def __init__(self, dt, periodT, tukey_param, zero="now"):  # noqa: N803
        if tukey_param <= 0 or tukey_param > 1:
            raise RuntimeError("Tukey parameter must be within (0, 1]")
        _shear_function.__init__(self, zero)
        self.cpp_function = _PSEv3.TukeyWindowFunction(periodT, tukey_param, self._offset, dt)


class windowed(_shear_function):  # noqa: N801
    def __init__(self, function_form, window):
        _shear_function.__init__(self, "now")
        self.cpp_function = _PSEv3.WindowedFunction(function_form.cpp_function, window.cpp_function)

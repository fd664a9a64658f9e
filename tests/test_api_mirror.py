"""The Python mirror of the plugin's API: integrate.PSEv3, shear_function,
variant and the _PSEv3 classes (integrate.py, shear_function.py, variant.py,
SpecificShearFunction.h, VariantShearFunction.cc and Stokes::OutputData of
the reference)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from fsd_b200 import _PSEv3, output, shear_function as sf, variant


def test_steady_and_sine_follow_the_reference_formulas():
    s = sf.steady(dt=1e-3, shear_rate=0.7, zero=0)
    assert s.get_shear_rate(123) == 0.7
    assert math.isclose(s.get_strain(500), 0.7 * 500 * 1e-3)
    o = sf.sine(dt=1e-3, shear_rate=2.0, shear_freq=0.5, zero=0)
    t = 400 * 1e-3
    assert math.isclose(o.get_shear_rate(400), 2.0 * math.cos(0.5 * 2 * 3.1415926536 * t))
    assert math.isclose(o.get_strain(400), 2.0 * math.sin(0.5 * 2 * 3.1415926536 * t) / 0.5 / 2 / 3.1415926536)


def test_offsets_wrap_like_unsigned_timesteps():
    """timestep - offset is unsigned in the reference: before the offset it wraps around."""
    f = _PSEv3.SteadyShearFunction(1.0, 10, 1.0)
    assert f.getStrain(9) == float(2 ** 32 - 1)


def test_chirp_uses_single_precision_log_ratio():
    c = sf.chirp(dt=1e-3, amplitude=0.1, omega_0=1.0, omega_f=10.0, periodT=5.0, zero=0)
    lr = float(np.log(np.float32(10.0), dtype=np.float32))
    phase = 5.0 * 1.0 / lr * (math.exp(1.0 * lr / 5.0) - 1)
    assert math.isclose(c.get_strain(1000), 0.1 * math.sin(phase), rel_tol=1e-12)


def test_tukey_window_and_windowed_product_rule():
    t = sf.tukey_window(dt=1e-3, periodT=1.0, tukey_param=0.5, zero=0)
    assert t.get_strain(0) == 0.0 and t.get_strain(500) == 1.0 and t.get_strain(1000) == 0.0
    assert math.isclose(t.get_strain(100), (1 + math.cos(2 * 3.1415926536 / 0.5 * (0.1 - 0.25))) / 2)
    s = sf.sine(dt=1e-3, shear_rate=2.0, shear_freq=0.5, zero=0)
    w = sf.windowed(s, t)
    assert math.isclose(w.get_strain(100), s.get_strain(100) * t.get_strain(100))
    assert math.isclose(w.get_shear_rate(100), s.get_shear_rate(100) * t.get_strain(100)
                        + s.get_strain(100) * t.get_shear_rate(100))
    with pytest.raises(RuntimeError):
        sf.tukey_window(dt=1e-3, periodT=1.0, tukey_param=1.5)
    with pytest.raises(RuntimeError):
        sf.sine(dt=1e-3, shear_rate=0.0, shear_freq=1.0)


def test_shear_variant_wraps_strain_into_the_box_range():
    v = variant.shear_variant(sf.steady(dt=1e-2, shear_rate=1.0, zero=0), total_timestep=1000, max_strain=0.5)
    cv = v.cpp_variant
    assert cv.getValue(0) == 0.0
    assert math.isclose(cv.getValue(40), 0.4)
    assert math.isclose(cv.getValue(60), -0.4)          # 0.6 wraps to -0.4
    assert math.isclose(cv.getValue(5000), cv.wrapValue(10.0))
    with pytest.raises(RuntimeError):
        variant.shear_variant(sf.steady(dt=1e-2, zero=0), total_timestep=0)


def test_output_files_have_the_reference_formats(tmp_path):
    N = 3
    pos = np.array([[0, 0, 0, 0], [2.05, 0, 0, 0], [0, 3.5, 0, 0]], np.float32)
    ori = np.tile([0, 0, 1.0], (N, 1))
    vel = np.arange(11 * N, dtype=np.float32)
    pair = dict(ndsr=0.1, kappa=20.0, k_n=1e4, beta_AF=0.0, epsq=1e-5)
    output.write_output(tmp_path, 7, (10.0, 10.0, 10.0, 0.0), pos, ori, pos, vel, pair, 5.0)
    lines = (tmp_path / "raw" / "stresslet.0000000007.txt").read_text().splitlines()
    assert len(lines) == N and lines[0].startswith("      0 ")
    vals = [float(v) for v in lines[1].split()]
    nden = N / 1000.0
    s = vel[6 * N + 5:6 * N + 10] * np.float32(nden)
    assert np.allclose(vals[1:], [s[0], s[1], s[2], s[4], s[3], -s[0] - s[4]], rtol=1e-3)
    ov = (tmp_path / "overlap.txt").read_text().split()
    assert ov[0] == "7" and float(ov[1]) == 0.0 and math.isclose(float(ov[4]), 0.05, rel_tol=1e-3)
    assert len((tmp_path / "raw" / "interparticle_stresslet.0000000007.txt").read_text().splitlines()) == N


def test_invalid_neighbour_list_kind_is_rejected():
    from fsd_b200.integrate import PSEv3
    from fsd_b200.system import System
    sysm = System(np.zeros((2, 4)), (20.0, 20.0, 20.0, 0.0), dt=1e-4, device="cpu")
    with pytest.raises(RuntimeError):
        PSEv3(sysm.all, T=1.0, nlist_type="octree", system=sysm)


def test_set_friction_follows_the_reference_types():
    """setFriction (Stokes.cc:1132-1191) takes NONE or TYPE1 with six
    strengths and must precede AllocateWorkSpaces; other types raise as the
    reference does."""
    from fsd_b200 import _PSEv3
    from fsd_b200.system import System
    sysm = System(np.zeros((2, 4)), (20.0, 20.0, 20.0, 0.0), dt=1e-4, device="cpu")
    st = _PSEv3.Stokes(sysm, sysm.all, lambda t: 1.0, 0, "CELL", 0.5, 1e-3, "stresslet", 0, 0.1, 20.0, 1e4, 0.0, 1e-5,
                       0.0, 0.0, 1, 1.0, 1.0, 0.0, 0.0, 0.0)
    st.setFriction("TYPE1", 0.05, [0.5, 0.3, 0.2, 0.1, 0.4, 0.25])
    assert st.solver["friction_type"] == 1 and st.solver["friction_h0"] == 0.05
    assert st.solver["friction_alpha"] == [0.5, 0.3, 0.2, 0.1, 0.4, 0.25]
    st.setFriction("none", 0.0, [0.0] * 6)
    assert st.solver["friction_type"] == 0
    with pytest.raises(RuntimeError):
        st.setFriction("TYPE2", 0.05, [0.0] * 6)


@pytest.mark.gpu
def test_psev3_steps_and_writes_output(cuda, tmp_path):
    from fsd_b200.configs import suspension
    from fsd_b200.integrate import PSEv3
    from fsd_b200.system import System, set_current
    pos, L = suspension(300, 0.3, 5)
    sysm = System(pos, (L, L, L, 0.0), dt=1e-4)
    set_current(sysm)
    try:
        integ = PSEv3(sysm.all, T=1.0, seed=3, function_form=sf.steady(dt=1e-4, shear_rate=0.5), period=2,
                      solver_tol=1e-4)
        integ.cpp_method.output_dir = tmp_path
        p0 = sysm.pos.cpu().numpy().copy()
        sysm.run(3)
        assert sysm.timestep == 3
        moved = np.abs(sysm.pos.cpu().numpy() - p0).max()
        assert 0 < moved < 1.0
        assert (tmp_path / "raw" / "stresslet.0000000000.txt").exists()
        assert (tmp_path / "raw" / "velocity.0000000002.txt").exists()
        assert len((tmp_path / "overlap.txt").read_text().splitlines()) == 2
        integ.set_params(T=0.5)
        sysm.run(1)
        assert integ.cpp_method.fsd.params.T == 0.5
    finally:
        set_current(None)

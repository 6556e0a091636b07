"""lbmpy's shear-wave scenario (tests/full_scenarios/shear_wave/scenario_shear_wave.py, after Geier et
al. 2015, section 5.1): a shear wave v = v0 l0/l sin(2 pi x / l) cos(4 pi z / (3 l)) carried by a
uniform u = u0 l0/l in a periodic l x 1 x 3l/2 box.  The viscosity follows from the decay of the
wave's largest Fourier amplitude; ER_nu = |nu_est - nu| / nu."""
import numpy as np

L0, U0, V0 = 32, 0.096, 0.1


def initial_velocity(l):
    n = (l, 1, 3 * l // 2)
    x, _, z = np.meshgrid(*[np.arange(s, dtype=float) for s in n], indexing="ij")
    u = np.zeros(n + (3,))
    u[..., 0] = U0 * L0 / l
    u[..., 1] = V0 * L0 / l * np.sin(2 * np.pi * x / l) * np.cos(4 * np.pi * z / (3 * l))
    return u


def schedule(l):
    """(initial steps, total steps, evaluation interval) of lbmpy's shortened integration test."""
    s = (l // L0) ** 2
    return 1100 * s, 2000 * s, 100 * s


def amplitude(vy_slice):
    return float(np.abs(np.fft.rfft2(vy_slice)).max())


def viscosity_error(amplitudes, interval, l, nu):
    x = np.arange(0, interval * len(amplitudes), interval)
    slope = np.polyfit(x, np.log(amplitudes), 1)[0]
    k2 = (2 * np.pi / l) ** 2 + (4 * np.pi / (3 * l)) ** 2
    return abs(-slope / k2 - nu) / nu

"""Analytic flow solutions used as physical checks of long runs (no lbmpy counterpart beyond the
plane Poiseuille profile of analytical_solutions.py:5-20)."""
import numpy as np


def duct_startup_velocity(ny, nz, nu, g, t, terms=199):
    """Axial velocity u(y, z, t) of flow in a rectangular duct started from rest by a constant
    body acceleration g at t = 0 (no-slip walls), at the cell centres of an ny x nz lattice whose
    halfway bounce-back walls sit half a cell outside the first and last cells (width ny, nz).

    Double sine series of du/dt = nu (u_yy + u_zz) + g:
        u = sum_{m,n odd} 16 g / (pi^2 m n nu lam) (1 - exp(-nu lam t)) sin(m pi y'/ny) sin(n pi z'/nz),
        lam = pi^2 (m^2/ny^2 + n^2/nz^2),  y' = y + 1/2,  z' = z + 1/2.
    As t -> infinity this is the steady rectangular-duct Poiseuille profile."""
    y = (np.arange(ny) + 0.5) / ny
    z = (np.arange(nz) + 0.5) / nz
    u = np.zeros((ny, nz))
    for m in range(1, terms + 1, 2):
        sy = np.sin(m * np.pi * y)
        for n in range(1, terms + 1, 2):
            lam = np.pi ** 2 * (m * m / ny ** 2 + n * n / nz ** 2)
            a = 16.0 * g / (np.pi ** 2 * m * n * nu * lam) * (1.0 - np.exp(-nu * lam * t))
            u += a * np.outer(sy, np.sin(n * np.pi * z))
    return u

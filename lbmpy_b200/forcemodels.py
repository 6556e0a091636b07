"""Force models with lbmpy's names (lbmpy ``forcemodels.py``).

The B200 sweep evaluates the forcing terms in registers; these classes only carry the force
vector and identify the model.  Supported: Simple, Luo, Guo (SRT/TRT/MRT) and CentralMoment
(cumulant).
"""
from __future__ import annotations


class AbstractForceModel:
    native_id = 0

    def __init__(self, force):
        force = tuple(force)
        self._force = force

    @property
    def symbolic_force_vector(self):
        return self._force

    @property
    def force(self):
        return self._force

    def macroscopic_velocity_shift(self, density):
        """u shift F/(2 rho) used by the density/velocity getter (forcemodels.py:592-593)."""
        return [f / (2 * density) for f in self._force]

    def macroscopic_momentum_density_shift(self, *_):
        return [f / 2 for f in self._force]

    def equilibrium_velocity_shift(self, density):
        return [0] * len(self._force)

    def __repr__(self):
        return f"{type(self).__name__}({self._force})"

    def __eq__(self, other):
        return type(self) is type(other) and self._force == other._force


class Simple(AbstractForceModel):
    """w_i c_i.F / c_s^2 added to the populations (forcemodels.py:179-211)."""
    native_id = 3


class Luo(AbstractForceModel):
    """Luo 1993 (forcemodels.py:235-271)."""
    native_id = 4


class Guo(AbstractForceModel):
    """Guo 2002, generalised to MRT (forcemodels.py:273-317); shifts the equilibrium velocity."""
    native_id = 1

    def equilibrium_velocity_shift(self, density):
        return [f / (2 * density) for f in self._force]


class CentralMoment(AbstractForceModel):
    """Symmetric forcing of the first central moments (forcemodels.py:213-233); cumulant only."""
    native_id = 2

    def equilibrium_velocity_shift(self, density):
        return [f / (2 * density) for f in self._force]


Schiller = Guo

"""Relaxation-rate helpers with lbmpy's names (lbmpy ``relaxationrates.py:6-20``)."""
from .methods import (lattice_viscosity_from_relaxation_rate, relaxation_rate_from_lattice_viscosity,  # noqa: F401
                      relaxation_rate_from_magic_number)

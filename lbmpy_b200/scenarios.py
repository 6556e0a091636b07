"""Scenario helpers with lbmpy's names (lbmpy ``scenarios.py:37-172``)."""
from __future__ import annotations

import numpy as np

from .boundaries import UBB, NoSlip, slice_from_direction
from .lbstep import LatticeBoltzmannStep


def create_fully_periodic_flow(initial_velocity, periodicity_in_kernel=False, lbm_kernel=None, data_handling=None,
                               parallel=False, **kwargs):
    """Periodic box initialised in equilibrium with `initial_velocity` ([x, y, z, 3]); scenarios.py:37-69.
    Periodicity is an index wrap in the sweep whether or not `periodicity_in_kernel` is set."""
    if parallel:
        raise NotImplementedError("use lbmpy_b200.distributed (DistributedLatticeBoltzmannStep) for multi-GPU domains")
    initial_velocity = np.asarray(initial_velocity)
    domain_size = initial_velocity.shape[:-1]
    step = LatticeBoltzmannStep(domain_size=domain_size, periodicity=True, lbm_kernel=lbm_kernel,
                                name="periodic_scenario", **kwargs)
    step.velocity_array[...] = initial_velocity
    step.set_pdf_fields_from_macroscopic_values()
    return step


def create_lid_driven_cavity(domain_size=None, lid_velocity=0.005, lbm_kernel=None, parallel=False,
                             data_handling=None, **kwargs):
    """UBB lid on the 'N' (y max) ghost layer, NoSlip on every other face (scenarios.py:72-102)."""
    if parallel:
        raise NotImplementedError("use lbmpy_b200.batched for many cavities")
    step = LatticeBoltzmannStep(domain_size=domain_size, periodicity=False, lbm_kernel=lbm_kernel, name="ldc",
                                **kwargs)
    step.boundary_handling.set_boundary(UBB(velocity=[lid_velocity, 0, 0]), slice_from_direction("N", 3))
    for d in ("W", "E", "S", "T", "B"):
        step.boundary_handling.set_boundary(NoSlip(), slice_from_direction(d, 3))
    return step


def create_channel(domain_size=None, force=None, pressure_difference=None, u_max=None, diameter_callback=None,
                   duct=False, wall_boundary=None, parallel=False, data_handling=None, **kwargs):
    """Force-driven channel periodic in x (scenarios.py:105-172).  duct=True: walls on the y and z
    faces; duct=False: circular pipe of diameter min(ny, nz)."""
    if [bool(p) for p in (force, pressure_difference, u_max)].count(True) != 1:
        raise ValueError("Please specify exactly one of the parameters 'force', 'pressure_difference' or 'u_max'")
    if not force:
        raise NotImplementedError("pressure- and velocity-driven channels need FixedDensity / inflow profiles, "
                                  "which are not built")
    if parallel:
        raise NotImplementedError("use lbmpy_b200.distributed (DistributedLatticeBoltzmannStep) for multi-GPU domains")
    wall_boundary = wall_boundary or NoSlip()
    kwargs["force"] = (force, 0, 0)
    step = LatticeBoltzmannStep(domain_size=domain_size, periodicity=(True, False, False),
                                name="force_driven_channel", **kwargs)
    for d in ("N", "S", "T", "B"):
        step.boundary_handling.set_boundary(wall_boundary, slice_from_direction(d, 3))
    if not duct:
        if diameter_callback is not None:
            raise NotImplementedError("diameter callbacks are not built")
        diameter = min(domain_size[1:])
        ny, nz = domain_size[1], domain_size[2]

        def outside(x, y, z):
            return np.sqrt((y - ny / 2) ** 2 + (z - nz / 2) ** 2) >= diameter / 2

        step.boundary_handling.set_boundary(wall_boundary, mask_callback=outside)
    return step

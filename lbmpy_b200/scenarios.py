"""Scenario helpers with lbmpy's names (lbmpy ``scenarios.py:37-172``)."""
from __future__ import annotations

import numpy as np

from .boundaries import UBB, FixedDensity, NoSlip, slice_from_direction
from .geometry import add_pipe_inflow_boundary, add_pipe_walls
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
    """Channel along x (scenarios.py:104-172), driven by exactly one of
    - force: periodic in x, body force (force, 0, 0);
    - pressure_difference: FixedDensity 1 + pressure_difference on W, FixedDensity 1 on E;
    - u_max: parabolic pipe inflow on W (add_pipe_inflow_boundary), FixedDensity 1 on E.
    duct=True: walls on the y and z faces only; duct=False: a pipe of diameter min(ny, nz) (or
    diameter_callback(x, shape)) inside them."""
    if [bool(p) for p in (force, pressure_difference, u_max)].count(True) != 1:
        raise ValueError("Please specify exactly one of the parameters 'force', 'pressure_difference' or 'u_max'")
    if parallel:
        raise NotImplementedError("use lbmpy_b200.distributed (DistributedLatticeBoltzmannStep) for multi-GPU domains")
    wall_boundary = wall_boundary or NoSlip()
    domain_size = tuple(int(s) for s in domain_size)
    periodicity = (True, False, False) if force else (False, False, False)
    if force:
        kwargs["force"] = (force, 0, 0)
        step = LatticeBoltzmannStep(domain_size=domain_size, periodicity=periodicity, name="force_driven_channel",
                                    **kwargs)
    elif pressure_difference:
        step = LatticeBoltzmannStep(domain_size=domain_size, periodicity=periodicity,
                                    name="pressure_driven_channel", **kwargs)
        step.boundary_handling.set_boundary(FixedDensity(1.0 + pressure_difference), slice_from_direction("W", 3))
        step.boundary_handling.set_boundary(FixedDensity(1.0), slice_from_direction("E", 3))
    else:
        if duct:
            raise NotImplementedError("Velocity inflow for duct flows not yet implemented")
        step = LatticeBoltzmannStep(domain_size=domain_size, periodicity=periodicity,
                                    name="velocity_driven_channel", **kwargs)
        diameter = diameter_callback(np.array([0]), domain_size)[0] if diameter_callback else min(domain_size[1:])
        add_pipe_inflow_boundary(step.boundary_handling, u_max, slice_from_direction("W", 3), flow_direction=0,
                                 diameter=diameter)
        step.boundary_handling.set_boundary(FixedDensity(1.0), slice_from_direction("E", 3))
    for d in ("N", "S", "T", "B"):
        step.boundary_handling.set_boundary(wall_boundary, slice_from_direction(d, 3))
    if duct and diameter_callback is not None:
        raise ValueError("For duct flows, passing a diameter callback does not make sense.")
    if not duct:
        add_pipe_walls(step.boundary_handling, diameter_callback if diameter_callback else min(domain_size[1:]),
                       wall_boundary)
    return step

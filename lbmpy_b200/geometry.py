"""Boundary set-up helpers with lbmpy's names (lbmpy ``geometry.py:8-191``) for the flag-field
boundary handling of this package."""
from __future__ import annotations

import numpy as np

from .boundaries import UBB, NoSlip, slice_from_direction


def add_box_boundary(boundary_handling, boundary=NoSlip(), replace=True):
    """Sets `boundary` on every face of the domain (geometry.py:8-26)."""
    flag = None
    for d in ("N", "S", "E", "W", "T", "B"):
        flag = boundary_handling.set_boundary(boundary, slice_from_direction(d, 3), replace=replace)
    return flag


def add_sphere(boundary_handling, midpoint, radius, boundary=NoSlip(), replace=True):
    """Sets `boundary` in the sphere (disc in x-y for a 2-D midpoint) around `midpoint`
    (geometry.py:29-33); coordinates are cell midpoints."""
    mid = tuple(midpoint)

    def inside(x, y, z):
        d = (x - mid[0]) ** 2 + (y - mid[1]) ** 2
        if len(mid) > 2:
            d = d + (z - mid[2]) ** 2
        return d < radius ** 2
    return boundary_handling.set_boundary(boundary, mask_callback=inside, replace=replace)


def _pipe_radius(shape, flow_direction, diameter):
    if diameter is None:
        return int(round(min(s for i, s in enumerate(shape) if i != flow_direction) / 2))
    return int(round(diameter / 2))


def add_pipe_inflow_boundary(boundary_handling, u_max, slice_obj, flow_direction=0, diameter=None):
    """Velocity inflow with the parabolic pipe profile u_max (1 - (r / R)^2) on `slice_obj`
    (geometry.py:36-86): a UBB whose callback sets one velocity per link from the link's midpoint."""
    shape = boundary_handling.shape

    def velocity_info_callback(boundary_data):
        for i in range(3):
            if i != flow_direction:
                boundary_data[f"vel_{i}"] = 0.0
        radius = _pipe_radius(shape, flow_direction, diameter)
        n1, n2 = (flow_direction + 1) % 3, (flow_direction + 2) % 3
        c1 = boundary_data.link_positions(n1) - int(round(shape[n1] / 2))
        c2 = boundary_data.link_positions(n2) - int(round(shape[n2] / 2))
        dist = np.sqrt(c1 ** 2 + c2 ** 2)
        boundary_data[f"vel_{flow_direction}"] = u_max * (1 - (dist / radius) ** 2)

    inflow = UBB(velocity_info_callback, dim=3)
    return boundary_handling.set_boundary(inflow, slice_obj=slice_obj, ghost_layers=True)


def add_pipe_walls(boundary_handling, diameter, boundary=NoSlip()):
    """Walls of a pipe along x (geometry.py:88-121): every cell whose midpoint lies outside the
    circle of `diameter` (a number, or a callback (x coordinates, domain shape) -> diameters)
    around the domain's y-z centre."""
    shape = boundary_handling.shape

    def outside(x, y, z):
        if callable(diameter):
            d = np.asarray(diameter(x[:, 0, 0], shape))[:, np.newaxis, np.newaxis]
        else:
            d = diameter
        mid = (shape[1] // 2, shape[2] // 2)
        return (y - mid[0]) ** 2 + (z - mid[1]) ** 2 > (d / 2) ** 2
    return boundary_handling.set_boundary(boundary, mask_callback=outside)


def get_pipe_velocity_field(domain_size, u_max, flow_direction=0, diameter=None):
    """Parabolic pipe profile on the cell midpoints of `domain_size` (geometry.py:124-163); values
    outside the pipe are not meaningful."""
    radius = _pipe_radius(domain_size, flow_direction, diameter)
    grid = np.meshgrid(*[np.arange(s) + 0.5 for s in domain_size], indexing="ij")
    dist = 0
    for i, s in enumerate(domain_size):
        if i != flow_direction:
            dist = dist + (grid[i] - int(round(s / 2))) ** 2
    dist = np.sqrt(dist)
    u = np.zeros(tuple(domain_size) + (len(domain_size),))
    u[..., flow_direction] = u_max * (1 - (dist / radius) ** 2)
    return u


def get_shear_flow_velocity_field(domain_size, u_max, random_y_factor=0.01, seed=None):
    """Two shear layers along the last axis (geometry.py:166-190): +u_max, then -u_max in the
    middle third, with a small random transverse component (seeded when `seed` is given)."""
    height = domain_size[-1]
    velocity = np.empty(tuple(domain_size) + (len(domain_size),))
    velocity[..., 0] = u_max
    velocity[..., height // 3: height // 3 * 2, 0] = -u_max
    rng = np.random.default_rng(seed)
    for j in range(1, len(domain_size)):
        velocity[..., j] = random_y_factor * u_max * (rng.random(domain_size) - 0.5)
    return velocity

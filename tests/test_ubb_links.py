"""UBB with per-link velocities (callbacks), prescribed wall density and adapt_velocity_to_force:
host-side link enumeration and the oracle's restatement (no GPU)."""
import numpy as np
import pytest

import lbmpy_b200 as L
from lbmpy_b200.boundaries import UBB, BoundaryData, LatticeBoltzmannBoundaryHandling, NoSlip, slice_from_direction
from lbmpy_b200.geometry import add_pipe_inflow_boundary, get_pipe_velocity_field
from oracle import oracle as O


def _handling(shape, stencil=L.Stencil.D3Q19, periodicity=(False, False, False)):
    m = L.create_lb_method(lbm_config=L.LBMConfig(stencil=stencil, method=L.Method.SRT, relaxation_rate=1.8))
    return LatticeBoltzmannBoundaryHandling(m, shape, periodicity, device="cpu")


def test_callback_needs_dim_and_density_is_positive():
    with pytest.raises(ValueError):
        UBB(lambda bd: None)
    with pytest.raises(ValueError):
        UBB((0.01, 0, 0), density=0.0)
    u = UBB(lambda bd: None, dim=3)
    assert u.velocity_is_callable and u.velocity == (0.0, 0.0, 0.0)


def test_links_of_a_west_inflow_sit_on_the_wall_plane():
    """Every link from the first interior x-plane into the W ghost plane: fluid cells at x = 0 (ghost
    index 1), directions with c_x = -1, link midpoints at x = 0 (the halfway wall)."""
    shape = (6, 5, 4)
    bh = _handling(shape)
    seen = {}

    def cb(bd: BoundaryData):
        seen["x"] = bd.link_positions(0)
        seen["y"] = bd.link_positions(1)
        seen["dirs"] = bd.link_offsets()
        bd["vel_0"] = 0.01 * bd.link_positions(1)
        bd["vel_1"] = 0.0
        bd["vel_2"] = 0.0

    bh.set_boundary(UBB(cb, dim=3), slice_from_direction("W", 3))
    links = bh.ubb_links()[0]
    assert len(links) == 5 * shape[1] * shape[2]          # 5 D3Q19 directions with c_x = -1
    assert (links["x"] == 1).all()
    np.testing.assert_array_equal(seen["x"], 0.0)
    assert (seen["dirs"][:, 0] == -1).all()
    np.testing.assert_allclose(seen["y"], links["y"] - 0.5 + 0.5 * seen["dirs"][:, 1])
    np.testing.assert_allclose(links["vel_0"], 0.01 * seen["y"])
    dense = bh.ubb_link_velocities_dense()
    assert dense.shape == shape + (19, 3)
    assert np.count_nonzero(dense[..., 0]) == np.count_nonzero(links["vel_0"])


def test_pipe_inflow_profile_matches_the_analytic_field():
    """add_pipe_inflow_boundary (geometry.py:36-86): the callback gives u_max (1 - r^2/R^2) at each
    link midpoint; at the links parallel to x (direction W) that is the cell's own profile value."""
    shape = (4, 10, 10)
    bh = _handling(shape)
    add_pipe_inflow_boundary(bh, 0.05, slice_from_direction("W", 3))
    links = bh.ubb_links()[0]
    straight = links["dir"] == 3                            # (-1, 0, 0)
    ref = get_pipe_velocity_field(shape, 0.05)[0, :, :, 0]
    got = links["vel_0"][straight]
    np.testing.assert_allclose(got, ref[links["y"][straight] - 1, links["z"][straight] - 1], atol=1e-15)


def _ldc_flags(n):
    fl = np.zeros(tuple(s + 2 for s in n), np.uint8)
    fl[:, -1, :] = 2
    fl[0] = fl[-1] = fl[:, 0] = fl[:, :, 0] = fl[:, :, -1] = 1
    return fl


def test_oracle_constant_link_velocities_equal_the_constant_ubb():
    n = (8, 7, 6)
    fl = _ldc_flags(n)
    for comp in (True, False):
        o = O.make("D3Q19", "trt", relaxation_rate=1.7, compressible=comp)
        f1, f2 = o.new_field(n), o.new_field(n)
        o.set_equilibrium(f1, np.ones(n), np.zeros(n + (3,)))
        f2[...] = f1
        link = np.zeros(n + (19, 3))
        link[..., 0] = 0.03
        r1, _ = o.run(f1, 20, "pull", 0, periodic=(0, 0, 0), flags=fl, ubb_velocity=(0.03, 0, 0))
        r2, _ = o.run(f2, 20, "pull", 0, periodic=(0, 0, 0), flags=fl, ubb_link=link)
        assert np.abs(r1 - r2).max() == 0.0


def test_oracle_adapt_velocity_shifts_by_half_the_force():
    """adapt_velocity_to_force (boundaryconditions.py:790-794): with wall velocity F/(2 rho) and the
    shift the lid is at rest, so the result equals a lid at rest (Guo force, incompressible)."""
    n = (8, 7, 6)
    fl = _ldc_flags(n)
    F = (2e-5, 0.0, 0.0)
    o = O.make("D3Q19", "trt", relaxation_rate=1.7, compressible=False, force=F)
    f1, f2 = o.new_field(n), o.new_field(n)
    o.set_equilibrium(f1, np.ones(n), np.zeros(n + (3,)))
    f2[...] = f1
    r1, _ = o.run(f1, 20, "pull", 0, periodic=(0, 0, 0), flags=fl, ubb_velocity=(0.5 * F[0], 0, 0), ubb_adapt=True)
    r2, _ = o.run(f2, 20, "pull", 0, periodic=(0, 0, 0), flags=fl, ubb_velocity=(0, 0, 0))
    assert np.abs(r1 - r2).max() < 1e-18
    f3 = o.new_field(n)
    o.set_equilibrium(f3, np.ones(n), np.zeros(n + (3,)))
    r3, _ = o.run(f3, 20, "pull", 0, periodic=(0, 0, 0), flags=fl, ubb_velocity=(0.5 * F[0], 0, 0))
    assert np.abs(r3 - r2).max() > 1e-9                     # without the shift the lid moves

"""Where a streaming pattern keeps a population: lbmpy's PDF field accessors (fieldaccess.py:66-318)
as plain offsets and slots, for host-side set-up that reads the PDF field (the initial state of
ExtrapolationOutflow links).  The sweep kernels restate the same rules on the device
(csrc/lbm_kernels.cuh, Access<PAT>)."""
from __future__ import annotations

from typing import Sequence, Tuple

# lbmpy's 'lehmann' ordering lists each direction right before its inverse; EsoPull / EsoPush
# stream the directions at even positions on one side of the collision (fieldaccess.py:184-318)
_LEHMANN_EVEN = {(0, 0, 0), (-1, 0, 0), (0, -1, 0), (0, 0, -1), (-1, -1, 0), (-1, 0, -1), (0, -1, -1),
                 (-1, 1, 0), (-1, 0, 1), (0, -1, 1), (-1, -1, -1), (-1, -1, 1), (-1, 1, -1), (1, -1, -1)}


def write_location(pattern: str, parity: int, dirs: Sequence[Tuple[int, int, int]], i: int):
    """(offset, slot) of the cell-relative location where a step of `pattern` with `parity`
    (0 EVEN, 1 ODD; ignored by two-field patterns) writes the outgoing population i of a cell."""
    c = tuple(dirs[i])
    inv = dirs.index(tuple(-v for v in c))
    zero = (0, 0, 0)
    if pattern == "pull":
        return zero, i
    if pattern == "push":
        return c, i
    if pattern == "aa":
        return (zero, inv) if parity == 0 else (c, i)
    if pattern == "esotwist":
        return tuple(max(v, 0) for v in c), (inv if parity == 0 else i)
    if pattern == "esopull":
        return (zero if c in _LEHMANN_EVEN else c), (inv if parity == 0 else i)
    if pattern == "esopush":
        return (c if c in _LEHMANN_EVEN else zero), (i if parity == 0 else inv)
    raise ValueError(f"unknown streaming pattern {pattern!r}")

"""``LBStencil`` with lbmpy's default 'walberla' direction order (lbmpy ``stencils.py:8-127``)."""
from __future__ import annotations

from .enums import Stencil
from . import methods as _m


class LBStencil:
    def __init__(self, stencil, ordering: str = "walberla"):
        if isinstance(stencil, LBStencil):
            entries, ordering = stencil.stencil_entries, stencil.ordering
        elif isinstance(stencil, tuple):
            entries, ordering = stencil, None
        else:
            name = stencil.name if isinstance(stencil, Stencil) else str(stencil)
            if ordering != "walberla":
                raise NotImplementedError("only the 'walberla' direction ordering is supported")
            if name not in _m.WALBERLA_ORDER:
                raise NotImplementedError(f"stencil {name} is not supported by the B200 sweep")
            entries = _m.WALBERLA_ORDER[name]
        if len({len(e) for e in entries}) != 1:
            raise ValueError("The stencil you have created is not valid. "
                             "It probably contains elements with different lengths")
        if len(set(entries)) < len(entries):
            raise ValueError("The stencil you have created is not valid. It contains duplicated elements")
        self._entries = tuple(tuple(e) for e in entries)
        self._ordering = ordering

    @property
    def D(self):
        return len(self._entries[0])

    @property
    def Q(self):
        return len(self._entries)

    @property
    def name(self):
        return f"D{self.D}Q{self.Q}"

    @property
    def ordering(self):
        return self._ordering

    @property
    def stencil_entries(self):
        return self._entries

    @property
    def inverse_stencil_entries(self):
        return tuple(tuple(-v for v in d) for d in self._entries)

    def index(self, direction):
        return self._entries.index(tuple(direction))

    def inverse_index(self, direction):
        return self._entries.index(tuple(-v for v in direction))

    def __getitem__(self, i):
        return self._entries[i]

    def __iter__(self):
        yield from self._entries

    def __len__(self):
        return len(self._entries)

    def __eq__(self, other):
        return isinstance(other, LBStencil) and self.ordering == other.ordering and \
            set(self._entries) == set(other._entries)

    def __hash__(self):
        return hash(self._entries)

    def __str__(self):
        return str(self._entries)

    __repr__ = __str__

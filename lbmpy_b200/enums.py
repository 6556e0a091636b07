"""Enumerations with lbmpy's names (lbmpy ``enums.py:4-238``, ``advanced_streaming/utility.py:18-38``)."""
from enum import Enum, IntEnum, auto


class Stencil(Enum):
    D2Q9 = auto()
    D2V17 = auto()
    D2V37 = auto()
    D3Q7 = auto()
    D3Q15 = auto()
    D3Q19 = auto()
    D3Q27 = auto()


class Method(Enum):
    SRT = auto()
    TRT = auto()
    MRT_RAW = auto()
    MRT = auto()
    CENTRAL_MOMENT = auto()
    TRT_KBC_N1 = auto()
    TRT_KBC_N2 = auto()
    TRT_KBC_N3 = auto()
    TRT_KBC_N4 = auto()
    CUMULANT = auto()
    MONOMIAL_CUMULANT = auto()


class CollisionSpace(Enum):
    POPULATIONS = auto()
    RAW_MOMENTS = auto()
    CENTRAL_MOMENTS = auto()
    CUMULANTS = auto()

    def compatible(self, method: Method) -> bool:
        """Which methods may be derived in this space (lbmpy enums.py:164-175)."""
        if self == CollisionSpace.POPULATIONS:
            return method in (Method.SRT, Method.TRT, Method.MRT_RAW, Method.MRT, Method.TRT_KBC_N1,
                              Method.TRT_KBC_N2, Method.TRT_KBC_N3, Method.TRT_KBC_N4)
        if self == CollisionSpace.RAW_MOMENTS:
            return method in (Method.SRT, Method.TRT, Method.MRT_RAW, Method.MRT)
        if self == CollisionSpace.CENTRAL_MOMENTS:
            return method in (Method.CENTRAL_MOMENT,)
        return method in (Method.MONOMIAL_CUMULANT, Method.CUMULANT)


class ForceModel(Enum):
    SIMPLE = auto()
    LUO = auto()
    GUO = auto()
    BUICK = auto()
    SILVA = auto()
    EDM = auto()
    KUPERSHTOKH = auto()
    HE = auto()
    SHANCHEN = auto()
    CENTRALMOMENT = auto()


class SubgridScaleModel(Enum):
    SMAGORINSKY = auto()
    QR = auto()
    LEARNED = auto()        # learned eddy viscosity (closure.MLPClosure); not an lbmpy model


class Target(Enum):
    """Where a kernel runs.  Only the GPU target exists in this package."""
    CPU = auto()
    GPU = auto()


class Timestep(IntEnum):
    """Parity of a time step for in-place streaming patterns (advanced_streaming/utility.py:18-38)."""
    EVEN = 0
    ODD = 1
    BOTH = 2

    def next(self):
        return self if self == Timestep.BOTH else Timestep((self + 1) % 2)

    @property
    def idx(self):
        return self % 2

    def __str__(self):
        return {0: "Even", 1: "Odd", 2: "Both"}[int(self)]


STREAMING_PATTERNS = ("pull", "push", "aa", "esotwist", "esopull", "esopush")


def is_inplace(streaming_pattern: str) -> bool:
    if streaming_pattern not in STREAMING_PATTERNS:
        raise ValueError("Invalid streaming pattern", streaming_pattern)
    return streaming_pattern in ("aa", "esotwist", "esopull", "esopush")


def get_timesteps(streaming_pattern: str):
    return (Timestep.EVEN, Timestep.ODD) if is_inplace(streaming_pattern) else (Timestep.BOTH,)

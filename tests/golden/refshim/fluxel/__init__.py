"""Minimal stand-in for the ``fluxel`` extension (names gridfoam imports)."""

from enum import IntEnum


class Direction(IntEnum):
    XMinus = 0
    XPlus = 1
    YMinus = 2
    YPlus = 3
    ZMinus = 4
    ZPlus = 5


class Axis(IntEnum):
    X = 0
    Y = 1
    Z = 2


class CfdAxisProjectedMesh:  # type-only placeholder
    pass


class ApibmSession:  # type-only placeholder
    pass


class BoundingBox:  # type-only placeholder
    def __init__(self, *args, **kwargs):
        pass


class FluxelManager:
    def __init__(self, *args, **kwargs):
        raise RuntimeError("fluxel is not available; use the synthetic builder")


def quaternion_from_axis_angle(axis, angle, degrees=False):
    raise RuntimeError("fluxel is not available")

"""Minimal stand-in for ``pyamg`` (the PyAMG solver is out of scope)."""


def smoothed_aggregation_solver(*args, **kwargs):
    raise RuntimeError("pyamg is not available")

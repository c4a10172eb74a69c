"""Minimal stand-in for ``graphlow`` (surface meshes are not used here)."""


class TensorMesh:
    def __class_getitem__(cls, item):
        return cls


def read(*args, **kwargs):
    raise RuntimeError("graphlow is not available")

"""Minimal stand-in for ``pyvista`` (VTU export is out of scope)."""


class UnstructuredGrid:
    def __init__(self, *args, **kwargs):
        raise RuntimeError("pyvista is not available")

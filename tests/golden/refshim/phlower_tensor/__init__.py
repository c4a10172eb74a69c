"""Minimal stand-in for ``phlower_tensor`` physical-dimension metadata."""


class PhysicalDimensions(dict):
    def __init__(self, value=None):
        super().__init__(
            {k: float(v) for k, v in (value or {}).items() if float(v) != 0.0}
        )

    def to_dict(self):
        return dict(self)


class _DimTensor:
    def __init__(self, dims):
        self.dims = dict(dims)

    def __mul__(self, other):
        out = dict(self.dims)
        for k, v in other.dims.items():
            out[k] = out.get(k, 0.0) + v
        return _DimTensor(out)

    def __truediv__(self, other):
        out = dict(self.dims)
        for k, v in other.dims.items():
            out[k] = out.get(k, 0.0) - v
        return _DimTensor(out)

    def __pow__(self, exponent):
        return _DimTensor({k: v * exponent for k, v in self.dims.items()})

    def to_physics_dimension(self):
        return PhysicalDimensions(self.dims)


def phlower_dimension_tensor(dims):
    return _DimTensor(dims)

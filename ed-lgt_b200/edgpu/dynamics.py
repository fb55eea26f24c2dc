"""Krylov time evolution (placeholder until the device kernels land)."""


def krylov_evolve(*args, **kwargs):
    raise NotImplementedError("Krylov time evolution is not built yet")

from .wavelets import fdgaus, ricker  # noqa: F401

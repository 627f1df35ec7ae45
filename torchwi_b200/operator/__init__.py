from .TimeOperator import Time2d, Time2dBatch, Time2dForward  # noqa: F401

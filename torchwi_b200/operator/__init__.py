from .TimeOperator import Time2d, Time2dBatch, Time2dForward, Time2dModels  # noqa: F401

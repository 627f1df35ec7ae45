"""Files either side of the propagator: RSF models, wavelets and shot tables,
and per-shot gather files (mirror of torchwi.io's time-domain part,
torchwi/io/__init__.py:1-13), plus batched loading of gathers into HBM."""

from . import rsf  # noqa: F401
from .shots import (  # noqa: F401
    SurveyFiles,
    TimeDataset,
    TimeForwardDataset,
    load_gathers,
    read_survey,
    save_gathers,
    time_dataloader,
    time_distributed_dataloader,
    time_forward_dataloader,
    time_forward_distributed_dataloader,
)

"""Shot gathers on disk: the reference's per-shot datasets and loaders, and a
batched loader that puts all of a rank's observed gathers into HBM at once.

Reference file conventions (examples/time/forward_modeling.py:20-22,52,
examples/time/inv_torch.py:115-116, torchwi/io/Dataset.py:6-64,
torchwi/io/Dataloader.py:7-15, torchwi/io/DistributedDataloader.py:7-20):

* model, wavelet and shot table are RSF files: `vel` has n1 = nz (fast),
  n2 = nx and d1 = h; the wavelet n1 = nt, d1 = dt; the shot table n1 = 2
  (sx, sy), n2 = nshot;
* observed gathers are one file per shot, `ftrue % ishot` (e.g.
  "seismo.%04d"), raw little-endian float32 of shape (nt, nx) -- or `.npy`.

The reference feeds shots one at a time through a DataLoader (batch size 1).
The batched plan wants every shot of a rank at once, so `load_gathers` reads
the rank's files in parallel threads into ONE pinned host buffer and copies it
to the device with a single asynchronous transfer; `save_gathers` does the
reverse for modelled data.
"""

from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np
import torch
import torch.distributed as dist

from . import rsf


# ----------------------------------------------------------------------------
# the reference's datasets and loaders (time domain)
# ----------------------------------------------------------------------------

def _load_shot(ftrue: str, index: int, data_type: str, shape=None) -> np.ndarray:
    path = ftrue % index
    if data_type in ("bin", "binary"):
        data = np.fromfile(path, dtype=np.float32)
        if shape:
            data = data.reshape(shape)
        return data
    if data_type == "npy":
        return np.load(path)
    raise ValueError(f"unknown data_type {data_type!r} (bin | binary | npy)")


class TimeDataset(torch.utils.data.Dataset):
    """(sx, sy, observed[, index]) per shot; observed read from `ftrue % index`."""

    def __init__(self, sxy, ftrue, with_index=False, data_type="bin", shape=None, transpose=False):
        super().__init__()
        self.sxy, self.ftrue, self.with_index = sxy, ftrue, with_index
        self.data_type, self.shape, self.transpose = data_type, shape, transpose

    def __len__(self):
        return len(self.sxy)

    def load_data(self, index):
        data = _load_shot(self.ftrue, index, self.data_type, self.shape)
        if self.transpose:
            data = data.T
        return torch.from_numpy(data)

    def __getitem__(self, index):
        observed = self.load_data(index)
        sx, sy = self.sxy[index]
        return (sx, sy, observed, index) if self.with_index else (sx, sy, observed)


class TimeForwardDataset(torch.utils.data.Dataset):
    """(sx, sy[, index]) per shot, for forward modelling."""

    def __init__(self, sxy, with_index=True):
        super().__init__()
        self.sxy, self.with_index = sxy, with_index
        self.nshot = len(sxy)

    def __len__(self):
        return self.nshot

    def __getitem__(self, index):
        sx, sy = self.sxy[index]
        return (sx, sy, index) if self.with_index else (sx, sy)


def time_forward_dataloader(sxy, **kwargs):
    return torch.utils.data.DataLoader(TimeForwardDataset(sxy, **kwargs), batch_size=1)


def time_dataloader(ftrue, sxy, **kwargs):
    return torch.utils.data.DataLoader(TimeDataset(sxy, ftrue, with_index=True, **kwargs), batch_size=1)


def _distributed(dataset, size=None, rank=None):
    # one shot per batch; ranks from torch.distributed (the reference asks Horovod)
    if size is None:
        size = dist.get_world_size() if dist.is_initialized() else 1
    if rank is None:
        rank = dist.get_rank() if dist.is_initialized() else 0
    sampler = torch.utils.data.distributed.DistributedSampler(dataset, num_replicas=size, rank=rank)
    return torch.utils.data.DataLoader(dataset, batch_size=1, sampler=sampler)


def time_forward_distributed_dataloader(sxy, size=None, rank=None, **kwargs):
    return _distributed(TimeForwardDataset(sxy, **kwargs), size, rank)


def time_distributed_dataloader(ftrue, sxy, size=None, rank=None, **kwargs):
    return _distributed(TimeDataset(sxy, ftrue, with_index=True, **kwargs), size, rank)


# ----------------------------------------------------------------------------
# survey inputs and batched gathers
# ----------------------------------------------------------------------------

@dataclass
class SurveyFiles:
    """Model, wavelet and shot table as the reference's examples read them."""
    nx: int
    ny: int
    h: float
    vel: np.ndarray      # (nx, ny), z fastest
    nt: int
    dt: float
    w: np.ndarray        # (nt,)
    nshot: int
    sxy: np.ndarray      # (nshot, 2): sx, sy

    @property
    def sx(self):
        return self.sxy[:, 0]

    @property
    def sy(self):
        return self.sxy[:, 1]


def read_survey(fvel: str, fwav: str, fshot: str) -> SurveyFiles:
    """`rsf.fromfile` calls of forward_modeling.py:20-22 / inv_torch.py:21,24,115."""
    nt, dt, w = rsf.fromfile(fwav, "n1 d1 data")
    ny, nx, h, vel = rsf.fromfile(fvel, "n1 n2 d1 data")
    nshot, sxy = rsf.fromfile(fshot, "n2 data")
    return SurveyFiles(nx, ny, h, vel, nt, dt, w, nshot, sxy.reshape(nshot, -1))


def _read_into(path: str, out: np.ndarray, data_type: str):
    if data_type == "npy":
        out[...] = np.load(path).reshape(out.shape)
        return
    with open(path, "rb") as fh:
        got = fh.readinto(memoryview(out).cast("B"))
    if got != out.nbytes:
        raise ValueError(f"{path}: {got} bytes, expected {out.nbytes} ({out.shape} float32)")


def load_gathers(ftrue: str, indices, nt: int, nx: int, device=None, data_type: str = "bin",
                 threads: int = 8) -> torch.Tensor:
    """Observed gathers of the shots `indices` as one [len(indices), nt, nx]
    float32 tensor on `device` (read in parallel into pinned memory, one
    asynchronous host-to-device copy on the current stream).  Each file holds
    exactly nt*nx float32 samples."""
    indices = [int(i) for i in indices]
    host = torch.empty((len(indices), nt, nx), dtype=torch.float32,
                       pin_memory=device is not None and torch.device(device).type == "cuda")
    view = host.numpy()
    with ThreadPoolExecutor(max_workers=max(1, threads)) as ex:
        list(ex.map(lambda k: _read_into(ftrue % indices[k], view[k], data_type), range(len(indices))))
    if device is None or torch.device(device).type == "cpu":
        return host
    return host.to(device, non_blocking=True)


def save_gathers(gathers: torch.Tensor, ftrue: str, indices, threads: int = 8):
    """Write gathers [S, nt, nx] as one raw float32 file per shot,
    `ftrue % indices[k]` (forward_modeling.py:52 writes "seismo.%04d")."""
    indices = [int(i) for i in indices]
    if gathers.shape[0] != len(indices):
        raise ValueError("one index per shot")
    if gathers.is_cuda:
        host = torch.empty(gathers.shape, dtype=torch.float32, pin_memory=True)
        host.copy_(gathers, non_blocking=True)
        torch.cuda.current_stream(gathers.device).synchronize()
    else:
        host = gathers.to(torch.float32)
    view = host.numpy()
    for k in indices:
        d = os.path.dirname(ftrue % k)
        if d:
            os.makedirs(d, exist_ok=True)
    with ThreadPoolExecutor(max_workers=max(1, threads)) as ex:
        list(ex.map(lambda k: view[k].tofile(ftrue % indices[k]), range(len(indices))))

"""Madagascar RSF datasets: a text header plus a data file.

The reference's examples read the velocity model, the wavelet and the shot
table from RSF files (examples/time/forward_modeling.py:20-22,
examples/time/inv_torch.py:21,24,115, through torchwi/io/rsf.py).  This
module reads and writes the same files, built from the format itself:

* Header: free text.  Every ``key=value`` token is an assignment; the value
  is a quoted string (``"..."`` or ``'...'``, blanks allowed) or a run of
  non-blank characters.  Programs append their own lines to a header, so a
  later assignment of a key overrides an earlier one.  Text without ``=``
  (program names between appended blocks) carries no keys.
* Keys: ``in`` (also ``_in``, ``infile``; infile over _in over in) names the
  data file; ``data_format`` is ``<form>_<type>`` with form ``native`` or
  ``ascii`` and type ``float``, ``int`` or ``complex`` (the keys ``form`` and
  ``type`` replace one half); ``esize`` is the sample size (4, 8 for complex,
  0 for ascii); ``n#``, ``o#``, ``d#`` are the sample count, origin and step
  of axis # (1 = fastest, up to 9); ``label#`` and ``unit#`` annotate it.
* Data: native files hold raw samples with axis 1 fastest (read here as an
  array of shape (n_k, ..., n2, n1): float32, int32 or complex64); ascii
  files hold whitespace-separated numbers.
* Written headers hold ``in``, ``esize`` and ``data_format`` (quoted
  strings), then one line per axis, ``n# o# d#`` plus quoted ``label#`` /
  ``unit#`` when set -- the lines TorchWI's writer emits, so files are
  interchangeable with it and with Madagascar.  Data go to ``<header>@``
  unless ``_in`` names another file.

Errors (an unknown keyword, no or a missing data file, an unsupported data
format) print their message to stderr and raise ``RSFError``, a
``SystemExit`` with status 1, so scripts end as they would with the
reference (which calls ``sys.exit(1)``) and library callers can catch it.
"""

from __future__ import annotations

import os
import re
import sys
import tempfile
from dataclasses import dataclass

import numpy as np

MAXDIM = 9
SAMPLE_TYPES = {"float": np.float32, "int": np.int32, "complex": np.complex64}
FORMS = ("native", "ascii")

# key = "quoted" | 'quoted' | bare-run ; the key may not follow a word character
_ASSIGNMENT = re.compile(r"""(?<![\w])([A-Za-z_]\w*)\s*=\s*("[^"]*"|'[^']*'|\S+)""")
_AXIS_KEY = re.compile(r"(n|o|d|label|unit)([1-9])")
_DATA_KEYS = ("in", "_in", "infile")   # lowest precedence first


class RSFError(SystemExit):
    """An RSF failure; exits with status 1 when not caught."""

    def __init__(self, message: str):
        sys.stderr.write(message + "\n")
        super().__init__(1)
        self.message = message

    def __str__(self):
        return self.message


def parse_header(text: str) -> dict[str, str]:
    """All assignments of a header as {key: value} (quotes removed); the
    last assignment of a key wins."""
    out: dict[str, str] = {}
    for key, value in _ASSIGNMENT.findall(text):
        if len(value) >= 2 and value[0] == value[-1] and value[0] in "\"'":
            value = value[1:-1]
        out[key] = value
    return out


@dataclass
class Axis:
    """One axis: n samples starting at o with step d, plus label and unit."""

    n: int = 0
    o: float = 0.0
    d: float = 0.0
    label: str = ""
    unit: str = ""

    def __post_init__(self):
        self.n, self.o, self.d = int(self.n), float(self.o), float(self.d)

    def line(self, i: int) -> str:
        parts = [f"n{i}={self.n}", f"o{i}={self.o}", f"d{i}={self.d}"]
        parts += [f'{k}{i}="{v}"' for k, v in (("label", self.label), ("unit", self.unit)) if v]
        return " ".join(parts)


def _typed_axis_value(field: str, raw):
    return int(raw) if field == "n" else float(raw) if field in ("o", "d") else str(raw)


class RSF:
    """One dataset: its header values and an open data file.  Use `input`
    to read one and `output` to write one."""

    def __init__(self, data_format: str | None = None):
        self.form, self.type = "native", "float"
        if data_format:
            self.data_format = data_format
        self.axes = [Axis() for _ in range(MAXDIM)]
        self.data_path = ""
        self.filename = ""   # the header file ("" = stdin / stdout)
        self.f = None
        self._header_written = False

    # -- format -----------------------------------------------------------------
    @property
    def data_format(self) -> str:
        return f"{self.form}_{self.type}"

    @data_format.setter
    def data_format(self, value: str):
        form, _, typ = str(value).partition("_")
        self.form, self.type = form.lower(), typ.lower()

    def _check_format(self):
        if self.type not in SAMPLE_TYPES:
            raise RSFError(f"Wrong type: {self.type}")
        if self.form not in FORMS:
            raise RSFError(f"Wrong format: {self.form}")

    @property
    def esize(self) -> int:
        return 0 if self.form == "ascii" else 8 if self.type == "complex" else 4

    @property
    def dtype(self):
        self._check_format()
        return SAMPLE_TYPES[self.type]

    # -- geometry ---------------------------------------------------------------
    @property
    def dimension(self) -> int:
        return max((i + 1 for i, ax in enumerate(self.axes) if ax.n > 0), default=0)

    @property
    def shape(self) -> tuple:
        return tuple(ax.n for ax in reversed(self.axes[:self.dimension]))

    def size(self, istart: int = 0) -> int:
        """Samples in the axes after the first `istart` (outermost first)."""
        return int(np.prod(self.shape[istart:], dtype=np.int64))

    # -- keys -------------------------------------------------------------------
    def set(self, **keys):
        """Set header keys: in/_in/infile, data_format/form/type, n#/o#/d#/
        label#/unit#, ax# (an Axis) or axes (a list of Axis); esize follows
        from the format."""
        for key, value in keys.items():
            axis = _AXIS_KEY.fullmatch(key)
            if key in _DATA_KEYS:
                self.data_path = str(value)
            elif key == "data_format":
                self.data_format = value
            elif key in ("form", "type"):
                setattr(self, key, str(value).lower())
            elif key == "esize":
                continue
            elif key == "axes":
                for i, ax in enumerate(value):
                    self.axes[i] = ax
            elif re.fullmatch(r"ax[1-9]", key):
                self.axes[int(key[2]) - 1] = value
            elif axis:
                field, i = axis.group(1), int(axis.group(2))
                setattr(self.axes[i - 1], field, _typed_axis_value(field, value))
            else:
                raise RSFError(f"Wrong keyword: {key}")

    def __setitem__(self, key, value):
        self.set(**{key: value})

    def get(self, key: str):
        """One value: in, esize, data_format, form, type, axes, ax#, n#, o#,
        d#, label#, unit#, header (a dict) or data (every sample)."""
        if key in _DATA_KEYS:
            return self.data_path
        if key in ("esize", "data_format", "form", "type", "axes"):
            return getattr(self, key)
        if key == "data":
            return self.read(read_all=True)
        if key == "header":
            return self.header_dict()
        if re.fullmatch(r"ax[1-9]", key):
            return self.axes[int(key[2]) - 1]
        axis = _AXIS_KEY.fullmatch(key)
        if axis:
            return getattr(self.axes[int(axis.group(2)) - 1], axis.group(1))
        raise RSFError(f"Wrong keyword: {key}")

    __getitem__ = get

    def gets(self, keys):
        """Several values (a list, or a blank-separated string); one key
        gives the value itself."""
        keys = keys.split() if isinstance(keys, str) else list(keys)
        values = [self.get(k) for k in keys]
        return values[0] if len(values) == 1 else values

    def header_dict(self, contain_in=False) -> dict:
        out = {"in": self.data_path} if contain_in else {}
        out.update({f"ax{i + 1}": self.axes[i] for i in range(self.dimension)})
        out.update(data_format=self.data_format, esize=self.esize)
        return out

    def header_text(self) -> str:
        lines = [f'in="{self.data_path}"', f"esize={self.esize}", f'data_format="{self.data_format}"']
        lines += [self.axes[i].line(i + 1) for i in range(self.dimension)]
        return "\n".join(lines) + "\n"

    # -- data -------------------------------------------------------------------
    def open_data(self, mode: str):
        try:
            self.f = open(self.data_path, mode)
        except OSError as e:
            raise RSFError(f"Error: cannot open data file {self.data_path}: {e.strerror}") from None

    def close(self):
        if self.f is not None:
            self.f.close()
            self.f = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def read(self, read_all=False):
        """Every sample, shaped (n_k, ..., n1), with read_all; else the next
        trace of n1 samples (empty at the end).  ascii data come whole."""
        if self.form == "ascii":
            data = np.loadtxt(self.f, dtype=self.dtype)
            return data.reshape(1) if data.ndim == 0 else data
        count = self.size() if read_all else self.axes[0].n
        data = np.fromfile(self.f, dtype=self.dtype, count=count)
        if read_all:
            self.close()
            return data.reshape(self.shape)
        return data

    def traces(self):
        """The data trace by trace (n1 samples each); ascii data as one."""
        if self.form == "ascii":
            yield self.read()
            return
        while True:
            trace = self.read()
            if trace.size == 0:
                return
            yield trace

    def write_header(self):
        if self._header_written:
            return
        text = self.header_text()
        if self.filename and self.filename.lower() != "stdout":
            with open(self.filename, "w") as fh:
                fh.write(text)
        else:
            sys.stdout.write(text)
        self._header_written = True

    def write(self, data, close=False, fmt="%.18e"):
        """Write the header (once) and append `data` to the data file."""
        self.write_header()
        data = np.asarray(data)
        if self.form == "native":
            data.astype(self.dtype).tofile(self.f)
        elif fmt:
            np.savetxt(self.f, data, fmt)
        else:
            np.savetxt(self.f, data)
        if close:
            self.close()


def input(filename="", mode=None, data_format=None) -> RSF:  # noqa: A001 - the reference's name
    """Read the header `filename` ("" or "stdin": standard input) and open
    its data file."""
    ds = RSF(data_format)
    ds.filename = filename
    if filename and filename.lower() != "stdin":
        with open(filename) as fh:
            text = fh.read()
    else:
        text = sys.stdin.read()
    values = parse_header(text)
    for key in _DATA_KEYS:
        if key in values:
            ds.data_path = values[key]
    if "data_format" in values:
        ds.data_format = values["data_format"]
    for key in ("type", "form"):
        if key in values:
            setattr(ds, key, values[key].lower())
    for key, value in values.items():
        if _AXIS_KEY.fullmatch(key):
            ds.set(**{key: value})
    if not ds.data_path:
        raise RSFError("Error: Cannot find 'in' keyword from rsf header")
    if not os.path.exists(ds.data_path):
        raise RSFError(f"Error: File not exists - {ds.data_path}")
    ds.open_data(mode or ("r" if ds.form == "ascii" else "rb"))
    return ds


def output(filename="", mode=None, data_format=None, _in=None, open_in=True, abspath=True,
           **keys) -> RSF:
    """Create a dataset for writing: header `filename` ("" or "stdout":
    standard output), data in `_in`, else `<filename>@`, else a temporary
    `./*.rsf@`; keyword arguments set header keys (`n1=`, `d1=`, `label1=`,
    `ax2=Axis(...)`, ...).  The path in the header is absolute with
    `abspath`."""
    ds = RSF(data_format)
    ds.filename = filename
    ds.set(**keys)
    to_file = bool(filename) and filename.lower() != "stdout"
    path = _in or (filename + "@" if to_file else None)
    if path is None:
        if not open_in:
            return ds
        ds.f = tempfile.NamedTemporaryFile(mode=mode or "wb", suffix=".rsf@", dir="./", delete=False)
        path = ds.f.name
    ds.data_path = os.path.abspath(path) if abspath else path
    if open_in and ds.f is None:
        ds.open_data(mode or "wb")
    return ds


def fromfile(filename, key):
    """`fromfile("vel.rsf", "n1 n2 d1 data")` -> [n1, n2, d1, array]; one key
    gives the value itself."""
    with input(filename) as ds:
        return ds.gets(key)


def tofile(filename, data, **keys):
    """Write `data` and its header in one call (keys as for `output`)."""
    with output(filename, **keys) as ds:
        ds.write(data)


__all__ = ["Axis", "RSF", "RSFError", "input", "output", "fromfile", "tofile", "parse_header",
           "MAXDIM", "SAMPLE_TYPES", "FORMS"]

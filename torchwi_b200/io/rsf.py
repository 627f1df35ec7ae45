"""Madagascar RSF files: a text header of `key=value` pairs plus a data file
named by its `in=` key (binary "native" or whitespace-separated "ascii").

Same reading and writing rules as TorchWI's RSF module (torchwi/io/rsf.py:1-409),
which the reference's examples use for the velocity model, the wavelet and
the shot table (examples/time/forward_modeling.py:20-22,
examples/time/inv_torch.py:21,24,115):

* reading: every known key is looked up in the header text and the LAST
  occurrence wins (appended histories override earlier entries); values may
  be quoted; `n*`/`esize` are integers, `o*`/`d*` floats;
* data come back as a numpy array of shape (n_k, ..., n2, n1) -- axis 1
  fastest -- with dtype float32 / int32 / complex64 from `data_format`
  (`native_float` by default);
* writing: the header holds `in`, `esize` and `data_format`, then one line
  per axis (`n o d` and, when set, quoted `label` and `unit`); the data go to
  `<header>@` unless `_in` names another file.

Errors (unknown keyword, missing or unreadable data file, bad data format)
print their message to stderr and raise `RSFError`, a `SystemExit` with
status 1 -- what the reference does with `sys.exit(1)` -- so scripts end the
same way and library callers can still catch it.
"""

from __future__ import annotations

import os
import re
import sys
import tempfile

import numpy as np

MAXDIM = 9
_AXIS_KEYS = [f"{f}{i}" for i in range(1, MAXDIM + 1) for f in ("n", "o", "d", "label", "unit")]
READ_KEYS = ["in", "esize", "data_format", "type", "form", "_in", "infile"] + _AXIS_KEYS
WRITE_KEYS = ["in", "esize", "data_format"]
_INT_KEYS = {"esize"} | {f"n{i}" for i in range(1, MAXDIM + 1)}
_FLOAT_KEYS = {f"{f}{i}" for i in range(1, MAXDIM + 1) for f in ("o", "d")}
_DTYPES = {"float": np.float32, "int": np.int32, "complex": np.complex64}
_FORMS = ("native", "ascii")


class RSFError(SystemExit):
    """An RSF failure; exits with status 1 when not caught."""

    def __init__(self, message: str):
        sys.stderr.write(message + "\n")
        super().__init__(1)
        self.message = message

    def __str__(self):
        return self.message


def _unquote(s: str) -> str:
    return s[1:-1] if s[:1] in ("'", '"') else s


def _quote(s: str) -> str:
    return f'"{s}"'


def _typed(key: str, raw: str):
    if key in _INT_KEYS:
        return int(raw)
    if key in _FLOAT_KEYS:
        return float(raw)
    return _unquote(raw)


def find_value(key: str, text: str, unquote: bool = True):
    """Last `key=value` of `text` (value up to whitespace, or a quoted string
    that may contain spaces), or None."""
    hits = re.findall(key + r"\s*=\s*(\S+)", text)
    if not hits:
        return None
    val = hits[-1]
    for q in ("'", '"'):
        if val.startswith(q) and not val.endswith(q):
            spaced = re.findall(key + "=" + q + "(.+?)" + q, text)
            if spaced:
                val = spaced[-1]
    return _unquote(val) if unquote else val


class Axis:
    """One axis: n samples starting at o with step d, plus label and unit."""

    def __init__(self, n=0, o=0.0, d=0.0, label="", unit=""):
        self.n, self.o, self.d = int(n), float(o), float(d)
        self.label, self.unit = _unquote(label), _unquote(unit)

    def to_str(self, idim: int) -> str:
        s = f"n{idim}={self.n} o{idim}={self.o} d{idim}={self.d}"
        if self.label:
            s += f' label{idim}="{self.label}"'
        if self.unit:
            s += f' unit{idim}="{self.unit}"'
        return s

    def __eq__(self, other):
        return isinstance(other, Axis) and (self.n, self.o, self.d, self.label, self.unit) == (
            other.n, other.o, other.d, other.label, other.unit)

    def __repr__(self):
        return f"Axis(n={self.n}, o={self.o}, d={self.d}, label={self.label!r}, unit={self.unit!r})"


class RSF:
    """An RSF dataset being read or written (use `input` / `output`)."""

    def __init__(self, mode=None, readonly=True, data_format=None):
        self._in = ""
        self._open = False
        self._data_format = data_format or "native_float"
        self._mode = mode or ("r" if readonly and self.form == "ascii" else "rb" if readonly else "wb")
        self.axes = [Axis() for _ in range(MAXDIM)]
        self.filename = ""
        self.wrote = False

    # --- format ------------------------------------------------------------
    @property
    def data_format(self) -> str:
        return self._data_format

    @data_format.setter
    def data_format(self, val):
        self._data_format = val
        if self.type not in _DTYPES:
            raise RSFError(f"Wrong type: {self.type}")
        if self.form not in _FORMS:
            raise RSFError(f"Wrong format: {self.form}")

    @property
    def form(self) -> str:
        return self._data_format.split("_")[0].lower()

    @form.setter
    def form(self, val):
        self._data_format = f"{val}_{self._data_format.split('_')[1]}"

    @property
    def type(self) -> str:
        return self._data_format.split("_")[1].lower()

    @type.setter
    def type(self, val):
        self._data_format = f"{self._data_format.split('_')[0]}_{val}"

    @property
    def esize(self) -> int:
        if self.form == "ascii":
            return 0
        return 8 if self.type == "complex" else 4

    @property
    def dtype(self):
        try:
            return _DTYPES[self.type]
        except KeyError:
            raise RSFError(f"Wrong type: {self.type}") from None

    # --- axes --------------------------------------------------------------
    @property
    def dimension(self) -> int:
        dim = 0
        for i, ax in enumerate(self.axes):
            if ax.n > 0:
                dim = i + 1
        return dim

    @property
    def shape(self) -> tuple:
        return tuple(self.axes[i].n for i in range(self.dimension - 1, -1, -1))

    def size(self, istart: int = 0) -> int:
        """Samples in dimensions istart+1 .. last (size(0) = all)."""
        return int(np.prod(self.shape[istart:], dtype=np.int64))

    # --- keys --------------------------------------------------------------
    def set_in(self, path, abspath=True):
        self._in = os.path.abspath(path) if abspath else path

    def set(self, **kwargs):
        for key, val in kwargs.items():
            if key in ("in", "infile", "_in"):
                self._in = val
            elif key == "esize":
                self._esize = val
            elif key in ("data_format", "form", "type"):
                setattr(self, key, val)
            elif key == "axes":
                for i, ax in enumerate(val):
                    self.axes[i] = ax
            elif key.startswith("ax"):
                self.axes[int(key[-1]) - 1] = val
            else:
                setattr(self.axes[int(key[-1]) - 1], key[:-1], val)

    def __setitem__(self, key, value):
        self.set(**{key: value})

    def get(self, key):
        if key == "in":
            return self._in
        if key in ("esize", "data_format", "form", "type"):
            return getattr(self, key)
        if key == "axes":
            return self.axes
        if key.startswith("ax"):
            return self.axes[int(key[-1]) - 1]
        if key == "data":
            return self.read(read_all=True)
        if key == "header":
            return self.header_dict()
        return getattr(self.axes[int(key[-1]) - 1], key[:-1])

    __getitem__ = get

    def gets(self, keys):
        if isinstance(keys, str):
            keys = keys.split()
        return self.get(keys[0]) if len(keys) == 1 else [self.get(k) for k in keys]

    def axes_dict(self) -> dict:
        return {f"ax{i}": self.axes[i - 1] for i in range(1, self.dimension + 1)}

    def header_dict(self, contain_in=False) -> dict:
        d = {"in": self._in} if contain_in else {}
        d.update(self.axes_dict())
        d["data_format"] = self.data_format
        d["esize"] = self.esize
        return d

    # --- files -------------------------------------------------------------
    def open_in(self, tmpfile=False, abspath=True):
        if tmpfile:
            self.f = tempfile.NamedTemporaryFile(mode=self._mode, suffix=".rsf@", dir="./", delete=False)
            self.set_in(self.f.name, abspath)
        else:
            try:
                self.f = open(self._in, self._mode)
            except OSError as e:
                raise RSFError(f"Error: cannot open data file {self._in}: {e.strerror}") from None
        self._open = True

    def close(self):
        if self._open:
            self.f.close()
            self._open = False

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def read_rsf(self, filename):
        if filename and filename.lower() != "stdin":
            with open(filename) as fh:
                text = fh.read()
        else:
            text = sys.stdin.read()
        for key in READ_KEYS:
            raw = find_value(key, text)
            if raw is not None:
                self.set(**{key: _typed(key, raw)})
        if not self._in:
            raise RSFError("Error: Cannot find 'in' keyword from rsf header")
        if not os.path.exists(self._in):
            raise RSFError(f"Error: File not exists - {self._in}")

    def read(self, read_all=False):
        """All samples (shaped) with read_all, else the next trace (n1 samples);
        ascii data are always read whole."""
        if self.form == "native":
            count = self.size() if read_all else self.axes[0].n
            data = np.fromfile(self.f, dtype=self.dtype, count=count)
            if read_all:
                data = data.reshape(self.shape)
                self.close()
            return data
        data = np.loadtxt(self.f, dtype=self.dtype)
        return data.reshape(1) if data.shape == () else data

    def traces(self):
        if self.form == "native":
            trc = self.read()
            while len(trc) > 0:
                yield trc
                trc = self.read()
        else:
            yield self.read()

    def header_text(self) -> str:
        lines = []
        for key in WRITE_KEYS:
            val = self.get(key)
            lines.append(f"{key}={val if key in _INT_KEYS or key in _FLOAT_KEYS else _quote(str(val))}")
        lines += [self.axes[i].to_str(i + 1) for i in range(self.dimension)]
        return "\n".join(lines) + "\n"

    def write_rsf(self):
        if self.wrote:
            return
        text = self.header_text()
        if self.filename and self.filename.lower() != "stdout":
            with open(self.filename, "w") as fh:
                fh.write(text)
        else:
            sys.stdout.write(text)
        self.wrote = True

    def write(self, data, close=False, fmt="%.18e"):
        self.write_rsf()
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
    """Open an RSF header and its data file for reading."""
    r = RSF(mode=mode, readonly=True, data_format=data_format)
    r.filename = filename
    r.read_rsf(filename)
    r.open_in()
    return r


def output(filename="", mode=None, data_format=None, _in=None, open_in=True, abspath=True,
           **kwargs) -> RSF:
    """Create an RSF dataset for writing; keyword arguments set header keys
    (`n1=`, `d1=`, `label1=`, `ax2=Axis(...)`, `data_format=` ...)."""
    r = RSF(mode=mode, readonly=False, data_format=data_format)
    r.filename = filename
    for key in kwargs:
        if key not in READ_KEYS and not re.fullmatch(r"ax[1-9]|axes", key):
            raise RSFError(f"Wrong keyword: {key}")
    r.set(**kwargs)
    r.wrote = False
    if filename and filename.lower() != "stdout":
        r.set_in(_in if _in else filename + "@", abspath)
        if open_in:
            r.open_in()
    elif _in:
        r.set_in(_in, abspath)
        if open_in:
            r.open_in()
    elif open_in:
        r.open_in(tmpfile=True, abspath=abspath)
    return r


def fromfile(filename, key):
    """`fromfile("vel.rsf", "n1 n2 d1 data")` -> [n1, n2, d1, array]; one key
    returns the value itself."""
    with input(filename) as f:
        return f.gets(key.split() if isinstance(key, str) else key)


def tofile(filename, data, **kwargs):
    with output(filename, **kwargs) as f:
        f.write(data)


__all__ = ["Axis", "RSF", "RSFError", "input", "output", "fromfile", "tofile", "find_value",
           "MAXDIM", "READ_KEYS", "WRITE_KEYS"]

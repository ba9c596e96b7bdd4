"""RSF/SEP file subset used by kirchmig2d_cig: a text header of ``key=value``
tokens plus a raw FP32 binary named by ``in=``.

Follows the reference's SEP handling in SEFILESYSTEM/src/se_fs_sep.cpp:
header parsing (:440-700: later tokens override earlier ones, ``n1..n9``,
``o*``, ``d*``, ``in``, ``esize``, ``data_format`` native_float/xdr_float),
new-file creation (:704-794: ``in="<header>@"``, native_float) and the header
writer (:796-977: history line, ``in``, ``data_format``, ``n``/``d``/``o``,
``esize``, then the remaining keys).  Doubles are printed as the reference's
``_sep_print_a_double`` does (:67-93): integers without a point, otherwise
``%.12f`` with trailing zeros removed.
"""
from __future__ import annotations

import datetime
import getpass
import os
import shlex
import socket

import numpy as np

__all__ = ["RsfHeader", "read_header", "read", "write", "format_double"]


def format_double(v: float) -> str:
    v = float(v)
    if v == int(v) and abs(v) < 9.2e18:
        return "%d" % int(v)
    s = "%.12f" % v
    if "." in s:
        s = s.rstrip("0")
    return s


class RsfHeader:
    def __init__(self, path: str):
        self.path = path
        self.n = [1] * 9
        self.o = [0.0] * 9
        self.d = [1.0] * 9
        self.ndim = 0
        self.esize = 4
        self.native = False  # a header without data_format is xdr (se_fs_sep.cpp:458)
        self.binary = ""
        self.extra: dict[str, str] = {}

    @property
    def shape_fortran(self):
        return tuple(self.n[: max(self.ndim, 1)])

    def data_path(self) -> str:
        if self.binary in ("stdin", "-"):
            raise ValueError("inline RSF data is not supported: %s" % self.path)
        if os.path.isabs(self.binary):
            return self.binary
        return os.path.join(os.path.dirname(os.path.abspath(self.path)), self.binary)


def _tokens(text: str):
    lex = shlex.shlex(text, posix=True)
    lex.whitespace_split = True
    lex.commenters = "#"
    try:
        return list(lex)
    except ValueError:
        return text.split()


def read_header(path: str) -> RsfHeader:
    h = RsfHeader(path)
    h.n[0] = 0
    with open(path, "rb") as f:
        raw = f.read()
    eot = raw.find(b"\x04")
    if eot >= 0:
        raw = raw[:eot]
    text = raw.decode("latin-1")
    for tok in _tokens(text):
        if "=" not in tok:
            continue
        key, val = tok.split("=", 1)
        key = key.strip()
        if not key:
            continue
        if key[0] in "nod" and key[1:].isdigit() and 1 <= int(key[1:]) <= 9:
            k = int(key[1:]) - 1
            try:
                dv = float(val)
            except ValueError:
                continue
            if key[0] == "n":
                if dv < 1.0:
                    continue
                h.n[k] = int(dv)
            elif key[0] == "o":
                h.o[k] = dv
            else:
                if dv == 0.0:
                    continue
                h.d[k] = dv
            h.ndim = max(h.ndim, k + 1)
            continue
        if key == "in":
            if val:
                h.binary = val
            continue
        if key == "esize":
            try:
                h.esize = int(val)
            except ValueError:
                pass
            continue
        if key == "data_format":
            if val == "native_float":
                h.native = True
            elif val == "xdr_float":
                h.native = False
            continue
        h.extra[key] = val
    if not h.binary:
        raise ValueError("Missing required SEP global header 'in' in file '%s'" % path)
    return h


def read(path: str, count: int | None = None, offset_elems: int = 0):
    """Return (header, data) with data as a 1-D float32 array in file order
    (axis 1 fastest).  ``count``/``offset_elems`` read a window."""
    h = read_header(path)
    if h.esize != 4:
        raise ValueError("only esize=4 float data is supported: %s" % path)
    total = 1
    for i in range(max(h.ndim, 1)):
        total *= h.n[i]
    if count is None:
        count = total - offset_elems
    dt = np.dtype("<f4") if h.native else np.dtype(">f4")
    with open(h.data_path(), "rb") as f:
        f.seek(4 * offset_elems)
        buf = f.read(4 * count)
    if len(buf) != 4 * count:
        raise ValueError("RSF data file %s is truncated" % h.data_path())
    arr = np.frombuffer(buf, dtype=dt).astype(np.float32)
    return h, arr


def write(path: str, data, n, o=None, d=None, extra: dict | None = None,
          tool: str = "kcig") -> None:
    """Write a new native_float RSF pair ``path`` + ``path@``."""
    ndim = len(n)
    o = list(o) if o is not None else [0.0] * ndim
    d = list(d) if d is not None else [1.0] * ndim
    arr = np.ascontiguousarray(np.asarray(data, dtype=np.float32)).reshape(-1)
    total = int(np.prod(n))
    if arr.size != total:
        raise ValueError("data size %d does not match n=%s" % (arr.size, n))
    bin_path = path + "@"
    arr.astype("<f4").tofile(bin_path)
    try:
        user = getpass.getuser()
    except Exception:
        user = "unknown_user"
    lines = ["", "%s\t\"%s\"\t%s@%s\t%s" % (tool, os.getcwd(), user, socket.gethostname(),
                                             datetime.datetime.now().ctime())]
    lines.append("\tin=\"%s\"" % os.path.basename(bin_path))
    lines.append("\tdata_format=\"native_float\"")
    for i in range(ndim):
        lines.append("\tn%d=%d" % (i + 1, int(n[i])))
    for i in range(ndim):
        lines.append("\td%d=%s" % (i + 1, format_double(d[i])))
    for i in range(ndim):
        lines.append("\to%d=%s" % (i + 1, format_double(o[i])))
    lines.append("\tesize=4")
    for k, v in (extra or {}).items():
        lines.append("\t%s=\"%s\"" % (k, v))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")

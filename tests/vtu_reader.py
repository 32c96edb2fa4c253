"""Minimal reader of the VTU files the writer produces (raw appended data,
a 4-byte length before each array), for the tests."""
import re

import numpy as np

_TYPES = {"Float64": np.float64, "Int32": np.int32}


def read_vtu(path):
    raw = open(path, "rb").read()
    marker = b'<AppendedData encoding="raw">\n_'
    head, data = raw.split(marker, 1)
    assert data.endswith(b" </AppendedData>\n</VTKFile>\n")
    text = head.decode()
    m = re.search(r'<Piece NumberOfPoints="(\d+)" NumberOfCells="(\d+)">', text)
    out = {"n_points": int(m.group(1)), "n_cells": int(m.group(2)), "arrays": {}}
    for a in re.finditer(r'<DataArray type="(\w+)" Name="([^"]+)"(?: NumberOfComponents="(\d+)")? '
                         r'format="appended" offset="(\d+)">', text):
        typ, name, comps, off = a.group(1), a.group(2), int(a.group(3) or 1), int(a.group(4))
        n = int(np.frombuffer(data[off:off + 4], np.int32)[0])
        arr = np.frombuffer(data[off + 4:off + 4 + n], _TYPES[typ])
        out["arrays"][name] = arr.reshape(-1, comps) if comps > 1 else arr
    return out

"""Reader of the legacy binary VTK files h3c_write_vtk writes (hom3's io::Vtk
layout, src/io/vtk.hpp:156-330): test helper."""
import numpy as np


def read(path):
    data = open(path, "rb").read()
    pos = 0

    def line():
        nonlocal pos
        e = data.index(b"\n", pos)
        s = data[pos:e].decode()
        pos = e + 1
        return s

    def block(count, dtype):
        nonlocal pos
        a = np.frombuffer(data, dtype=dtype, count=count, offset=pos)
        pos += 4 * count
        assert data[pos:pos + 1] == b"\n", "block not followed by a newline"
        pos += 1
        return a

    out = {"header": [line() for _ in range(4)]}
    kw, n, _ = line().split()
    assert kw == "POINTS"
    out["points"] = block(3 * int(n), ">f4").reshape(-1, 3)
    kw, ncell, total = line().split()
    assert kw == "CELLS"
    ncell = int(ncell)
    out["cells"] = block(int(total), ">i4").reshape(ncell, -1)
    kw, n = line().split()
    assert kw == "CELL_TYPES" and int(n) == ncell
    out["cell_types"] = block(ncell, ">i4")
    kw, n = line().split()
    assert kw == "CELL_DATA" and int(n) == ncell
    fields = []
    while pos < len(data):
        kw, name, typ = line().split()
        assert kw == "SCALARS"
        assert line() == "LOOKUP_TABLE default"
        fields.append((name, block(ncell, ">i4" if typ == "int" else ">f4")))
    out["fields"] = fields
    return out

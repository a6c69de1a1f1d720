"""VTK XML output of device results: the file side of neon's post-processing.

neon writes, per output step, an unstructured grid (``vtkXMLUnstructuredGridWriter``) with the
mesh, the nodal displacement and the requested internal variables averaged to the nodes, and
keeps a ``.pvd`` collection that maps time steps to files (io/file_output.cpp:49-180, fields from
mesh/mechanics/solid/mesh.cpp:174-214, node order from node_ordering_adapter.cpp:236-244).
This module writes the same two file kinds as plain XML (ASCII data arrays) -- no VTK library and
no rendering: the nodal values come from ``SolidMesh.nodal_averaged`` on the device.
"""
from __future__ import annotations

import os
from xml.sax.saxutils import quoteattr

import numpy as np

# VTK cell types of the element topologies on the path
VTK_TETRA, VTK_HEXAHEDRON = 10, 12


def vtk_connectivity(conn: np.ndarray) -> np.ndarray:
    """neon's local node order -> VTK's (convert_to_vtk: tet4 swaps its first two nodes; hex8
    corners are already in VTK order)."""
    conn = np.asarray(conn)
    if conn.shape[1] == 4:
        return conn[:, [1, 0, 2, 3]]
    if conn.shape[1] == 8:
        return conn
    raise ValueError("only tet4 and hex8 elements are written")


def _array(name, values, components, vtk_type="Float64"):
    flat = np.asarray(values).reshape(-1)
    fmt = "%.17g" if vtk_type == "Float64" else "%d"
    body = " ".join(fmt % v for v in flat)
    head = f'<DataArray type="{vtk_type}" Name={quoteattr(name)}'
    if components > 1:
        head += f' NumberOfComponents="{components}"'
    return f'{head} format="ascii">{body}</DataArray>'


def write_vtu(path: str, X: np.ndarray, conn: np.ndarray, point_data: dict | None = None):
    """One unstructured grid: points X [N][3], cells conn [E][4 or 8] (neon order), point arrays
    name -> [N] or [N][k]."""
    X = np.asarray(X, dtype=np.float64)
    cells = vtk_connectivity(conn).astype(np.int64)
    E, npe = cells.shape
    ctype = VTK_TETRA if npe == 4 else VTK_HEXAHEDRON
    parts = ['<?xml version="1.0"?>',
             '<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian">',
             "<UnstructuredGrid>",
             f'<Piece NumberOfPoints="{X.shape[0]}" NumberOfCells="{E}">',
             "<PointData>"]
    for name, values in (point_data or {}).items():
        v = np.asarray(values, dtype=np.float64)
        if v.shape[0] != X.shape[0]:
            raise ValueError(f"point array {name} has {v.shape[0]} rows for {X.shape[0]} points")
        parts.append(_array(name, v, 1 if v.ndim == 1 else v.shape[1]))
    parts += ["</PointData>", "<Points>", _array("Points", X, 3), "</Points>", "<Cells>",
              _array("connectivity", cells, 1, "Int64"),
              _array("offsets", npe * np.arange(1, E + 1), 1, "Int64"),
              _array("types", np.full(E, ctype), 1, "UInt8"),
              "</Cells>", "</Piece>", "</UnstructuredGrid>", "</VTKFile>"]
    with open(path, "w") as fh:
        fh.write("\n".join(parts) + "\n")


class VtkOutput:
    """neon's vtk_file_output: files ``<directory>/<name>_<step>.vtu`` and the collection
    ``<name>.pvd`` written every ``write_every`` steps with the requested ``fields`` (any of
    "displacement" and the names of ``SolidMesh.NODAL``)."""

    directory = "visualisation"

    def __init__(self, name: str, fields, write_every: int = 1, root: str = "."):
        if not name:
            raise ValueError('"name" field for file IO must be specified')
        self.name = name
        self.fields = list(fields)
        self.write_every = int(write_every)
        self.root = root
        self.entries = []
        os.makedirs(os.path.join(root, self.directory), exist_ok=True)

    def write(self, time_step: int, time: float, mesh, X, conn, displacement=None):
        """Write one step from a SolidMesh whose last update holds the state to output."""
        if time_step % self.write_every:
            return None
        data = {}
        for f in self.fields:
            if f == "displacement":
                u = mesh.displacement() if displacement is None else displacement
                data[f] = np.asarray(u).reshape(-1, 3)
            else:
                data[f] = mesh.nodal_averaged(f)
        rel = f"{self.directory}/{self.name}_{time_step}.vtu"
        write_vtu(os.path.join(self.root, rel), X, conn, data)
        self.entries.append((time, rel))
        self._write_pvd()
        return os.path.join(self.root, rel)

    def _write_pvd(self):
        lines = ['<?xml version="1.0"?>', '<VTKFile type="Collection" version="0.1">',
                 "  <Collection>"]
        lines += [f'    <DataSet timestep="{t!r}" file="{f}" />' for t, f in self.entries]
        lines += ["  </Collection>", "</VTKFile>"]
        with open(os.path.join(self.root, self.name + ".pvd"), "w") as fh:
            fh.write("\n".join(lines) + "\n")

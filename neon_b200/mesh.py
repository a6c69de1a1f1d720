"""Synthetic meshes in neon's data model.

neon reads a ``.mesh`` JSON file (``Nodes[0].Coordinates``, ``Elements[{Name, Type,
NodalConnectivity}]``; mesh/basic_mesh.cpp:8-19, mesh/nodal_coordinates.cpp:13-33) and converts
gmsh element ordering to its own local ordering (mesh/node_ordering_adapter.cpp:46-68).  The
generators here produce the same in-memory result directly:

* nodal coordinates ``X`` as ``float64[N, 3]`` (node-major, so DOF ``3*node + k`` indexes a
  flattened copy, mesh/dof_allocator.hpp:39-47),
* connectivity ``conn`` as ``int32[E, npe]`` in neon's local ordering (hex8: Hughes corner order of
  interpolations/hexahedron.cpp:21-28; tet4: gmsh (1,2,3,0)),
* named boundary node sets (faces) from which the Dirichlet DOF lists are built.
"""
from __future__ import annotations

import dataclasses
import json

import numpy as np


@dataclasses.dataclass
class Mesh:
    X: np.ndarray              # float64 [N, 3]
    conn: np.ndarray           # int32 [E, npe] (neon local ordering)
    faces: dict                # name -> int32 [F, 4] quad4 (or [F, 3] tri3) boundary faces
    shape: tuple = ()          # structured (nx, ny, nz) cells, informational

    @property
    def num_nodes(self) -> int:
        return int(self.X.shape[0])

    @property
    def num_elements(self) -> int:
        return int(self.conn.shape[0])

    @property
    def nodes_per_element(self) -> int:
        return int(self.conn.shape[1])

    def boundary_nodes(self, name: str) -> np.ndarray:
        """Sorted unique node indices of a boundary group (dof_allocator.hpp:19-37)."""
        return np.unique(self.faces[name].reshape(-1)).astype(np.int32)


def _node_id(i, j, k, nx, ny):
    return i + (nx + 1) * (j + (ny + 1) * k)


def _box_faces(nx, ny, nz):
    """quad4 faces of the six sides of a structured box, outward-facing ordering."""
    faces = {}
    I, J = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    I, J = I.ravel(), J.ravel()
    for name, k in (("bottom", 0), ("top", nz)):
        f = np.stack([_node_id(I, J, k, nx, ny), _node_id(I + 1, J, k, nx, ny),
                      _node_id(I + 1, J + 1, k, nx, ny), _node_id(I, J + 1, k, nx, ny)], axis=1)
        faces[name] = f if name == "top" else f[:, ::-1]
    J, K = np.meshgrid(np.arange(ny), np.arange(nz), indexing="ij")
    J, K = J.ravel(), K.ravel()
    for name, i in (("x0", 0), ("x1", nx)):
        f = np.stack([_node_id(i, J, K, nx, ny), _node_id(i, J + 1, K, nx, ny),
                      _node_id(i, J + 1, K + 1, nx, ny), _node_id(i, J, K + 1, nx, ny)], axis=1)
        faces[name] = f if name == "x1" else f[:, ::-1]
    I, K = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    I, K = I.ravel(), K.ravel()
    for name, j in (("y0", 0), ("y1", ny)):
        f = np.stack([_node_id(I, j, K, nx, ny), _node_id(I, j, K + 1, nx, ny),
                      _node_id(I + 1, j, K + 1, nx, ny), _node_id(I + 1, j, K, nx, ny)], axis=1)
        faces[name] = f if name == "y1" else f[:, ::-1]
    return {k: v.astype(np.int32) for k, v in faces.items()}


def structured_hex8(nx: int, ny: int | None = None, nz: int | None = None,
                    size=(1.0, 1.0, 1.0), jitter: float = 0.0, seed: int | None = None) -> Mesh:
    """Box [0,Lx]x[0,Ly]x[0,Lz] split into nx*ny*nz hex8 cells.

    Nodes are numbered i fastest, then j, then k.  ``jitter`` perturbs every *interior* node
    coordinate by U(-jitter*h, +jitter*h) per component (numpy PCG64 with ``seed``), so the
    faces stay planar and the symmetry boundary conditions stay exact.
    """
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    xs = np.linspace(0.0, size[0], nx + 1)
    ys = np.linspace(0.0, size[1], ny + 1)
    zs = np.linspace(0.0, size[2], nz + 1)
    Z, Y, Xg = np.meshgrid(zs, ys, xs, indexing="ij")
    X = np.stack([Xg.ravel(), Y.ravel(), Z.ravel()], axis=1).astype(np.float64)
    if jitter > 0.0:
        rng = np.random.Generator(np.random.PCG64(seed))
        h = np.array([size[0] / nx, size[1] / ny, size[2] / nz])
        k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1),
                              indexing="ij")
        interior = ((i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)).ravel()
        d = rng.uniform(-jitter, jitter, size=(int(interior.sum()), 3)) * h
        X[interior] += d
    K, J, I = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    n = lambda a, b, c: _node_id(I + a, J + b, K + c, nx, ny)  # noqa: E731
    conn = np.stack([n(0, 0, 0), n(1, 0, 0), n(1, 1, 0), n(0, 1, 0),
                     n(0, 0, 1), n(1, 0, 1), n(1, 1, 1), n(0, 1, 1)], axis=1).astype(np.int32)
    return Mesh(X=X, conn=conn, faces=_box_faces(nx, ny, nz), shape=(nx, ny, nz))


# Six tetrahedra around the cube diagonal 0-6 (corner numbering of the hex8 above).  Every cube
# uses the same diagonal, so neighbouring cubes split their shared faces identically.
_KUHN = ((0, 1, 2, 6), (0, 2, 3, 6), (0, 3, 7, 6), (0, 7, 4, 6), (0, 4, 5, 6), (0, 5, 1, 6))


def structured_tet4(nx: int, ny: int | None = None, nz: int | None = None,
                    size=(1.0, 1.0, 1.0)) -> Mesh:
    """Box split into nx*ny*nz cubes of 6 tet4 each (conforming), neon local tet4 ordering.

    neon's tet4 shape functions are N = (r, s, t, 1-r-s-t) (interpolations/tetrahedron.cpp:6-45),
    so the local Jacobian columns are x0-x3, x1-x3, x2-x3; nodes are ordered so that it is
    positive.
    """
    hexm = structured_hex8(nx, ny, nz, size=size)
    tets = np.concatenate([hexm.conn[:, list(t)] for t in _KUHN], axis=0)
    # cell-major ordering: all 6 tets of cell 0, then cell 1, ...
    E = hexm.conn.shape[0]
    tets = tets.reshape(6, E, 4).transpose(1, 0, 2).reshape(-1, 4)
    X = hexm.X
    a = X[tets[:, 0]] - X[tets[:, 3]]
    b = X[tets[:, 1]] - X[tets[:, 3]]
    c = X[tets[:, 2]] - X[tets[:, 3]]
    det = np.einsum("ij,ij->i", a, np.cross(b, c))
    neg = det < 0
    tets[neg, 0], tets[neg, 1] = tets[neg, 1].copy(), tets[neg, 0].copy()
    faces = {}
    for name, q in hexm.faces.items():
        faces[name] = q  # quad4 node sets are enough for Dirichlet DOF lists
    return Mesh(X=X, conn=tets.astype(np.int32), faces=faces, shape=(nx, ny, nz))


# gmsh element type codes (mesh/element_topology.hpp:9-46)
_GMSH_NPE = {5: 8, 4: 4, 3: 4, 2: 3}


def convert_from_gmsh(conn: np.ndarray, gmsh_type: int) -> np.ndarray:
    """neon's gmsh->local reordering (node_ordering_adapter.cpp:46-68): tet4 -> (1,2,3,0)."""
    if gmsh_type == 4:
        return conn[:, [1, 2, 3, 0]]
    return conn


def read_neon_mesh(path: str, part: str) -> Mesh:
    """Read a neon ``.mesh`` JSON file (basic_mesh.cpp:8-19, basic_submesh.cpp:12-53).

    The volume group named ``part`` becomes the element list; every other group is a boundary.
    """
    with open(path) as fh:
        data = json.load(fh)
    X = np.asarray(data["Nodes"][0]["Coordinates"], dtype=np.float64)
    conn = None
    faces = {}
    for group in data["Elements"]:
        c = np.asarray(group["NodalConnectivity"], dtype=np.int32)
        c = convert_from_gmsh(c, int(group["Type"]))
        if group["Name"] == part:
            conn = c if conn is None else np.concatenate([conn, c])
        else:
            faces[group["Name"]] = c if group["Name"] not in faces else np.concatenate(
                [faces[group["Name"]], c])
    if conn is None:
        raise ValueError(f"part {part!r} not found in {path}")
    return Mesh(X=X, conn=conn.astype(np.int32), faces=faces)


def quad4_consistent_forces(mesh: Mesh, face: str, traction) -> tuple[np.ndarray, np.ndarray]:
    """Consistent nodal forces of a uniform traction on quad4 faces (2x2 Gauss).

    Restates neon's non-follower surface load (mesh/boundary/neumann.hpp:69-133) for a constant
    traction vector: f_a = sum_l N_a(l) t |J_s(l)| w_l.  Returns (dofs, values).
    """
    q = mesh.faces[face]
    g = 1.0 / np.sqrt(3.0)
    pts = [(-g, -g), (g, -g), (g, g), (-g, g)]
    t = np.asarray(traction, dtype=np.float64)
    f = np.zeros((mesh.num_nodes, 3))
    Xf = mesh.X[q]  # [F, 4, 3]
    for xi, eta in pts:
        N = 0.25 * np.array([(1 - xi) * (1 - eta), (1 + xi) * (1 - eta),
                             (1 + xi) * (1 + eta), (1 - xi) * (1 + eta)])
        dxi = 0.25 * np.array([-(1 - eta), (1 - eta), (1 + eta), -(1 + eta)])
        deta = 0.25 * np.array([-(1 - xi), -(1 + xi), (1 + xi), (1 - xi)])
        a = np.einsum("a,fak->fk", dxi, Xf)
        b = np.einsum("a,fak->fk", deta, Xf)
        jac = np.linalg.norm(np.cross(a, b), axis=1)
        for k in range(4):
            np.add.at(f, q[:, k], (N[k] * jac)[:, None] * t[None, :])
    nodes = np.unique(q.reshape(-1))
    dofs, vals = [], []
    for comp in range(3):
        if t[comp] != 0.0:
            dofs.append(3 * nodes + comp)
            vals.append(f[nodes, comp])
    if not dofs:
        return np.zeros(0, np.int32), np.zeros(0)
    return np.concatenate(dofs).astype(np.int32), np.concatenate(vals)

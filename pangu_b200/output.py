"""Output of a job's primitive fields for analysis and visualisation tools.

The reference writes Parthenon ``.phdf`` files (HDF5) with an ``.xdmf``
description. Its analysis script reads, per field, the dataset named after
the primitive field as [block][k][j][i] over the interior cells, the cell
centres ``VolumeLocations/{x,y,z}`` as [block][i] (and j, k) and the block
lattice ``LogicalLocations`` as [block][3] (scripts/python/xzplot.py:35-58).

* ``write_xdmf`` writes those arrays as one raw little-endian binary file
  described by an XDMF file (one rectilinear grid per block, cell-centred
  attributes), which ParaView and VisIt read without HDF5.
* ``write_phdf`` writes the ``.phdf`` layout itself through h5py, where that
  package is installed (it is not a dependency of the engine).

Vector fields (weighted_velocity, magnetic_field) are [block][3][k][j][i].
"""
from __future__ import annotations

import os
import xml.etree.ElementTree as ET

import numpy as np

from . import abi
from .params import primitive_field_names


def _components(name: str) -> int:
    return 3 if name in ("weighted_velocity", "magnetic_field") else 1


def _geometry(mesh: abi.Mesh):
    from .problems import Geometry
    return Geometry(mesh)


def interior_fields(prim: np.ndarray, mesh: abi.Mesh, enable_B: bool,
                    enable_heating: bool) -> dict[str, np.ndarray]:
    """The primitive fields of prim ([block][var][k][j][i] with ghosts) over
    the interior cells: scalars [block][k][j][i], vectors [block][3][k][j][i]."""
    geo = _geometry(mesh)
    s = geo.interior()
    out, v = {}, 0
    for name in primitive_field_names(enable_B, enable_heating):
        n = _components(name)
        a = np.ascontiguousarray(prim[:, v:v + n, s[0], s[1], s[2]], dtype=np.float64)
        out[name] = a[:, 0] if n == 1 else a
        v += n
    return out


def block_locations(mesh: abi.Mesh):
    """Per block: cell-centre and face coordinates along x1, x2, x3 (interior
    only) and the lattice position (b1, b2, b3)."""
    geo = _geometry(mesh)
    nb = geo.nb
    centres, faces = [[], [], []], [[], [], []]
    for b in range(nb):
        for d in range(3):
            st, n = geo.start[d], geo.nx[d]
            xc = geo.xc(b, d)[st:st + n]
            o = geo.origin(b, d) + st * geo.dx[d]
            xf = o + np.arange(n + 1, dtype=np.float64) * geo.dx[d]
            centres[d].append(xc)
            faces[d].append(xf)
    lattice = np.array([geo.block_lattice(b) for b in range(nb)], dtype=np.int64)
    return ([np.array(c) for c in centres], [np.array(f) for f in faces], lattice)


def write_xdmf(prefix: str, prim: np.ndarray, mesh: abi.Mesh, enable_B: bool,
               enable_heating: bool, cycle: int = 0, time: float = 0.0) -> str:
    """Writes <prefix>.xdmf and <prefix>.bin; returns the .xdmf path."""
    fields = interior_fields(prim, mesh, enable_B, enable_heating)
    _, faces, _ = block_locations(mesh)
    nb = prim.shape[0]
    nx = [mesh.nx1, mesh.nx2, mesh.nx3]
    binpath = prefix + ".bin"
    binname = os.path.basename(binpath)
    root = ET.Element("Xdmf", Version="3.0")
    dom = ET.SubElement(root, "Domain")
    coll = ET.SubElement(dom, "Grid", Name="mesh", GridType="Collection",
                         CollectionType="Spatial")
    ET.SubElement(coll, "Time", Value=repr(float(time)))
    ET.SubElement(coll, "Information", Name="NCycle", Value=str(int(cycle)))
    offset = 0
    with open(binpath, "wb") as fb:
        def item(parent, arr, dims):
            nonlocal offset
            a = np.ascontiguousarray(arr, dtype="<f8")
            fb.write(a.tobytes())
            el = ET.SubElement(parent, "DataItem", Format="Binary", NumberType="Float",
                               Precision="8", Endian="Little", Seek=str(offset),
                               Dimensions=dims)
            el.text = binname
            offset += a.nbytes
        for b in range(nb):
            g = ET.SubElement(coll, "Grid", Name=f"block{b}", GridType="Uniform")
            ET.SubElement(g, "Topology", TopologyType="3DRectMesh",
                          Dimensions=f"{nx[2] + 1} {nx[1] + 1} {nx[0] + 1}")
            geo = ET.SubElement(g, "Geometry", GeometryType="VXVYVZ")
            for d in range(3):
                item(geo, faces[d][b], str(nx[d] + 1))
            for name, a in fields.items():
                if a.ndim == 4:
                    at = ET.SubElement(g, "Attribute", Name=name, AttributeType="Scalar",
                                       Center="Cell")
                    item(at, a[b], f"{nx[2]} {nx[1]} {nx[0]}")
                else:
                    for c in range(a.shape[1]):
                        at = ET.SubElement(g, "Attribute", Name=f"{name}_{c + 1}",
                                           AttributeType="Scalar", Center="Cell")
                        item(at, a[b, c], f"{nx[2]} {nx[1]} {nx[0]}")
    ET.ElementTree(root).write(prefix + ".xdmf", encoding="unicode", xml_declaration=True)
    return prefix + ".xdmf"


def write_phdf(path: str, prim: np.ndarray, mesh: abi.Mesh, enable_B: bool,
               enable_heating: bool, cycle: int = 0, time: float = 0.0) -> str:
    """Writes the Parthenon .phdf layout the reference's analysis scripts read
    (field datasets, VolumeLocations, Locations, LogicalLocations, Info).
    Needs h5py."""
    try:
        import h5py
    except ImportError as exc:  # h5py is optional
        raise ImportError("write_phdf needs h5py; write_xdmf needs nothing") from exc
    fields = interior_fields(prim, mesh, enable_B, enable_heating)
    centres, faces, lattice = block_locations(mesh)
    with h5py.File(path, "w") as h:
        for name, a in fields.items():
            h.create_dataset(name, data=a)
        vol, loc = h.create_group("VolumeLocations"), h.create_group("Locations")
        for d, axis in enumerate("xyz"):
            vol.create_dataset(axis, data=centres[d])
            loc.create_dataset(axis, data=faces[d])
        h.create_dataset("LogicalLocations", data=lattice)
        info = h.create_group("Info")
        info.attrs["NumMeshBlocks"] = prim.shape[0]
        info.attrs["MeshBlockSize"] = np.array([mesh.nx1, mesh.nx2, mesh.nx3], dtype=np.int64)
        info.attrs["NCycle"] = int(cycle)
        info.attrs["Time"] = float(time)
        info.attrs["OutputFormatVersion"] = -1  # not produced by Parthenon
    return path

"""Output files on CPU: the XDMF + raw binary description of a job's
primitives reads back to the interior cells of every block, and the .phdf
layout (written through a stand-in for h5py, which is not installed here)
holds the datasets the reference's analysis script reads, with the shapes it
expects: a global map assembled from the blocks by their lattice positions
equals the mesh's interior field."""
import sys
import types
import xml.etree.ElementTree as ET

import numpy as np

from pangu_b200 import output
from pangu_b200 import params as prm
from pangu_b200 import problems


def _state(**kw):
    pin, gen = problems.make_problem("torus", **kw)
    mesh = prm.mesh_struct(pin)
    pk = prm.process_packages(pin)
    prim = gen(problems.Geometry(mesh), pk, pin)
    return mesh, prim


def test_xdmf_reads_back(tmp_path):
    mesh, prim = _state(nx1=32, nx2=16, nx3=4, bx=(16, 8, 4))
    path = output.write_xdmf(str(tmp_path / "out"), prim, mesh, True, True, cycle=7, time=1.5)
    fields = output.interior_fields(prim, mesh, True, True)
    raw = open(str(tmp_path / "out.bin"), "rb").read()
    root = ET.parse(path).getroot()
    grids = root.find("Domain").find("Grid").findall("Grid")
    assert len(grids) == prim.shape[0]
    for b, g in enumerate(grids):
        for at in g.findall("Attribute"):
            di = at.find("DataItem")
            dims = [int(x) for x in di.get("Dimensions").split()]
            n = int(np.prod(dims))
            a = np.frombuffer(raw, dtype="<f8", count=n, offset=int(di.get("Seek"))).reshape(dims)
            name = at.get("Name")
            if name in fields:
                np.testing.assert_array_equal(a, fields[name][b])
            else:
                base, c = name.rsplit("_", 1)
                np.testing.assert_array_equal(a, fields[base][b, int(c) - 1])
        xs = g.find("Geometry").findall("DataItem")
        assert [int(x.get("Dimensions")) for x in xs] == [mesh.nx1 + 1, mesh.nx2 + 1, mesh.nx3 + 1]


class _FakeH5:
    """Records what write_phdf stores (the h5py calls it makes)."""

    def __init__(self, store, prefix=""):
        self.store, self.prefix, self.attrs = store, prefix, {}

    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False

    def create_dataset(self, name, data):
        self.store[self.prefix + name] = np.array(data)

    def create_group(self, name):
        g = _FakeH5(self.store, self.prefix + name + "/")
        self.store[self.prefix + name + "/@attrs"] = g.attrs
        return g


def test_phdf_layout_matches_the_analysis_script(monkeypatch, tmp_path):
    store = {}
    fake = types.ModuleType("h5py")
    fake.File = lambda path, mode: _FakeH5(store)
    monkeypatch.setitem(sys.modules, "h5py", fake)
    mesh, prim = _state(nx1=64, nx2=32, bx=(16, 16, 1))
    output.write_phdf(str(tmp_path / "x.phdf"), prim, mesh, True, True, cycle=3)
    nb = prim.shape[0]
    rho = store["density"]
    assert rho.shape == (nb, 1, 16, 16)  # (nb, nz, ny, nx)
    assert store["weighted_velocity"].shape == (nb, 3, 1, 16, 16)
    assert store["VolumeLocations/x"].shape == (nb, 16)
    assert store["VolumeLocations/y"].shape == (nb, 16)
    ll = store["LogicalLocations"]
    assert ll.shape == (nb, 3)
    # the analysis script's assembly (xzplot.py:45-70): blocks placed by lattice position
    nbx, nby = int(ll[:, 0].max()) + 1, int(ll[:, 1].max()) + 1
    glob = np.zeros((nby * 16, nbx * 16))
    for b in range(nb):
        bx, by = ll[b, 0], ll[b, 1]
        glob[by * 16:(by + 1) * 16, bx * 16:(bx + 1) * 16] = rho[b].mean(axis=0)
    geo = problems.Geometry(mesh)
    s = geo.interior()
    want = np.zeros_like(glob)
    for b in range(nb):
        bx, by, _ = geo.block_lattice(b)
        want[by * 16:(by + 1) * 16, bx * 16:(bx + 1) * 16] = prim[b, 0, s[0], s[1], s[2]][0]
    np.testing.assert_array_equal(glob, want)
    x = np.concatenate([store["VolumeLocations/x"][b] for b in range(nb) if ll[b, 1] == 0])
    assert np.all(np.diff(x) > 0)
    assert store["Info/@attrs"]["NCycle"] == 3

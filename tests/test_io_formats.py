"""The file formats of the reference's input and output path, read and written
without vtk or h5py (mpmwarpydw_b200.vtkio, mpmwarpydw_b200.hdf5io,
utils.fs5PlotUtils):

* tests/golden/block_particles.h5 and block_particles.vtp are the reference's
  example domain (exampleDomains/), unmodified: the same 100,000-particle block
  written by h5py and by VTK.  Each reader decodes its file, and the two agree
  on every coordinate (two independent formats and parsers).
* The writer's VTP/VTI files read back exactly; so do the inline-ascii and
  appended (raw and base64) encodings VTK also writes.
* A checkpoint written by save_grid_and_particles_vti_vtp comes back from
  load_restart_from_vtp with the reference's keys and defaults.
"""
import base64
import os
import zlib

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_reference_example_domain_hdf5_and_vtp_agree():
    from mpmwarpydw_b200 import hdf5io, vtkio
    f = hdf5io.HDF5File(os.path.join(HERE, "block_particles.h5"))
    assert sorted(f.keys()) == ["particle_volume", "x"]
    x = f["x"]
    vol = f["particle_volume"]
    assert x.shape == (3, 100000) and x.dtype == np.float64
    assert vol.shape == (100000,) and vol.dtype == np.int64 and (vol == 1).all()
    v = vtkio.read_vtp(os.path.join(HERE, "block_particles.vtp"))
    assert v["points"].shape == (100000, 3) and v["points"].dtype == np.float64
    assert np.array_equal(v["points"], x.T)
    assert np.array_equal(v["point_data"]["volume"], vol)
    assert float(x.min()) == 25.0 and float(x.max()) == 124.5
    with pytest.raises(KeyError):
        f["E"]


def test_driver_loads_the_reference_hdf5_domain():
    from mpmwarpydw_b200.runMPMYDW import load_domain
    x, vol, props, over, dom = load_domain(os.path.join(HERE, "block_particles.h5"), None)
    assert x.shape == (100000, 3) and x.dtype == np.float32 and vol.shape == (100000,)
    assert props == {} and dom is None


def test_vtp_vti_round_trip(tmp_path):
    from mpmwarpydw_b200 import vtkio
    rng = np.random.default_rng(0)
    n = 70_001                                   # several zlib blocks, a partial last one
    pts = rng.normal(size=(n, 3)).astype(np.float32)
    pd = {"radius": rng.random(n).astype(np.float32), "velocity": rng.normal(size=(n, 3)).astype(np.float32),
          "stress_tensor": rng.normal(size=(n, 6)).astype(np.float32),
          "material_label": rng.integers(0, 3, n).astype(np.int32), "ids": np.arange(n, dtype=np.int64)}
    fd = {"sim_time": np.array([0.25], np.float32), "bigStep": np.array([3.0], np.float32)}
    p = str(tmp_path / "a.vtp")
    vtkio.write_vtp(p, pts, pd, fd)
    r = vtkio.read_vtp(p)
    assert np.array_equal(r["points"], pts)
    for k, a in pd.items():
        assert r["point_data"][k].dtype == a.dtype and np.array_equal(r["point_data"][k], a), k
    assert float(r["field_data"]["sim_time"][0]) == 0.25 and float(r["field_data"]["bigStep"][0]) == 3.0
    g = rng.random((7, 5, 3)).astype(np.float32)
    q = str(tmp_path / "g.vti")
    vtkio.write_vti(q, g.shape, (1.0, -2.0, 0.5), 0.25, {"grid_mass": g})
    gr = vtkio.read_vti(q)
    assert gr["dims"] == (7, 5, 3) and np.allclose(gr["origin"], [1.0, -2.0, 0.5]) and np.allclose(gr["spacing"], 0.25)
    assert np.array_equal(gr["point_data"]["grid_mass"], g)


def _payload(a, compressed, header=np.uint32):
    raw = a.tobytes()
    if not compressed:
        return np.array([len(raw)], header).tobytes() + raw, None
    blocks = [raw[i:i + 1000] for i in range(0, len(raw), 1000)]
    comp = [zlib.compress(b) for b in blocks]
    head = np.array([len(blocks), 1000, len(blocks[-1])] + [len(c) for c in comp], header).tobytes()
    return head, b"".join(comp)


@pytest.mark.parametrize("mode", ["ascii", "appended-raw", "appended-base64", "appended-raw-zlib",
                                  "binary-uint64", "binary-uncompressed"])
def test_vtp_reader_encodings(tmp_path, mode):
    """The other encodings VTK writes: ascii, appended raw / base64 (with and
    without zlib), UInt64 headers, uncompressed inline binary."""
    from mpmwarpydw_b200 import vtkio
    rng = np.random.default_rng(1)
    n = 1234
    pts = rng.normal(size=(n, 3)).astype(np.float64)
    rad = rng.random(n).astype(np.float32)
    compressed = mode in ("appended-raw-zlib", "binary-uint64")
    header = np.uint64 if mode == "binary-uint64" else np.uint32
    comp_attr = ' compressor="vtkZLibDataCompressor"' if compressed else ""
    htype = "UInt64" if header is np.uint64 else "UInt32"
    top = f'<?xml version="1.0"?>\n<VTKFile type="PolyData" version="1.0" byte_order="LittleEndian" header_type="{htype}"{comp_attr}>\n'
    piece = f'<PolyData><Piece NumberOfPoints="{n}" NumberOfVerts="0" NumberOfLines="0" NumberOfStrips="0" NumberOfPolys="0">'
    if mode == "ascii":
        body = (f'<PointData><DataArray type="Float32" Name="radius" format="ascii">{" ".join(map(repr, rad.tolist()))}'
                f'</DataArray></PointData><Points><DataArray type="Float64" Name="Points" NumberOfComponents="3" '
                f'format="ascii">{" ".join(map(repr, pts.ravel().tolist()))}</DataArray></Points>')
        xml = (top + piece + body + "</Piece></PolyData></VTKFile>").encode()
    elif mode.startswith("binary"):
        def inline(a):
            h, c = _payload(a, compressed, header)
            return base64.b64encode(h).decode() + (base64.b64encode(c).decode() if c is not None else "")
        body = (f'<PointData><DataArray type="Float32" Name="radius" format="binary">{inline(rad)}</DataArray>'
                f'</PointData><Points><DataArray type="Float64" Name="Points" NumberOfComponents="3" format="binary">'
                f'{inline(pts)}</DataArray></Points>')
        xml = (top + piece + body + "</Piece></PolyData></VTKFile>").encode()
    else:
        enc = "base64" if mode == "appended-base64" else "raw"
        chunks, offs, off = [], [], 0
        for a in (rad, pts):
            h, c = _payload(a, compressed, header)
            blob = h + (c or b"")
            blob = base64.b64encode(blob) if enc == "base64" else blob
            offs.append(off)
            chunks.append(blob)
            off += len(blob)
        body = (f'<PointData><DataArray type="Float32" Name="radius" format="appended" offset="{offs[0]}"/></PointData>'
                f'<Points><DataArray type="Float64" Name="Points" NumberOfComponents="3" format="appended" '
                f'offset="{offs[1]}"/></Points>')
        xml = (top + piece + body + "</Piece></PolyData>").encode() + \
            f'<AppendedData encoding="{enc}">\n   _'.encode() + b"".join(chunks) + b"\n</AppendedData>\n</VTKFile>\n"
    p = tmp_path / "e.vtp"
    p.write_bytes(xml)
    r = __import__("mpmwarpydw_b200.vtkio", fromlist=["read_vtp"]).read_vtp(str(p))
    assert np.array_equal(r["points"], pts)
    assert np.array_equal(r["point_data"]["radius"], rad)


def test_checkpoint_round_trip(tmp_path):
    """save_grid_and_particles_vti_vtp with restart data, then
    load_restart_from_vtp: every restart array comes back (FP32), the stress
    tensor rebuilt symmetric from its 6 components, the field data restored."""
    from mpmwarpydw_b200.utils import fs5PlotUtils as P
    rng = np.random.default_rng(2)
    n = 5000
    f = lambda *s: rng.normal(size=(n,) + s).astype(np.float32)  # noqa: E731
    sig = f(3, 3)
    sig = 0.5 * (sig + sig.transpose(0, 2, 1))
    rd = {"sim_time": 1.25, "bigStep": 2, "dx": 0.5, "particle_F": f(3, 3), "particle_C": f(3, 3),
          "particle_accumulated_strain": f(), "ys_base": f(), "particle_vol": f(), "particle_mass": f(),
          "particle_density": f(), "particle_x_initial_xpbd": f(3), "particle_cumDist_xpbd": f()}
    for p in P.MATERIAL_PROPERTIES:
        rd[p] = f()
    x, v, r, ys, dmg = f(3), f(3), f(), f(), f()
    ml = rng.integers(0, 3, n).astype(np.int32)
    al = rng.integers(0, 2, n).astype(np.int32)
    path = P.save_grid_and_particles_vti_vtp(str(tmp_path / "out" / "sim_step_x"), np.ones((4, 5, 6), np.float32),
                                             (0, 0, 0), 0.5, x, r, v, ys, ys, dmg, dmg, dmg, sig, al, ml, rd)
    assert os.path.exists(str(tmp_path / "out" / "sim_step_x_grid.vti"))
    back = P.load_restart_from_vtp(path)
    assert np.array_equal(back["particle_x"], x) and np.array_equal(back["particle_v"], v)
    assert np.array_equal(back["particle_radius"], r) and np.array_equal(back["ys"], ys)
    assert np.array_equal(back["particle_damage"], dmg)
    assert np.array_equal(back["materialLabel"], ml) and np.array_equal(back["activeLabel"], al)
    assert np.array_equal(back["particle_stress"], sig)
    for k in ("particle_F", "particle_C", "particle_accumulated_strain", "ys_base", "particle_vol", "particle_mass",
              "particle_density", "particle_x_initial_xpbd", "particle_cumDist_xpbd", *P.MATERIAL_PROPERTIES):
        assert np.array_equal(back[k], rd[k]), k
    assert back["sim_time"] == 1.25 and back["bigStep"] == 2 and back["dx"] == 0.5

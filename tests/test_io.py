"""Headless particle export (VTK XML .vtu / .pvd) and checkpoint-file checks
that need no GPU: the files written by the library parse back to the
particle arrays given, with dead particles left out."""
import os
import re
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import amk

VTK_TYPES = {"Float64": np.float64, "Int64": np.int64, "Int32": np.int32, "UInt32": np.uint32, "UInt8": np.uint8}


def read_vtu(path):
    """Arrays of a .vtu written by amk_write_vtu (ASCII or appended raw)."""
    raw = open(path, "rb").read()
    head, sep, tail = raw.partition(b"<AppendedData encoding=\"raw\">\n_")
    xml_text = head.decode() + ("</VTKFile>\n" if sep else "")
    if sep:
        xml_text = xml_text.replace("</VTKFile>\n</VTKFile>", "</VTKFile>")
    root = ET.fromstring(xml_text if sep else raw.decode())
    out = {}
    for da in root.iter("DataArray"):
        name = da.get("Name") or "Points"
        dt = VTK_TYPES[da.get("type")]
        comps = int(da.get("NumberOfComponents", "1"))
        if da.get("format") == "appended":
            off = int(da.get("offset"))
            n = int(np.frombuffer(tail[off:off + 8], np.uint64)[0])
            arr = np.frombuffer(tail[off + 8:off + 8 + n], dt)
        else:
            arr = np.array(da.text.split(), dtype=dt)
        out[name] = arr.reshape(-1, comps) if comps > 1 else arr
    piece = root.find(".//Piece")
    out["_n"] = int(piece.get("NumberOfPoints"))
    out["_time"] = float(root.find(".//FieldData/DataArray").text)
    return out


@pytest.mark.parametrize("binary", [True, False])
def test_write_vtu_round_trip(tmp_path, binary):
    rng = np.random.default_rng(1)
    n = 257
    x, y, z = rng.normal(0, 1e-4, (3, n))
    vx, vy, vz = rng.normal(0, 1e3, (3, n))
    sp = rng.integers(0, 5, n).astype(np.uint8)
    alive = (rng.random(n) < 0.8).astype(np.uint8)
    ids = np.arange(n, dtype=np.uint32) * 3
    path = str(tmp_path / "p.vtu")
    amk.write_vtu(path, x, y, z, sp, vx, vy, vz, alive=alive, ids=ids, time=1.25e-9, binary=binary)
    d = read_vtu(path)
    live = alive.astype(bool)
    m = int(live.sum())
    assert d["_n"] == m and d["_time"] == 1.25e-9
    assert np.array_equal(d["Points"], np.stack([x, y, z], 1)[live])
    assert np.array_equal(d["velocity"], np.stack([vx, vy, vz], 1)[live])
    assert np.array_equal(d["species_id"], sp[live].astype(np.int32))
    assert np.array_equal(d["id"], ids[live])
    assert np.array_equal(d["connectivity"], np.arange(m)) and np.array_equal(d["offsets"], np.arange(1, m + 1))
    assert np.all(d["types"] == 1)  # VTK_VERTEX


def test_write_pvd_lists_the_series(tmp_path):
    path = str(tmp_path / "s.pvd")
    amk.write_pvd(path, ["a_0.vtu", "a_10.vtu"], [0.0, 1e-10])
    root = ET.parse(path).getroot()
    ds = root.findall(".//DataSet")
    assert [d.get("file") for d in ds] == ["a_0.vtu", "a_10.vtu"]
    assert [float(d.get("timestep")) for d in ds] == [0.0, 1e-10]


def test_checkpoint_info_rejects_foreign_and_missing_files(tmp_path):
    bad = tmp_path / "x.ckpt"
    bad.write_bytes(b"not a checkpoint at all")
    with pytest.raises(amk.AmkError):
        amk.checkpoint_info(str(bad))
    with pytest.raises(amk.AmkError):
        amk.checkpoint_info(str(tmp_path / "missing.ckpt"))
    assert "checkpoint" in amk.lib().amk_last_error().decode()

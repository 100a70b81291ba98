"""The HDF5 writer behind light.h5 and events.h5: the lookup3 checksum against
its published self-test values, the encodings against the format
specification, and the reference's file layouts (dataset names, Julia
column-major shapes, dtypes, root attributes) written and read back.  No GPU."""
import os
import struct

import numpy as np
import pytest

from crysplight_b200 import hdf5


def test_lookup3_known_answers():
    # the self-test values published with lookup3.c (hashlittle)
    assert hdf5.lookup3(b"") == 0xDEADBEEF
    assert hdf5.lookup3(b"", 0xDEADBEEF) == 0xBD5B7DDE
    assert hdf5.lookup3(b"Four score and seven years ago", 0) == 0x17770551
    assert hdf5.lookup3(b"Four score and seven years ago", 1) == 0xCD628161


def test_datatype_encodings():
    # IEEE little-endian float32/64, signed and unsigned integers (version 1 messages)
    assert hdf5._datatype(np.float32) == bytes.fromhex("11201f00" "04000000" "00002000" "1708" "0017" "7f000000")
    assert hdf5._datatype(np.float64) == bytes.fromhex("11203f00" "08000000" "00004000" "340b" "0034" "ff030000")
    assert hdf5._datatype(np.int16) == bytes.fromhex("10080000" "02000000" "0000" "1000")
    assert hdf5._datatype(np.uint32) == bytes.fromhex("10000000" "04000000" "0000" "2000")
    assert hdf5._datatype(None, strlen=5) == bytes.fromhex("13100000" "05000000")


def test_superblock_and_checksums(tmp_path):
    p = str(tmp_path / "a.h5")
    hdf5.write_h5(p, {"x": np.arange(10, dtype=np.int32)}, {"tag": "t"})
    buf = open(p, "rb").read()
    assert buf[:8] == b"\x89HDF\r\n\x1a\n" and buf[8] == 2 and buf[9] == 8 and buf[10] == 8
    base, ext, eof, root = struct.unpack_from("<QQQQ", buf, 12)
    assert base == 0 and ext == hdf5.UNDEF and eof == len(buf) and root == 48
    assert hdf5.lookup3(buf[:44]) == struct.unpack_from("<I", buf, 44)[0]
    assert buf[48:52] == b"OHDR"
    # corrupting one byte of an object header is detected
    bad = bytearray(buf)
    bad[60] ^= 0xFF
    q = str(tmp_path / "bad.h5")
    open(q, "wb").write(bytes(bad))
    with pytest.raises(hdf5.H5FormatError):
        hdf5.read_h5(q)


def test_julia_order_round_trip(tmp_path):
    p = str(tmp_path / "b.h5")
    n = 7
    maps = np.asfortranarray(np.random.default_rng(0).integers(0, 60000, (8, 8, n)).astype(np.uint16))
    tmin = np.full((8, 8, n), np.inf, np.float32, order="F")
    tmin[2, 3, 4] = 12.5
    xyz = np.asfortranarray(np.random.default_rng(1).uniform(0, 48, (3, n)).astype(np.float32))
    ds = {"maps": maps, "tmin_ns": tmin, "xyz1_mm": xyz, "int_type": np.array([-1, 0, 1, 2, 3, 0, 1], np.int8),
          "n_int": np.arange(n, dtype=np.int16), "npe": np.arange(n, dtype=np.int32) * 1000,
          "edep_kev": np.linspace(0, 511, n).astype(np.float32)}
    at = {"tag": "gammas_t", "n_events": np.int64(n), "seed": np.int64(11), "pde": np.float32(0.4),
          "sigma_alpha_deg": np.float64(1.3), "backend": "cuda", "nbins": np.int32(80)}
    hdf5.write_h5(p, ds, at)
    d2, a2 = hdf5.read_h5(p)
    for k, v in ds.items():
        assert d2[k].dtype == v.dtype and d2[k].shape == v.shape
        assert np.array_equal(d2[k], v), k
    assert a2["tag"] == "gammas_t" and a2["n_events"] == n and a2["pde"] == np.float32(0.4)
    assert a2["nbins"].dtype == np.int32 and a2["sigma_alpha_deg"] == 1.3
    # the dataspace lists Julia's dimensions in reverse: h5py reads maps as (n, ny, nx)
    raw_c, _ = hdf5.read_h5(p, julia_order=False)
    assert raw_c["maps"].shape == (n, 8, 8) and raw_c["xyz1_mm"].shape == (n, 3)
    assert np.array_equal(raw_c["maps"][4, 3, 2], maps[2, 3, 4])


def test_events_h5_layout(tmp_path):
    from crysplight_b200.events import EventsResult
    from crysplight_b200.shoot_gammas import INT_TYPE_KEY, events_h5_contents, load_gamma_setup
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    st = load_gamma_setup(os.path.join(root, "crysplight_b200", "runs", "gammas_csitl_50k.toml"))
    assert st.tb.nbins == 80 and abs(st.op.pde - 0.4) < 1e-7 and st.yield_per_mev == 54000
    assert st.n_events == 50000 and st.seed == 11 and st.box.L[2] == np.float32(37.2)
    n = 5
    r = EventsResult(np.full(n, 511, np.float32), np.arange(n, dtype=np.int32),
                     np.zeros((8, 8, n), np.uint16, order="F"), np.full((8, 8, n), np.inf, np.float32, order="F"),
                     np.zeros((3, n), np.float32, order="F"), np.zeros(n, np.float32),
                     np.zeros((3, n), np.float32, order="F"), np.zeros(n, np.float32), np.zeros(n, np.float32),
                     np.full(n, -1, np.int8), np.zeros(n, np.int16))
    st.n_events = n
    ds, at = events_h5_contents(st, r, "cuda")
    p = str(tmp_path / "events.h5")
    hdf5.write_h5(p, ds, at)
    d2, a2 = hdf5.read_h5(p)
    assert list(d2) == ["edep_kev", "npe", "maps", "tmin_ns", "xyz1_mm", "e1_kev", "xyz2_mm", "e2_kev",
                        "er_kev", "int_type", "n_int"]
    assert d2["maps"].dtype == np.uint16 and d2["tmin_ns"].dtype == np.float32
    assert d2["int_type"].dtype == np.int8 and d2["n_int"].dtype == np.int16 and d2["npe"].dtype == np.int32
    assert np.isinf(d2["tmin_ns"]).all()
    assert a2 == {**a2, "tag": "gammas_csitl_50k", "crystal": "csitl", "backend": "cuda",
                  "int_type_key": INT_TYPE_KEY, "tmin_nohit": "Inf"}
    assert a2["n_events"] == n and a2["seed"] == 11


def test_light_h5_from_write_output(tmp_path):
    import shutil
    from crysplight_b200.config import load_setup
    from crysplight_b200.output import write_output
    from crysplight_b200.params import Accumulator
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    runs = tmp_path / "runs"
    runs.mkdir()
    cfg = runs / "point_csitl_teflon.toml"
    shutil.copy(os.path.join(root, "crysplight_b200", "runs", "point_csitl_teflon.toml"), cfg)
    st = load_setup(str(cfg), data_dir=os.path.join(root, "crysplight_b200", "data"))
    acc = Accumulator.empty(st.grid, st.tb)
    acc.counts[1, 6, 0] = 5
    acc.first_ns[1, 6] = np.float32(0.25)
    acc.ndet = 5
    write_output(st, acc, 0.1)
    d, a = hdf5.read_h5(os.path.join(st.outdir, "light.h5"))
    assert d["counts"].shape == (8, 8, 81) and d["counts"].dtype == acc.counts.dtype
    assert d["counts"][1, 6, 0] == 5 and d["first_time_ns"][1, 6] == np.float32(0.25)
    assert a["tag"] == st.tag and a["n_photons"] == st.n_photons and a["ndet"] == 5
    assert a["crystal"] == "csitl" and a["wrap"] == "teflon" and a["finish"] == "backpainted"
    assert os.path.exists(os.path.join(st.outdir, "point_csitl_teflon.toml"))

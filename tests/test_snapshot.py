"""The snapshot file format (save_to_disk, io.rs:5-196, as a DGSNAP01 file)
written by the library's host writer and read back by deepgreen.snapshot."""
import json
import struct

import numpy as np
import pytest

from deepgreen import capi, snapshot

NAMES = ["primitives/rho", "primitives/vx", "primitives/vy", "primitives/vz", "primitives/pressure",
         "conserved/mass", "conserved/momentum_x", "conserved/momentum_y", "conserved/momentum_z",
         "conserved/energy"]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_host_writer_round_trip(tmp_path, dtype):
    rng = np.random.default_rng(3)
    shape = (6, 7, 9)
    arrays = {n: rng.standard_normal(shape).astype(dtype) for n in NAMES}
    path = tmp_path / "state.00000.dgsnap"
    snapshot.write_host(path, arrays, steps=17, attrs={"ds": 0.125, "bcs": [0, 0, 1, 1, 2, 2]})
    got = snapshot.read(path)
    assert got["meta"]["steps"] == 17 and got["meta"]["shape"] == list(shape)
    assert got["meta"]["attrs"] == {"ds": 0.125, "bcs": [0, 0, 1, 1, 2, 2]}
    assert got["meta"]["dtype"] == np.dtype(dtype).name
    for n, a in arrays.items():
        g, f = n.split("/")
        assert got[g][f].dtype == dtype and np.array_equal(got[g][f], a)
    eager = snapshot.read(path, mmap=False)
    assert np.array_equal(eager["conserved"]["energy"], arrays["conserved/energy"])


def test_layout_is_page_aligned(tmp_path):
    a = {"conserved/mass": np.arange(5 * 5 * 5, dtype=np.float32).reshape(5, 5, 5),
         "conserved/energy": np.ones((5, 5, 5), np.float32)}
    path = tmp_path / "s.dgsnap"
    snapshot.write_host(path, a)
    raw = path.read_bytes()
    assert raw[:8] == b"DGSNAP01"
    (hl,) = struct.unpack("<Q", raw[8:16])
    h = json.loads(raw[16:16 + hl])
    offs = [d["offset"] for d in h["datasets"]]
    assert all(o % 4096 == 0 for o in offs) and offs[0] == 16 + hl
    assert np.array_equal(np.frombuffer(raw[offs[0]:offs[0] + 500], np.float32), np.arange(125, dtype=np.float32))
    assert len(raw) == offs[1] + 500


def test_host_writer_rejects_bad_input(tmp_path):
    with pytest.raises(ValueError):
        snapshot.write_host(tmp_path / "x", {"a/b": np.zeros((2, 2), np.float32)})
    with pytest.raises(capi.DgError):
        snapshot.write_host(tmp_path / "no_such_dir" / "x", {"a/b": np.zeros((2, 2, 2), np.float32)})
    bad = tmp_path / "bad"
    bad.write_bytes(b"NOTASNAP" + bytes(8))
    with pytest.raises(ValueError):
        snapshot.read(bad)


def test_reader_rejects_truncated_files(tmp_path):
    a = {"conserved/mass": np.ones((4, 4, 4), np.float32), "conserved/energy": np.ones((4, 4, 4), np.float32)}
    path = tmp_path / "s.dgsnap"
    snapshot.write_host(path, a)
    raw = path.read_bytes()
    cut = tmp_path / "cut.dgsnap"
    cut.write_bytes(raw[:-10])           # last dataset short
    with pytest.raises(ValueError, match="truncated"):
        snapshot.read(cut)
    cut.write_bytes(raw[:20])            # header short
    with pytest.raises(ValueError, match="truncated"):
        snapshot.read_header(cut)

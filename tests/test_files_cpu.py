"""The reference's input files on CPU: the gen_vector array format
(evaluation/util/gen_vector.c:21-60: size_t n, int32[n]) and the CSR binary of
the BFS examples (asynchronous_bfs_thread.cu:69-84: int N, int M, row[N+1],
col[M]).  Files laid out byte by byte here (struct, as the reference's
fwrite/fread produce them on a 64-bit little-endian host) must read back; the
library's writers must produce the same bytes; malformed files are refused."""
import struct

import numpy as np
import pytest

import gtap_b200 as gt


def test_array_file_layout_and_round_trip(tmp_path):
    a = gt.gen_keys(42, 1000)
    p = tmp_path / "a.bin"
    p.write_bytes(struct.pack("<Q", len(a)) + a.astype("<i4").tobytes())
    assert np.array_equal(gt.read_array(p), a)
    q = tmp_path / "b.bin"
    gt.write_array(q, a)
    assert q.read_bytes() == p.read_bytes()
    gt.write_array(tmp_path / "e.bin", np.empty(0, np.int32))
    assert len(gt.read_array(tmp_path / "e.bin")) == 0


def test_csr_file_layout_and_round_trip(tmp_path):
    row, col = gt.gen_rmat(9, 16, 5)
    p = tmp_path / "g.csr"
    p.write_bytes(struct.pack("<ii", len(row) - 1, len(col)) + row.astype("<i4").tobytes() + col.astype("<i4").tobytes())
    r2, c2 = gt.read_csr(p)
    assert np.array_equal(r2, row) and np.array_equal(c2, col)
    q = tmp_path / "h.csr"
    gt.write_csr(q, row, col)
    assert q.read_bytes() == p.read_bytes()


def test_malformed_files_are_refused(tmp_path):
    a = np.arange(10, dtype=np.int32)
    p = tmp_path / "short.bin"
    p.write_bytes(struct.pack("<Q", 11) + a.tobytes())           # header says 11, file holds 10
    with pytest.raises(gt.GtapError):
        gt.read_array(p)
    row = np.array([0, 2, 1, 3], np.int32)                       # offsets decrease
    col = np.array([0, 1, 2], np.int32)
    bad = tmp_path / "bad.csr"
    bad.write_bytes(struct.pack("<ii", 3, 3) + row.tobytes() + col.tobytes())
    with pytest.raises(gt.GtapError):
        gt.read_csr(bad)
    row = np.array([0, 1, 2, 3], np.int32)
    col = np.array([0, 1, 7], np.int32)                          # vertex 7 of 3
    bad.write_bytes(struct.pack("<ii", 3, 3) + row.tobytes() + col.tobytes())
    with pytest.raises(gt.GtapError):
        gt.read_csr(bad)
    with pytest.raises(gt.GtapError):
        gt.read_array(tmp_path / "missing.bin")

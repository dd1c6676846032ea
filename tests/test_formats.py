"""The reference drivers' text formats (graph file and <prefix>.batch.<i>),
host only."""
import numpy as np
import pytest

import meerkat_b200 as mk


def test_graph_and_batch_round_trip(tmp_path):
    s, d, _ = mk.gen_rmat(12, 20000, seed=4)
    p = tmp_path / "g.txt"
    mk.write_edge_list(p, 4096, s, d)
    V, s2, d2 = mk.read_edge_list(p)
    assert V == 4096 and (s2 == s).all() and (d2 == d).all()
    first = p.read_text().splitlines()[:2]
    assert first[0] == "4096 20000" and first[1] == f"{s[0]} {d[0]}"
    for i in range(3):
        b = tmp_path / f"upd.batch.{i}"
        mk.write_batch(b, s[i * 100:(i + 1) * 100], d[i * 100:(i + 1) * 100])
        bs, bd = mk.read_batch(b)
        assert (bs == s[i * 100:(i + 1) * 100]).all() and (bd == d[i * 100:(i + 1) * 100]).all()
        assert b.read_text().splitlines()[0] == "100"


def test_any_whitespace_between_tokens(tmp_path):
    p = tmp_path / "g.txt"
    p.write_text("5\t3\r\n0 1\n\n  2\t\t3\r\n4\n0")
    V, s, d = mk.read_edge_list(p)
    assert V == 5 and s.tolist() == [0, 2, 4] and d.tolist() == [1, 3, 0]
    e = tmp_path / "x.batch.0"
    e.write_text("0\n")
    bs, bd = mk.read_batch(e)
    assert len(bs) == 0 and len(bd) == 0


@pytest.mark.parametrize("text,needle", [
    ("4 3\n0 1\n1 2\n", "edge 2 of 3"),         # file ends early
    ("4 2\n0 1\n1 9\n", "out of range"),        # id >= V
    ("4 2\n0 1\n1 x\n", "malformed"),           # not a number
    ("4 2\n0 1\n1 4294967296\n", "malformed"),  # above 32 bits
    ("4\n", "edge count"),                      # header cut short
    ("", "vertex count"),
])
def test_malformed_graph_files_are_rejected(tmp_path, text, needle):
    p = tmp_path / "bad.txt"
    p.write_text(text)
    with pytest.raises(mk.MeerkatError) as ei:
        mk.read_edge_list(p)
    assert needle in str(ei.value)


def test_missing_file_and_out_of_range_write(tmp_path):
    with pytest.raises(mk.MeerkatError):
        mk.read_batch(tmp_path / "none.batch.0")
    with pytest.raises(mk.MeerkatError):
        mk.write_edge_list(tmp_path / "w.txt", 3, np.array([0, 3], np.uint32),
                           np.array([1, 1], np.uint32))

"""The reference's cache files and perfect spatial hash, on the host (no GPU).

Golden fixtures (tests/golden/make_golden.py): a .grid file written by the
reference's own Grid constructor through cereal, with its tables and every
lattice vertex looked up by the reference's hash; a .star file written by
the reference's StarProcessor through cereal.  The library's reader must
return those tables and arrays bit for bit, and its writer must reproduce
the reference's bytes; where the reference harness is built, files written
here are also read back through the reference's cereal and hash.
"""
import os
import tempfile

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def gold(name):
    return os.path.join(GOLD, name)


def lookup(psh, keys):
    """hashLookup (BT/kernel.cuh:713-733) restated in numpy: value per key,
    (-2, -2) where the slot holds another key."""
    hw, ow = psh["hash_width"], psh["offset_width"]
    keys = np.asarray(keys, np.int64)
    o = psh["offset_table"][(keys[:, 0] % ow) * ow + keys[:, 1] % ow].astype(np.int64)
    s = ((keys[:, 0] % hw + o[:, 0]) % hw) * hw + (keys[:, 1] % hw + o[:, 1]) % hw
    hit = (psh["pos_tag"][s] == keys).all(1)
    out = np.full((len(keys), 2), -2.0, np.float32)
    out[hit] = psh["hash_table"][s[hit]]
    return out, s


def test_grid_file_reader_matches_reference_fixture(bt):
    ref = np.load(gold("ref_c2_l6s4_decoded.npz"))
    got = bt.read_grid_file(gold("ref_c2_l6s4.grid"))
    assert (got["MAXLEVEL"], got["N"], got["M"]) == (int(ref["maxlevel"]), int(ref["N"]),
                                                     int(ref["M"]))
    assert (got["hash_width"], got["offset_width"]) == (int(ref["hash_width"]),
                                                        int(ref["offset_width"]))
    assert np.array_equal(got["hash_table"].view(np.uint32), ref["hash_table"].view(np.uint32))
    assert np.array_equal(got["pos_tag"], ref["pos_tag"])
    assert np.array_equal(got["offset_table"], ref["offset_table"])
    # the numpy restatement of the lookup gives the reference's dense decode
    N, M = got["N"], got["M"]
    ii, jj = np.meshgrid(np.arange(N), np.arange(M), indexing="ij")
    dense, _ = lookup(got, np.stack([ii.ravel(), jj.ravel()], 1))
    assert np.array_equal(dense.view(np.uint32), ref["dense"].view(np.uint32))
    assert int((dense[:, 0] != -2).sum()) == int(ref["entries"])


def test_grid_file_writer_reproduces_reference_bytes(bt):
    t = bt.read_grid_file(gold("ref_c2_l6s4.grid"))
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "x.grid")
        bt.write_grid_file(p, t["MAXLEVEL"], t["N"], t["M"], t)
        assert open(p, "rb").read() == open(gold("ref_c2_l6s4.grid"), "rb").read()


def test_psh_of_reference_grid_reads_back_in_reference(bt, oracle_mod):
    ref = np.load(gold("ref_c2_l6s4_decoded.npz"))
    N, M = int(ref["N"]), int(ref["M"])
    dense = ref["dense"]
    ex = dense[:, 0] != -2
    ii, jj = np.nonzero(ex.reshape(N, M))
    keys = np.stack([ii, jj], 1).astype(np.int32)
    psh = bt.psh_build(keys, dense[ex])
    # the reference's table widths for the same key count
    assert (psh["hash_width"], psh["offset_width"]) == (int(ref["hash_width"]),
                                                        int(ref["offset_width"]))
    allk = np.stack(np.meshgrid(np.arange(N), np.arange(M), indexing="ij"), -1).reshape(-1, 2)
    got, _ = lookup(psh, allk)
    assert np.array_equal(got.view(np.uint32), dense.view(np.uint32))
    again = bt.psh_build(keys, dense[ex])
    for k in ("hash_table", "pos_tag", "offset_table"):
        assert np.array_equal(again[k], psh[k]), "the table is not reproducible"
    if not oracle_mod.have_ref():
        pytest.skip("reference harness not built")
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "ours.grid")
        bt.write_grid_file(p, int(ref["maxlevel"]), N, M, psh)
        back = oracle_mod.ref_grid_file_decode(p)
    assert (back["N"], back["M"], back["MAXLEVEL"]) == (N, M, int(ref["maxlevel"]))
    assert np.array_equal(back["dense"].view(np.uint32), dense.view(np.uint32))


@pytest.mark.parametrize("shape", [(65, 128, 1.0), (129, 256, 0.35), (257, 512, 0.1),
                                   (3, 4, 1.0), (1, 1, 1.0)])
def test_psh_build_is_perfect(bt, shape):
    N, M, frac = shape
    rng = np.random.default_rng(N * M)
    allk = np.stack(np.meshgrid(np.arange(N), np.arange(M), indexing="ij"), -1).reshape(-1, 2)
    keys = allk[rng.random(len(allk)) < frac] if frac < 1 else allk
    vals = rng.standard_normal((len(keys), 2)).astype(np.float32)
    psh = bt.psh_build(keys, vals)
    got, slots = lookup(psh, keys)
    assert len(np.unique(slots)) == len(keys), "two keys share a slot"
    assert np.array_equal(got, vals)
    absent = np.setdiff1d(allk[:, 0] * M + allk[:, 1], keys[:, 0] * M + keys[:, 1])
    if len(absent):
        miss, _ = lookup(psh, np.stack([absent // M, absent % M], 1))
        assert (miss == -2).all()


def test_psh_build_rejects_bad_keys(bt):
    with pytest.raises(bt.BtError):
        bt.psh_build([[1, 2], [3, 4], [1, 2]], np.zeros((3, 2)))
    with pytest.raises(bt.BtError):
        bt.psh_build([[1, -2]], np.zeros((1, 2)))
    empty = bt.psh_build(np.zeros((0, 2)), np.zeros((0, 2)))
    assert empty["hash_width"] >= 1


def test_star_file_reader_and_writer_match_reference(bt, oracle_mod):
    ref = np.load(gold("ref_stars_l6.npz"))
    pos, mag, tree, lv = bt.read_star_file(gold("ref_stars_l6.star"))
    assert lv == int(ref["tree_level"])
    assert np.array_equal(pos, ref["pos"]) and np.array_equal(mag, ref["mag"])
    assert np.array_equal(tree, ref["tree"])
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "s.star")
        bt.write_star_file(p, pos, mag, tree, lv)
        assert open(p, "rb").read() == open(gold("ref_stars_l6.star"), "rb").read()
        if oracle_mod.have_ref():
            rp, rm, rt, rl = oracle_mod.ref_stars_file_read(p)
            assert rl == lv and np.array_equal(rp, pos) and np.array_equal(rt, tree)


def test_malformed_files_are_rejected(bt):
    raw = open(gold("ref_c2_l6s4.grid"), "rb").read()
    sraw = open(gold("ref_stars_l6.star"), "rb").read()
    with tempfile.TemporaryDirectory() as d:
        cases = {
            "truncated.grid": raw[:-3],
            "trailing.grid": raw + b"\0",
            "badlevel.grid": (7).to_bytes(4, "little") + raw[4:],
            "huge.grid": raw[:12] + (1 << 60).to_bytes(8, "little") + raw[20:],
        }
        for name, data in cases.items():
            p = os.path.join(d, name)
            open(p, "wb").write(data)
            with pytest.raises(bt.BtError):
                bt.read_grid_file(p)
        with pytest.raises(bt.BtError):
            bt.read_grid_file(os.path.join(d, "missing.grid"))
        p = os.path.join(d, "bad.star")
        open(p, "wb").write(sraw[:-4] + (9).to_bytes(4, "little"))
        with pytest.raises(bt.BtError):
            bt.read_star_file(p)

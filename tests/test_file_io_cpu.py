"""HReadSDPA (include/hdsdp_file_io.h) against the compiled reference reader
(interface/hdsdp_file_io.c) on the same SDPA files: identical sizes, right-hand
sides and CSC arrays (column order, entry order within columns, values). Host only.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from hdsdp_b200 import api, instances
from hdsdp_b200.build import build
from oracle import ref_api
from make_golden import SMALL


def write_sdpa(path, inst, header_style=0):
    """An instance as an SDPA file: F0 = -C, F_k = A_k, c = b (the inverse of the reader's
    conversion), entries in the upper triangle, 1-based."""
    n, m = inst.n, inst.m
    lines = ['"generated from %s' % inst.name, "* comment line"]
    if header_style == 0:
        lines += ["%d = mDIM" % m, "1 = nBLOCK", "%d = bLOCKsTRUCT" % n,
                  " ".join("%.17g" % v for v in inst.b)]
    else:
        lines += ["%d" % m, "1", "{%d}" % n, "{" + ", ".join("%.17g" % v for v in inst.b) + "}"]
    starts = instances.pack_idx(n, np.arange(n), np.arange(n))
    for k in range(m + 1):
        rows, vals = inst.column(k)
        j = np.searchsorted(starts, rows, side="right") - 1
        i = rows - starts[j] + j
        sign = -1.0 if k == 0 else 1.0
        for a, c, v in zip(j, i, vals):  # a = column (<= row c): upper entry (a, c)
            lines.append("%d 1 %d %d %.17g" % (k, a + 1, c + 1, sign * v))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_sdpa_lp(path, inst, lp):
    """An instance and an LP cone (n_lp, Ap, Ai, Ax) as an SDPA file with a diagonal LP block
    (negative block size): LP column k is diagonal entry (k, k) of block 2."""
    write_sdpa(path, inst)
    nlp, Ap, Ai, Ax = lp
    lines = open(path).read().splitlines()
    lines[3] = "2 = nBLOCK"
    lines[4] = "%d %d = bLOCKsTRUCT" % (inst.n, -nlp)
    for k in range(inst.m + 1):
        sign = -1.0 if k == 0 else 1.0
        for e in range(Ap[k], Ap[k + 1]):
            lines.append("%d 2 %d %d %.17g" % (k, Ai[e] + 1, Ai[e] + 1, sign * Ax[e]))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_sdpa_problem(path, prob):
    """A multi-cone problem (instances.ConicProblem) as an SDPA file: its SDP blocks in
    order, then its LP cone as a diagonal block (negative size); F0 = -C_k, 1-based upper
    entries."""
    sdp = [c for c in prob.cones if c[0] == "sdp"]
    lps = [c for c in prob.cones if c[0] == "lp"]
    assert len(lps) <= 1 and prob.cones[:len(sdp)] == sdp
    sizes = [str(c[1]) for c in sdp] + ["-%d" % c[1] for c in lps]
    lines = ['"generated from %s' % prob.name, "%d = mDIM" % prob.m, "%d = nBLOCK" % len(sizes),
             " ".join(sizes) + " = bLOCKsTRUCT", " ".join("%.17g" % v for v in prob.b)]
    for blk, (kind, n, Ap, Ai, Ax) in enumerate(prob.cones):
        for k in range(prob.m + 1):
            sign = -1.0 if k == 0 else 1.0
            rows, vals = Ai[Ap[k]:Ap[k + 1]], Ax[Ap[k]:Ap[k + 1]]
            if kind == "lp":
                for q, v in zip(rows, vals):
                    lines.append("%d %d %d %d %.17g" % (k, blk + 1, q + 1, q + 1, sign * v))
                continue
            starts = instances.pack_idx(n, np.arange(n), np.arange(n))
            j = np.searchsorted(starts, rows, side="right") - 1
            i = rows - starts[j] + j
            for a, c, v in zip(j, i, vals):
                lines.append("%d %d %d %d %.17g" % (k, blk + 1, a + 1, c + 1, sign * v))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


@pytest.fixture(scope="module")
def libs():
    build()
    if not ref_api.available():
        pytest.skip("oracle/_ref not built")
    return api._lib.load(), ref_api.lib()


def same(a, b):
    assert a["m"] == b["m"] and a["n_cols"] == b["n_cols"] and a["n_elems"] == b["n_elems"]
    np.testing.assert_array_equal(a["b"], b["b"])
    assert len(a["blocks"]) == len(b["blocks"])
    for (n1, p1, i1, x1), (n2, p2, i2, x2) in zip(a["blocks"], b["blocks"]):
        assert n1 == n2
        np.testing.assert_array_equal(p1, p2)
        np.testing.assert_array_equal(i1, i2)
        np.testing.assert_array_equal(x1, x2)
    assert (a["lp"] is None) == (b["lp"] is None)
    if a["lp"] is not None:
        for u, v in zip(a["lp"][1:], b["lp"][1:]):
            np.testing.assert_array_equal(u, v)
        assert a["lp"][0] == b["lp"][0]


@pytest.mark.parametrize("name", sorted(SMALL))
def test_instances_round_trip(libs, tmp_path, name):
    ours, ref = libs
    inst = SMALL[name]()
    path = tmp_path / ("%s.dat-s" % name)
    write_sdpa(path, inst, 0)
    a = api.read_sdpa_with(ours, path)
    same(a, api.read_sdpa_with(ref, path))
    # braces and commas in the size and right-hand-side lines read the same (the
    # reference itself misreads a braced last block size, so it is not asked here)
    path1 = tmp_path / ("%s_braces.dat-s" % name)
    write_sdpa(path1, inst, 1)
    same(api.read_sdpa_with(ours, path1), a)
    # and the data is the instance's (entry order may differ within a column)
    n, Ap, Ai, Ax = a["blocks"][0]
    np.testing.assert_array_equal(a["b"], inst.b)
    for k in range(inst.m + 1):
        r0, v0 = inst.column(k)
        r1, v1 = Ai[Ap[k]:Ap[k + 1]], Ax[Ap[k]:Ap[k + 1]]
        o0, o1 = np.argsort(r0, kind="stable"), np.argsort(r1, kind="stable")
        np.testing.assert_array_equal(np.asarray(r0)[o0], r1[o1])
        np.testing.assert_array_equal(np.asarray(v0)[o0], v1[o1])


def test_blocks_lp_tiny_duplicates(libs, tmp_path):
    """Two SDP blocks and an LP block, lower-triangle entries (swapped to upper), a tiny
    entry (dropped), a repeated position (kept twice), the BEGIN.COMMENT terminator (the
    reference wants the line exactly as "BEGIN.COMMENT" and two spaces)."""
    ours, ref = libs
    text = """* three constraints
3
3
2 3 -4
1.0, -2.5, 3.0
0 1 1 1 1.5
0 1 2 1 -0.25
1 1 1 2 2.0
1 2 3 3 1.0
2 2 2 1 4.0
2 2 2 1 4.0
3 2 1 3 1e-14
3 1 2 2 -7.0
0 3 1 1 2.0
1 3 2 2 -1.0
3 3 4 4 0.5
BEGIN.COMMENT  
anything after this is ignored
"""
    path = tmp_path / "mixed.dat-s"
    path.write_text(text)
    a = api.read_sdpa_with(ours, path)
    same(a, api.read_sdpa_with(ref, path))
    assert len(a["blocks"]) == 2 and a["lp"][0] == 4 and a["n_elems"] == 10


def test_last_line_without_newline(libs, tmp_path):
    ours, ref = libs
    path = tmp_path / "nonl.dat-s"
    path.write_text("1\n1\n2\n1.0\n0 1 1 1 1.0\n1 1 1 2 0.5")
    same(api.read_sdpa_with(ours, path), api.read_sdpa_with(ref, path))


@pytest.mark.parametrize("text", ["1\n1\n2\n1.0\n0 1 1 1 1.0\n\n1 1 1 2 0.5\n",   # blank line inside the data
                                  "1\n1\n2\n1.0\n0 1 1 1 1.0\n1 1 x 2 0.5\n"])   # a malformed entry
def test_bad_files_fail_like_the_reference(libs, tmp_path, text):
    ours, ref = libs
    path = tmp_path / "bad.dat-s"
    path.write_text(text)
    with pytest.raises(RuntimeError):
        api.read_sdpa_with(ours, path)
    with pytest.raises(RuntimeError):
        api.read_sdpa_with(ref, path)


def test_missing_file(libs, tmp_path):
    ours, _ = libs
    with pytest.raises(RuntimeError):
        api.read_sdpa_with(ours, tmp_path / "absent.dat-s")


def test_sdpa_instance(libs, tmp_path):
    inst = SMALL[sorted(SMALL)[0]]()
    path = tmp_path / "one.dat-s"
    write_sdpa(path, inst)
    got = api.sdpa_instance(path)
    assert got.n == inst.n and got.m == inst.m
    np.testing.assert_array_equal(got.b, inst.b)


def test_sdpa_with_lp_block(libs, tmp_path):
    """An SDP block plus an LP cone written as SDPA and read back: the same LP arrays as the
    reference reader, and the LP cone the solver takes."""
    from make_golden import lp_case
    ours, ref = libs
    inst, lp = lp_case("theta40+lp25")
    path = tmp_path / "lp.dat-s"
    write_sdpa_lp(path, inst, lp)
    a = api.read_sdpa_with(ours, path)
    same(a, api.read_sdpa_with(ref, path))
    got_inst, got_lp = api.sdpa_problem(path)
    assert got_lp[0] == lp[0]
    for k in range(inst.m + 1):
        lo, hi = lp[1][k], lp[1][k + 1]
        glo, ghi = got_lp[1][k], got_lp[1][k + 1]
        np.testing.assert_array_equal(np.sort(lp[2][lo:hi]), np.sort(got_lp[2][glo:ghi]))
        np.testing.assert_array_equal(lp[3][lo:hi][np.argsort(lp[2][lo:hi])],
                                      got_lp[3][glo:ghi][np.argsort(got_lp[2][glo:ghi])])


@pytest.mark.parametrize("name", ["mb5_sparse", "mb2_lp"])
def test_sdpa_multiblock(libs, tmp_path, name):
    """Several SDP blocks (and an LP block) written as SDPA: both readers give the same
    arrays, and sdpa_cones() gives back the problem's cones (entry order within a column
    may differ)."""
    ours, ref = libs
    prob = instances.multiblock_case(name)
    path = tmp_path / ("%s.dat-s" % name)
    write_sdpa_problem(path, prob)
    same(api.read_sdpa_with(ours, path), api.read_sdpa_with(ref, path))
    got = api.sdpa_cones(path)
    assert got.m == prob.m and len(got.cones) == len(prob.cones)
    np.testing.assert_array_equal(got.b, prob.b)
    for (k0, n0, p0, i0, x0), (k1, n1, p1, i1, x1) in zip(prob.cones, got.cones):
        assert (k0, n0) == (k1, n1)
        np.testing.assert_array_equal(p0, p1)
        for k in range(prob.m + 1):
            o0 = np.argsort(i0[p0[k]:p0[k + 1]], kind="stable")
            o1 = np.argsort(i1[p1[k]:p1[k + 1]], kind="stable")
            np.testing.assert_array_equal(i0[p0[k]:p0[k + 1]][o0], i1[p1[k]:p1[k + 1]][o1])
            np.testing.assert_array_equal(x0[p0[k]:p0[k + 1]][o0], x1[p1[k]:p1[k + 1]][o1])


def test_sizes_over_several_lines(libs, tmp_path):
    """Block sizes (and the right-hand side) spread over several lines read as the same file
    on one line. The reference counts one line for each and then misplaces the data."""
    ours, ref = libs
    one = tmp_path / "one.dat-s"
    one.write_text('"c\n1\n3\n2 2 -1\n1.0\n0 1 1 1 1.0\n1 1 1 2 0.5\n1 3 1 1 2.0\n')
    multi = tmp_path / "multi.dat-s"
    multi.write_text('"c\n1\n3\n2\n2\n-1\n1.0\n0 1 1 1 1.0\n1 1 1 2 0.5\n1 3 1 1 2.0\n')
    same(api.read_sdpa_with(ours, multi), api.read_sdpa_with(ref, one))
    with pytest.raises(RuntimeError):
        api.read_sdpa_with(ref, multi)


def test_index_outside_block_is_an_error(libs, tmp_path):
    """An entry whose row or column exceeds its block's size is an error here; the reference
    stores it at a packed index outside the block."""
    ours, _ = libs
    path = tmp_path / "oob.dat-s"
    path.write_text("1\n1\n2\n1.0\n0 1 1 1 1.0\n1 1 3 1 0.5\n")
    with pytest.raises(RuntimeError):
        api.read_sdpa_with(ours, path)


def test_lp_block_not_last_fails_like_the_reference(libs, tmp_path):
    ours, ref = libs
    path = tmp_path / "lpfirst.dat-s"
    path.write_text("1\n2\n-2 2\n1.0\n0 2 1 1 1.0\n1 1 1 1 1.0\n1 2 1 2 0.5\n")
    for L in (ours, ref):
        with pytest.raises(RuntimeError):
            api.read_sdpa_with(L, path)

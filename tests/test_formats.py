"""Byte formats pinned to the reference converter's own output.

tests/golden/toy.{csr,csc,wcsr} and toy_w.csr were written by the reference
converter (converter/converter.cpp, built from its sources by oracle/Makefile)
from tests/golden/toy_edges.txt; make_golden.py regenerates them.  The
converter keeps duplicates and self-loops, numbers vertices 0..max id, and
writes weight 20 unless built with -DWEIGHTED (converter.cpp:9,80,93-95).
"""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load_edges():
    a = np.loadtxt(os.path.join(GOLD, "toy_edges.txt"), dtype=np.int64)
    return a[:, 0], a[:, 1], a[:, 2]


def converter_csr(src, dst, w, by_dst=False):
    nv = int(max(src.max(), dst.max())) + 1
    order = np.lexsort((src, dst)) if by_dst else np.lexsort((dst, src))
    key = dst if by_dst else src
    off = np.zeros(nv + 1, np.uint64)
    np.add.at(off, key + 1, 1)
    off = np.cumsum(off).astype(np.uint64)
    other = src if by_dst else dst
    return nv, off, other[order].astype(np.uint32), w[order].astype(np.uint32)


def read(name):
    with open(os.path.join(GOLD, name), "rb") as f:
        return f.read()


def test_csr_bytes_match_converter(O, tmp_path):
    s, d, w = load_edges()
    nv, off, adj, _ = converter_csr(s, d, w)
    g = O.CSR(off, adj, None)
    p = str(tmp_path / "x.csr")
    O.write_csr(p, g)  # default weight 20, like the unweighted converter
    assert open(p, "rb").read() == read("toy.csr")


def test_weighted_csr_bytes_match_converter(O, tmp_path):
    s, d, w = load_edges()
    nv, off, adj, ww = converter_csr(s, d, w)
    g = O.CSR(off, adj, ww)
    p = str(tmp_path / "x.csr")
    O.write_csr(p, g)
    assert open(p, "rb").read() == read("toy_w.csr")


def test_wcsr_bytes_match_converter(O, tmp_path):
    s, d, w = load_edges()
    nv, off, adj, _ = converter_csr(s, d, w)
    g = O.CSR(off, adj, None)
    p = str(tmp_path / "x.wcsr")
    O.write_wcsr(p, g)
    assert open(p, "rb").read() == read("toy.wcsr")


def test_csc_bytes_match_converter(O, tmp_path):
    s, d, w = load_edges()
    nv, off, adj, _ = converter_csr(s, d, w)
    # oracle transpose of the converter CSR == converter CSC
    g = O.CSR(off, adj, None)
    p = str(tmp_path / "x.csc")
    O.write_csc(p, g)
    assert open(p, "rb").read() == read("toy.csc")


def test_golden_header_layout():
    b = read("toy.csr")
    nv, ne = np.frombuffer(b[:16], np.uint64)
    assert len(b) == 16 + 8 * nv + 4 * ne + 4 * ne
    b = read("toy.csc")
    nv, ne = np.frombuffer(b[:16], np.uint64)
    assert len(b) == 16 + 8 * nv + 4 * ne + 4 * nv
    b = read("toy.wcsr")
    nv, ne = np.frombuffer(b[:16], np.uint64)
    assert len(b) == 16 + 8 * nv + 8 * ne

"""thv_convert: text edge lists to the converter's byte formats, sorted on
the GPU.  Pinned to the files the reference converter wrote for
tests/golden/toy_edges.txt, and to a restatement of the converter's line
parsing (a field that fails keeps the previous line's value) below."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
ROOT = os.path.join(os.path.dirname(__file__), "..")


def gold(name):
    return open(os.path.join(GOLD, name), "rb").read()


@pytest.mark.parametrize("fmt,weighted,name", [("csr", False, "toy.csr"), ("csc", False, "toy.csc"),
                                               ("wcsr", False, "toy.wcsr"), ("csr", True, "toy_w.csr")])
def test_matches_reference_converter_output(T, tmp_path, fmt, weighted, name):
    out = str(tmp_path / f"g.{fmt}")
    nv, ne = T.convert(os.path.join(GOLD, "toy_edges.txt"), out, fmt, skip=0, weighted=weighted)
    assert open(out, "rb").read() == gold(name)
    assert nv == 45


def test_cli_names_and_bytes(T, tmp_path):
    txt = tmp_path / "g.txt"
    txt.write_bytes(open(os.path.join(GOLD, "toy_edges.txt"), "rb").read())
    for kind, name in (("csr", "toy.csr"), ("wcsr", "toy.wcsr"), ("csc", "toy.csc")):
        r = subprocess.run([os.path.join(ROOT, "convert"), "--input", str(txt), "--type", kind,
                            "--skip", "0"], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        assert (tmp_path / f"g.{kind}").read_bytes() == gold(name)


def parse_like_converter(text, skip, weighted, undirected):
    """istream semantics per line: src, dst, then w (weighted); the first
    field that fails stops the line and every unread field keeps its value."""
    src = dst = 0
    w = 20
    out = []
    lines = text.split("\n")
    if text.endswith("\n"):
        lines = lines[:-1]
    for line in lines[skip:]:
        toks = line.replace("\r", " ").replace("\t", " ").split(" ")
        toks = [t for t in toks if t != ""]
        vals = []
        for t in toks:
            t2 = t[1:] if t.startswith("+") else t
            digits = ""
            for ch in t2:
                if ch.isdigit():
                    digits += ch
                else:
                    break
            if not digits:
                break
            vals.append(int(digits))
            if len(digits) < len(t2):
                break  # the next extraction starts inside this token and fails
        if len(vals) >= 1:
            src = vals[0]
            if len(vals) >= 2:
                dst = vals[1]
                if weighted and len(vals) >= 3:
                    w = vals[2]
        out.append((src, dst, w))
        if undirected:
            out.append((dst, src, w))
    return out


def expected_bytes(edges, fmt):
    e = np.array(edges, dtype=np.int64).reshape(-1, 3)
    nv = int(e[:, :2].max()) + 1 if len(e) else 1
    key, other = (e[:, 1], e[:, 0]) if fmt == "csc" else (e[:, 0], e[:, 1])
    order = np.lexsort((other, key))  # stable: duplicates keep input order
    off = np.zeros(nv + 1, np.uint64)
    np.add.at(off, key + 1, 1)
    off = np.cumsum(off).astype(np.uint64)[:nv]
    hdr = np.array([nv, len(e)], np.uint64).tobytes() + off.tobytes()
    o = other[order].astype(np.uint32)
    w = e[order, 2].astype(np.uint32)
    if fmt == "csr":
        return hdr + o.tobytes() + w.tobytes()
    if fmt == "wcsr":
        return hdr + np.stack([o, w], axis=1).tobytes()
    outdeg = np.bincount(e[:, 0], minlength=nv).astype(np.uint32)
    return hdr + o.tobytes() + outdeg.tobytes()


QUIRKY = ("# header line 1\n% header 2\n\nheader 4\n"
          "1 2 7\n3 4\n\n# a comment keeps the previous edge\n5\t6\t9\r\n"
          "  7 8 +3\n9 x 5\n10 11 12 13\n2 2 2\n1 2 7\n")


@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("undirected", [False, True])
@pytest.mark.parametrize("fmt", ["csr", "wcsr", "csc"])
def test_line_parsing_matches_the_converter_stream(T, tmp_path, weighted, undirected, fmt):
    txt = tmp_path / "q.txt"
    txt.write_text(QUIRKY)
    out = str(tmp_path / f"q.{fmt}")
    T.convert(str(txt), out, fmt, skip=4, weighted=weighted, undirected=undirected)
    want = expected_bytes(parse_like_converter(QUIRKY, 4, weighted, undirected), fmt)
    assert open(out, "rb").read() == want


def test_random_list_and_round_trip(T, O, tmp_path):
    rng = np.random.default_rng(3)
    n = 200_000
    s = rng.integers(0, 5000, n)
    d = rng.integers(0, 5000, n)
    w = rng.integers(1, 100, n)
    txt = tmp_path / "r.txt"
    with open(txt, "w") as f:
        f.write("src dst w\n")
        for a, b, c in zip(s, d, w):
            f.write(f"{a} {b} {c}\n")
    edges = list(zip(s.tolist(), d.tolist(), w.tolist()))
    for fmt in ("csr", "wcsr", "csc"):
        out = str(tmp_path / f"r.{fmt}")
        nv, ne = T.convert(str(txt), out, fmt, skip=1, weighted=True)
        assert ne == n
        assert open(out, "rb").read() == expected_bytes(edges, fmt)
    # the engine opens the converted file and traverses it
    with T.Graph.open(str(tmp_path / "r.wcsr"), "wcsr") as g:
        off, ed, _ = g.host_arrays()
        csr = O.CSR(np.array(off, np.uint64), np.array(ed[:, 0]), np.array(ed[:, 1]))
        g.plan()
        src = int(O.sources(csr, 1)[0])
        got, _ = g.run("sssp", source=src, timeout_ms=20000)
        assert np.array_equal(got, O.sssp(csr, src))


def test_errors(T, tmp_path):
    with pytest.raises(T.ThvError):
        T.convert(str(tmp_path / "missing.txt"), str(tmp_path / "o.csr"))
    big = tmp_path / "big.txt"
    big.write_text("1 4294967296\n")
    with pytest.raises(T.ThvError):
        T.convert(str(big), str(tmp_path / "o.csr"), skip=0)
    empty = tmp_path / "e.txt"
    empty.write_text("")
    nv, ne = T.convert(str(empty), str(tmp_path / "e.csr"), skip=0)
    assert (nv, ne) == (1, 0)
    assert open(tmp_path / "e.csr", "rb").read() == np.array([1, 0, 0], np.uint64).tobytes()

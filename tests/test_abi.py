"""C ABI surface and host-side error paths (no GPU needed)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest


def declared_functions(root):
    src = open(os.path.join(root, "include", "thv.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return set(re.findall(r"\b(thv_[a-z_0-9]+)\s*\(", src))


def test_library_exports_every_declared_symbol(T, root):
    lib = T.load_library()
    decl = declared_functions(root)
    assert decl == set(T.ABI_FUNCTIONS)
    for name in decl:
        assert hasattr(lib, name), name


def test_version_and_status_strings(T):
    lib = T.load_library()
    assert lib.thv_abi_version() == 4
    assert lib.thv_status_str(0) == b"ok"
    assert lib.thv_status_str(3) == b"malformed graph file"


def test_missing_file_is_eio(T, tmp_path):
    with pytest.raises(T.ThvError) as e:
        T.Graph.open(str(tmp_path / "nope.csr"))
    assert e.value.status == T.THV_EIO


def test_truncated_header_is_eformat(T, tmp_path):
    p = tmp_path / "t.csr"
    p.write_bytes(b"\x01\x00\x00")
    with pytest.raises(T.ThvError) as e:
        T.Graph.open(str(p))
    assert e.value.status == T.THV_EFORMAT


def test_truncated_edges_is_eformat(T, tmp_path):
    p = tmp_path / "t.csr"
    hdr = np.array([4, 100], np.uint64).tobytes() + np.zeros(4, np.uint64).tobytes()
    p.write_bytes(hdr + np.zeros(10, np.uint32).tobytes())
    with pytest.raises(T.ThvError) as e:
        T.Graph.open(str(p))
    assert e.value.status == T.THV_EFORMAT


def test_csr_weights_section_required_for_sssp(T, root, tmp_path):
    # golden toy.csr has its weight section: size check passes; cut it off
    b = open(os.path.join(root, "tests", "golden", "toy.csr"), "rb").read()
    nv, ne = np.frombuffer(b[:16], np.uint64)
    p = tmp_path / "cut.csr"
    p.write_bytes(b[: 16 + 8 * int(nv) + 4 * int(ne)])
    with pytest.raises(T.ThvError) as e:
        T.Graph.open(str(p), "csr", weights=True)
    assert e.value.status == T.THV_EFORMAT


def test_write_values_roundtrip(T, tmp_path):
    lib = T.load_library()
    v = np.arange(10, dtype=np.uint32)
    p = str(tmp_path / "values.bin")
    assert lib.thv_write_values(p.encode(), ctypes.c_void_p(v.ctypes.data), 10, 4) == 0
    assert np.array_equal(np.fromfile(p, np.uint32), v)


def test_neighbour_gpus_rejected(T):
    with pytest.raises(T.ThvError) as e:
        T.BFS32("x.csr", 1, 1, n_neighbor_gpus=1)
    assert e.value.status == T.THV_EUNSUPPORTED


def run_main(root, *args, cwd=None):
    return subprocess.run([os.path.join(root, "main"), *args], capture_output=True, text=True,
                          cwd=cwd, timeout=60)


def test_cli_without_input_prints_usage(root):
    r = run_main(root)
    assert r.returncode == 0 and "Usage" in r.stdout


def test_cli_rejects_neighbour_gpus(root):
    r = run_main(root, "--input", "x.csr", "--gpus", "2")
    assert r.returncode == 1 and "--gpus" in r.stderr


def test_cli_missing_file(root, tmp_path):
    r = run_main(root, "--input", str(tmp_path / "none.csr"))
    assert r.returncode == 1 and "cannot open" in r.stderr


def test_cli_bad_edge_size(root):
    r = run_main(root, "--input", "x.csr", "--edgeSize", "3")
    assert r.returncode == 1


def test_convert_input_errors_before_any_device_work(T, tmp_path):
    """thv_convert checks its arguments and parses the whole text file on
    the host before it touches a GPU: these errors come back on any host."""
    with pytest.raises(T.ThvError) as e:
        T.convert(str(tmp_path / "missing.txt"), str(tmp_path / "o.csr"))
    assert e.value.status == T.THV_EIO
    txt = tmp_path / "g.txt"
    txt.write_text("0 1\n1 4294967295\n")
    with pytest.raises(T.ThvError) as e:
        T.convert(str(txt), str(tmp_path / "o.csr"), skip=0)
    assert e.value.status == T.THV_EUNSUPPORTED
    assert not (tmp_path / "o.csr").exists()

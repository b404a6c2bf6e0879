"""The values.bin comparer (thievory_b200/csrc/compare.cpp), a drop-in for
the reference's comparer/compare.cpp with its flags: exact integers,
absolute tolerance for doubles, and the fixes (u32 read size, 64-bit
indices, short files, exit status)."""
import os
import subprocess

import numpy as np
import pytest

SRC = os.path.join(os.path.dirname(__file__), "..", "thievory_b200", "csrc", "compare.cpp")


@pytest.fixture(scope="module")
def cmp_bin(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("cmp") / "compare")
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-o", out, SRC], check=True)
    return out


def run(cmp_bin, a, b, n, kind=0, *extra):
    r = subprocess.run([cmp_bin, "--input1", a, "--input2", b, "--type", str(kind),
                        "--vertices", str(n), *map(str, extra)],
                       capture_output=True, text=True)
    return r.returncode, r.stdout + r.stderr


def write(tmp_path, name, arr):
    p = str(tmp_path / name)
    arr.tofile(p)
    return p


def test_u32_equal_and_mismatch(cmp_bin, tmp_path):
    a = np.arange(1000, dtype=np.uint32)
    b = a.copy()
    pa, pb = write(tmp_path, "a", a), write(tmp_path, "b", b)
    rc, out = run(cmp_bin, pa, pb, 1000)
    assert rc == 0 and "Mismatches: 0 of 1000" in out
    b[3] = 7
    b[999] = 0
    pb = write(tmp_path, "b", b)
    rc, out = run(cmp_bin, pa, pb, 1000)
    assert rc == 1
    assert "Arrays do not match at: 3\n3 | 7" in out
    assert "Mismatches: 2 of 1000" in out


def test_u32_reads_four_bytes_per_value(cmp_bin, tmp_path):
    # the reference read n * 8 bytes for u32 files; a file of exactly n u32
    # values must compare cleanly
    a = np.full(17, 5, np.uint32)
    pa = write(tmp_path, "a", a)
    assert os.path.getsize(pa) == 17 * 4
    assert run(cmp_bin, pa, pa, 17)[0] == 0


def test_doubles_tolerance_and_nan(cmp_bin, tmp_path):
    a = np.linspace(0, 1, 64)
    b = a + 5e-4
    pa, pb = write(tmp_path, "a", a), write(tmp_path, "b", b)
    assert run(cmp_bin, pa, pb, 64, 2)[0] == 0
    assert run(cmp_bin, pa, pb, 64, 2, "--tolerance", "1e-4")[0] == 1
    b[10] = np.nan
    pb = write(tmp_path, "b", b)
    rc, out = run(cmp_bin, pa, pb, 64, 2)
    assert rc == 1 and "Mismatches: 1 of 64" in out


def test_u64_and_report_limit(cmp_bin, tmp_path):
    a = np.arange(100, dtype=np.uint64) << np.uint64(33)
    b = a + np.uint64(1)
    pa, pb = write(tmp_path, "a", a), write(tmp_path, "b", b)
    rc, out = run(cmp_bin, pa, pb, 100, 1, "--max-report", "3")
    assert rc == 1 and out.count("Arrays do not match") == 3 and "Mismatches: 100 of 100" in out


def test_short_file_and_bad_arguments(cmp_bin, tmp_path):
    pa = write(tmp_path, "a", np.zeros(10, np.uint32))
    pb = write(tmp_path, "b", np.zeros(5, np.uint32))
    rc, out = run(cmp_bin, pa, pb, 10)
    assert rc == 2 and "holds 5 values" in out
    assert run(cmp_bin, pa, str(tmp_path / "missing"), 10)[0] == 2
    assert run(cmp_bin, pa, pa, 10, 7)[0] == 2
    r = subprocess.run([cmp_bin, "--input1", pa], capture_output=True, text=True)
    assert r.returncode == 2

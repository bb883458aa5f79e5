"""The .field / .vfield / DAT / VTS formats, byte for byte against the
reference, with no GPU: tests/cxx/io_format.cu writes scalar and vector
fields (2-D and 3-D) in every format, reads them back through every reader
and writes them again, and prints the message of each reader error; it is
built once against the reference library and once against libphix_cxx.so
(oracle/Makefile `dropin`).  Both builds must write the same files and print
the same lines.  The binaries are built where the reference tree exists;
without them the test skips.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROP = os.path.join(ROOT, "oracle", "_ref", "dropin")


def _run(name, cwd):
    exe = os.path.join(DROP, name)
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built (needs the reference tree at build time)")
    r = subprocess.run([exe], cwd=cwd, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def test_io_formats_match_reference_bytes(tmp_path):
    ref, ours = tmp_path / "ref", tmp_path / "ours"
    ref.mkdir()
    ours.mkdir()
    out_ref = _run("iofmt_ref", ref)
    out_ours = _run("iofmt_phix", ours)
    assert out_ours == out_ref
    assert out_ref.count(": no error") == 0 and "io_format done" in out_ref
    names = sorted(os.listdir(ref))
    assert sorted(os.listdir(ours)) == names
    # 2 meshes x (3 scalar + 2 scalar re-reads + 3 vector + 3 vector re-reads) + 3 truncated copies
    assert len(names) == 2 * 11 + 3
    for n in names:
        assert (ref / n).read_bytes() == (ours / n).read_bytes(), n

"""Drop-in check of the C++ API: the reference's own drivers, unmodified, built
once against the reference library and once against include/phix +
libphix_cxx.so (oracle/Makefile `dropin`), must print the same verdicts and
write the same fields bit for bit.

  * tutorials/quickstart/main.cu: 2-D Allen-Cahn, 256^2, RK4, 10000 steps,
    a .field file every 500 steps (the fused single-equation Solver path).
  * develop/fieldOperation/test_fieldops.cu: the reference's own known-answer
    checks of pw / field arithmetic / composite products (tolerance 1e-12).

The binaries are built where the reference tree exists; without them the
tests skip.
"""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROP = os.path.join(ROOT, "oracle", "_ref", "dropin")


def _bin(name):
    p = os.path.join(DROP, name)
    if not os.path.exists(p):
        pytest.skip(f"{p} not built (needs the reference tree at build time)")
    return p


def _run(binary, cwd):
    r = subprocess.run([binary], cwd=cwd, capture_output=True, text=True, timeout=900)
    return r.returncode, r.stdout + r.stderr


def _read_field(path):
    raw = open(path, "rb").read()
    cut = raw.index(b"---\n") + 4
    return raw[:cut], np.frombuffer(raw[cut:], dtype="<f8")


def test_quickstart_fields_identical(cuda, tmp_path):
    ref_dir, our_dir = tmp_path / "ref", tmp_path / "ours"
    ref_dir.mkdir()
    our_dir.mkdir()
    rc_r, out_r = _run(_bin("quickstart_ref"), ref_dir)
    rc_o, out_o = _run(_bin("quickstart_phix"), our_dir)
    assert rc_r == 0, out_r[-2000:]
    assert rc_o == 0, out_o[-2000:]
    ref_files = sorted(os.listdir(ref_dir / "output"))
    our_files = sorted(os.listdir(our_dir / "output"))
    assert ref_files == our_files and len(ref_files) == 21
    worst = 0.0
    for name in ref_files:
        hr, dr = _read_field(ref_dir / "output" / name)
        ho, do = _read_field(our_dir / "output" / name)
        assert hr == ho, name
        assert dr.shape == do.shape == (256 * 256,)
        worst = max(worst, float(np.abs(dr - do).max()))
        assert np.array_equal(dr, do), f"{name}: max-abs {np.abs(dr - do).max():.3e}"
    print(f"quickstart: {len(ref_files)} fields identical (max-abs {worst:.1e})")


def test_fieldops_known_answers(cuda, tmp_path):
    rc_r, out_r = _run(_bin("fieldops_ref"), tmp_path)
    rc_o, out_o = _run(_bin("fieldops_phix"), tmp_path)
    assert rc_r == 0, out_r[-2000:]
    assert rc_o == 0 and "ALL TESTS PASSED" in out_o, out_o[-3000:]
    verdicts = lambda s: [l.strip() for l in s.splitlines() if "[PASS]" in l or "[FAIL]" in l]
    assert verdicts(out_o) == verdicts(out_r)

"""Drop-in check of the C++ API: the reference's own drivers, unmodified, built
once against the reference library and once against include/phix +
libphix_cxx.so (oracle/Makefile `dropin`), must print the same verdicts and
write the same fields bit for bit.

  * tutorials/quickstart/main.cu: 2-D Allen-Cahn, 256^2, RK4, 10000 steps,
    a .field file every 500 steps (the fused single-equation Solver path).
  * develop/fieldOperation/test_fieldops.cu: the reference's own known-answer
    checks of pw / field arithmetic / composite products (tolerance 1e-12).
  * applications/solvers/Cahn-Hillard_double-well/2D: the CH application
    (config file, BC factory, multi-step STEADY/TRANSIENT Euler Solver,
    OutputWriter in all three formats).  Ours runs twice: with the default
    asynchronous OutputWriter and with "async": false (the reference's
    synchronous order); those two runs must write the same bytes, and both
    must match the reference's files to 1e-12.
  * applications/solvers/glass_formation/2D/GFA.cu: the glass-formation
    application (six SolverSteps over c, phi, eta, mu, D: pw terms of two
    and three fields, D lap(mu) + grad(D) . grad(mu), pw + lap), which runs
    as one fused launch per step here; its files must equal the reference's
    byte for byte.

  * applications/solvers/Cahn-Hillard+Allen-Cahn_double-well/2D: the coupled
    CH+AC application (three SolverSteps: mu STEADY from pw of c and of eta
    and lap c; c and eta TRANSIENT), all files equal the reference's.
  * develop/Spinodal Decomposition/Cahn-Hillard.cu and
    develop/Ostwald_Ripening/AC-CH.cu: the develop drivers' manual loops
    (BCs by applyOnGPU, Equation::computeRHS called directly, single-equation
    Euler Solvers on other fields).  They run 1e8 steps; the test stops each
    after its step-10000 output and compares every file written up to then.

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


CH_SETTINGS = """{{
    // written by tests/test_gpu_dropin.py
    "mesh": {{"nx": {nx}, "ny": {ny}, "dx": 1.0, "dy": 1.0, "x0": 0.0, "y0": 0.0}},
    "initialize": {{"start_from": "initial_field", "dt": 0.01, "nSteps": {nsteps}}},
    "boundary_conditions": {{"x_min": "Periodic", "x_max": "Periodic", "y_min": "NoFlux", "y_max": "NoFlux"}},
    "constants": {{"M": 1.0, "kappa": 0.5, "rho": 1.0, "ca": 0.0, "cb": 1.0}},
    "output": {{"print_interval": {every}, "write_interval": {every}, "format": "ALL"{extra}}}
}}
"""


def _write_field(path, name, a):
    """A 2-D .field file in the reference's binary format (physical cells,
    little-endian FP64, x fastest)."""
    ny, nx = a.shape
    hdr = f"# PhiX ScalarField\nname    {name}\nnx {nx}  ny {ny}  nz 1\nghost   1\n---\n".encode()
    with open(path, "wb") as f:
        f.write(hdr + np.ascontiguousarray(a, dtype="<f8").tobytes())


def _numbers_close(a, b, tol):
    """Two text files with the same lines, numbers allowed to differ by tol."""
    la, lb = a.decode().splitlines(), b.decode().splitlines()
    if len(la) != len(lb):
        return False
    worst = 0.0
    for x, y in zip(la, lb):
        if x == y:
            continue
        tx, ty = x.split(), y.split()
        if len(tx) != len(ty):
            return False
        for u, v in zip(tx, ty):
            if u != v:
                worst = max(worst, abs(float(u) - float(v)))
    return worst <= tol


def test_ch_app_output_identical(cuda, tmp_path):
    exes = {"ref": _bin("chapp_ref"), "async": _bin("chapp_phix"), "sync": _bin("chapp_phix")}
    nx, ny, nsteps, every = 160, 96, 1000, 100
    rng = np.random.default_rng(4)
    c0 = 0.5 + rng.uniform(-0.01, 0.01, size=(ny, nx))
    out, files = {}, {}
    for tag, exe in exes.items():
        d = tmp_path / tag
        (d / "settings" / "initial_field").mkdir(parents=True)
        extra = ', "async": false' if tag == "sync" else ""
        (d / "settings" / "settings.jsonc").write_text(
            CH_SETTINGS.format(nx=nx, ny=ny, nsteps=nsteps, every=every, extra=extra))
        _write_field(d / "settings" / "initial_field" / "c.field", "c", c0)
        _write_field(d / "settings" / "initial_field" / "mu.field", "mu", np.zeros_like(c0))
        rc, text = _run(exe, d)
        assert rc == 0, text[-2000:]
        out[tag] = [l for l in text.splitlines() if "written:" in l]
        files[tag] = {n: (d / "output" / n).read_bytes() for n in sorted(os.listdir(d / "output"))}
    names = sorted(files["ref"])
    assert len(names) == 3 * (nsteps // every + 1)
    assert sorted(files["async"]) == sorted(files["sync"]) == names
    assert out["async"] == out["sync"] == out["ref"] and len(out["ref"]) == nsteps // every + 1
    for n in names:
        assert files["async"][n] == files["sync"][n], f"{n}: async and sync output differ"
    worst = 0.0
    for n in names:
        a, b = files["ref"][n], files["async"][n]
        if n.endswith(".field"):
            cut = a.index(b"---\n") + 4
            assert a[:cut] == b[:cut], n
            da, db = np.frombuffer(a[cut:], "<f8"), np.frombuffer(b[cut:], "<f8")
            assert da.shape == db.shape == (nx * ny,)
            worst = max(worst, float(np.abs(da - db).max()))
        else:
            assert _numbers_close(a, b, 1e-12), f"{n}: text differs beyond 1e-12"
    assert worst <= 1e-12, worst
    print(f"CH app: {len(names)} files, async == sync byte for byte, max-abs vs reference {worst:.1e}")


GFA_SETTINGS = """{{
    // written by tests/test_gpu_dropin.py; constants of an Fe-B alloy
    "mesh": {{"nx": {nx}, "ny": {ny}, "dx": 3.0e-4, "dy": 3.0e-4, "x0": 0.0, "y0": 0.0}},
    "initialize": {{"start_from": "initial_field", "dt": 1.0e-6, "nSteps": {nsteps}}},
    "boundary_conditions": {{"x_min": "NoFlux", "x_max": "NoFlux", "y_min": "NoFlux", "y_max": "NoFlux"}},
    "constants": {{"M_eta": 1.0, "D_Am": 3.0e-12, "eps_sq": 2.86e-3, "beta_sq": 1.0e-4, "w_phi": 441.0,
                   "w_eta": 10.0, "w_ex": 100.0, "T": 1000.0, "T_g": 710.0, "alpha": 0.45,
                   "V_m_L": 2.64e-5, "V_m_S": 2.44e-5}},
    "output": {{"print_interval": {every}, "write_interval": {every}, "format": "ALL"}}
}}
"""


def test_gfa_app_identical(cuda, tmp_path):
    exes = {"ref": _bin("gfa_ref"), "ours": _bin("gfa_phix")}
    nx, ny, nsteps, every = 96, 64, 300, 100
    # an amorphous matrix (eta = 1, c = 0.25) around a crystalline disc of
    # radius 3 cells (phi = 1, eta = 0, c = 0.33 + noise)
    rng = np.random.default_rng(5)
    jj, ii = np.mgrid[0:ny, 0:nx]
    disc = (ii + 0.5 - nx / 2) ** 2 + (jj + 0.5 - ny / 2) ** 2 <= 9.0
    c0 = np.where(disc, 0.33 + rng.uniform(-0.01, 0.01, size=(ny, nx)), 0.25)
    phi0 = np.where(disc, 1.0, 0.0)
    eta0 = np.where(disc, 0.0, 1.0)
    out, files, logs = {}, {}, {}
    for tag, exe in exes.items():
        d = tmp_path / tag
        (d / "settings" / "initial_field").mkdir(parents=True)
        (d / "settings" / "settings.jsonc").write_text(GFA_SETTINGS.format(nx=nx, ny=ny, nsteps=nsteps, every=every))
        for name, a in (("c", c0), ("phi", phi0), ("eta", eta0), ("mu", np.zeros_like(c0))):
            _write_field(d / "settings" / "initial_field" / f"{name}.field", name, a)
        rc, text = _run(exe, d)
        assert rc == 0, text[-2000:]
        logs[tag] = text.splitlines()
        out[tag] = [l for l in text.splitlines() if "written:" in l]
        files[tag] = {n: (d / "output" / n).read_bytes() for n in sorted(os.listdir(d / "output"))}
    names = sorted(files["ref"])
    assert sorted(files["ours"]) == names and len(names) == 3 * 3 * (nsteps // every + 1)
    assert out["ours"] == out["ref"]
    worst = 0.0
    for n in names:
        a, b = files["ref"][n], files["ours"][n]
        if n.endswith(".field"):
            cut = a.index(b"---\n") + 4
            da, db = np.frombuffer(a[cut:], "<f8"), np.frombuffer(b[cut:], "<f8")
            assert np.isfinite(da).all(), f"{n}: the reference wrote non-finite values\n" + "\n".join(logs["ref"][-12:])
            worst = max(worst, float(np.abs(da - db).max()))
    for n in names:
        assert files["ours"][n] == files["ref"][n], f"{n}: differs from the reference (field max-abs {worst:.3e})"
    print(f"GFA app: {len(names)} files identical to the reference's")


CHAC_SETTINGS = """{{
    // written by tests/test_gpu_dropin.py
    "mesh": {{"nx": {nx}, "ny": {ny}, "dx": 1.0, "dy": 1.0, "x0": 0.0, "y0": 0.0}},
    "initialize": {{"start_from": "initial_field", "dt": 0.005, "nSteps": {nsteps}}},
    "boundary_conditions": {{"x_min": "Periodic", "x_max": "Periodic", "y_min": "NoFlux", "y_max": "NoFlux"}},
    "constants": {{"rho": 1.4142135623730951, "ca": 0.3, "cb": 0.7, "kappa_c": 3.0, "kappa_eta": 3.0,
                   "M": 5.0, "L": 5.0, "w": 1.0}},
    "output": {{"print_interval": {every}, "write_interval": {every}, "format": "ALL"}}
}}
"""


def test_chac_app_identical(cuda, tmp_path):
    exes = {"ref": _bin("chacapp_ref"), "ours": _bin("chacapp_phix")}
    nx, ny, nsteps, every = 128, 96, 600, 200
    rng = np.random.default_rng(6)
    c0 = 0.5 + rng.uniform(-0.05, 0.05, size=(ny, nx))
    eta0 = rng.uniform(0.0, 0.1, size=(ny, nx))
    out, files = {}, {}
    for tag, exe in exes.items():
        d = tmp_path / tag
        (d / "settings" / "initial_field").mkdir(parents=True)
        (d / "settings" / "settings.jsonc").write_text(CHAC_SETTINGS.format(nx=nx, ny=ny, nsteps=nsteps, every=every))
        for name, a in (("c", c0), ("eta", eta0), ("mu", np.zeros_like(c0))):
            _write_field(d / "settings" / "initial_field" / f"{name}.field", name, a)
        rc, text = _run(exe, d)
        assert rc == 0, text[-2000:]
        out[tag] = [l for l in text.splitlines() if "written:" in l]
        files[tag] = {n: (d / "output" / n).read_bytes() for n in sorted(os.listdir(d / "output"))}
    names = sorted(files["ref"])
    assert sorted(files["ours"]) == names and len(names) == 2 * 3 * (nsteps // every + 1)
    assert out["ours"] == out["ref"]
    for n in names:
        if n.endswith(".field") and files["ours"][n] != files["ref"][n]:
            a, b = files["ref"][n], files["ours"][n]
            cut = a.index(b"---\n") + 4
            da, db = np.frombuffer(a[cut:], "<f8"), np.frombuffer(b[cut:], "<f8")
            pytest.fail(f"{n}: max-abs {np.abs(da - db).max():.3e} against the reference")
        assert files["ours"][n] == files["ref"][n], n
    print(f"CH+AC app: {len(names)} files identical to the reference's")


def _run_until(binary, cwd, marker, timeout=600):
    """Runs a driver until a line containing `marker` is printed, then stops
    it (the develop drivers loop for 1e8 steps); returns the printed lines."""
    import time
    p = subprocess.Popen([binary], cwd=cwd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    lines, t0 = [], time.time()
    try:
        for line in p.stdout:
            lines.append(line.rstrip("\n"))
            if marker in line or time.time() - t0 > timeout:
                break
    finally:
        p.terminate()
        try:
            p.wait(timeout=60)
        except subprocess.TimeoutExpired:
            p.kill()
            p.wait()
    return lines


@pytest.mark.parametrize("driver,marker", [("devch", "written: output/c_10000.field"),
                                           ("ostwald", "written: output/eta_10000.field")])
def test_develop_manual_loop_drivers_identical(cuda, tmp_path, driver, marker):
    logs, files = {}, {}
    for tag in ("ref", "phix"):
        d = tmp_path / tag
        d.mkdir()
        lines = _run_until(_bin(f"{driver}_{tag}"), d, marker)
        assert any(marker in l for l in lines), "\n".join(lines[-20:])
        logs[tag] = [l for l in lines if "written:" in l or "progress" in l]
        files[tag] = {n: (d / "output" / n).read_bytes() for n in sorted(os.listdir(d / "output"))}
    assert logs["phix"] == logs["ref"]
    names = [n for n in sorted(files["ref"]) if int(n.split("_")[1].split(".")[0]) <= 10000]
    assert len(names) >= (4 if driver == "devch" else 8)
    for n in names:
        a, b = files["ref"][n], files["phix"].get(n)
        assert b is not None, n
        if a != b:
            cut = a.index(b"---\n") + 4
            da, db = np.frombuffer(a[cut:], "<f8"), np.frombuffer(b[cut:], "<f8")
            pytest.fail(f"{driver} {n}: max-abs {np.abs(da - db).max():.3e} against the reference")
    print(f"{driver}: {len(names)} files identical to the reference's")

"""FP64 parity with the reference's own GPU build at the benchmark step counts.

tests/golden/fullsteps_ref_gpu.json holds, per case, the digest of the final
state of the reference library's Solver / VectorSolver GPU path (compiled from
its sources for sm_100a, run once on a B200 by tests/golden/gen_fullsteps.py):
the SHA-256 of the physical cells, a strided sample, mass and moments.  These
tests run the library's fused FP64 path for the same full step counts from the
same seeded inputs and require the same bits (equal hashes; the sample is
compared to <= 1e-12 first, so a mismatch reports its size), mass conserved to
<= 1e-12 relative, and (CH+AC) the FP32 path's relative L2 error against the
FP64 result, which is printed.

    CH 1024^2, periodic, single-equation RK4, dt 0.005, 20000 steps (seed 1)
    CH+AC 256^3, zero-flux x, periodic y/z, RK4, dt 0.002, 5000 steps (seed 2)
"""
import hashlib
import json
import os

import numpy as np
import pytest
import torch

import phix_b200 as px
from phix_b200 import workloads

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(__file__), "golden", "fullsteps_ref_gpu.json")


def _fixture(name):
    if not os.path.exists(FIXTURE):
        pytest.fail(f"{FIXTURE} missing (generated by tests/golden/gen_fullsteps.py on a B200)")
    with open(FIXTURE) as f:
        cases = json.load(f)["cases"]
    if name not in cases:
        pytest.fail(f"case {name} not in {FIXTURE}")
    return cases[name]


def _phys(g, a):
    gh = g.ghost
    return np.ascontiguousarray(a[gh:gh + g.n[2], gh:gh + g.n[1], gh:gh + g.n[0]], dtype="<f8")


def _run(name, precision):
    g, phys, prm, scheme, dt, nsteps, fields = getattr(workloads, name)()
    st = px.Stepper(phys, scheme, precision, prm, dt, g)
    d = [torch.from_numpy(f).cuda() for f in fields]
    st.load(d)
    st.set_graph(50)
    st.advance(nsteps)
    st.store(d)
    torch.cuda.synchronize()
    st.status()
    st.close()
    return g, fields, [x.cpu().numpy() for x in d], nsteps


def _check_against_fixture(name):
    rec = _fixture(name)
    g, fields, out, nsteps = _run(name, px.F64)
    assert nsteps == rec["nsteps"]
    vol = float(np.prod([g.d[i] for i in range(g.dim)]))
    for f, (a, want) in enumerate(zip(out, rec["fields"])):
        p = _phys(g, a).reshape(-1)
        sample = p[want["offset"]::want["stride"]][:len(want["sample"])]
        dev = float(np.abs(sample - np.asarray(want["sample"])).max())
        print(f"{name} field {f}: sample max-abs vs reference GPU {dev:.3e}")
        assert dev <= 1e-12
        assert hashlib.sha256(p.tobytes()).hexdigest() == want["sha256"], "bits differ from the reference GPU build"
        mass = float(np.sum(p) * vol)
        assert mass == pytest.approx(want["mass"], rel=1e-14, abs=0.0)
    # conserved field (c): mass drift over the whole run
    m0 = rec["mass0"][0]
    drift = abs(float(np.sum(_phys(g, out[0])) * vol) - m0) / abs(m0)
    print(f"{name}: mass drift of c over {nsteps} steps {drift:.2e} (relative)")
    assert drift <= 1e-12
    return g, out


def test_ch2d_1024_20000_steps_equals_reference_gpu(cuda):
    _check_against_fixture("ch2d")


def test_chac3d_256_5000_steps_equals_reference_gpu(cuda):
    g, out64 = _check_against_fixture("chac3d")
    # FP32 stencils (compensated state, FP64 reductions) against that result
    _, _, out32, _ = _run("chac3d", px.F32)
    for f, (a, b) in enumerate(zip(out32, out64)):
        pa, pb = _phys(g, a), _phys(g, b)
        rel = float(np.linalg.norm(pa - pb) / np.linalg.norm(pb))
        print(f"chac3d field {f}: FP32 rel-L2 vs FP64 after 5000 steps {rel:.2e}")
        assert rel <= 1e-5

"""Fixtures of the reference GPU build at the benchmark step counts.

Runs the reference library compiled from its sources (oracle/_ref, its own
Solver / VectorSolver GPU path built for sm_100a) once per case, from the same
seeded inputs as phix_b200.workloads, and writes for every field of the final
state:
  * the SHA-256 of the physical cells (FP64, C order (z, y, x), little endian);
  * a strided sample of the physical cells (every `stride`-th cell in that
    order, from offset `stride // 2`);
  * mass (numpy float64 sum of the physical cells times the cell volume),
    min, max and the sum of squares;
plus the initial mass of every field.

Cases (the benchmark configurations' full sizes and step counts):
  ch2d    CH 1024^2 periodic, single-equation RK4, dt=0.005, 20000 steps, seed 1
  chac3d  CH+AC 256^3, zero-flux x, periodic y/z, RK4, dt=0.002, 5000 steps, seed 2

The reference's CH step takes about 58 ms at 1024^2 and the coupled 3-D step
far longer, so this is run once on a B200 and the JSON is committed; the -m
gpu tests (tests/test_gpu_fullsteps.py) compare the library's fused FP64 path
against it at the same step counts.

    python tests/golden/gen_fullsteps.py --out tests/golden/fullsteps_ref_gpu.json [--case ch2d] [--check-mine]

--check-mine also runs the library's fused FP64 stepper and prints whether
its bits equal the reference's (max-abs over every physical cell).
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

SAMPLES = 1024


def phys_view(g, a):
    gh = g.ghost
    return a[gh:gh + g.n[2], gh:gh + g.n[1], gh:gh + g.n[0]]


def summarize(g, a, samples=SAMPLES):
    """Digest of one stored FP64 field: hash, sample, mass and moments of its physical cells."""
    p = np.ascontiguousarray(phys_view(g, a), dtype="<f8")
    flat = p.reshape(-1)
    stride = max(1, flat.size // samples)
    vol = float(np.prod([g.d[i] for i in range(g.dim)]))
    return {
        "sha256": hashlib.sha256(p.tobytes()).hexdigest(),
        "stride": stride,
        "offset": stride // 2,
        "sample": [float(v) for v in flat[stride // 2::stride][:samples]],
        "mass": float(np.sum(flat) * vol),
        "min": float(flat.min()),
        "max": float(flat.max()),
        "sumsq": float(np.dot(flat, flat)),
    }


def case_inputs(name):
    from phix_b200 import workloads
    return getattr(workloads, name)()


def run_reference(name, nsteps_override=0):
    from oracle.oracle import Grid, Reference
    g, phys, prm, scheme, dt, nsteps, fields = case_inputs(name)
    nsteps = nsteps_override or nsteps
    grid = Grid(n=tuple(g.n[a] for a in range(g.dim)), d=tuple(g.d[a] for a in range(g.dim)), ghost=g.ghost,
                bc=tuple(g.bc_type), bc_val=tuple(g.bc_val))
    ref = [f.copy() for f in fields]
    vol = float(np.prod([g.d[i] for i in range(g.dim)]))
    mass0 = [float(np.sum(phys_view(g, f)) * vol) for f in fields]
    t0 = time.time()
    ms = Reference().advance(ref, phys, prm, scheme, dt, nsteps, grid, use_gpu=True)
    wall = time.time() - t0
    out = {
        "case": name,
        "n": [int(g.n[a]) for a in range(g.dim)],
        "phys": int(phys), "prm": [float(v) for v in prm], "scheme": int(scheme), "dt": float(dt),
        "nsteps": int(nsteps),
        "bc": [int(v) for v in g.bc_type],
        "mass0": mass0,
        "fields": [summarize(g, a) for a in ref],
        "reference_ms_per_step": ms / nsteps,
        "reference_wall_s": wall,
    }
    return out, ref


def run_mine(name):
    import torch
    import phix_b200 as px
    g, phys, prm, scheme, dt, nsteps, fields = case_inputs(name)
    st = px.Stepper(phys, scheme, px.F64, prm, dt, g)
    d = [torch.from_numpy(f).cuda() for f in fields]
    st.load(d)
    st.set_graph(50)
    st.advance(nsteps)
    st.store(d)
    torch.cuda.synchronize()
    st.close()
    return g, [x.cpu().numpy() for x in d]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out")
    ap.add_argument("--case", action="append", choices=["ch2d", "chac3d"])
    ap.add_argument("--check-mine", action="store_true")
    ap.add_argument("--probe", type=int, default=0, help="time N reference steps per case, write nothing")
    args = ap.parse_args()
    cases = args.case or ["ch2d", "chac3d"]
    if args.probe:
        for name in cases:
            rec, _ = run_reference(name, args.probe)
            print(f"{name}: reference {args.probe} steps, {rec['reference_ms_per_step']:.3f} ms/step", flush=True)
        return
    if not args.out:
        ap.error("--out is required")
    doc = {}
    if os.path.exists(args.out):
        with open(args.out) as f:
            doc = json.load(f)
    doc.setdefault("generator", "tests/golden/gen_fullsteps.py")
    doc.setdefault("source", "reference library compiled from its sources (oracle/_ref), Solver/VectorSolver GPU path, sm_100a")
    doc.setdefault("cases", {})
    for name in cases:
        rec, ref = run_reference(name)
        print(f"{name}: reference {rec['nsteps']} steps, {rec['reference_ms_per_step']:.3f} ms/step, "
              f"wall {rec['reference_wall_s']:.1f} s", flush=True)
        if args.check_mine:
            g, mine = run_mine(name)
            d = max(float(np.abs(phys_view(g, a) - phys_view(g, b)).max()) for a, b in zip(mine, ref))
            same = all(summarize(g, a)["sha256"] == s["sha256"] for a, s in zip(mine, rec["fields"]))
            print(f"{name}: fused FP64 path vs reference max-abs {d:.3e}, sha256 equal: {same}", flush=True)
            rec["fused_f64_max_abs"] = d
        doc["cases"][name] = rec
        with open(args.out, "w") as f:
            json.dump(doc, f, indent=1)
            f.write("\n")


if __name__ == "__main__":
    main()

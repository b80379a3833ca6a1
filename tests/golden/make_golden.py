"""Generates the golden fixtures in tests/golden/.

The reference runs only as WebGL2 shaders (no graphics stack here) and ships
no golden vectors, so the fixtures come from this repository's restatements:
the host setup (grid, cut-cell geometry, parameter block, initial state) and
the CPU oracle's state after a few steps, for three small seeded cases. They
pin both restatements against regressions and give the GPU tests a fixed
target. Run from the repository root:

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

CASES = {
    "plain": ("plain_small", dict(Nx=96, Nr=36), 300),
    "viscous": ("viscous_plume", dict(Nx=96, Nr=36), 300),
    "spray": ("injector_spray", dict(Nx=96, Nr=36), 200),
}


def digest(a):
    a = np.ascontiguousarray(a)
    return hashlib.sha256(a.tobytes()).hexdigest()


def case_setup(rn, name):
    from rocket_nozzle_cfd_solver_b200 import configs
    fn, kw, steps = CASES[name]
    cfg = getattr(configs, fn)(**kw)[0]
    return rn.build_sim_setup(cfg), steps


def setup_record(s):
    init = s.initialState()
    P = {k: v for k, v in s.P.items() if k not in ("injData", "spray")}
    rec = {
        "Nx": s.Nx, "Nr": s.Nr, "dx": s.dx, "iExit": s.iExit, "jExit": s.jExit, "iChamber": s.iChamber,
        "iThroat": s.iThroat, "nCut": s.geo["nCut"], "nMerged": s.geo["nMerged"],
        "sha256": {"mask": digest(s.mask), "geoA": digest(s.geo["geoA"]), "geoG": digest(s.geo["geoG"]),
                   "geoM": digest(s.geo["geoM"]), "jWall": digest(s.geo["jWall"]), "A0": digest(init["A"]),
                   "B0": digest(init["B"])},
        "P": json.loads(json.dumps(P, default=float)),
    }
    if s.injector is not None:
        rec["sha256"]["injector"] = digest(s.injector["tab"])
    return rec


def main():
    import __graft_entry__ as ge
    rn = ge.load_package()
    oracle = ge.load_oracle()
    oracle.set_threads(1)
    records = {}
    for name in CASES:
        s, steps = case_setup(rn, name)
        records[name] = setup_record(s)
        o = oracle.OracleSolver(s.Nx, s.Nr)
        o.setGeometry(s.geo)
        init = s.initialState()
        o.setState(init["A"], init["B"])
        if s.injector is not None:
            o.setInjector(s.injector)
        o.step(steps, s.P)
        st = o.readAll()
        out = {"A": st["A"].astype(np.float32), "B": st["B"].astype(np.float32),
               "stepinfo": o.readStepInfo().astype(np.float32), "steps": np.int32(steps)}
        if s.injector is not None:
            par = o.readParcels()
            out["PA"] = par["PA"].astype(np.float32)
            out["PB"] = par["PB"].astype(np.float32)
            out["src"] = o.readSrc().astype(np.float32)
        np.savez_compressed(os.path.join(HERE, f"oracle_{name}.npz"), **out)
        records[name]["oracle_steps"] = steps
        print(name, s.Nx, s.Nr, steps, "steps")
    with open(os.path.join(HERE, "setup_golden.json"), "w") as f:
        json.dump(records, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()

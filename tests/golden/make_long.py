"""Oracle references for the configuration-length parity tests
(tests/test_gpu_long_parity.py): the viscous plume 512 x 192 to 10k steps from
cold starts at 0 km and 20 km, and the injector + spray chamber 512 x 192 with
its ring pre-populated with 65,536 parcels to about 2 ms of simulated time.

The CPU oracle (oracle/, the restatement of the reference's shader passes) is
deterministic: the same library gives the same bits on any host, whatever the
thread count (its only cross-row reduction, the CFL maximum, is exact). The
full horizons take the oracle minutes (10k steps of 98,304 cells per run), so
they are computed once here and committed: per checkpoint the exit thrust,
exhaust mass flow and chamber pressure (FP32 oracle; at the last checkpoint
also the FP64 oracle's), and every 4th cell of the state in each direction
(FP32 oracle) for the per-field relative L2 on that subsample.

Run from the repository root: python tests/golden/make_long.py
(about 25 minutes on 8 cores). Writes tests/golden/long_runs.npz."""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import __graft_entry__ as ge  # noqa: E402

STRIDE = 4
PLUME_CHECKPOINTS = (1000, 2500, 5000, 10000)
SPRAY_T_END_S = 2e-3
SPRAY_CHUNK = 50


def readouts(rn, s, state):
    """Exit thrust (N), exhaust mass flow (kg/s) and chamber pressure (Pa)."""
    A = np.asarray(state["A"]).reshape(s.Nr, s.Nx, 4)
    B = np.asarray(state["B"]).reshape(s.Nr, s.Nx, 4)
    col = {"A": A[:, s.iExit].ravel(), "B": B[:, s.iExit].ravel()}
    perf = rn.exit_performance(s, col)
    ch = rn.cell_prim_si(s, A[0, s.iChamber], B[0, s.iChamber])
    return np.array([perf["F"], perf["mdot"], ch["p"]])


def subsample(s, state):
    A = np.asarray(state["A"], np.float32).reshape(s.Nr, s.Nx, 4)[::STRIDE, ::STRIDE]
    B = np.asarray(state["B"], np.float32).reshape(s.Nr, s.Nx, 4)[::STRIDE, ::STRIDE]
    return np.concatenate([A, B], axis=-1)


def plume_case(rn, oracle, alt_km):
    from rocket_nozzle_cfd_solver_b200 import configs
    s = rn.build_sim_setup(configs.viscous_plume(alt_km=alt_km)[0])
    init = s.initialState()
    out = {}
    o = oracle.OracleSolver(s.Nx, s.Nr)
    o.setGeometry(s.geo)
    o.setState(init["A"], init["B"])
    done, ro, sub = 0, [], []
    for n in PLUME_CHECKPOINTS:
        o.step(n - done, s.P)
        done = n
        st = o.readAll()
        ro.append(readouts(rn, s, st))
        sub.append(subsample(s, st))
        print(f"  plume {alt_km} km: {n} steps", flush=True)
    o.close()
    out["readouts"] = np.array(ro)
    out["sub"] = np.array(sub)
    o = oracle.OracleSolver(s.Nx, s.Nr, fp64=True)
    o.setGeometry(s.geo)
    o.setState(init["A"], init["B"])
    o.step(PLUME_CHECKPOINTS[-1], s.P)
    out["fp64_readouts"] = readouts(rn, s, o.readAll())
    o.close()
    return out


def spray_case(rn, oracle):
    from rocket_nozzle_cfd_solver_b200 import configs
    s = rn.build_sim_setup(configs.injector_spray(512, 192)[0])
    PA, PB, head = configs.prepopulated_parcels(s, 65536)
    init = s.initialState()
    o = oracle.OracleSolver(s.Nx, s.Nr)
    o.setGeometry(s.geo)
    o.setState(init["A"], init["B"])
    o.setInjector(s.injector)
    o.setParcels(PA, PB, head)
    steps, t = 0, 0.0
    t_end = SPRAY_T_END_S / s.tScale
    while t < t_end:
        o.step(SPRAY_CHUNK, s.P)
        steps += SPRAY_CHUNK
        t = float(o.readStepInfo()[2])
    st = o.readAll()
    pb = np.asarray(o.readParcels()["PB"]).reshape(-1, 4)
    live = pb[:, 1] > 0
    parcels = np.array([live.sum(), pb[live & (pb[:, 2] < 0.5), 1].sum(), pb[live & (pb[:, 2] >= 0.5), 1].sum()])
    o.close()
    print(f"  spray: {steps} steps, t = {t * s.tScale * 1e3:.4f} ms", flush=True)
    return {"steps": np.array(steps), "t": np.array(t), "readouts": readouts(rn, s, st), "sub": subsample(s, st),
            "parcels": parcels}


def main():
    rn = ge.load_package()
    oracle = ge.load_oracle()
    oracle.set_threads(os.cpu_count() or 1)
    t0 = time.time()
    arrays = {"stride": np.array(STRIDE), "plume_checkpoints": np.array(PLUME_CHECKPOINTS)}
    for alt in (0, 20):
        for k, v in plume_case(rn, oracle, alt).items():
            arrays[f"plume{alt}_{k}"] = v
    for k, v in spray_case(rn, oracle).items():
        arrays[f"spray_{k}"] = v
    np.savez_compressed(os.path.join(HERE, "long_runs.npz"), **arrays)
    print(f"wrote long_runs.npz in {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()

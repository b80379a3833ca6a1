"""Synthetic, seeded workloads with the shapes of the benchmark configurations.

Each function returns a ``cfg`` dict for :func:`build_sim_setup` (SI units,
the keys of the reference's ``cfgFromS``, app.js:201-211) plus the step count
the configuration is quoted on. No dataset is involved: every input is built
by the setup pipeline from these parameters.
"""
import math

from .physics import ENGINE_PRESETS, PROPELLANTS

BASE = dict(base=False, bodyRatio=1.5, mach=0.0, startMode="ramp", rampMs=0.12, order2=True, wallModel="cut",
            minCells=8, Tw=800, inletAbsorb=1.0, injMode=False, hllBlend=1.0)


def plain_small(Nx=256, Nr=96):
    """Cold-gas conical nozzle: gamma 1.4, R 287 (Mw 28.97), p0 20 bar, T0 300 K,
    contraction 4, 15-degree cone, expansion 8, sea level; inviscid MUSCL-HLLC,
    CFL 0.5, 2000 steps."""
    cfg = dict(BASE, prop="coldgas", Dt=0.020, De=0.020 * math.sqrt(8.0), type="cone", bellPct=80, coneAngle=15,
               CR=4, chamberLen=1.4, Pc=20e5, Tc=300.0, gamma=1.4, Mw=28.97, alt=0.0, domainL=0.6, Nx=Nx,
               aspect=Nr / Nx, cfl=0.5, viscous=False, afterburn=False, qAb=0.0, sAir=1.0)
    return cfg, 2000


def viscous_plume(Nx=512, Nr=192, alt_km=0.0):
    """Methalox products, gamma 1.2, T0 3500 K, p0 70 bar, 80 % bell with
    expansion 20 (throat 30 mm); Sutherland + eddy viscosity, wall model at
    800 K, afterburning scalars; 10k steps."""
    Dt = 0.030
    cfg = dict(BASE, prop="methalox", Dt=Dt, De=Dt * math.sqrt(20.0), type="bell", bellPct=80, coneAngle=15,
               CR=5, chamberLen=1.5, Pc=70e5, Tc=3500.0, gamma=1.2, Mw=20.5, alt=alt_km * 1000.0, domainL=1.2,
               Nx=Nx, aspect=Nr / Nx, cfl=0.6, viscous=True, afterburn=True, qAb=3.0, sAir=0.8)
    return cfg, 10000


def injector_spray(Nx=512, Nr=192):
    """Coaxial methalox injector chamber (preset injCoax) at 70 bar with the
    65,536-parcel spray ring; about 2 ms of simulated time."""
    e = ENGINE_PRESETS["injCoax"]
    p = PROPELLANTS[e["prop"]]
    cfg = dict(BASE, prop=e["prop"], Dt=e["Dt"] / 1000, De=max(e["De"], e["Dt"] * 1.02) / 1000, type=e["type"],
               bellPct=e["bellPct"], coneAngle=e["coneAngle"], CR=e["CR"], chamberLen=e["chamberLen"],
               Pc=e["Pc"] * 1e5, Tc=p["Tc"], gamma=p["gamma"], Mw=p["Mw"], alt=e["alt"] * 1000.0,
               domainL=e["domain"], Nx=Nx, aspect=Nr / Nx, cfl=0.6, viscous=True, afterburn=True, qAb=p["qAb"],
               sAir=p["sAir"], OF=p["spray"]["OF"], injTMR=1, injAngle=30)
    cfg.update(e["inj"])
    return cfg, None


def preset(key, Nx, aspect=0.28):
    """Any of the reference's engine presets (physics.js:233-309) as applied by
    app.js:1108-1122 with the app's default settings."""
    e = ENGINE_PRESETS[key]
    p = PROPELLANTS[e["prop"]]
    cfg = dict(BASE, prop=e["prop"], Dt=e["Dt"] / 1000, De=max(e["De"], e["Dt"] * 1.02) / 1000, type=e["type"],
               bellPct=e["bellPct"], coneAngle=e["coneAngle"], CR=e["CR"], chamberLen=e["chamberLen"],
               Pc=e["Pc"] * 1e5, Tc=p["Tc"], gamma=p["gamma"], Mw=p["Mw"], alt=e["alt"] * 1000.0,
               mach=e["mach"], base=e["base"], domainL=e["domain"], Nx=Nx, aspect=aspect, cfl=0.6, viscous=True,
               afterburn=True, qAb=p["qAb"], sAir=p["sAir"], injTMR=1, injAngle=30)
    if p.get("spray"):
        cfg["OF"] = p["spray"]["OF"]
    if "inj" in e:
        cfg.update(e["inj"])
    return cfg


BATCH_SIZES = ((128, 48), (256, 96), (512, 192), (1024, 384))


def batched_instance(rng, size=None):
    """One nozzle of the batched workload: grid uniform over BATCH_SIZES,
    expansion ratio uniform 4-40, p0 log-uniform 10-100 bar, gamma 1.2 or 1.4,
    altitude uniform 0-30 km; viscous with the afterburning scalars (every
    instance has the same physics flags, so all share one batch)."""
    Nx, Nr = size if size is not None else BATCH_SIZES[int(rng.integers(len(BATCH_SIZES)))]
    eps = float(rng.uniform(4.0, 40.0))
    Pc = float(10.0 ** rng.uniform(1.0, 2.0)) * 1e5
    gamma = (1.2, 1.4)[int(rng.integers(2))]
    alt = float(rng.uniform(0.0, 30.0)) * 1000.0
    Dt = 0.030
    cfg = dict(BASE, prop="methalox", Dt=Dt, De=Dt * math.sqrt(eps), type="bell", bellPct=80, coneAngle=15,
               CR=5, chamberLen=1.5, Pc=Pc, Tc=3500.0, gamma=gamma, Mw=20.5, alt=alt, domainL=1.2,
               Nx=Nx, aspect=Nr / Nx, cfl=0.6, viscous=True, afterburn=True, qAb=3.0, sAir=0.8)
    return cfg


def batched(count=64, seed=2024):
    """The batched workload: `count` seeded instances (batched_instance)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    return [batched_instance(rng) for _ in range(count)]


def prepopulated_parcels(setup, n, seed=20261203):
    """A parcel ring already holding ``n`` parcels, for the injector chamber
    ``setup``: each on a seeded uniform draw of the injector table's rows
    (position on that element across its width), diameter lognormal (median
    60 um, sigma 0.4), axial speed 30 m/s (oxidiser) or 120 m/s (fuel) times
    U(0.9, 1.1), and the mass the reference gives a spawned parcel at the
    initial time step (mhat dt / 4). Returns (PA, PB, head) in the ring's
    layout: 65,536 x 4 float32 each, free slots dead, spawning resumes at n."""
    import numpy as np
    from .physics import U_REF
    N = 65536
    if not (0 <= n <= N):
        raise ValueError("parcel count out of range")
    rng = np.random.default_rng(seed)
    tab = np.asarray(setup.injector["tab"], dtype=np.float64).reshape(3, 256, 4)
    P = setup.P
    init = setup.initialState()
    A = init["A"].reshape(-1, 4).astype(np.float64)
    B = init["B"].reshape(-1, 4).astype(np.float64)
    fluid = np.asarray(setup.mask) == 0
    rho = np.maximum(A[:, 0], 1e-7)
    u, v = A[:, 1] / rho, A[:, 2] / rho
    G = np.maximum(B[:, 2], 0.5)
    p = np.maximum((A[:, 3] - 0.5 * rho * (u * u + v * v)) / G, 1e-7)
    w = np.abs(u) + np.abs(v) + 2 * np.sqrt((1 + 1 / G) * p / rho)
    dt = min(P["cfl"] / max(float(w[fluid].max()), P["wFloor"]), P["dtMax"])
    m = P["spray"]["mhat"] * dt / 4
    PA = np.zeros((N, 4), np.float32)
    PB = np.zeros((N, 4), np.float32)
    PA[:, 0] = PA[:, 1] = -1
    rows = rng.integers(0, 256, size=n)
    typ = tab[1, rows, 0]
    PA[:n, 0] = tab[0, rows, 0]
    PA[:n, 1] = np.maximum(tab[0, rows, 1] + (rng.uniform(size=n) - 0.5) * tab[1, rows, 3], 0.05)
    PA[:n, 2] = np.where(typ >= 0.5, 30.0, 120.0) * rng.uniform(0.9, 1.1, size=n) / U_REF
    PB[:n, 0] = 60e-6 * np.exp(0.4 * rng.standard_normal(n))
    PB[:n, 1] = m
    PB[:n, 2] = typ
    PB[:n, 3] = tab[2, rows, 0]
    return PA.reshape(-1), PB.reshape(-1), n % N

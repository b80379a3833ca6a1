"""Grid, wall mask, initial condition and the normalised parameter block.

Host-side restatement of the reference's ``source/simsetup.js``:
``buildSimSetup`` (simsetup.js:7-126), the injector helpers (133-237),
``computeParams`` (257-311) and the read-outs ``exitPerformance`` (314-337),
``chamberPerformance`` (239-250), ``cellPrimSI`` (338-348),
``wallSeparation`` (352-373) and ``summerfieldPoint`` (375-383).

Doubles throughout as in JavaScript; every array the reference keeps in a
``Float32Array`` is a float32 numpy array here.
"""
import math

import numpy as np

from .physics import (CHEM_TAU0, G0, GAMMA_AIR, P_REF, PROPELLANTS, R_REF, RHO_REF, RU,
                      SPRAY_FLUIDS, T_REF, U_REF, atmosphere, build_contour, js_round,
                      mach_from_area_ratio, nozzle_theory)
from .cutcell import build_cut_geometry

f32 = np.float32


def injector_active(cfg):
    """simsetup.js:133-135"""
    p = PROPELLANTS.get(cfg.get("prop")) if cfg.get("prop") else None
    return bool(cfg.get("injMode") and p and p.get("spray"))


def injector_thermo(cfg, ReN, Ge):
    """Single global reaction; heat set so the design O/F reaches Tc (simsetup.js:138-153)."""
    sp = PROPELLANTS[cfg["prop"]]["spray"]
    f, o = SPRAY_FLUIDS[sp["fuel"]], SPRAY_FLUIDS[sp["ox"]]

    def Rn(Mw):
        return (RU / Mw) / R_REF

    Rf, Ro = Rn(f["Mw"]), Rn(o["Mw"])

    def Leff(x):
        return x["L"] + x["cl"] * (x["Tb"] - x["Tinj"])

    eF = Rf * Ge * f["Tb"] / T_REF - Leff(f) / (U_REF * U_REF)
    eO = Ro * Ge * o["Tb"] / T_REF - Leff(o) / (U_REF * U_REF)
    Yo = sp["OF"] / (1 + sp["OF"])
    Yf = 1 - Yo
    burnt = min(Yf, Yo / sp["s"])
    Fres = Yf - burnt
    Rp = (ReN - Fres * Rf) / max(1 - Fres, 1e-3)
    qHat = (ReN * (Ge + 1) * cfg["Tc"] / T_REF - (Yf * eF + Yo * eO)) / burnt
    return {"Rf": Rf, "Ro": Ro, "Rp": Rp, "eF": eF, "eO": eO, "Fres": Fres, "qHat": qHat,
            "s": sp["s"], "fuel": f, "ox": o, "Ge": Ge,
            "fuelVec": [f["rho"], f["Tb"], Leff(f), f["sigma"]],
            "oxVec": [o["rho"], o["Tb"], Leff(o), o["sigma"]]}


def chamber_hardware_contour(c, cfg, on):
    """Annular acoustic cavity next to the injector face (simsetup.js:155-159)."""
    if not on or not ((cfg.get("cavD") or 0) > 0):
        return c
    w = (cfg.get("cavW") or 0) / 100 * c.Rc
    d = cfg["cavD"] / 100 * c.Rc
    base = c._base_radius
    return c.copy_with(lambda x: base(x) + (d if x < w else 0))


def chamber_solids(cfg, c, dx):
    """Pintle post, ring baffles and cavity back wall snapped to cells (simsetup.js:161-175)."""
    out = []

    def snap(v):
        return js_round(v / dx) * dx

    if cfg.get("injType") == "pintle":
        out.append({"x0": -dx, "x1": snap(0.5 * c.Rc), "r0": -dx, "r1": snap(0.22 * c.Rc)})
    n = js_round(cfg.get("baffles") or 0)
    h = snap((cfg.get("baffleH") or 0) / 100 * c.Rc)
    t = max(2 * dx, snap(0.04 * c.Rc))
    k = 1
    while k <= n and h > 0:
        r = snap(k / (n + 1) * c.Rc)
        out.append({"x0": -dx, "x1": h, "r0": r - t / 2, "r1": r + t / 2})
        k += 1
    if (cfg.get("cavD") or 0) > 0:
        w = snap((cfg.get("cavW") or 0) / 100 * c.Rc)
        d = (cfg["cavD"] / 100) * c.Rc
        out.append({"x0": w, "x1": w + max(3 * dx, 0.12 * c.Rt), "r0": c.Rc,
                    "r1": c.Rc + d + max(3 * dx, 0.12 * c.Rt)})
    return out


def build_injector_table(cfg, c, dx, P):
    """Weighted 256 x 3 table of spray elements, filled by largest remainder
    (simsetup.js:181-237). Rows: (x0, r0, angle, speed), (type, drop, cone,
    width), (impingement x, 0, 0, 0); lengths in cells, speeds in U_REF."""
    d = P["injData"]
    Pc = cfg["Pc"]
    dp = (cfg.get("injDP") or 20) / 100 * Pc
    OF = cfg["OF"] if (cfg.get("OF") or 0) > 0 else PROPELLANTS[cfg["prop"]]["spray"]["OF"]
    Vf = 0.8 * math.sqrt(2 * dp / d["fuel"]["rho"]) / U_REF
    Vo = 0.8 * math.sqrt(2 * dp / d["ox"]["rho"]) / U_REF
    Do = (cfg.get("injD") or 1.5) * 1e-3
    n = max(1, js_round(cfg.get("injRings") or 4))
    mf, mo = 1 / (1 + OF), OF / (1 + OF)
    film = min((cfg.get("film") or 0) / 100, 0.5)
    Ri = 0.9 * c.Rc
    deg = math.pi / 180
    C = 1 / dx
    el = []

    def add(type_, weight, x, r, angle, speed, drop, cone, width, xi=0):
        el.append({"type": type_, "weight": weight, "x": x * C, "r": r * C, "angle": angle,
                   "speed": speed, "drop": drop, "cone": cone, "width": width * C, "xi": xi * C})

    x0 = 0.5 * dx

    def ringR(k, m):
        return (k + 0.5) / m * Ri

    def share_of(rs):
        s = 0
        for r in rs:
            s = s + r
        s = s or 1
        return [r / s for r in rs]

    t_ = cfg.get("injType")
    if t_ == "coax":
        rs = [ringR(k, n) for k in range(n)]
        w = share_of(rs)
        g = 1.2 * Do
        for k, r in enumerate(rs):
            add(1, mo * w[k], x0, r, 0, Vo, 0.035 * Do, 3 * deg, 0.5 * Do)
            add(0, 0.5 * mf * (1 - film) * w[k], x0, r + g, 0, 3 * Vf, 0.015 * Do, 8 * deg, 0.4 * Do)
            add(0, 0.5 * mf * (1 - film) * w[k], x0, max(r - g, 0.2 * Do), 0, 3 * Vf, 0.015 * Do, 8 * deg, 0.4 * Do)
    elif t_ == "impinge":
        th = (cfg.get("injAngle") or 30) * deg
        xi = 6 * Do
        dl = xi * math.tan(th)
        rs = [max(ringR(k, n), dl + Do) for k in range(n)]
        w = share_of(rs)
        for k, r in enumerate(rs):
            add(0, mf * (1 - film) * w[k], x0, r + dl, -th, Vf, 0.12 * Do, 1 * deg, 0.5 * Do, xi)
            add(1, mo * w[k], x0, r - dl, th, Vo, 0.12 * Do, 1 * deg, 0.5 * Do, xi)
    elif t_ == "pintle":
        Rp = 0.22 * c.Rc
        Lp = 0.5 * c.Rc
        th = math.atan(math.sqrt(max(cfg.get("injTMR") or 1, 0.01)))
        xt = Lp + 1.5 * dx
        add(1, mo, xt, Rp, th, Vo, 0.04 * Do, 6 * deg, 0.6 * Do)
        add(0, mf * (1 - film), xt, Rp + Do, th, Vf, 0.04 * Do, 6 * deg, 0.6 * Do)
    else:
        m = max(2, n)
        rs = [ringR(k, m) for k in range(m)]
        f = share_of([r for k, r in enumerate(rs) if k % 2 == 0])
        o = share_of([r for k, r in enumerate(rs) if k % 2 == 1])
        a = b = 0
        for k, r in enumerate(rs):
            if k % 2 == 0:
                add(0, mf * (1 - film) * f[a], x0, r, 0, Vf, 0.03 * Do, 4 * deg, 0.6 * Do)
                a += 1
            else:
                add(1, mo * o[b], x0, r, 0, Vo, 0.03 * Do, 4 * deg, 0.6 * Do)
                b += 1
    if film > 0:
        add(0, mf * film, x0, 0.97 * c.Rc, 2 * deg, 0.5 * Vf, 80e-6, 1 * deg, 0.015 * c.Rc)
    total = 0
    for e in el:
        total = total + e["weight"]
    N = 256
    slots = [{"e": e, "q": e["weight"] / total * N} for e in el]
    for s in slots:
        s["n"] = math.floor(s["q"])
    used = sum(s["n"] for s in slots)
    for s in sorted(slots, key=lambda s: -(s["q"] - s["n"])):   # stable, like Array.prototype.sort
        if used < N:
            s["n"] += 1
            used += 1
    tab = np.zeros(N * 3 * 4, dtype=f32)
    t = 0
    for s in slots:
        e = s["e"]
        for _ in range(s["n"]):
            tab[t * 4:t * 4 + 4] = [e["x"], e["r"], e["angle"], e["speed"]]
            tab[(N + t) * 4:(N + t) * 4 + 4] = [e["type"], e["drop"], e["cone"], e["width"]]
            tab[(2 * N + t) * 4:(2 * N + t) * 4 + 4] = [e["xi"], 0, 0, 0]
            t += 1
    return {"tab": tab, "elements": el, "OF": OF}


def chamber_inflow_speed(cfg, c0):
    """1-D subsonic inflow speed for the contraction ratio (simsetup.js:251-254)."""
    M = mach_from_area_ratio(max(cfg["CR"], 1.05), cfg["gamma"], False)
    return M * c0 / math.sqrt(1 + 0.5 * (cfg["gamma"] - 1) * M * M)


def compute_params(cfg, contour, dx, PcSi, pStartSi):
    """Normalised solver parameter block ``P`` (simsetup.js:257-311)."""
    g = cfg["gamma"]
    Ge = 1 / (g - 1)
    Ga = 1 / (GAMMA_AIR - 1)
    atm = atmosphere(cfg.get("alt", 0))
    pa = atm["p"] / P_REF
    rhoa = pa / (atm["T"] / T_REF)
    ca = math.sqrt(GAMMA_AIR * pa / rhoa)
    uinf = cfg.get("mach", 0) * ca
    ReN = (RU / cfg["Mw"]) / R_REF
    TcN = cfg["Tc"] / T_REF
    PcN = PcSi / P_REF
    c0 = math.sqrt(g * ReN * TcN)
    uLim = math.sqrt(2 * g / (g - 1) * ReN * TcN)
    tScale = dx / U_REF
    injOn = injector_active(cfg)
    injData = injector_thermo(cfg, ReN, Ge) if injOn else None
    chem = injOn or (cfg.get("afterburn") is not False and (cfg.get("qAb") or 0) > 0)
    PcTheory = nozzle_theory({"Pc": PcSi, "Tc": cfg["Tc"], "gamma": g, "Mw": cfg["Mw"], "Dt": cfg["Dt"],
                              "De": cfg["De"], "pa": atm["p"]}) if injOn else None
    return {
        "inj": injOn,
        "injData": injData,
        "Rs": [injData["Rf"], injData["Ro"], injData["Rp"]] if injOn else [ReN, ReN, ReN],
        "chamberNu": ([0.01 * chamber_inflow_speed(cfg, c0) * contour.Rc / dx, contour.xt / dx]
                      if injOn else [0, 0]),
        "cap": [1.02 * cfg["Tc"], 1.25 * cfg["Tc"]] if injOn else [2400, 2800],
        "spray": ({"mhat": PcTheory["mdot"] / (2 * math.pi * RHO_REF * U_REF * dx * dx),
                   "mdot": PcTheory["mdot"], "tScale": dx / U_REF, "dx": dx} if injOn else None),
        "gamma": g,
        "amb": [rhoa, uinf, 0, pa],
        "ambCons": [rhoa, rhoa * uinf, 0, pa * Ga + 0.5 * rhoa * uinf * uinf],
        "ambB": [0, 0, Ga, 0],
        "gamR": [min(Ge, Ga), max(Ge, Ga)],
        "inlet": [c0 / (6 * contour.xt / dx), 1 if cfg.get("inletAbsorb") is None else cfg["inletAbsorb"], Ge, Ga],
        "uInlet0": chamber_inflow_speed(cfg, c0),
        "visc": cfg.get("viscous") is not False,
        "chem": chem,
        "gas": [1.0, ReN, T_REF, U_REF / (dx * P_REF)],
        "chemK": ([injData["qHat"], injData["s"], (dx / U_REF) / CHEM_TAU0, pa] if injOn else
                  [(cfg.get("qAb") or 0) * 1e6 / (U_REF * U_REF), max(cfg.get("sAir") or 1, 0.05),
                   (dx / U_REF) / CHEM_TAU0, pa]),
        "Tw": min(cfg.get("Tw") or 800, max(cfg["Tc"], 1)) / T_REF,
        "res": [PcN, TcN, ReN],
        "pStart": min(pStartSi / P_REF, PcN),
        "ramp": 0 if cfg.get("startMode") == "burst" else (cfg["rampMs"] * 1e-3) / tScale,
        "RcCells": (contour.Rc + ((cfg.get("cavD") or 0) / 100 * contour.Rc if injOn else 0)) / dx + 0.5,
        "cfl": cfg.get("cfl") or 0.6,
        "dtMax": 10.0,
        "wFloor": 2.0 * c0 + abs(uinf),
        "vMax": 3.0 * (uLim + c0 + abs(uinf) + ca),
        "hllBlend": 1.0 if cfg.get("hllBlend") is None else cfg["hllBlend"],
        "order2": True if cfg.get("order2") is None else cfg["order2"],
        "ReN": ReN, "RaN": 1.0, "Ta": atm["T"], "pa": atm["p"], "uinf": uinf, "uLimN": uLim,
    }


class SimSetup(dict):
    """Result of :func:`build_sim_setup`; keys mirror the reference's object,
    also readable as attributes."""

    def __getattr__(self, k):
        try:
            return self[k]
        except KeyError:
            raise AttributeError(k)


def build_sim_setup(cfg):
    """User-facing engine parameters -> grid, geometry, P and initial state
    (simsetup.js:7-126). ``cfg`` (SI): Dt, De, type, bellPct, coneAngle, CR,
    chamberLen, Pc, Tc, gamma, Mw, alt, mach, base, bodyRatio, domainL, Nx,
    aspect, startMode, rampMs, minCells, viscous, afterburn, qAb, sAir, Tw,
    inletAbsorb, cfl, order2, hllBlend, wallModel and the injector keys."""
    cfg = dict(cfg)
    Nx = cfg["Nx"]
    Nr = max(16, js_round(Nx * cfg["aspect"]))
    injOn = injector_active(cfg)
    contour = chamber_hardware_contour(build_contour(cfg), cfg, injOn)
    if injOn and not cfg.get("dx"):
        cfg["domainL"] = max(1.3 * contour.xe,
                             1.25 * (contour.Re + max(contour.Rc, contour.Re) * 0.12) / cfg["aspect"])
    dx = cfg["domainL"] / Nx
    nt = 0
    gridLimited = False
    if cfg.get("dx"):
        dx = cfg["dx"]
    else:
        minCells = cfg.get("minCells") or 8
        want = max(minCells, js_round(contour.Rt / dx))
        fit = math.floor(contour.Rt / (contour.xe / (0.75 * Nx)))
        nt = max(3, min(want, max(fit, min(js_round(contour.Rt / dx), want))))
        gridLimited = nt < minCells
        dx = contour.Rt / nt
    atm = atmosphere(cfg.get("alt", 0))
    g = cfg["gamma"]
    Ge = 1 / (g - 1)
    Ga = 1 / (GAMMA_AIR - 1)
    theory = nozzle_theory({"Pc": cfg["Pc"], "Tc": cfg["Tc"], "gamma": g, "Mw": cfg["Mw"],
                            "Dt": cfg["Dt"], "De": cfg["De"], "pa": atm["p"]})

    # wall mask (simsetup.js:37-47)
    tw = max(2.6 * dx, 0.12 * contour.Rt)
    bodyR = max(contour.Rc, contour.Re) * (cfg.get("bodyRatio") or 1.5) + tw if cfg.get("base") else 0
    xBase = contour.xt
    RinCol = np.empty(Nx, dtype=f32)
    for i in range(Nx):
        x = (i + 0.5) * dx
        RinCol[i] = contour.radiusAt(x) if x <= contour.xe else math.inf
    hw = chamber_solids(cfg, contour, dx) if injOn else []
    cut_input = {"Nx": Nx, "Nr": Nr, "dx": dx, "contour": contour, "tw": tw, "base": cfg.get("base"),
                 "xBase": xBase, "bodyR": bodyR, "mode": cfg.get("wallModel") or "cut", "solids": hw}
    geo = build_cut_geometry(cut_input)
    mask = geo["mask"]
    # turbulence length scale and boundary-layer band flag in geoM (simsetup.js:51-63)
    CS, KAPPA = 0.17, 0.41
    geoM = geo["geoM"].reshape(Nr, Nx, 4)
    for i in range(Nx):
        x = (i + 0.5) * dx
        Rin = float(RinCol[i])
        inside = x <= contour.xe
        for j in range(Nr):
            r = (j + 0.5) * dx
            l = CS
            if inside and r < Rin:
                s = x - contour.xt if x > contour.xt else x
                delta = 0.025 * s + (0.05 * contour.Rt if x > contour.xt else 0)
                l = max(CS, min(KAPPA * (Rin - r), 0.09 * delta) / dx)
                if x > contour.xt + 0.5 * contour.Rt and Rin - r < max(2 * dx, delta):
                    geoM[j, i, 2] = f32(float(geoM[j, i, 2]) + 16)
            geoM[j, i, 3] = l

    tScale = dx / U_REF
    P = compute_params(cfg, contour, dx, cfg["Pc"], atm["p"])
    pa, rhoa = P["amb"][3], P["amb"][0]
    ReN, TcN, PcN = P["ReN"], P["res"][1], P["res"][0]

    def initial_state():
        """Initial A, B (simsetup.js:72-102)."""
        A = np.zeros((Nr, Nx, 4), dtype=f32)
        B = np.zeros((Nr, Nx, 4), dtype=f32)
        rho0 = PcN / (ReN * TcN)
        E0 = PcN * Ge
        xs = (np.arange(Nx) + 0.5) * dx
        for j in range(Nr):
            r = (j + 0.5) * dx
            for i in range(Nx):
                x = float(xs[i])
                inNozzle = x <= contour.xe and r < float(RinCol[i])
                if injOn and inNozzle and x < contour.xt:
                    A[j, i] = (rho0, 0, 0, E0)
                    B[j, i, 0] = rho0
                    B[j, i, 1] = rho0 * P["injData"]["Fres"]
                    B[j, i, 2] = Ge
                elif cfg.get("startMode") == "burst" and inNozzle and x < contour.xt:
                    A[j, i] = (rho0, 0, 0, E0)
                    B[j, i, 0] = rho0
                    B[j, i, 1] = rho0
                    B[j, i, 2] = Ge
                elif inNozzle:
                    A[j, i] = (rhoa, 0, 0, pa * Ga)
                    B[j, i, 2] = Ga
                else:
                    A[j, i] = (P["ambCons"][0], P["ambCons"][1], 0, P["ambCons"][3])
                    B[j, i, 2] = Ga
        if not injOn:
            B[:, 0, 3] = P["uInlet0"]
        Af, Bf = A.reshape(-1, 4), B.reshape(-1, 4)
        gm = geo["geoM"].reshape(-1, 4)
        for k in range(Nx * Nr):
            hx, hy = gm[k, 0], gm[k, 1]
            if mask[k] or (hx == 0 and hy == 0):
                continue
            h = k + int(hy) * Nx + int(hx)
            Af[k] = Af[h]
            Bf[k] = Bf[h]
        return {"A": Af.reshape(-1), "B": Bf.reshape(-1)}

    iExit = max(1, min(Nx - 1, math.floor(contour.xe / dx) - 1))
    jExit = 0
    while jExit < Nr and not mask[jExit * Nx + iExit]:
        jExit += 1
    iChamber = max(1, math.floor(0.5 * contour.Lc / dx))
    for s in hw:
        if s["r0"] <= 0:
            iChamber = max(iChamber, math.ceil(s["x1"] / dx) + 2)
    iThroat = math.floor(contour.xt / dx)
    jWall = np.zeros(Nx * 4, dtype=f32)
    for i in range(iExit + 1):
        j = min(Nr - 1, math.floor(float(RinCol[i]) / dx))
        while j > 0 and (mask[j * Nx + i] or geo["kappa"][j * Nx + i] < 0.5):
            j -= 1
        jWall[i * 4] = j
    geo["jWall"] = jWall
    return SimSetup(
        cfg=cfg, Nx=Nx, Nr=Nr, dx=dx, tw=tw, bodyR=bodyR, xBase=xBase, contour=contour, atm=atm,
        theory=theory, mask=mask, geo=geo, P=P, initialState=initial_state, solids=hw,
        cutInput=cut_input, rinCol=RinCol,
        injector=build_injector_table(cfg, contour, dx, P) if injOn else None,
        iExit=iExit, jExit=jExit, iChamber=iChamber, iThroat=iThroat, tScale=tScale,
        resolution={"throatCells": contour.Rt / dx, "exitCells": contour.Re / dx,
                    "gridLimited": gridLimited,
                    "shortened": (not cfg.get("dx")) and Nx * dx < 0.98 * cfg["domainL"]},
    )


def chamber_performance(setup, col):
    """Throat-plane mass flow and unburnt fractions (simsetup.js:239-250)."""
    dx, geo, iThroat, P = setup["dx"], setup["geo"], setup["iThroat"], setup["P"]
    m = mO = mF = 0.0
    Nx = setup["Nx"]
    for j in range(setup["Nr"]):
        if setup["mask"][j * Nx + iThroat]:
            break
        k = j * 4
        rho = max(float(col["A"][k]), 1e-9)
        u = float(col["A"][k + 1]) / rho
        dA = 2 * math.pi * abs(float(geo["Ax"][j * geo["W1"] + iThroat])) * dx * dx
        m += rho * u * dA
        mO += float(col["B"][k + 3]) * u * dA
        mF += float(col["B"][k + 1]) * u * dA
    f = RHO_REF * U_REF
    target = P["spray"]["mdot"] if P["spray"] else 1
    return {"mdot": m * f, "unburntOx": mO * f / max(target, 1e-9), "fuelVapour": mF * f / max(target, 1e-9)}


def exit_performance(setup, col):
    """Exit-plane thrust, mass flow, Mach, pressure and Isp in SI (simsetup.js:314-337)."""
    dx, P = setup["dx"], setup["P"]
    F = mdot = Mw = pw = A = 0.0
    geo = setup.get("geo")
    for j in range(setup["jExit"]):
        k = j * 4
        a0, a1, a2, a3 = (float(col["A"][k + c]) for c in range(4))
        rho = max(a0, 1e-9)
        u = a1 / rho
        v = a2 / rho
        G = float(col["B"][k + 2])
        g = 1 + 1 / G
        p = max((a3 - 0.5 * rho * (u * u + v * v)) / G, 1e-9)
        if geo is not None:
            dA = 2 * math.pi * abs(float(geo["Ax"][j * geo["W1"] + setup["iExit"] + 1])) * dx * dx
        else:
            dA = 2 * math.pi * (j + 0.5) * dx * dx
        c = math.sqrt(g * p / rho)
        m = float(col["B"][k]) * u * dA
        F += (rho * u * u + p - P["amb"][3]) * dA
        mdot += m
        Mw += m * math.sqrt(u * u + v * v) / c
        pw += p * dA
        A += dA
    Fsi = F * P_REF
    mdotSi = mdot * RHO_REF * U_REF
    return {"F": Fsi, "mdot": mdotSi, "Me": Mw / mdot if mdot > 1e-12 else 0,
            "pe": (pw / A if A > 0 else 0) * P_REF,
            "Isp": Fsi / (mdotSi * G0) if mdotSi > 1e-9 else 0}


def cell_prim_si(setup, a, b):
    """One cell's primitive state in SI (simsetup.js:338-348)."""
    G = float(b[2])
    g = 1 + 1 / G
    rho = max(float(a[0]), 1e-9)
    u = float(a[1]) / rho
    v = float(a[2]) / rho
    p = max((float(a[3]) - 0.5 * rho * (u * u + v * v)) / G, 1e-9)
    Y = min(max(float(b[0]) / rho, 0), 1)
    P = setup["P"]
    R = P["Rs"]
    Fv = max(float(b[1]) / rho, 0)
    Ov = max(float(b[3]) / rho, 0) if P["inj"] else 0
    Rmix = (1 - Y) * P["RaN"] + Fv * R[0] + Ov * R[1] + max(Y - Fv - Ov, 0) * R[2]
    T = p / (rho * Rmix) * T_REF
    c = math.sqrt(g * p / rho)
    return {"rho": rho * RHO_REF, "u": u * U_REF, "v": v * U_REF, "p": p * P_REF, "T": T, "Y": Y,
            "M": math.hypot(u, v) / c}


def wall_separation(setup, row, paSi):
    """Separation point from the near-wall row, walking upstream from the exit
    while the flow next to the wall runs backwards (simsetup.js:352-373)."""
    dx, contour, iThroat, iExit = setup["dx"], setup["contour"], setup["iThroat"], setup["iExit"]
    i, gaps, last = iExit, 0, -1
    while i > iThroat + 2 and gaps <= 2:
        k = i * 4
        x = (i + 0.5) * dx
        slope = (contour.radiusAt(x + 0.5 * dx) - contour.radiusAt(x - 0.5 * dx)) / dx
        ut = (float(row[k]) + slope * float(row[k + 1])) / math.hypot(1, slope)
        if ut < 0 or math.hypot(float(row[k]), float(row[k + 1])) < 0.6 * float(row[k + 3]):
            last = i
            gaps = 0
        elif last >= 0 or iExit - i > 2:
            gaps += 1
        i -= 1
    if last < 0 or iExit - last < 3:
        return None
    pSep, kS = math.inf, last * 4
    q = last
    while q >= max(iThroat + 1, last - 30):
        if float(row[q * 4 + 2]) < pSep:
            pSep = float(row[q * 4 + 2])
            kS = q * 4
        q -= 1
    Msep = math.hypot(float(row[kS]), float(row[kS + 1])) / max(float(row[kS + 3]), 1e-6)
    if Msep < 1.05:
        return None
    x = (last + 0.5) * dx
    R = contour.radiusAt(x)
    return {"x": x, "frac": (x - contour.xt) / (contour.xe - contour.xt),
            "eps": (R * R) / (contour.Rt * contour.Rt), "pRatio": pSep * P_REF / max(paSi, 1e-6),
            "Msep": Msep}


def summerfield_point(contour, Pc, g, pa):
    """Where 1-D theory reaches wall p = 0.4 pa (simsetup.js:375-383)."""
    nS = 200
    for k in range(nS + 1):
        x = contour.xt + (contour.xe - contour.xt) * k / nS
        R = contour.radiusAt(x)
        M = mach_from_area_ratio(max((R * R) / (contour.Rt * contour.Rt), 1.0001), g, True)
        if Pc * math.pow(1 + 0.5 * (g - 1) * M * M, -g / (g - 1)) < 0.4 * pa:
            return k / nS
    return None

"""Atmosphere, 1-D isentropic nozzle theory, nozzle contour and presets.

Host-side restatement of the reference's ``source/physics.js`` (all SI units).
JavaScript numbers are IEEE doubles, as are Python floats, so every formula here
is evaluated in the same precision and order as the reference. ``js_round``
reproduces ``Math.round`` (ties toward +infinity), which differs from Python's
``round``.
"""
import math

G0 = 9.80665
RU = 8314.462618            # J/(kmol K)
R_AIR = 287.053             # J/(kg K)
# Normalisation used by the solver (physics.js:10-16)
P_REF = 101325.0
T_REF = 288.15
R_REF = R_AIR
RHO_REF = P_REF / (R_REF * T_REF)     # 1.225 kg/m^3
U_REF = math.sqrt(P_REF / RHO_REF)    # ~287.6 m/s
GAMMA_AIR = 1.4
CHEM_TAU0 = 5.5e-8                    # physics.js:19


def js_round(x):
    """``Math.round``: nearest integer, ties toward +infinity."""
    f = math.floor(x)
    return f + 1 if x - f >= 0.5 else f


# US Standard Atmosphere 1976 (physics.js:24-50)
ISA_LAYERS = [
    (0, 288.15, -0.0065, 101325.0),
    (11000, 216.65, 0.0, 22632.06),
    (20000, 216.65, 0.001, 5474.889),
    (32000, 228.65, 0.0028, 868.0187),
    (47000, 270.65, 0.0, 110.9063),
    (51000, 270.65, -0.0028, 66.93887),
    (71000, 214.65, -0.002, 3.956420),
    (86000, 186.87, 0.0, 0.3734),
]


def atmosphere(h):
    """ISA 1976 temperature/pressure at geopotential altitude ``h`` (physics.js:35-50)."""
    h = max(0.0, min(h, 120000.0))
    L = ISA_LAYERS[0]
    for layer in ISA_LAYERS:
        if h >= layer[0]:
            L = layer
    hb, Tb, lapse, pb = L
    k = G0 / R_AIR
    if abs(lapse) < 1e-12:
        T = Tb
        p = pb * math.exp(-k * (h - hb) / Tb)
    else:
        T = Tb + lapse * (h - hb)
        p = pb * math.pow(Tb / T, k / lapse)
    return {"T": T, "p": p, "rho": p / (R_AIR * T), "a": math.sqrt(1.4 * R_AIR * T)}


def area_ratio_from_mach(M, g):
    """physics.js:55-58"""
    t = (2 / (g + 1)) * (1 + 0.5 * (g - 1) * M * M)
    return math.pow(t, (g + 1) / (2 * (g - 1))) / M


def mach_from_area_ratio(eps, g, supersonic=True):
    """Bisection, 200 iterations (physics.js:59-69)."""
    if eps <= 1.0:
        return 1.0
    lo, hi = (1.0, 100.0) if supersonic else (1e-6, 1.0)
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        f = area_ratio_from_mach(mid, g) - eps
        if supersonic:
            if f > 0:
                hi = mid
            else:
                lo = mid
        else:
            if f > 0:
                lo = mid
            else:
                hi = mid
    return 0.5 * (lo + hi)


def mach_from_pressure_ratio(p0_over_p, g):
    """physics.js:70-72"""
    return math.sqrt(max(0.0, (math.pow(p0_over_p, (g - 1) / g) - 1) * 2 / (g - 1)))


def nozzle_theory(o):
    """Ideal 1-D frozen-gamma performance (physics.js:75-106).

    ``o``: dict with Pc, Tc, gamma, Mw, Dt, De, pa (SI).
    """
    g = o["gamma"]
    R = RU / o["Mw"]
    At = math.pi * 0.25 * o["Dt"] * o["Dt"]
    Ae = math.pi * 0.25 * o["De"] * o["De"]
    eps = Ae / At
    Me = mach_from_area_ratio(eps, g, True)
    fT = 1 + 0.5 * (g - 1) * Me * Me
    pe = o["Pc"] * math.pow(fT, -g / (g - 1))
    Te = o["Tc"] / fT
    ue = Me * math.sqrt(g * R * Te)
    Gam = math.sqrt(g) * math.pow(2 / (g + 1), (g + 1) / (2 * (g - 1)))
    cstar = math.sqrt(R * o["Tc"]) / Gam
    mdot = o["Pc"] * At / cstar
    pa = o["pa"]
    F = mdot * ue + (pe - pa) * Ae
    Fvac = mdot * ue + pe * Ae
    Mopt = mach_from_pressure_ratio(o["Pc"] / max(pa, 1e-3), g)
    epsOpt = area_ratio_from_mach(max(Mopt, 1.0001), g) if pa > 1 else math.inf
    ratio = pe / max(pa, 1e-9)
    if pa < 1:
        state = "vacuum"
    elif ratio > 1.08:
        state = "under-expanded"
    elif ratio < 0.92:
        state = "over-expanded"
    else:
        state = "near-ideal"
    separation = (pa > 1) and pe < 0.4 * pa
    uLim = math.sqrt(2 * g / (g - 1) * R * o["Tc"])
    return {"At": At, "Ae": Ae, "eps": eps, "Me": Me, "pe": pe, "Te": Te, "ue": ue,
            "cstar": cstar, "mdot": mdot, "F": F, "Fvac": Fvac, "Cf": F / (o["Pc"] * At),
            "Isp": F / (mdot * G0), "IspVac": Fvac / (mdot * G0), "epsOpt": epsOpt,
            "ratio": ratio, "state": state, "separation": separation,
            "c0": math.sqrt(g * R * o["Tc"]), "uLim": uLim, "R": R}


def rao_angles(eps, pct):
    """Fits to the Rao 80 % bell charts (physics.js:112-122)."""
    le = math.log10(max(eps, 2))
    thn = 14.5 + 11.0 * le
    the = 16.5 - 5.3 * le
    d = 80 - pct
    thn += d * 0.30
    the += d * 0.22
    thn = min(max(thn, 12), 48)
    the = min(max(the, 2), thn - 4)
    return thn * math.pi / 180, the * math.pi / 180


class Contour:
    """Inner-wall radius against axial position (physics.js:124-199)."""

    def __init__(self, pts, Rt, Re, Rc, Lc, xt, xe, eps, thn, the):
        self.pts = pts
        self.Rt, self.Re, self.Rc, self.Lc = Rt, Re, Rc, Lc
        self.xt, self.xe, self.eps, self.thn, self.the = xt, xe, eps, thn, the
        self.xs = [p[0] for p in pts]
        self.rs = [p[1] for p in pts]
        self._radius_override = None

    def radiusAt(self, x):
        if self._radius_override is not None:
            return self._radius_override(x)
        return self._base_radius(x)

    def _base_radius(self, x):
        """Linear interpolation with a binary search, x monotone (physics.js:190-197)."""
        if x <= 0:
            return self.Rc
        if x >= self.xe:
            return self.Re
        xs = self.xs
        lo, hi = 0, len(xs) - 1
        while hi - lo > 1:
            m = (lo + hi) >> 1
            if xs[m] <= x:
                lo = m
            else:
                hi = m
        t = (x - xs[lo]) / (xs[hi] - xs[lo])
        return self.rs[lo] + t * (self.rs[hi] - self.rs[lo])

    def copy_with(self, radius_fn):
        c = Contour(self.pts, self.Rt, self.Re, self.Rc, self.Lc, self.xt, self.xe,
                    self.eps, self.thn, self.the)
        c._radius_override = radius_fn
        return c


def build_contour(o):
    """Chamber cylinder, fillet, converging cone, throat arcs and a cone or Rao
    parabola (physics.js:124-199). ``o``: Dt, De, type, bellPct, coneAngle, CR, chamberLen."""
    Rt = 0.5 * o["Dt"]
    Re = max(0.5 * o["De"], Rt * 1.001)
    Rc = Rt * math.sqrt(max(o["CR"], 1.5))
    Lc = max(o["chamberLen"] * Rc, 1.5 * Rt)
    thc = 35 * math.pi / 180
    Ru = 1.5 * Rt
    Rf = min(0.6 * Rc, 1.0 * Rt * 1.5)
    pts = []

    def push(x, r):
        if not pts or x > pts[-1][0] + 1e-12:
            pts.append((x, r))

    push(0, Rc)
    push(Lc, Rc)
    nA = 24
    for k in range(1, nA + 1):
        ph = thc * k / nA
        push(Lc + Rf * math.sin(ph), Rc - Rf * (1 - math.cos(ph)))
    x1, r1 = pts[-1]
    r2 = Rt + Ru * (1 - math.cos(thc))
    if r1 > r2:
        x2 = x1 + (r1 - r2) / math.tan(thc)
        push(x2, r2)
        x1, r1 = x2, r2
    xt = x1 + Ru * math.sin(thc)
    for k in range(1, nA + 1):
        ph = thc * (1 - k / nA)
        push(xt - Ru * math.sin(ph), Rt + Ru * (1 - math.cos(ph)))
    Rd = 0.382 * Rt
    eps = (Re * Re) / (Rt * Rt)
    bellPct = o.get("bellPct") or 80
    if o.get("type") == "cone":
        thn = (o.get("coneAngle") or 15) * math.pi / 180
        the = thn
    else:
        thn, the = rao_angles(eps, bellPct)
    for k in range(1, nA + 1):
        ph = thn * k / nA
        push(xt + Rd * math.sin(ph), Rt + Rd * (1 - math.cos(ph)))
    xN, rN = pts[-1]
    if o.get("type") == "cone":
        xe = xN + (Re - rN) / math.tan(thn)
        n = 40
        for k in range(1, n + 1):
            push(xN + (xe - xN) * k / n, rN + (Re - rN) * k / n)
    else:
        L15 = (Re - Rt) / math.tan(15 * math.pi / 180)
        xe = xt + bellPct / 100 * L15
        xe = max(xe, xN + (Re - rN) / math.tan(thn) * 1.02)
        tn, te = math.tan(thn), math.tan(the)
        qx = (Re - rN + xN * tn - xe * te) / (tn - te)
        qx = min(max(qx, xN + 1e-6), xe - 1e-6)
        qr = rN + tn * (qx - xN)
        qr = min(max(qr, rN), Re * 1.2)
        n = 80
        for k in range(1, n + 1):
            s = k / n
            a, b, c = (1 - s) * (1 - s), 2 * s * (1 - s), s * s
            push(a * xN + b * qx + c * xe, a * rN + b * qr + c * Re)
    xe = pts[-1][0]
    return Contour(pts, Rt, Re, Rc, Lc, xt, xe, eps, thn, the)


# Presets (physics.js:215-309)
SPRAY_FLUIDS = {
    "rp1": {"rho": 810, "Tb": 650, "Tinj": 300, "L": 250e3, "cl": 2000, "sigma": 0.02, "Mw": 100},
    "ch4": {"rho": 420, "Tb": 190, "Tinj": 112, "L": 300e3, "cl": 3500, "sigma": 0.005, "Mw": 16},
    "h2": {"rho": 40, "Tb": 60, "Tinj": 40, "L": 20e3, "cl": 14000, "sigma": 0.001, "Mw": 2},
    "lox": {"rho": 1140, "Tb": 155, "Tinj": 90, "L": 150e3, "cl": 1700, "sigma": 0.005, "Mw": 32},
}
PROPELLANTS = {
    "kerolox": {"Tc": 3670, "gamma": 1.22, "Mw": 22.0, "qAb": 6.8, "sAir": 1.8,
                "spray": {"OF": 2.3, "s": 3.4, "fuel": "rp1", "ox": "lox"}},
    "methalox": {"Tc": 3550, "gamma": 1.21, "Mw": 20.5, "qAb": 3.0, "sAir": 0.8,
                 "spray": {"OF": 3.0, "s": 4.0, "fuel": "ch4", "ox": "lox"}},
    "hydrolox": {"Tc": 3400, "gamma": 1.20, "Mw": 13.5, "qAb": 4.2, "sAir": 1.2,
                 "spray": {"OF": 6.0, "s": 8.0, "fuel": "h2", "ox": "lox"}},
    "hybrid": {"Tc": 3150, "gamma": 1.23, "Mw": 26.0, "qAb": 2.0, "sAir": 0.5},
    "solid": {"Tc": 3100, "gamma": 1.20, "Mw": 25.0, "qAb": 4.6, "sAir": 1.2},
    "hydrazine": {"Tc": 1150, "gamma": 1.28, "Mw": 13.0, "qAb": 14.0, "sAir": 4.2},
    "coldgas": {"Tc": 300, "gamma": 1.40, "Mw": 28.0, "qAb": 0, "sAir": 1},
    "custom": {"Tc": 3000, "gamma": 1.22, "Mw": 22.0, "qAb": 3.0, "sAir": 1},
}
CHAMBER_HW = {"film": 0, "baffles": 0, "baffleH": 30, "cavD": 0, "cavW": 40}


def _preset(prop, Pc, Dt, De, type_, CR, chamberLen, alt, mach, base, domain, inj=None, bellPct=80, coneAngle=15):
    e = {"prop": prop, "Pc": Pc, "Dt": Dt, "De": De, "type": type_, "bellPct": bellPct,
         "coneAngle": coneAngle, "CR": CR, "chamberLen": chamberLen, "alt": alt, "mach": mach,
         "base": base, "domain": domain}
    if inj is not None:
        e["inj"] = inj
    return e


ENGINE_PRESETS = {
    "injShower": _preset("kerolox", 70, 30, 85, "bell", 5, 6, 0, 0, False, 0.5,
                         {"injMode": True, "injType": "shower", "injRings": 6, "injDP": 20, "injD": 1.5, **CHAMBER_HW}),
    "injCoax": _preset("methalox", 70, 30, 85, "bell", 5, 6, 0, 0, False, 0.5,
                       {"injMode": True, "injType": "coax", "injRings": 4, "injDP": 15, "injD": 2, **CHAMBER_HW}),
    "injImpinge": _preset("kerolox", 70, 30, 85, "bell", 5, 6, 0, 0, False, 0.5,
                          {"injMode": True, "injType": "impinge", "injRings": 4, "injDP": 20, "injD": 1.2,
                           "injAngle": 30, **CHAMBER_HW}),
    "injPintle": _preset("kerolox", 70, 30, 85, "bell", 5, 6, 0, 0, False, 0.5,
                         {"injMode": True, "injType": "pintle", "injRings": 1, "injDP": 20, "injD": 1,
                          "injTMR": 0.4, **CHAMBER_HW}),
    "injHardware": _preset("kerolox", 70, 30, 85, "bell", 5, 6, 0, 0, False, 0.5,
                           {"injMode": True, "injType": "impinge", "injRings": 4, "injDP": 20, "injD": 1.2,
                            "injAngle": 30, **CHAMBER_HW, "film": 10, "baffles": 1, "baffleH": 30,
                            "cavD": 12, "cavW": 40}),
    "demo": _preset("kerolox", 196, 23, 119, "bell", 6, 1.6, 0, 0, False, 1.2),
    "overexp": _preset("hydrolox", 120, 20, 160, "bell", 5, 1.4, 0, 0, False, 1.4),
    "diamonds": _preset("methalox", 90, 30, 125, "bell", 5, 1.5, 0, 0, False, 1.2),
    "ideal": _preset("kerolox", 70, 34, 99, "bell", 5, 1.5, 0, 0, False, 1.2),
    "underexp": _preset("kerolox", 80, 30, 70, "bell", 5, 1.5, 22, 0, False, 1.4),
    "coldgas": _preset("coldgas", 20, 20, 30, "cone", 4, 1.4, 0, 0, False, 0.6),
    "hybrid": _preset("hybrid", 30, 30, 64, "cone", 4, 2.0, 0, 0, False, 1.0, coneAngle=12),
    "upper": _preset("hydrolox", 100, 16, 100, "bell", 5, 1.5, 30, 0, False, 1.4),
    "flight": _preset("kerolox", 100, 26, 90, "bell", 5, 1.5, 12, 2.0, True, 1.2),
}

"""Host-side setup restatement (physics.js, cutcell.js, simsetup.js) on CPU.

Known answers: ISA 1976 table values, isentropic relations; structural
invariants of the cut-cell topology the reference builds (cutcell.js); and the
committed golden digests of the setup for the three small cases.
"""
import json
import math
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_js_round(rn):
    from rocket_nozzle_cfd_solver_b200.physics import js_round
    assert js_round(0.5) == 1 and js_round(1.5) == 2 and js_round(2.5) == 3
    assert js_round(-0.5) == 0 and js_round(-1.5) == -1 and js_round(-2.6) == -3
    assert js_round(0.49999999999999994) == 0


@pytest.mark.parametrize("h,T,p", [(0, 288.15, 101325.0), (11000, 216.65, 22632.06), (20000, 216.65, 5474.889),
                                   (32000, 228.65, 868.0187)])
def test_atmosphere_layer_bases(rn, h, T, p):
    from rocket_nozzle_cfd_solver_b200.physics import atmosphere
    a = atmosphere(h)
    assert a["T"] == pytest.approx(T, rel=1e-12)
    assert a["p"] == pytest.approx(p, rel=2e-4)      # layer base pressures are rounded in the table


def test_isentropic_round_trip(rn):
    from rocket_nozzle_cfd_solver_b200.physics import area_ratio_from_mach, mach_from_area_ratio
    for g in (1.2, 1.4):
        for eps in (1.5, 4.0, 8.0, 40.0):
            Ms = mach_from_area_ratio(eps, g, True)
            Mu = mach_from_area_ratio(eps, g, False)
            assert Ms > 1 > Mu
            assert area_ratio_from_mach(Ms, g) == pytest.approx(eps, rel=1e-9)
            assert area_ratio_from_mach(Mu, g) == pytest.approx(eps, rel=1e-9)
    # isentropic tables, gamma 1.4: A/A* = 4.2346 at M = 3, 1.6875 at M = 2
    assert mach_from_area_ratio(4.2346, 1.4) == pytest.approx(3.0, abs=2e-4)
    assert mach_from_area_ratio(1.6875, 1.4) == pytest.approx(2.0, abs=2e-4)


def test_nozzle_theory_cold_gas(rn):
    from rocket_nozzle_cfd_solver_b200.physics import nozzle_theory
    t = nozzle_theory({"Pc": 20e5, "Tc": 300, "gamma": 1.4, "Mw": 28.97, "Dt": 0.02, "De": 0.02 * math.sqrt(8),
                       "pa": 101325.0})
    # choked mass flow: Pc At / c*, c* = sqrt(R Tc) / Gamma
    R = 8314.462618 / 28.97
    Gam = math.sqrt(1.4) * (2 / 2.4) ** (2.4 / 0.8)
    assert t["cstar"] == pytest.approx(math.sqrt(R * 300) / Gam, rel=1e-12)
    assert t["mdot"] == pytest.approx(20e5 * math.pi * 1e-4 / t["cstar"], rel=1e-12)
    assert t["eps"] == pytest.approx(8.0, rel=1e-12)
    assert t["state"] == "over-expanded"


@pytest.mark.parametrize("kind", ["cone", "bell"])
def test_contour_shape(rn, kind):
    from rocket_nozzle_cfd_solver_b200.physics import build_contour
    c = build_contour({"Dt": 0.03, "De": 0.03 * math.sqrt(20), "type": kind, "bellPct": 80, "coneAngle": 15,
                       "CR": 5, "chamberLen": 1.5})
    xs = np.array(c.xs)
    assert np.all(np.diff(xs) > 0)
    assert c.radiusAt(0.0) == c.Rc and c.radiusAt(c.xe) == pytest.approx(c.Re)
    r = np.array([c.radiusAt(x) for x in np.linspace(0, c.xe, 2001)])
    assert r.min() == pytest.approx(c.Rt, rel=2e-3)
    assert abs(np.linspace(0, c.xe, 2001)[r.argmin()] - c.xt) < 0.02 * c.xe


def cases(rn):
    from rocket_nozzle_cfd_solver_b200 import configs
    return [rn.build_sim_setup(configs.plain_small(96, 36)[0]), rn.build_sim_setup(configs.viscous_plume(96, 36)[0]),
            rn.build_sim_setup(configs.injector_spray(96, 36)[0]), rn.build_sim_setup(configs.plain_small()[0])]


def test_cut_cell_topology_invariants(rn):
    for s in cases(rn):
        Nx, Nr = s.Nx, s.Nr
        g = s.geo
        gm = g["geoM"].reshape(Nr, Nx, 4)
        gg = g["geoG"].reshape(Nr, Nx, 4)
        gA = g["geoA"].reshape(Nr + 1, Nx + 1, 4)
        mask = s.mask.reshape(Nr, Nx)
        kap = g["kappa"].reshape(Nr, Nx)
        for j in range(Nr):
            for i in range(Nx):
                if mask[j, i]:
                    assert gg[j, i, 0] == 1 and np.all(gm[j, i, :2] == 0)
                    # solid cells have all four faces closed
                    assert gA[j, i, 2] == 0 and gA[j, i + 1, 2] == 0 and gA[j, i, 3] == 0 and gA[j + 1, i, 3] == 0
                    continue
                hx, hy = int(gm[j, i, 0]), int(gm[j, i, 1])
                assert abs(hx) + abs(hy) <= 1
                if hx or hy:
                    Hi, Hj = i + hx, j + hy
                    assert not mask[Hj, Hi]
                    assert kap[Hj, Hi] >= 0.5 and kap[j, i] < 0.5       # slivers merge into full cells
                    assert gm[Hj, Hi, 0] == 0 and gm[Hj, Hi, 1] == 0     # hosts are not slaves
                    bit = 1 if i < Hi else 2 if i > Hi else 4 if j < Hj else 8
                    assert int(gm[Hj, Hi, 2]) & bit
                    assert np.all(gg[j, i] == gg[Hj, Hi])              # members share the group sums
                sm = int(gm[j, i, 2]) & 15
                for bit, (di, dj) in ((1, (-1, 0)), (2, (1, 0)), (4, (0, -1)), (8, (0, 1))):
                    if sm & bit:
                        assert (int(gm[j + dj, i + di, 0]), int(gm[j + dj, i + di, 1])) == (-di, -dj)


def test_group_sums_and_closure(rn):
    for s in cases(rn):
        Nx, Nr = s.Nx, s.Nr
        g = s.geo
        Ax = g["Ax"].reshape(Nr + 1, Nx + 1)
        Ar = g["Ar"].reshape(Nr + 1, Nx + 1)
        gA = g["geoA"].reshape(Nr + 1, Nx + 1, 4)
        gg = g["geoG"].reshape(Nr, Nx, 4)
        gm = g["geoM"].reshape(Nr, Nx, 4)
        mask = s.mask.reshape(Nr, Nx)
        for j in range(Nr):
            for i in range(Nx):
                if mask[j, i] or gm[j, i, 0] or gm[j, i, 1] or int(gm[j, i, 2]) & 15:
                    continue
                # a cell that is its own group: group volume = its volume, wall vector by closure
                assert gg[j, i, 0] == gA[j, i, 0]
                wx = np.float32(float(Ax[j, i]) - float(Ax[j, i + 1]))
                wr = np.float32(float(gA[j, i, 1]) - (float(Ar[j + 1, i]) - float(Ar[j, i])))
                wx = np.float32(0) if abs(wx) < 1e-6 else wx
                wr = np.float32(0) if abs(wr) < 1e-6 else wr
                assert gg[j, i, 2] == wx and gg[j, i, 3] == wr
        # open areas carry their sign as the first-order flag only
        assert np.all(np.abs(gA[:Nr, :, 2]) == Ax[:Nr, :])
        assert np.all(np.abs(gA[:, :Nx, 3]) == Ar[:, :Nx])


def test_setup_golden(rn):
    from test_setup_helpers import setup_digests
    with open(os.path.join(HERE, "golden", "setup_golden.json")) as f:
        gold = json.load(f)
    for name, rec in gold.items():
        got = setup_digests(rn, name)
        for k in ("Nx", "Nr", "iExit", "jExit", "iChamber", "iThroat", "nCut", "nMerged"):
            assert got[k] == rec[k], (name, k)
        assert got["dx"] == pytest.approx(rec["dx"], rel=0, abs=0)
        assert got["sha256"] == rec["sha256"], name
        for k, v in rec["P"].items():
            assert got["P"][k] == v, (name, k)


def test_injector_table(rn):
    from rocket_nozzle_cfd_solver_b200 import configs
    s = rn.build_sim_setup(configs.injector_spray(96, 36)[0])
    tab = s.injector["tab"].reshape(3, 256, 4)
    types = tab[1, :, 0]
    assert set(np.unique(types)) <= {0.0, 1.0}
    # slots are filled in proportion to element mass: oxidiser share = OF / (1 + OF) within 1 slot per element
    OF = s.injector["OF"]
    n_ox = int((types == 1).sum())
    assert abs(n_ox - 256 * OF / (1 + OF)) <= len(s.injector["elements"])
    assert np.all(tab[0, :, 0] > 0) and np.all(tab[1, :, 1] > 0)


def test_params_rounding(rn):
    """rn_params carries P rounded to float32 exactly as gl.uniform*fv does."""
    from rocket_nozzle_cfd_solver_b200 import configs
    s = rn.build_sim_setup(configs.viscous_plume(96, 36)[0])
    p = rn.params_from_P(s.P)
    P = s.P
    for n in ("amb", "ambCons", "inlet", "res", "gas", "Rs", "chemK", "cap"):
        assert [float(x) for x in getattr(p, n)] == [float(np.float32(v)) for v in P[n]], n
    assert p.bar[1] == float(np.float32(1.6 * P["uInlet0"]))
    assert p.cfl == float(np.float32(P["cfl"])) and p.visc == 1 and p.chem == 1 and p.inj == 0

"""GPUSolver / GPUSpray: the reference's JavaScript solver API over librn.so.

Mirrors ``GPUSolver`` (source/solver.js:677-1076) and ``GPUSpray``
(source/spray.js:211-321) method for method, with the CUDA library declared in
``include/rn.h`` in place of the WebGL2 context. Textures are named by the
``RN_TEX_*`` ids; ``state`` returns ``{"A": RN_TEX_A, "B": RN_TEX_B}`` so a
caller can build ``requestAsync`` requests exactly as ``app.js`` does.

There is no CPU fallback: constructing a solver without the library or
without a CUDA device raises.
"""
import ctypes
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librn.so")

RN_OK, RN_NOT_READY, RN_BUSY = 0, 1, 2
RN_TEX_A, RN_TEX_B, RN_TEX_STEPINFO, RN_TEX_WALLROW = 0, 1, 2, 3
RN_TEX_PARCEL_A, RN_TEX_PARCEL_B, RN_TEX_PARCEL_C, RN_TEX_INJECTOR = 4, 5, 6, 7
SPRAY_W = SPRAY_H = 256
SPRAY_N = SPRAY_W * SPRAY_H

EXPORTS = ("rn_create", "rn_destroy", "rn_resize", "rn_set_mask", "rn_set_geometry", "rn_set_state",
           "rn_get_state", "rn_step", "rn_rescale_ambient", "rn_draw_wall_row", "rn_read_rect",
           "rn_read_step_info", "rn_request_async", "rn_poll_async", "rn_cancel_async", "rn_spray_set_injector",
           "rn_spray_reset", "rn_spray_stats", "rn_integrals", "rn_sync", "rn_wait", "rn_kernel_launches",
           "rn_set_precision", "rn_get_precision", "rn_get_stream", "rn_profile", "rn_profile_read",
           "rn_integrals_static", "rn_set_tile", "rn_get_tile", "rn_autotune", "rn_batch_create",
           "rn_batch_destroy", "rn_batch_add", "rn_batch_remove", "rn_batch_set_params", "rn_batch_size",
           "rn_batch_step", "rn_batch_run", "rn_batch_sync", "rn_batch_set_tile", "rn_batch_autotune", "rn_batch_stream",
           "rn_batch_kernel_launches", "rn_residual_mark", "rn_residual", "rn_server_default_opts",
           "rn_server_create", "rn_server_destroy", "rn_serve_submit", "rn_serve_poll", "rn_serve_wait",
           "rn_serve_stats", "rn_solve_bytes", "rn_set_wall_profile", "rn_wall_separation", "rn_derived",
           "rn_derived_buffer", "rn_build_geometry", "rn_get_geometry", "rn_spray_build_injector",
           "rn_spray_set_parcels", "rn_serve_inject", "rn_spray_parcel_steps",
           "rn_last_error")
PRECISION = {"fast": 0, "exact": 1}
TILES = {"16x16": 0, "16x8": 1, "16x15": 2, "32x15": 3, "14x16": 4}
KERNEL_KINDS = ("reduce", "stage1", "stage2", "physics", "parcels", "apply", "other", "stage2_physics")


class RnError(RuntimeError):
    """A librn.so call returned an error code."""

    def __init__(self, code, msg):
        super().__init__(f"librn error {code}: {msg}")
        self.code = code


class RnParams(ctypes.Structure):
    """``rn_params`` (include/rn.h): the float32 uniforms of P."""
    _fields_ = [
        ("amb", ctypes.c_float * 4), ("ambCons", ctypes.c_float * 4), ("ambB", ctypes.c_float * 4),
        ("gamR", ctypes.c_float * 2), ("inlet", ctypes.c_float * 4), ("bar", ctypes.c_float * 3),
        ("res", ctypes.c_float * 3), ("gas", ctypes.c_float * 4), ("Rs", ctypes.c_float * 3),
        ("chemK", ctypes.c_float * 4), ("cap", ctypes.c_float * 2), ("chamberNu", ctypes.c_float * 2),
        ("Tw", ctypes.c_float), ("cfl", ctypes.c_float), ("dtMax", ctypes.c_float), ("wFloor", ctypes.c_float),
        ("vMax", ctypes.c_float), ("hllBlend", ctypes.c_float), ("ramp", ctypes.c_float),
        ("pStart", ctypes.c_float), ("RcCells", ctypes.c_float),
        ("order2", ctypes.c_int), ("inj", ctypes.c_int), ("visc", ctypes.c_int), ("chem", ctypes.c_int),
        ("mhat", ctypes.c_float), ("tScale", ctypes.c_float),
        ("fuel", ctypes.c_float * 4), ("ox", ctypes.c_float * 4),
        ("eF", ctypes.c_float), ("eO", ctypes.c_float), ("Ge", ctypes.c_float), ("fan", ctypes.c_float),
    ]


class RnReadReq(ctypes.Structure):
    _fields_ = [("tex", ctypes.c_int), ("x", ctypes.c_int), ("y", ctypes.c_int), ("w", ctypes.c_int),
                ("h", ctypes.c_int)]


class RnIntegralSpec(ctypes.Structure):
    _fields_ = [("iExit", ctypes.c_int), ("jExit", ctypes.c_int), ("iThroat", ctypes.c_int),
                ("iChamber", ctypes.c_int), ("dx", ctypes.c_double), ("pAmb", ctypes.c_double),
                ("Rs", ctypes.c_double * 3), ("RaN", ctypes.c_double), ("inj", ctypes.c_int)]


class RnIntegralsOut(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("F", "mdot", "Mw", "pw", "A", "throat_mdot", "throat_mO",
                                               "throat_mF", "chamber_p", "chamber_T", "dt", "t")]


class RnServerOpts(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_size_t), ("max_active", ctypes.c_int), ("check_every", ctypes.c_int),
                ("precision", ctypes.c_int), ("tile", ctypes.c_int), ("max_active_cells", ctypes.c_longlong)]


class RnSolveRequest(ctypes.Structure):
    _fields_ = [("Nx", ctypes.c_int), ("Nr", ctypes.c_int), ("mask", ctypes.c_void_p), ("geoA", ctypes.c_void_p),
                ("geoG", ctypes.c_void_p), ("geoM", ctypes.c_void_p), ("jWall", ctypes.c_void_p),
                ("A", ctypes.c_void_p), ("B", ctypes.c_void_p), ("injTab", ctypes.c_void_p), ("P", RnParams),
                ("spec", RnIntegralSpec), ("drop", ctypes.c_double), ("t_end", ctypes.c_double),
                ("max_steps", ctypes.c_longlong), ("parcelsA", ctypes.c_void_p), ("parcelsB", ctypes.c_void_p),
                ("parcelHead", ctypes.c_int)]


class RnSolveResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("pad_", ctypes.c_int), ("steps", ctypes.c_longlong),
                ("t", ctypes.c_double), ("residual0", ctypes.c_double), ("residual", ctypes.c_double),
                ("submit_ms", ctypes.c_double), ("admit_ms", ctypes.c_double), ("done_ms", ctypes.c_double),
                ("integrals", RnIntegralsOut)]


class RnServeStatus(ctypes.Structure):
    _fields_ = [(n, ctypes.c_longlong) for n in ("queued", "active", "finished", "bytes_used", "bytes_budget",
                                                  "ticks", "admitted", "failed", "evicted")]


class RnSeparationSpec(ctypes.Structure):
    _fields_ = [("iThroat", ctypes.c_int), ("iExit", ctypes.c_int)] + \
               [(n, ctypes.c_double) for n in ("dx", "xt", "xe", "Rt", "paSi", "pRef")]


class RnSeparationOut(ctypes.Structure):
    _fields_ = [("found", ctypes.c_int), ("last", ctypes.c_int)] + \
               [(n, ctypes.c_double) for n in ("x", "frac", "eps", "pRatio", "Msep")]


class RnDerivedSpec(ctypes.Structure):
    _fields_ = [("field", ctypes.c_int), ("range", ctypes.c_float * 2), ("RaN", ctypes.c_float),
                ("Rs", ctypes.c_float * 3), ("chemV", ctypes.c_float * 4), ("Tscale", ctypes.c_float * 4),
                ("schlGain", ctypes.c_float), ("velScale", ctypes.c_float), ("dx", ctypes.c_float)]


# the reference's display fields in uField order (render.js:8-23)
FIELDS = ("temp", "mach", "schl", "pres", "dens", "vel", "vort", "exh", "flame", "turb", "burn", "fuel", "ox",
          "heat")


def derived_spec(setup, field, value_range=(0.0, 1.0), schl_gain=10.0, Tc=None):
    """Uniforms of the derived-field pass as app.js sets them (app.js:376-383,
    render.js:427-434): gas constants and chemistry of P, (T_REF, Tc, Ta),
    the schlieren gain, U_REF and dx. ``field`` is a FIELDS name or index."""
    from .physics import T_REF, U_REF
    P = setup["P"]
    return {"field": FIELDS.index(field) if isinstance(field, str) else int(field),
            "range": tuple(value_range), "RaN": P["RaN"], "Rs": tuple(P["Rs"]), "chemV": tuple(P["chemK"]),
            "Tscale": (T_REF, Tc if Tc is not None else setup["cfg"]["Tc"], P["Ta"], 0.0),
            "schlGain": schl_gain, "velScale": U_REF, "dx": setup["dx"]}


class RnCutSpec(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("Nx", "Nr", "cut", "base", "nSolids", "iExit")] + \
               [(n, ctypes.c_double) for n in ("xeC", "twC", "xBaseC", "bodyC", "dx", "xt", "xe", "Rt")] + \
               [("Rtab", ctypes.c_void_p), ("rin", ctypes.c_void_p), ("solids", ctypes.c_void_p),
                ("rinCol", ctypes.c_void_p)]


class RnCutStats(ctypes.Structure):
    _fields_ = [("nCut", ctypes.c_int), ("nMerged", ctypes.c_int)]


class RnInjectorElement(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("type", "weight", "x", "r", "angle", "speed", "drop", "cone",
                                               "width", "xi")]


SOLVE_STATUS = {0: "converged", 1: "time", 2: "max_steps", -1: "rejected", -2: "failed"}


def integral_spec(setup):
    """rn_integral_spec of a setup from build_sim_setup: the exit and throat
    columns, the chamber probe and the gas constants of the read-outs."""
    P = setup["P"]
    s = RnIntegralSpec()
    s.iExit, s.jExit, s.iThroat, s.iChamber = setup["iExit"], setup["jExit"], setup["iThroat"], setup["iChamber"]
    s.dx = setup["dx"]
    s.pAmb = P["amb"][3]
    for k in range(3):
        s.Rs[k] = P["Rs"][k]
    s.RaN = P["RaN"]
    s.inj = 1 if P["inj"] else 0
    return s


def params_from_P(P):
    """Round the reference's parameter block ``P`` to the uniforms the shaders
    receive (``gl.uniform*fv`` converts JavaScript doubles to float32)."""
    p = RnParams()
    for n in ("amb", "ambCons", "ambB", "gamR", "inlet", "res", "gas", "Rs", "chemK", "cap", "chamberNu"):
        arr = getattr(p, n)
        for k, v in enumerate(P[n]):
            arr[k] = float(v)
    # uBar = (inlet[0], 1.6 uInlet0, max(ramp, 0)) formed in doubles (solver.js:935)
    p.bar[0] = float(P["inlet"][0])
    p.bar[1] = 1.6 * float(P["uInlet0"])
    p.bar[2] = max(float(P["ramp"]), 0.0)
    for n in ("Tw", "cfl", "dtMax", "wFloor", "vMax", "hllBlend", "ramp", "pStart", "RcCells"):
        setattr(p, n, float(P[n]))
    p.order2 = 1 if P["order2"] else 0
    p.inj = 1 if P["inj"] else 0
    p.visc = 1 if P["visc"] else 0
    p.chem = 1 if P["chem"] else 0
    p.fan = 25 * math.pi / 180                   # spray.js:271
    if P.get("inj"):
        d = P["injData"]
        p.mhat = P["spray"]["mhat"]
        p.tScale = P["spray"]["tScale"]
        for k in range(4):
            p.fuel[k] = d["fuelVec"][k]
            p.ox[k] = d["oxVec"][k]
        p.eF, p.eO, p.Ge = d["eF"], d["eO"], d["Ge"]
    return p


_lib = None


def lib():
    """Load librn.so once; raise if it is missing (no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RnError(-100, f"{LIB_PATH} is not built; run __graft_entry__.build()")
    L = ctypes.CDLL(LIB_PATH)
    H = ctypes.c_void_p
    i, f = ctypes.c_int, ctypes.c_float
    fp = ctypes.POINTER(ctypes.c_float)
    L.rn_create.argtypes = [i, i, ctypes.POINTER(H)]
    L.rn_destroy.argtypes = [H]
    L.rn_resize.argtypes = [H, i, i]
    L.rn_set_mask.argtypes = [H, ctypes.c_void_p]
    L.rn_set_geometry.argtypes = [H, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_void_p]
    L.rn_set_state.argtypes = [H, ctypes.c_void_p, ctypes.c_void_p]
    L.rn_get_state.argtypes = [H, ctypes.c_void_p, ctypes.c_void_p]
    L.rn_step.argtypes = [H, i, ctypes.POINTER(RnParams)]
    L.rn_rescale_ambient.argtypes = [H, f, f, f, ctypes.POINTER(RnParams)]
    L.rn_draw_wall_row.argtypes = [H]
    L.rn_read_rect.argtypes = [H, i, i, i, i, i, ctypes.c_void_p]
    L.rn_read_step_info.argtypes = [H, fp]
    L.rn_request_async.argtypes = [H, ctypes.POINTER(RnReadReq), i, i]
    L.rn_poll_async.argtypes = [H, ctypes.POINTER(i), ctypes.c_void_p, ctypes.c_size_t]
    L.rn_cancel_async.argtypes = [H]
    L.rn_spray_set_injector.argtypes = [H, ctypes.c_void_p]
    L.rn_spray_reset.argtypes = [H]
    L.rn_spray_stats.argtypes = [H, ctypes.POINTER(ctypes.c_double)]
    L.rn_integrals.argtypes = [H, ctypes.POINTER(RnIntegralSpec), ctypes.POINTER(RnIntegralsOut)]
    # read-outs from caller-owned device buffers, no device allocation (include/rn.h)
    L.rn_integrals_static.argtypes = [ctypes.c_void_p] * 4 + [i, i, ctypes.c_void_p, ctypes.POINTER(RnIntegralSpec),
                                                              ctypes.POINTER(RnIntegralsOut), ctypes.c_void_p]
    L.rn_sync.argtypes = [H]
    L.rn_wait.argtypes = [H, i]
    L.rn_kernel_launches.argtypes = [H, ctypes.POINTER(ctypes.c_longlong)]
    L.rn_get_stream.argtypes = [H, ctypes.POINTER(ctypes.c_void_p)]
    L.rn_set_precision.argtypes = [H, i]
    L.rn_get_precision.argtypes = [H, ctypes.POINTER(i)]
    L.rn_profile.argtypes = [H, i]
    L.rn_profile_read.argtypes = [H, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong)]
    L.rn_set_tile.argtypes = [H, i]
    L.rn_get_tile.argtypes = [H, ctypes.POINTER(i)]
    L.rn_autotune.argtypes = [H, ctypes.POINTER(RnParams), i, ctypes.POINTER(i)]
    L.rn_batch_create.argtypes = [ctypes.POINTER(H)]
    L.rn_batch_destroy.argtypes = [H]
    L.rn_batch_add.argtypes = [H, H, ctypes.POINTER(RnParams), ctypes.POINTER(i)]
    L.rn_batch_remove.argtypes = [H, H]
    L.rn_batch_set_params.argtypes = [H, H, ctypes.POINTER(RnParams)]
    L.rn_batch_size.argtypes = [H, ctypes.POINTER(i), ctypes.POINTER(ctypes.c_longlong)]
    L.rn_batch_step.argtypes = [H, i]
    L.rn_batch_run.argtypes = [H, ctypes.POINTER(ctypes.c_double), i, ctypes.c_longlong,
                               ctypes.POINTER(ctypes.c_longlong)]
    L.rn_batch_sync.argtypes = [H]
    L.rn_batch_set_tile.argtypes = [H, i]
    L.rn_batch_autotune.argtypes = [H, i, ctypes.POINTER(i)]
    L.rn_batch_stream.argtypes = [H, ctypes.POINTER(ctypes.c_void_p)]
    L.rn_batch_kernel_launches.argtypes = [H, ctypes.POINTER(ctypes.c_longlong)]
    L.rn_residual_mark.argtypes = [H]
    L.rn_residual.argtypes = [H, ctypes.POINTER(ctypes.c_double)]
    L.rn_server_default_opts.argtypes = [ctypes.POINTER(RnServerOpts)]
    L.rn_server_create.argtypes = [ctypes.POINTER(RnServerOpts), ctypes.POINTER(H)]
    L.rn_server_destroy.argtypes = [H]
    L.rn_serve_submit.argtypes = [H, ctypes.POINTER(RnSolveRequest), ctypes.POINTER(ctypes.c_longlong)]
    L.rn_serve_poll.argtypes = [H, ctypes.c_longlong, ctypes.POINTER(RnSolveResult), ctypes.c_void_p,
                                ctypes.c_void_p]
    L.rn_serve_wait.argtypes = [H, ctypes.c_longlong, i, ctypes.POINTER(RnSolveResult), ctypes.c_void_p,
                                ctypes.c_void_p]
    L.rn_serve_stats.argtypes = [H, ctypes.POINTER(RnServeStatus)]
    L.rn_solve_bytes.argtypes = [i, i, ctypes.POINTER(ctypes.c_longlong)]
    L.rn_serve_inject.argtypes = [H, i]
    L.rn_spray_parcel_steps.argtypes = [H, ctypes.POINTER(ctypes.c_longlong)]
    dp = ctypes.POINTER(ctypes.c_double)
    L.rn_set_wall_profile.argtypes = [H, dp, dp, dp]
    L.rn_wall_separation.argtypes = [H, ctypes.POINTER(RnSeparationSpec), ctypes.POINTER(RnSeparationOut)]
    L.rn_derived.argtypes = [H, ctypes.POINTER(RnDerivedSpec), ctypes.POINTER(RnParams), ctypes.c_void_p]
    L.rn_derived_buffer.argtypes = [H, ctypes.POINTER(ctypes.c_void_p)]
    L.rn_build_geometry.argtypes = [H, ctypes.POINTER(RnCutSpec), ctypes.POINTER(RnCutStats)]
    L.rn_get_geometry.argtypes = [H] + [ctypes.c_void_p] * 5
    L.rn_spray_build_injector.argtypes = [H, ctypes.POINTER(RnInjectorElement), i]
    L.rn_spray_set_parcels.argtypes = [H, ctypes.c_void_p, ctypes.c_void_p, i]
    L.rn_last_error.restype = ctypes.c_char_p
    for n in EXPORTS[:-1]:
        getattr(L, n).restype = ctypes.c_int
    _lib = L
    return L


def _check(rc, allowed=(RN_OK,)):
    if rc in allowed:
        return rc
    raise RnError(rc, lib().rn_last_error().decode())


def _f32(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} floats, got {a.size}")
    return a


class GPUSolver:
    """The reference's ``GPUSolver`` (solver.js:677) on a B200 via librn.so."""

    def __init__(self, Nx=0, Nr=0):
        self.h = ctypes.c_void_p()
        self.Nx = self.Nr = 0
        self.stepCount = 0
        self.spray = None
        self._async = None
        if Nx and Nr:
            self.resize(Nx, Nr)

    # ---- lifetime
    def resize(self, Nx, Nr):
        """solver.js:759-789"""
        L = lib()
        if self.h.value:
            _check(L.rn_resize(self.h, int(Nx), int(Nr)))
        else:
            _check(L.rn_create(int(Nx), int(Nr), ctypes.byref(self.h)))
        self.Nx, self.Nr = int(Nx), int(Nr)
        self._async = None
        if self.spray is not None:
            self.spray.resize()

    def close(self):
        if self.h.value:
            lib().rn_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- uploads
    def setMask(self, u8):
        """solver.js:791-799"""
        m = np.ascontiguousarray(u8, dtype=np.uint8)
        _check(lib().rn_set_mask(self.h, m.ctypes.data))
        self.maskData = u8

    def setGeometry(self, geo):
        """solver.js:801-814"""
        N, NF = self.Nx * self.Nr, (self.Nx + 1) * (self.Nr + 1)
        m = np.ascontiguousarray(geo["mask"], dtype=np.uint8)
        gA, gG, gM = _f32(geo["geoA"], NF * 4), _f32(geo["geoG"], N * 4), _f32(geo["geoM"], N * 4)
        jw = geo.get("jWall")
        jwp = None
        if jw is not None:
            jw = _f32(jw, self.Nx * 4)
            jwp = jw.ctypes.data
        _check(lib().rn_set_geometry(self.h, m.ctypes.data, gA.ctypes.data, gG.ctypes.data, gM.ctypes.data, jwp))
        self.maskData = geo["mask"]

    def buildGeometry(self, setup):
        """Build the cut-cell geometry of ``setup`` on the device
        (rn_build_geometry: buildCutGeometry, cutcell.js:14-186, and the geoM
        post-pass, simsetup.js:51-63) in place of setGeometry(setup.geo).
        Returns {nCut, nMerged}."""
        from .cutcell import device_inputs
        d = device_inputs(setup["cutInput"])
        c = setup["contour"]
        keep = [np.ascontiguousarray(d["Rtab"], np.float32), np.ascontiguousarray(d["rin"], np.float64),
                np.ascontiguousarray(d["solids"], np.float64), np.ascontiguousarray(setup["rinCol"], np.float32)]
        sp = RnCutSpec()
        sp.Nx, sp.Nr, sp.cut, sp.base = self.Nx, self.Nr, 1 if d["cut"] else 0, 1 if d["base"] else 0
        sp.nSolids, sp.iExit = len(d["solids"]), setup["iExit"]
        sp.xeC, sp.twC, sp.xBaseC, sp.bodyC = d["xeC"], d["twC"], d["xBaseC"], d["bodyC"]
        sp.dx, sp.xt, sp.xe, sp.Rt = setup["dx"], c.xt, c.xe, c.Rt
        sp.Rtab, sp.rin, sp.solids, sp.rinCol = (a.ctypes.data if a.size else None for a in keep)
        st = RnCutStats()
        _check(lib().rn_build_geometry(self.h, ctypes.byref(sp), ctypes.byref(st)))
        return {"nCut": st.nCut, "nMerged": st.nMerged}

    def readGeometry(self):
        """The handle's geometry planes: {mask, geoA, geoG, geoM, jWall} (host copies)."""
        N, NF = self.Nx * self.Nr, (self.Nx + 1) * (self.Nr + 1)
        out = {"mask": np.empty(N, np.uint8), "geoA": np.empty(NF * 4, np.float32),
               "geoG": np.empty(N * 4, np.float32), "geoM": np.empty(N * 4, np.float32),
               "jWall": np.empty(self.Nx * 4, np.float32)}
        _check(lib().rn_get_geometry(self.h, *(out[k].ctypes.data for k in ("mask", "geoA", "geoG", "geoM",
                                                                           "jWall"))))
        return out

    def setState(self, A, B):
        """solver.js:816-828: every state slot; clears dt/t and the spray ring."""
        N = self.Nx * self.Nr * 4
        a, b = _f32(A, N), _f32(B, N)
        _check(lib().rn_set_state(self.h, a.ctypes.data, b.ctypes.data))
        self.stepCount = 0

    # ---- the hot path
    def step(self, n, P):
        """solver.js:849-891 (+ GPUSpray.step when P.inj): queued, returns at once."""
        p = P if isinstance(P, RnParams) else params_from_P(P)
        if p.inj and self.spray is None:
            # the app attaches a GPUSpray on every restart (app.js:239); the
            # handle always owns the parcel ring, so attach its front end here
            GPUSpray(self).resize()
        _check(lib().rn_step(self.h, int(n), ctypes.byref(p)))
        self.stepCount += int(n)

    def rescaleAmbient(self, fp, fT, du, P):
        """solver.js:998-1010"""
        p = P if isinstance(P, RnParams) else params_from_P(P)
        _check(lib().rn_rescale_ambient(self.h, float(fp), float(fT), float(du), ctypes.byref(p)))

    def drawWallRow(self):
        """solver.js:986-996: returns the wall-row texture id."""
        _check(lib().rn_draw_wall_row(self.h))
        return RN_TEX_WALLROW

    @property
    def state(self):
        return {"A": RN_TEX_A, "B": RN_TEX_B}

    @property
    def stepInfoTex(self):
        return RN_TEX_STEPINFO

    # ---- read-backs (solver.js:1016-1075)
    def _readRect(self, tex, x, y, w, h):
        out = np.empty(int(w) * int(h) * 4, dtype=np.float32)
        _check(lib().rn_read_rect(self.h, int(tex), int(x), int(y), int(w), int(h), out.ctypes.data))
        return out

    def readStepInfo(self):
        return self._readRect(RN_TEX_STEPINFO, 0, 0, 1, 1)

    def readColumn(self, i):
        return {"A": self._readRect(RN_TEX_A, i, 0, 1, self.Nr), "B": self._readRect(RN_TEX_B, i, 0, 1, self.Nr)}

    def readCell(self, i, j):
        return {"A": self._readRect(RN_TEX_A, i, j, 1, 1), "B": self._readRect(RN_TEX_B, i, j, 1, 1)}

    def readAll(self):
        N = self.Nx * self.Nr * 4
        A, B = np.empty(N, dtype=np.float32), np.empty(N, dtype=np.float32)
        _check(lib().rn_get_state(self.h, A.ctypes.data, B.ctypes.data))
        return {"A": A, "B": B}

    def requestAsync(self, reqs, tag):
        """solver.js:1028-1048. reqs: [{name, tex, x, y, w, h}]; False while a read is in flight."""
        arr = (RnReadReq * len(reqs))()
        offs, floats = [], 0
        for k, r in enumerate(reqs):
            arr[k].tex, arr[k].x, arr[k].y, arr[k].w, arr[k].h = r["tex"], r["x"], r["y"], r["w"], r["h"]
            offs.append(floats)
            floats += r["w"] * r["h"] * 4
        rc = _check(lib().rn_request_async(self.h, arr, len(reqs), int(tag)), (RN_OK, RN_BUSY))
        if rc == RN_BUSY:
            return False
        self._async = {"reqs": reqs, "offs": offs, "floats": floats, "tag": tag}
        return True

    def pollAsync(self):
        """solver.js:1050-1065: {tag, data: {name: array}} once ready, else None."""
        a = self._async
        if a is None:
            return None
        out = np.empty(max(a["floats"], 1), dtype=np.float32)
        tag = ctypes.c_int()
        rc = _check(lib().rn_poll_async(self.h, ctypes.byref(tag), out.ctypes.data, out.size), (RN_OK, RN_NOT_READY))
        if rc == RN_NOT_READY:
            return None
        self._async = None
        data = {r["name"]: out[o:o + r["w"] * r["h"] * 4] for r, o in zip(a["reqs"], a["offs"])}
        return {"tag": tag.value, "data": data, "probe": a.get("probe")}

    def cancelAsync(self):
        """solver.js:1066-1070"""
        if self.h.value:
            lib().rn_cancel_async(self.h)
        self._async = None

    # ---- extras of the C-ABI
    def integrals(self, setup):
        """FP64 exit/throat/chamber read-outs (rn_integrals) in the reference's
        normalised units, for ``setup`` from build_sim_setup."""
        o = RnIntegralsOut()
        _check(lib().rn_integrals(self.h, ctypes.byref(integral_spec(setup)), ctypes.byref(o)))
        return {n: getattr(o, n) for n, _ in RnIntegralsOut._fields_}

    def wallSeparation(self, setup, paSi):
        """Separation point of the current state, evaluated on the device
        (wallSeparation, simsetup.js:352-373): None where the reference returns
        null, else {x, frac, eps, pRatio, Msep}. The wall profile of ``setup``
        is uploaded on first use."""
        from .physics import P_REF
        c, dx, Nx = setup["contour"], setup["dx"], self.Nx
        if getattr(self, "_wall_profile_of", None) is not setup:
            slope = np.empty(Nx)
            hyp = np.empty(Nx)
            rad = np.empty(Nx)
            for i in range(Nx):
                x = (i + 0.5) * dx
                slope[i] = (c.radiusAt(x + 0.5 * dx) - c.radiusAt(x - 0.5 * dx)) / dx
                hyp[i] = math.hypot(1, slope[i])
                rad[i] = c.radiusAt(x)
            dp = ctypes.POINTER(ctypes.c_double)
            _check(lib().rn_set_wall_profile(self.h, slope.ctypes.data_as(dp), hyp.ctypes.data_as(dp),
                                             rad.ctypes.data_as(dp)))
            self._wall_profile_of = setup
        sp = RnSeparationSpec()
        sp.iThroat, sp.iExit = setup["iThroat"], setup["iExit"]
        sp.dx, sp.xt, sp.xe, sp.Rt = dx, c.xt, c.xe, c.Rt
        sp.paSi, sp.pRef = float(paSi), float(P_REF)
        o = RnSeparationOut()
        _check(lib().rn_wall_separation(self.h, ctypes.byref(sp), ctypes.byref(o)))
        if not o.found:
            return None
        return {"x": o.x, "frac": o.frac, "eps": o.eps, "pRatio": o.pRatio, "Msep": o.Msep}

    def derived(self, spec, P=None, read=True):
        """Derived display field (FS_DERIVED, render.js:60-134) into the
        handle's device buffer; returns it as Nx*Nr*4 float32 (t, Z, Tn, M)
        when ``read``. ``spec`` from derived_spec(); fields 'turb' and 'heat'
        need the step's parameter block P."""
        sp = RnDerivedSpec()
        sp.field = int(spec["field"])
        sp.range[0], sp.range[1] = spec["range"]
        sp.RaN = spec["RaN"]
        for k in range(3):
            sp.Rs[k] = spec["Rs"][k]
        for k in range(4):
            sp.chemV[k] = spec["chemV"][k]
            sp.Tscale[k] = spec["Tscale"][k]
        sp.schlGain, sp.velScale, sp.dx = spec["schlGain"], spec["velScale"], spec["dx"]
        p = None if P is None else ctypes.byref(P if isinstance(P, RnParams) else params_from_P(P))
        out = np.empty(self.Nx * self.Nr * 4, np.float32) if read else None
        _check(lib().rn_derived(self.h, ctypes.byref(sp), p, out.ctypes.data if read else None))
        return out

    def derivedBuffer(self):
        """Device address of the derived-field buffer (0 before the first derived())."""
        v = ctypes.c_void_p()
        _check(lib().rn_derived_buffer(self.h, ctypes.byref(v)))
        return v.value or 0

    def residualMark(self):
        """Snapshot the current state for residual()."""
        _check(lib().rn_residual_mark(self.h))

    def residual(self):
        """FP64 RMS of dU/dt since residualMark() over fluid cells:
        {rho, rhou, rhov, E, span, cells}."""
        out = (ctypes.c_double * 6)()
        _check(lib().rn_residual(self.h, out))
        return dict(zip(("rho", "rhou", "rhov", "E", "span", "cells"), list(out)))

    def sync(self):
        _check(lib().rn_sync(self.h))

    def wait(self, timeout_ms):
        """Bounded wait for the queued work: True when done, False on timeout."""
        return _check(lib().rn_wait(self.h, int(timeout_ms)), (RN_OK, RN_NOT_READY)) == RN_OK

    def setPrecision(self, mode):
        """'fast' (default: hardware approximate division/sqrt, GLSL highp
        latitude) or 'exact' (IEEE division/sqrt: bit for bit with the CPU
        oracle except where pow/exp/log/sin/cos differ in the last bit)."""
        _check(lib().rn_set_precision(self.h, PRECISION[mode]))

    @property
    def precision(self):
        v = ctypes.c_int()
        _check(lib().rn_get_precision(self.h, ctypes.byref(v)))
        return {b: a for a, b in PRECISION.items()}[v.value]

    def setTile(self, shape):
        """Tile shape of the stage/physics kernels: '16x15', '16x16', '16x8', '32x15' or '14x16' (a new handle
        starts with '14x16' when its tiles number at most 3 per SM, else '16x15')."""
        _check(lib().rn_set_tile(self.h, TILES[shape]))

    @property
    def tile(self):
        v = ctypes.c_int()
        _check(lib().rn_get_tile(self.h, ctypes.byref(v)))
        return {b: a for a, b in TILES.items()}[v.value]

    def autotune(self, P, steps=20):
        """Time `steps` steps with each tile shape on the current state (which
        is restored afterwards), keep the fastest and return its name."""
        p = P if isinstance(P, RnParams) else params_from_P(P)
        v = ctypes.c_int()
        _check(lib().rn_autotune(self.h, ctypes.byref(p), int(steps), ctypes.byref(v)))
        return {b: a for a, b in TILES.items()}[v.value]

    def stream(self):
        """The handle's CUDA stream as an integer handle (cudaStream_t)."""
        v = ctypes.c_void_p()
        _check(lib().rn_get_stream(self.h, ctypes.byref(v)))
        return v.value or 0

    def profile(self, enable, in_graph=False):
        """Bracket every kernel with CUDA events on the handle's stream:
        launch by launch, or (in_graph) inside replays of the step graph,
        as event-record nodes around each kernel of the replayed period."""
        _check(lib().rn_profile(self.h, (2 if in_graph else 1) if enable else 0))

    def profileRead(self):
        """{kind: (milliseconds, launches)} since the last read."""
        ms = (ctypes.c_double * len(KERNEL_KINDS))()
        n = (ctypes.c_longlong * len(KERNEL_KINDS))()
        _check(lib().rn_profile_read(self.h, ms, n))
        return {k: (ms[q], n[q]) for q, k in enumerate(KERNEL_KINDS)}

    def kernelLaunches(self):
        v = ctypes.c_longlong()
        _check(lib().rn_kernel_launches(self.h, ctypes.byref(v)))
        return v.value


class GPUSpray:
    """The reference's ``GPUSpray`` (spray.js:211-321): the parcel ring lives in
    the solver handle; this object carries the injector table and read-outs."""

    def __init__(self, solver):
        self.s = solver
        self.blendOk = True          # the deposit is a sorted reduction, no float blending needed
        self.ready = False
        solver.spray = self

    def resize(self):
        """spray.js:224-235 (the ring is allocated with the solver)."""
        self.ready = True
        self.reset()

    def setInjector(self, inj):
        """spray.js:236-241"""
        if not inj or not self.ready:
            return
        tab = _f32(inj["tab"], 256 * 3 * 4)
        _check(lib().rn_spray_set_injector(self.s.h, tab.ctypes.data))

    def buildInjector(self, inj):
        """The injector table of ``inj`` (build_injector_table's result) built on
        the device from its element list (rn_spray_build_injector)."""
        el = inj["elements"]
        arr = (RnInjectorElement * len(el))()
        for q, e in enumerate(el):
            for n in ("type", "weight", "x", "r", "angle", "speed", "drop", "cone", "width", "xi"):
                setattr(arr[q], n, float(e[n]))
        _check(lib().rn_spray_build_injector(self.s.h, arr, len(el)))

    def setParcels(self, PA, PB, head):
        """Pre-populate the parcel ring: PA = (x, r, u, v), PB = (d, m, type,
        x_imp), 65,536 x 4 floats each; ``head`` is where spawning continues."""
        a, b = _f32(PA, SPRAY_N * 4), _f32(PB, SPRAY_N * 4)
        _check(lib().rn_spray_set_parcels(self.s.h, a.ctypes.data, b.ctypes.data, int(head)))

    def reset(self):
        """spray.js:242-254"""
        if not self.ready:
            return
        _check(lib().rn_spray_reset(self.s.h))

    def stats(self, P=None):
        """spray.js:312-320: {fuel, ox, parcels, meanD}."""
        out = (ctypes.c_double * 4)()
        _check(lib().rn_spray_stats(self.s.h, out))
        return {"fuel": out[0], "ox": out[1], "parcels": int(out[2]), "meanD": out[3]}

    def parcelSteps(self):
        """Live parcels summed over every spray step since the ring was last
        set (counted on the device; waits for the queued steps)."""
        v = ctypes.c_longlong()
        _check(lib().rn_spray_parcel_steps(self.s.h, ctypes.byref(v)))
        return v.value

    def readParcels(self):
        """The current parcel textures PA, PB, PC (65,536 x 4 each)."""
        r = self.s._readRect
        return {"PA": r(RN_TEX_PARCEL_A, 0, 0, 256, 256), "PB": r(RN_TEX_PARCEL_B, 0, 0, 256, 256),
                "PC": r(RN_TEX_PARCEL_C, 0, 0, 256, 256)}


class SolverBatch:
    """Steps many GPUSolver handles together: one launch per kernel kind per
    step covers every tile of every member (no reference counterpart; the
    reference runs one grid per page). Members share the physics flags and
    the precision; each keeps its own grid, geometry, state, dt and P."""

    def __init__(self):
        self.b = ctypes.c_void_p()
        _check(lib().rn_batch_create(ctypes.byref(self.b)))
        self.members = []

    def add(self, solver, P):
        p = P if isinstance(P, RnParams) else params_from_P(P)
        slot = ctypes.c_int()
        _check(lib().rn_batch_add(self.b, solver.h, ctypes.byref(p), ctypes.byref(slot)))
        self.members.append(solver)
        return slot.value

    def remove(self, solver):
        _check(lib().rn_batch_remove(self.b, solver.h))
        self.members.remove(solver)

    def setParams(self, solver, P):
        p = P if isinstance(P, RnParams) else params_from_P(P)
        _check(lib().rn_batch_set_params(self.b, solver.h, ctypes.byref(p)))

    def size(self):
        """(members, cells)"""
        m, c = ctypes.c_int(), ctypes.c_longlong()
        _check(lib().rn_batch_size(self.b, ctypes.byref(m), ctypes.byref(c)))
        return m.value, c.value

    def step(self, n):
        """n steps of every member, queued on the batch's stream."""
        _check(lib().rn_batch_step(self.b, int(n)))
        for s in self.members:
            s.stepCount += int(n)

    def run(self, t_end, chunk=60, max_steps=0):
        """Steps every member in chunks of `chunk` steps until its simulated
        time (step info t_new, solver units) reaches its entry of t_end, or
        the run has taken max_steps (> 0), both checked on the device before
        each chunk: the steps of `while t < t_end: solver.step(chunk, P)` run
        for each member alone. Returns the steps each member took."""
        n = len(self.members)
        if len(t_end) != n:
            raise ValueError("t_end needs one entry per member")
        te = (ctypes.c_double * max(n, 1))(*[float(v) for v in t_end])
        out = (ctypes.c_longlong * max(n, 1))()
        _check(lib().rn_batch_run(self.b, te, int(chunk), int(max_steps), out))
        steps = [int(out[k]) for k in range(n)]
        for s, k in zip(self.members, steps):
            s.stepCount += k
        return steps

    def sync(self):
        _check(lib().rn_batch_sync(self.b))

    def setTile(self, shape):
        _check(lib().rn_batch_set_tile(self.b, TILES[shape]))

    def autotune(self, steps=12):
        """Time `steps` batch steps with each tile shape (member states are
        restored afterwards), keep the fastest and return its name."""
        v = ctypes.c_int()
        _check(lib().rn_batch_autotune(self.b, int(steps), ctypes.byref(v)))
        return {b: a for a, b in TILES.items()}[v.value]

    @property
    def tile(self):
        return self.members[0].tile if self.members else None

    def stream(self):
        v = ctypes.c_void_p()
        _check(lib().rn_batch_stream(self.b, ctypes.byref(v)))
        return v.value or 0

    def kernelLaunches(self):
        v = ctypes.c_longlong()
        _check(lib().rn_batch_kernel_launches(self.b, ctypes.byref(v)))
        return v.value

    def close(self):
        if self.b.value:
            lib().rn_batch_destroy(self.b)
            self.b = ctypes.c_void_p()
            self.members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SolveServer:
    """Continuous batching of whole solves on one GPU (rn_server_*): submit
    setups from build_sim_setup with stop criteria, collect results with their
    FP64 read-outs, latencies and (optionally) final states. No reference
    counterpart: the reference runs one interactive solve per page."""

    def __init__(self, budget_bytes=0, max_active=0, check_every=60, precision="fast", tile="16x15",
                 max_active_cells=0):
        o = RnServerOpts()
        _check(lib().rn_server_default_opts(ctypes.byref(o)))
        o.hbm_budget = int(budget_bytes)
        o.max_active = int(max_active)
        o.check_every = int(check_every)
        o.precision = PRECISION[precision]
        o.tile = TILES[tile]
        o.max_active_cells = int(max_active_cells)
        self.s = ctypes.c_void_p()
        _check(lib().rn_server_create(ctypes.byref(o), ctypes.byref(self.s)))
        self.shapes = {}

    @staticmethod
    def solve_bytes(Nx, Nr):
        v = ctypes.c_longlong()
        _check(lib().rn_solve_bytes(int(Nx), int(Nr), ctypes.byref(v)))
        return v.value

    def submit(self, setup, drop=1e-4, t_end_s=2e-3, max_steps=0, state=None, parcels=None):
        """Queue a solve of ``setup`` from its initial state (or ``state``);
        stop at a density-residual drop of ``drop``, ``t_end_s`` seconds of
        simulated time or ``max_steps`` steps. ``parcels`` = (PA, PB, head)
        pre-populates the spray ring. Returns the request id."""
        s = setup
        N, NF = s.Nx * s.Nr, (s.Nx + 1) * (s.Nr + 1)
        geo = s.geo
        keep = [np.ascontiguousarray(geo["mask"], dtype=np.uint8), _f32(geo["geoA"], NF * 4),
                _f32(geo["geoG"], N * 4), _f32(geo["geoM"], N * 4)]
        jw = geo.get("jWall")
        keep.append(_f32(jw, s.Nx * 4) if jw is not None else None)
        init = state if state is not None else s.initialState()
        keep += [_f32(init["A"], N * 4), _f32(init["B"], N * 4)]
        tab = None
        if s.P["inj"]:
            tab = _f32(s.injector["tab"], 256 * 3 * 4)
        keep.append(tab)
        r = RnSolveRequest()
        r.Nx, r.Nr = s.Nx, s.Nr
        for name, a in zip(("mask", "geoA", "geoG", "geoM", "jWall", "A", "B", "injTab"), keep):
            setattr(r, name, a.ctypes.data if a is not None else None)
        r.P = params_from_P(s.P)
        r.spec = integral_spec(s)
        r.drop = float(drop or 0.0)
        r.t_end = float(t_end_s) / float(s.tScale) if t_end_s else 0.0
        r.max_steps = int(max_steps or 0)
        if parcels is not None:
            pa, pb = _f32(parcels[0], SPRAY_N * 4), _f32(parcels[1], SPRAY_N * 4)
            keep += [pa, pb]
            r.parcelsA, r.parcelsB, r.parcelHead = pa.ctypes.data, pb.ctypes.data, int(parcels[2])
        rid = ctypes.c_longlong()
        _check(lib().rn_serve_submit(self.s, ctypes.byref(r), ctypes.byref(rid)))
        self.shapes[rid.value] = (s.Nx, s.Nr)
        return rid.value

    def _result(self, rid, res, A, B, state):
        out = {"id": rid, "status": SOLVE_STATUS.get(res.status, res.status), "steps": res.steps, "t": res.t,
               "residual0": res.residual0, "residual": res.residual, "submit_ms": res.submit_ms,
               "admit_ms": res.admit_ms, "done_ms": res.done_ms,
               "latency_ms": res.done_ms - res.submit_ms,
               "integrals": {n: getattr(res.integrals, n) for n, _ in RnIntegralsOut._fields_}}
        if state:
            out["A"], out["B"] = A, B
        self.shapes.pop(rid, None)
        return out

    def _bufs(self, rid, state):
        if not state:
            return None, None
        Nx, Nr = self.shapes[rid]
        return np.empty(Nx * Nr * 4, np.float32), np.empty(Nx * Nr * 4, np.float32)

    def poll(self, rid, state=False):
        """The result of request ``rid`` once it has finished, else None."""
        A, B = self._bufs(rid, state)
        res = RnSolveResult()
        rc = _check(lib().rn_serve_poll(self.s, int(rid), ctypes.byref(res), A.ctypes.data if state else None,
                                        B.ctypes.data if state else None), (RN_OK, RN_NOT_READY))
        return None if rc == RN_NOT_READY else self._result(rid, res, A, B, state)

    def wait(self, rid, timeout_s=600.0, state=False):
        A, B = self._bufs(rid, state)
        res = RnSolveResult()
        rc = _check(lib().rn_serve_wait(self.s, int(rid), int(timeout_s * 1000), ctypes.byref(res),
                                        A.ctypes.data if state else None, B.ctypes.data if state else None),
                    (RN_OK, RN_NOT_READY))
        return None if rc == RN_NOT_READY else self._result(rid, res, A, B, state)

    def inject(self, where):
        """Host-side fault injection for tests: the next submitted request
        fails as a device allocation would, at its admission ("admit") or in
        its first tick ("tick"); the server evicts it alone."""
        _check(lib().rn_serve_inject(self.s, {"admit": 1, "tick": 2}[where]))

    def stats(self):
        st = RnServeStatus()
        _check(lib().rn_serve_stats(self.s, ctypes.byref(st)))
        return {n: getattr(st, n) for n, _ in RnServeStatus._fields_}

    def close(self):
        if self.s.value:
            lib().rn_server_destroy(self.s)
            self.s = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

"""ctypes front end of the CPU oracle (test infrastructure only).

Loads ``oracle/librn_oracle.so`` (built by ``oracle/Makefile``). Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this file;
the product never does. The oracle restates the reference's shader passes;
parity against the reference itself is unpinned (the reference runs only as
WebGL2 shaders, which need a graphics stack).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librn_oracle.so")


class RnoParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double * k) for n, k in (
        ("amb", 4), ("ambCons", 4), ("ambB", 4), ("gamR", 2), ("inlet", 4), ("res", 3), ("gas", 4),
        ("Rs", 3), ("chemK", 4), ("cap", 2), ("chamberNu", 2))] + [
        (n, ctypes.c_double) for n in ("uInlet0", "Tw", "cfl", "dtMax", "wFloor", "vMax", "hllBlend",
                                       "ramp", "pStart", "RcCells")] + [
        (n, ctypes.c_int) for n in ("order2", "inj", "visc", "chem")] + [
        ("mhat", ctypes.c_double), ("tScale", ctypes.c_double), ("fuelVec", ctypes.c_double * 4),
        ("oxVec", ctypes.c_double * 4), ("eF", ctypes.c_double), ("eO", ctypes.c_double), ("Ge", ctypes.c_double)]


def params_from_P(P):
    """Pack the reference's parameter block ``P`` (a dict of doubles)."""
    p = RnoParams()
    for n in ("amb", "ambCons", "ambB", "gamR", "inlet", "res", "gas", "Rs", "chemK", "cap", "chamberNu"):
        arr = getattr(p, n)
        for k, v in enumerate(P[n]):
            arr[k] = float(v)
    for n in ("uInlet0", "Tw", "cfl", "dtMax", "wFloor", "vMax", "hllBlend", "ramp", "pStart", "RcCells"):
        setattr(p, n, float(P[n]))
    p.order2 = 1 if P["order2"] else 0
    p.inj = 1 if P["inj"] else 0
    p.visc = 1 if P["visc"] else 0
    p.chem = 1 if P["chem"] else 0
    if P.get("inj"):
        d = P["injData"]
        p.mhat = P["spray"]["mhat"]
        p.tScale = P["spray"]["tScale"]
        for k in range(4):
            p.fuelVec[k] = d["fuelVec"][k]
            p.oxVec[k] = d["oxVec"][k]
        p.eF, p.eO, p.Ge = d["eF"], d["eO"], d["Ge"]
    return p


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        fptr = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
        dptr = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        u8 = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
        L.rno_create.restype = vp
        L.rno_create.argtypes = [i, i, i]
        L.rno_destroy.argtypes = [vp]
        L.rno_set_threads.argtypes = [i]
        L.rno_set_geometry.argtypes = [vp, u8, fptr, fptr, fptr, ctypes.c_void_p]
        L.rno_set_state.argtypes = [vp, fptr, fptr]
        L.rno_set_injector.argtypes = [vp, fptr]
        L.rno_step.argtypes = [vp, i, ctypes.POINTER(RnoParams)]
        L.rno_rescale_ambient.argtypes = [vp, d, d, d, ctypes.POINTER(RnoParams)]
        L.rno_get_state.argtypes = [vp, dptr, dptr]
        L.rno_get_step_info.argtypes = [vp, dptr]
        L.rno_get_wall_row.argtypes = [vp, dptr]
        L.rno_get_t2.argtypes = [vp, dptr]
        fptr32 = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
        L.rno_set_parcels.argtypes = [vp, fptr32, fptr32, i]
        L.rno_get_parcels.argtypes = [vp, dptr, dptr, dptr]
        L.rno_get_spray_counters.argtypes = [vp, np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")]
        L.rno_get_src.argtypes = [vp, dptr]
        _lib = L
    return _lib


def set_threads(n):
    lib().rno_set_threads(int(n))


class OracleSolver:
    """CPU oracle with the reference GPUSolver's call shape (FP32 or FP64)."""

    def __init__(self, Nx, Nr, fp64=False):
        self.Nx, self.Nr, self.fp64 = Nx, Nr, fp64
        self.h = lib().rno_create(Nx, Nr, 1 if fp64 else 0)

    def close(self):
        if self.h:
            lib().rno_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def setGeometry(self, geo):
        jw = geo.get("jWall")
        jwp = None
        if jw is not None:
            self._jw = np.ascontiguousarray(jw, dtype=np.float32)
            jwp = self._jw.ctypes.data
        lib().rno_set_geometry(self.h, np.ascontiguousarray(geo["mask"], dtype=np.uint8),
                               np.ascontiguousarray(geo["geoA"], dtype=np.float32),
                               np.ascontiguousarray(geo["geoG"], dtype=np.float32),
                               np.ascontiguousarray(geo["geoM"], dtype=np.float32), jwp)

    def setState(self, A, B):
        lib().rno_set_state(self.h, np.ascontiguousarray(A, dtype=np.float32), np.ascontiguousarray(B, dtype=np.float32))

    def setInjector(self, inj):
        if inj is not None:
            lib().rno_set_injector(self.h, np.ascontiguousarray(inj["tab"], dtype=np.float32))

    def step(self, n, P):
        p = params_from_P(P)
        lib().rno_step(self.h, int(n), ctypes.byref(p))

    def rescaleAmbient(self, fp, fT, du, P):
        p = params_from_P(P)
        lib().rno_rescale_ambient(self.h, float(fp), float(fT), float(du), ctypes.byref(p))

    def readAll(self):
        n = self.Nx * self.Nr * 4
        A, B = np.empty(n), np.empty(n)
        lib().rno_get_state(self.h, A, B)
        return {"A": A, "B": B}

    def readStepInfo(self):
        o = np.empty(4)
        lib().rno_get_step_info(self.h, o)
        return o

    def readWallRow(self):
        o = np.empty(self.Nx * 4)
        lib().rno_get_wall_row(self.h, o)
        return o

    def setParcels(self, PA, PB, head):
        """A pre-populated parcel ring (65,536 x 4 each) and its head."""
        lib().rno_set_parcels(self.h, np.ascontiguousarray(PA, dtype=np.float32),
                              np.ascontiguousarray(PB, dtype=np.float32), int(head))

    def readT2(self):
        """T2 of the last physics pass (effective viscosity, h, strain, laminar viscosity)."""
        o = np.empty(self.Nx * self.Nr * 4)
        lib().rno_get_t2(self.h, o)
        return o

    def readParcels(self):
        n = 65536 * 4
        PA, PB, PC = np.empty(n), np.empty(n), np.empty(n)
        lib().rno_get_parcels(self.h, PA, PB, PC)
        return {"PA": PA, "PB": PB, "PC": PC}

    def sprayCounters(self):
        o = np.zeros(2, dtype=np.uint32)
        lib().rno_get_spray_counters(self.h, o)
        return int(o[0]), int(o[1])

    def readSrc(self):
        o = np.empty(self.Nx * self.Nr * 4)
        lib().rno_get_src(self.h, o)
        return o

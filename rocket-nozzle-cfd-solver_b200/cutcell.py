"""Embedded-boundary ("cut-cell") geometry for the solver.

Host-side restatement of the reference's ``source/cutcell.js:14-186``
(``buildCutGeometry``). For every cell: r-weighted fluid volume V and
meridional area Am from an 8x8 sub-sample; for every face: the r-weighted open
area from a 12-point sub-sample; solid classification (kappa < 0.02); sliver
merge (kappa < 0.5) into the neighbour with the largest open face, in two
sequential passes; negated areas flag first-order faces next to cut cells;
wall vectors by closure; group sums and the slave bitmask.

Arithmetic follows the JavaScript exactly: doubles everywhere, with every
value that the reference keeps in a ``Float32Array`` rounded to float32 at the
same point and re-read as a double. The topology (``mask``, host offsets and
slave bits) therefore comes out bit-identical. O(N) loops that have no
sequential dependency are evaluated with numpy, whose elementwise float64
operations are the same IEEE operations in the same order.
"""
import math

import numpy as np

f32 = np.float32
SUB = 8          # radius table entries per cell (cutcell.js:20)
NC = 8           # volume sub-samples per direction (cutcell.js:69)
NF = 12          # face sub-samples (cutcell.js:69)
KMERGE = 0.5     # cutcell.js:123


class _Walls:
    """Wall description in cell units with scalar and column-vector tests."""

    def __init__(self, o):
        Nx, dx, contour = o["Nx"], o["dx"], o["contour"]
        self.contour, self.dx = contour, dx
        self.xeC = contour.xe / dx
        self.twC = o["tw"] / dx
        self.xBaseC = o["xBase"] / dx
        self.bodyC = o["bodyR"] / dx
        self.base = bool(o.get("base"))
        self.nTab = Nx * SUB + 1
        tab = np.empty(self.nTab, dtype=np.float64)
        for k in range(self.nTab):
            X = (k / SUB) * dx
            tab[k] = contour.radiusAt(X) / dx if X <= contour.xe else -1e9
        self.Rtab = tab.astype(f32)          # Float32Array (cutcell.js:22)
        self.solids = [{"x0": s["x0"] / dx, "x1": s["x1"] / dx, "r0": s["r0"] / dx, "r1": s["r1"] / dx}
                       for s in (o.get("solids") or [])]

    def RinAt(self, xc):
        """Interpolated inner-wall radius in cells (cutcell.js:27-34)."""
        if xc > self.xeC:
            return -1e9
        f = min(max(xc * SUB, 0), self.nTab - 1)
        k = min(math.floor(f), self.nTab - 2)
        t = f - k
        a, b = float(self.Rtab[k]), float(self.Rtab[k + 1])
        if a < -1e8 or b < -1e8:
            return self.contour.radiusAt(min(xc * self.dx, self.contour.xe)) / self.dx
        return a + (b - a) * t

    def fluid(self, xc, rc):
        """cutcell.js:36-44"""
        for s in self.solids:
            if xc >= s["x0"] and xc <= s["x1"] and rc >= s["r0"] and rc <= s["r1"]:
                return False
        if xc <= self.xeC:
            ri = self.RinAt(xc)
            if rc >= ri and rc <= ri + self.twC:
                return False
            if self.base and xc < self.xBaseC and rc >= ri and rc < self.bodyC:
                return False
        return True

    def fluid_col(self, xc, rc):
        """``fluid`` for one x and a vector of radii (same double operations)."""
        ok = np.ones(rc.shape, dtype=bool)
        for s in self.solids:
            if xc >= s["x0"] and xc <= s["x1"]:
                ok &= ~((rc >= s["r0"]) & (rc <= s["r1"]))
        if xc <= self.xeC:
            ri = self.RinAt(xc)
            ok &= ~((rc >= ri) & (rc <= ri + self.twC))
            if self.base and xc < self.xBaseC:
                ok &= ~((rc >= ri) & (rc < self.bodyC))
        return ok


CUT_SAMPLES = 23     # RinAt abscissae per column handed to the device builder (rn.h RN_CUT_SAMPLES)


def sample_abscissae(i):
    """The x (cells) at which the builder evaluates RinAt in column i: the
    x-face, the centre, the 8 volume and 12 r-face sub-samples, the next x-face."""
    return ([float(i), i + 0.5] + [i + (a + 0.5) / NC for a in range(NC)] +
            [i + (b + 0.5) / NF for b in range(NF)] + [float(i + 1)])


def device_inputs(o):
    """Inputs of the device builder (rn_build_geometry) for the same ``o`` as
    build_cut_geometry: the float32 radius table, RinAt at every sampled
    abscissa (-1e9 beyond the exit, where it is not read), solids in cells."""
    w = _Walls(o)
    Nx = o["Nx"]
    rin = np.full((Nx, CUT_SAMPLES), -1e9, dtype=np.float64)
    for i in range(Nx):
        for s, xc in enumerate(sample_abscissae(i)):
            if xc <= w.xeC:
                rin[i, s] = w.RinAt(xc)
    solids = np.array([[s["x0"], s["x1"], s["r0"], s["r1"]] for s in w.solids], dtype=np.float64).reshape(-1, 4)
    return {"Rtab": w.Rtab, "rin": rin, "solids": solids, "xeC": w.xeC, "twC": w.twC, "xBaseC": w.xBaseC,
            "bodyC": w.bodyC, "base": w.base, "cut": o.get("mode") != "stair"}


def build_cut_geometry(o):
    """Cut-cell geometry (cutcell.js:14-186).

    ``o``: dict with Nx, Nr, dx, contour, tw, base, xBase, bodyR, mode
    ('cut' | 'stair') and solids [{x0, x1, r0, r1}] in metres.
    Returns a dict with mask, geoA, geoG, geoM, Ax, Ar, W1, kappa, nCut, nMerged;
    the float arrays are float32 like the reference's typed arrays.
    """
    Nx, Nr = o["Nx"], o["Nr"]
    cut = o.get("mode") != "stair"
    w = _Walls(o)
    # per column: radius range of the inner wall over [i, i+1] (cutcell.js:46-51)
    colMin = np.empty(Nx, dtype=f32)
    colMax = np.empty(Nx, dtype=f32)
    for i in range(Nx):
        seg = w.Rtab[i * SUB:i * SUB + SUB + 1].astype(np.float64)
        seg = seg[seg > -1e8]
        colMin[i] = seg.min() if seg.size else 1e9
        colMax[i] = seg.max() if seg.size else -1e9

    # maybeCut for every cell (cutcell.js:52-67), evaluated column by column
    jr = np.arange(Nr, dtype=np.float64)
    r0v, r1v = jr, jr + 1

    def ov(a0, a1, b0, b1):
        return (a0 < b1) & (a1 > b0)

    MC = np.zeros((Nr, Nx), dtype=bool)
    if cut:
        for i in range(Nx):
            x0, x1 = float(i), float(i + 1)
            m = np.zeros(Nr, dtype=bool)
            for s in w.solids:
                if x0 < s["x1"] + 1e-6 and x1 > s["x0"] - 1e-6:
                    m |= ov(r0v, r1v, s["r0"] - 1e-6, s["r1"] + 1e-6)
            if not (float(colMax[i]) < -1e8):
                mn, mx = float(colMin[i]), float(colMax[i])
                m |= ov(r0v, r1v, mn - 1e-6, mx + 1e-6)
                m |= ov(r0v, r1v, mn + w.twC - 1e-6, mx + w.twC + 1e-6)
                if w.xeC >= x0 and w.xeC <= x1:
                    m |= ov(r0v, r1v, mn, mx + w.twC)
                if w.base:
                    if w.xBaseC >= x0 and w.xBaseC <= x1:
                        m |= ov(r0v, r1v, mn, w.bodyC)
                    if x0 < w.xBaseC:
                        m |= (w.bodyC >= r0v) & (w.bodyC <= r1v)
            MC[:, i] = m

    # volumes and meridional areas (cutcell.js:70-82)
    V = np.zeros((Nr, Nx), dtype=f32)
    Am = np.zeros((Nr, Nx), dtype=f32)
    isCut = np.zeros((Nr, Nx), dtype=np.uint8)
    rc_mid = jr + 0.5
    for i in range(Nx):
        fl = w.fluid_col(i + 0.5, rc_mid)
        Am[:, i] = np.where(fl, 1.0, 0.0)
        V[:, i] = np.where(fl, rc_mid, 0.0)
    for j, i in zip(*np.nonzero(MC)):
        j, i = int(j), int(i)
        am, v = 0, 0.0
        for b in range(NC):
            rc = j + (b + 0.5) / NC
            for a in range(NC):
                if w.fluid(i + (a + 0.5) / NC, rc):
                    am += 1
                    v += rc
        Am[j, i] = am / (NC * NC)
        V[j, i] = v / (NC * NC)
        isCut[j, i] = 1 if (Am[j, i] > 0 and Am[j, i] < 1) else 0

    # faces on the (Nx+1) x (Nr+1) lattice (cutcell.js:84-104)
    W1 = Nx + 1
    Ax = np.zeros((Nr + 1, W1), dtype=f32)
    Ar = np.zeros((Nr + 1, W1), dtype=f32)
    cutPad = np.zeros((Nr + 2, Nx + 2), dtype=bool)   # cutAt with a zero border
    cutPad[1:-1, 1:-1] = isCut.astype(bool)
    mcPad = np.zeros((Nr + 2, Nx + 2), dtype=bool)
    mcPad[1:-1, 1:-1] = MC
    # x-faces at x = i
    for i in range(Nx + 1):
        sel = cutPad[1:-1, i] | cutPad[1:-1, i + 1] | MC[:, min(i, Nx - 1)]
        if i > 0:
            sel = sel | MC[:, i - 1]
        if not cut:
            sel[:] = False
        fl = w.fluid_col(float(i), rc_mid)
        Ax[:Nr, i] = np.where(fl, rc_mid, 0.0)
        for j in np.nonzero(sel)[0]:
            j = int(j)
            a = 0.0
            for b in range(NF):
                rc = j + (b + 0.5) / NF
                if w.fluid(i, rc):
                    a += rc
            Ax[j, i] = a / NF
    # r-faces at r = j
    jf = np.arange(Nr + 1, dtype=np.float64)
    for i in range(Nx):
        sel = cutPad[0:Nr + 1, i + 1] | cutPad[1:Nr + 2, i + 1]
        sel = sel | np.concatenate([MC[:, i], [False]]) | np.concatenate([[False], MC[:, i]])
        if not cut:
            sel[:] = False
        fl = w.fluid_col(i + 0.5, jf)
        Ar[:, i] = np.where(fl, jf, 0.0)
        for j in np.nonzero(sel)[0]:
            j = int(j)
            f = 0
            for b in range(NF):
                if w.fluid(i + (b + 0.5) / NF, j):
                    f += 1
            Ar[j, i] = j * f / NF

    # classification (cutcell.js:107-120)
    kap = (V.astype(np.float64) / rc_mid[:, None]).astype(f32)
    kap64 = kap.astype(np.float64)               # Float32Array values compared as doubles
    solid = (kap64 < 0.02).astype(np.uint8)

    def zero_solid_faces():
        js, is_ = np.nonzero(solid)
        Ax[js, is_] = 0
        Ax[js, is_ + 1] = 0
        Ar[js, is_] = 0
        Ar[js + 1, is_] = 0

    zero_solid_faces()
    # merge slivers into a neighbour with kappa >= 0.5 (cutcell.js:122-142); sequential scan order
    host = np.full((Nr, Nx), -1, dtype=np.int64)
    slivers = [(int(j), int(i)) for j, i in zip(*np.nonzero(kap < KMERGE))]   # row-major order
    for pas in range(2):
        for j, i in slivers:
            if solid[j, i] or kap[j, i] >= KMERGE or host[j, i] >= 0:
                continue
            best, bestA = -1, 0.0
            cand = [
                (i - 1, j, float(Ax[j, i]) / (j + 0.5)),
                (i + 1, j, float(Ax[j, i + 1]) / (j + 0.5)),
                (i, j - 1, float(Ar[j, i]) / j if j > 0 else 0.0),
                (i, j + 1, float(Ar[j + 1, i]) / (j + 1)),
            ]
            for ii, jj, a in cand:
                if ii < 0 or ii >= Nx or jj < 0 or jj >= Nr:
                    continue
                if solid[jj, ii] or kap[jj, ii] < KMERGE or host[jj, ii] >= 0:
                    continue
                if a > bestA + 1e-9:
                    bestA = a
                    best = jj * Nx + ii
            if best >= 0 and bestA > 0.02:
                host[j, i] = best
            elif pas == 1:
                solid[j, i] = 1
    zero_solid_faces()

    # first-order flag for faces next to cut cells: store the area negated (cutcell.js:145-153)
    partial = (solid == 0) & ((kap64 < 0.98) | (host >= 0))
    pp = np.zeros((Nr + 2, Nx + 2), dtype=bool)
    pp[1:-1, 1:-1] = partial
    geoA = np.zeros((Nr + 1, W1, 4), dtype=f32)
    geoA[:Nr, :Nx, 0] = V
    geoA[:Nr, :Nx, 1] = Am
    negx = pp[1:-1, 0:Nx + 1] | pp[1:-1, 1:Nx + 2]           # partial(i-1,j) | partial(i,j), j < Nr
    geoA[:Nr, :, 2] = np.where(negx, -Ax[:Nr, :], Ax[:Nr, :])
    negr = pp[0:Nr + 1, 1:-1] | pp[1:Nr + 2, 1:-1]           # partial(i,j-1) | partial(i,j), i < Nx
    geoA[:, :Nx, 3] = np.where(negr, -Ar[:, :Nx], Ar[:, :Nx])

    # wall vectors by closure (cutcell.js:155-163)
    A64x = Ax.astype(np.float64)
    A64r = Ar.astype(np.float64)
    Wx = (A64x[:Nr, :Nx] - A64x[:Nr, 1:Nx + 1]).astype(f32)
    Wr = (Am.astype(np.float64) - (A64r[1:Nr + 1, :Nx] - A64r[:Nr, :Nx])).astype(f32)
    Wx[np.abs(Wx.astype(np.float64)) < 1e-6] = 0
    Wr[np.abs(Wr.astype(np.float64)) < 1e-6] = 0
    Wx[solid != 0] = 0
    Wr[solid != 0] = 0

    # group sums, accumulated in float32 in ascending cell order (cutcell.js:165-174)
    N = Nx * Nr
    hostf = host.reshape(N)
    solidf = solid.reshape(N)
    Vf, Amf, Wxf, Wrf = V.reshape(N), Am.reshape(N), Wx.reshape(N), Wr.reshape(N)
    gV = np.where(solidf == 0, Vf, 0).astype(f32)
    gA = np.where(solidf == 0, Amf, 0).astype(f32)
    gX = np.where(solidf == 0, Wxf, 0).astype(f32)
    gR = np.where(solidf == 0, Wrf, 0).astype(f32)
    members = {}
    for k in np.nonzero((hostf >= 0) & (solidf == 0))[0]:
        members.setdefault(int(hostf[k]), []).append(int(k))
    for h, ks in members.items():
        order = sorted(ks + [h])
        acc = [f32(0), f32(0), f32(0), f32(0)]
        for k in order:
            acc[0] = f32(float(acc[0]) + float(Vf[k]))
            acc[1] = f32(float(acc[1]) + float(Amf[k]))
            acc[2] = f32(float(acc[2]) + float(Wxf[k]))
            acc[3] = f32(float(acc[3]) + float(Wrf[k]))
        gV[h], gA[h], gX[h], gR[h] = acc
    slaveMask = np.zeros(N, dtype=np.uint8)
    for h, ks in members.items():
        hi = h % Nx
        hj = (h - hi) // Nx
        for k in ks:
            i, j = k % Nx, k // Nx
            bit = 1 if i < hi else 2 if i > hi else 4 if j < hj else 8
            slaveMask[h] |= bit

    geoG = np.zeros((N, 4), dtype=f32)
    geoM = np.zeros((N, 4), dtype=f32)
    kapf = kap.reshape(N)
    fluid_idx = np.nonzero(solidf == 0)[0]
    hsel = np.where(hostf >= 0, hostf, np.arange(N))
    geoG[solidf != 0, 0] = 1
    geoG[fluid_idx, 0] = gV[hsel[fluid_idx]]
    geoG[fluid_idx, 1] = gA[hsel[fluid_idx]]
    geoG[fluid_idx, 2] = gX[hsel[fluid_idx]]
    geoG[fluid_idx, 3] = gR[hsel[fluid_idx]]
    ii = np.arange(N) % Nx
    jj = np.arange(N) // Nx
    hi = hsel % Nx
    hj = hsel // Nx
    geoM[fluid_idx, 0] = (hi - ii)[fluid_idx]
    geoM[fluid_idx, 1] = (hj - jj)[fluid_idx]
    geoM[fluid_idx, 2] = slaveMask[fluid_idx]
    geoM[fluid_idx, 3] = kapf[fluid_idx]
    nCut = int(np.count_nonzero(kapf[fluid_idx].astype(np.float64) < 0.98))
    nMerged = int(np.count_nonzero(hostf[fluid_idx] >= 0))
    return {"mask": solidf.copy(), "geoA": geoA.reshape(-1), "geoG": geoG.reshape(-1),
            "geoM": geoM.reshape(-1), "Ax": Ax.reshape(-1), "Ar": Ar.reshape(-1), "W1": W1,
            "kappa": kapf.copy(), "host": hostf.copy(), "nCut": nCut, "nMerged": nMerged}

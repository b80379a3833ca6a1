"""NumPy restatement of the reference's derived-field shader (test infrastructure
only: tests/ compare the device's rn_derived against it).

Follows FS_DERIVED, source/render.js:60-134, in float32 (GLSL highp): the
field value v of every fluid cell, its display mapping t, and the output
(t, Z, normalised T, Mach); walls give (0, 0, 0, -1). ``T2`` is the split
step's cell data (the oracle's T2 texture, FS_VCELL solver.js:458-488).
"""
import numpy as np

f = np.float32


def to_prim(A, B):
    """toPrim (solver.js:33-39) on (..., 4) float32 arrays."""
    rho = np.maximum(A[..., 0], f(1e-7))
    vx, vy = A[..., 1] / rho, A[..., 2] / rho
    G = np.maximum(B[..., 2], f(0.5))
    p = np.maximum((A[..., 3] - f(0.5) * rho * (vx * vx + vy * vy)) / G, f(1e-7))
    s = np.stack([np.clip(B[..., 0] / rho, f(0), f(1)), np.clip(B[..., 1] / rho, f(0), f(1)), G,
                  np.clip(B[..., 3] / rho, f(0), f(1))], axis=-1)
    return np.stack([rho, vx, vy, p], axis=-1), s


def derived(A, B, mask, Nx, Nr, spec, T2=None):
    """spec: dict with field, range (2), RaN, Rs (3), chemV (4), Tscale (4), schlGain, velScale, dx."""
    A = np.asarray(A, f).reshape(Nr, Nx, 4)
    B = np.asarray(B, f).reshape(Nr, Nx, 4)
    solid = np.asarray(mask).reshape(Nr, Nx) != 0
    T2 = np.zeros((Nr, Nx, 4), f) if T2 is None else np.asarray(T2, f).reshape(Nr, Nx, 4)
    F = int(spec["field"])
    rng = [f(v) for v in spec["range"]]
    Rs = [f(v) for v in spec["Rs"]]
    chemV = [f(v) for v in spec["chemV"]]
    Ts = [f(v) for v in spec["Tscale"]]
    w, s = to_prim(A, B)
    rho, p = w[..., 0], w[..., 3]
    c = np.sqrt((f(1) + f(1) / s[..., 2]) * p / rho)
    spd = np.sqrt(w[..., 1] * w[..., 1] + w[..., 2] * w[..., 2])
    M = spd / c
    Rm = (f(1) - s[..., 0]) * f(spec["RaN"]) + s[..., 1] * Rs[0] + s[..., 3] * Rs[1] + \
        np.maximum(s[..., 0] - s[..., 1] - s[..., 3], f(0)) * Rs[2]
    T = p / (rho * Rm) * Ts[0]
    jj, ii = np.meshgrid(np.arange(Nr), np.arange(Nx), indexing="ij")

    def clampi(i, j):
        return np.clip(i, 0, Nx - 1), np.clip(j, 0, Nr - 1)

    def lrho(i, j):
        ci, cj = clampi(i, j)
        cj = np.where(j < 0, -j - 1, cj)
        return np.log(np.maximum(A[cj, ci, 0], f(1e-7)))

    def solid_c(i, j):
        ci, cj = clampi(i, j)
        return solid[cj, ci]

    if F == 1:
        v = M
    elif F == 2:
        l0 = lrho(ii, jj)
        le = np.where(solid_c(ii + 1, jj), l0, lrho(ii + 1, jj))
        lw = np.where(solid_c(ii - 1, jj), l0, lrho(ii - 1, jj))
        ln = np.where(solid_c(ii, jj + 1), l0, lrho(ii, jj + 1))
        below = np.where(jj > 0, solid[np.maximum(jj - 1, 0), ii], False)
        ls = np.where(below, l0, lrho(ii, jj - 1))
        gr = np.sqrt((le - lw) * (le - lw) + (ln - ls) * (ln - ls)) * f(0.5)
        v = f(1) - np.exp(-f(spec["schlGain"]) * gr)
    elif F == 3:
        v = np.log(p * f(101325.0)) / np.log(f(10.0))
    elif F == 4:
        v = np.log(rho * f(1.225)) / np.log(f(10.0))
    elif F == 5:
        v = spd * f(spec["velScale"])
    elif F == 6:
        def wy(i, j, comp):
            ci, cj = clampi(i, j)
            return w[cj, ci, comp]
        e_v, w_v, n_u = wy(ii + 1, jj, 2), wy(ii - 1, jj, 2), wy(ii, jj + 1, 1)
        s_u = np.where(jj > 0, wy(ii, jj - 1, 1), w[..., 1])
        om = f(0.5) * (e_v - w_v) - f(0.5) * (n_u - s_u)
        v = np.abs(om) * f(spec["velScale"]) / f(spec["dx"])
    elif F == 7:
        v = s[..., 0]
    elif F == 9:
        m = T2
        with np.errstate(divide="ignore", invalid="ignore"):
            v = np.where(m[..., 3] > 0, np.log(np.maximum(m[..., 0] / m[..., 3], f(1))) / np.log(f(10.0)), f(0))
    elif F == 10:
        with np.errstate(divide="ignore", invalid="ignore"):
            v = np.where(s[..., 0] > f(0.003), (s[..., 0] - s[..., 1]) / s[..., 0], f(0))
    elif F == 11:
        v = s[..., 1]
    elif F == 12:
        v = s[..., 3]
    elif F == 13:
        m = T2
        avail = np.minimum(s[..., 1], (s[..., 3] + f(0.233) * np.maximum(f(1) - s[..., 0], f(0))) / chemV[1])
        kin = chemV[2] * p * np.exp(f(-9000.0) / np.maximum(T, f(200.0)))
        v = np.log(f(1) + f(1e5) * avail * np.minimum(np.maximum(m[..., 2], f(4) * m[..., 0] / rho), kin)) / \
            np.log(f(10.0))
    else:
        v = T
    v = v.astype(f)
    t = (v - rng[0]) / (rng[1] - rng[0])
    if F == 2:
        t = v
    if F == 6:
        t = np.log(f(1) + f(20) * np.maximum(v, f(0)) / rng[1]) / np.log(f(21.0))
    out = np.stack([t, s[..., 0], (T - Ts[2]) / np.maximum(Ts[1] - Ts[2], f(1)), M], axis=-1).astype(f)
    out[solid] = (0, 0, 0, -1)
    return out.reshape(-1)

"""CPU restatement of the reference's near-to-far-field transform (test
infrastructure: the checker of fdtd_ntff, never part of the product path).

Follows Source/Scheme/SchemeHelper.h:1036-2121 (ntffN3D_x/y/z over the H
fields averaged over two time levels, ntffL3D_x/y/z over the current E
fields, per layout) and Source/Scheme/Scheme.inc.h:4037-4095 (Pointing_scat
over Pointing_inc), with numpy complex arithmetic over whole faces.

fields: {"Ex": complex array (nx, ny, nz), ...} at the current level;
h_prev: {"Hx": ..., "Hy": ..., "Hz": ...} one time level earlier.
"""
import numpy as np

MU0 = 4 * np.pi * 0.0000001
EPS0 = 1 / (MU0 * 299792458.0 ** 2)

# first positions of the components (Source/Layout/YeeGridLayout.cpp:1937-2035)
MIN_FP = {
    0: {"Ex": (1.0, 0.5, 0.5), "Ey": (0.5, 1.0, 0.5), "Ez": (0.5, 0.5, 1.0),
        "Hx": (0.5, 1.0, 1.0), "Hy": (1.0, 0.5, 1.0), "Hz": (1.0, 1.0, 0.5)},
    1: {"Ex": (0.5, 1.0, 1.0), "Ey": (1.0, 0.5, 1.0), "Ez": (1.0, 1.0, 0.5),
        "Hx": (1.0, 0.5, 0.5), "Hy": (0.5, 1.0, 0.5), "Hz": (0.5, 0.5, 1.0)},
}


def _sample(f, prev, comp, pos, avg_axis, layout):
    """comp at positions pos (list of 3 arrays); avg over -/+1/2 along avg_axis;
    over two time levels when prev is given (the N sums)."""
    mn = MIN_FP[layout][comp]
    q = [pos[a] - mn[a] for a in range(3)]

    def at(arr, qq):
        return arr[tuple(np.asarray(v, dtype=np.int64) for v in qq)]

    if avg_axis is None:
        v = at(f[comp], q)
        return (v + at(prev[comp], q)) / 2.0 if prev is not None else v
    q1, q2 = list(q), list(q)
    q1[avg_axis] = q1[avg_axis] - 0.5
    q2[avg_axis] = q2[avg_axis] + 0.5
    if prev is not None:
        return (at(f[comp], q1) + at(f[comp], q2) + at(prev[comp], q1) + at(prev[comp], q2)) / 4.0
    return (at(f[comp], q1) + at(f[comp], q2)) / 2.0


def _face(f, h_prev, layout, axis, x0, left, right, n, dx, k, teta, phi, is_n):
    tb = 1 if axis == 0 else 0
    tc = 1 if axis == 2 else 2
    ub = left[tb] + 0.5 + np.arange(right[tb] - left[tb])
    uc = left[tc] + 0.5 + np.arange(right[tc] - left[tc])
    gb, gc = np.meshgrid(ub, uc, indexing="ij")
    pos = [None, None, None]
    pos[axis] = np.full(gb.shape, float(x0))
    pos[tb], pos[tc] = gb, gc
    hc = layout == 1
    avg = axis if (is_n == hc) else None
    sa, sb = (tc, tb) if hc else (tb, tc)
    comps = {(0, True): ("Hz", "Hy"), (1, True): ("Hz", "Hx"), (2, True): ("Hy", "Hx"),
             (0, False): ("Ey", "Ez"), (1, False): ("Ex", "Ez"), (2, False): ("Ex", "Ey")}[(axis, is_n)]
    prev = h_prev if is_n else None
    a1, a2, b1, b2 = ([p.copy() for p in pos] for _ in range(4))
    a1[sa] = a1[sa] - 0.5
    # H_CENTERED z faces: the first component is sampled twice at -1/2
    a2[sa] = a2[sa] + (-0.5 if (hc and axis == 2) else 0.5)
    b1[sb] = b1[sb] - 0.5
    b2[sb] = b2[sb] + 0.5
    A = (_sample(f, prev, comps[0], a1, avg, layout) + _sample(f, prev, comps[0], a2, avg, layout)) / 2.0
    B = (_sample(f, prev, comps[1], b1, avg, layout) + _sample(f, prev, comps[1], b2, avg, layout)) / 2.0
    st, ct, sp, cp = np.sin(teta), np.cos(teta), np.sin(phi), np.cos(phi)
    d0 = [float(v // 2) for v in n]
    arg = ((pos[0] - d0[0]) * st * cp + (pos[1] - d0[1]) * st * sp + (pos[2] - d0[2]) * ct) * dx
    e = np.exp(1j * k * arg)
    s = 1.0 if x0 == right[axis] else -1.0
    w = e * dx * dx * s
    if is_n:
        if axis == 0:
            return np.sum((A * ct * sp + B * st) * w * -1.0), np.sum(A * cp * w * -1.0)
        if axis == 1:
            return np.sum((A * ct * cp + B * st) * w), np.sum(A * sp * w * -1.0)
        return np.sum((-A * ct * cp + B * ct * sp) * w), np.sum((A * sp + B * cp) * w)
    if axis == 0:
        return np.sum((B * ct * sp + A * st) * w), np.sum(B * cp * w)
    if axis == 1:
        return np.sum((B * ct * cp + A * st) * w * -1.0), np.sum(B * sp * w)
    return np.sum((B * ct * cp - A * ct * sp) * w), np.sum((B * sp + A * cp) * w * -1.0)


def ntff_values(fields, h_prev, layout, left, right, dx, wavelength, teta, phis):
    """The reference's "NTFF value" per azimuth in phis."""
    n = fields["Ex"].shape
    k = 2 * np.pi / wavelength
    out = []
    for phi in phis:
        tot = {True: [0j, 0j], False: [0j, 0j]}
        for is_n in (True, False):
            for axis in range(3):
                for x0 in (left[axis], right[axis]):
                    t, p = _face(fields, h_prev, layout, axis, x0, left, right, n, dx, k, teta, phi, is_n)
                    tot[is_n][0] += t
                    tot[is_n][1] += p
        n_t, n_p = tot[True]
        l_t, l_p = tot[False]
        n0 = np.sqrt(MU0 / EPS0)
        first = l_p + n_t * n0
        second = l_t - n_p * n0
        val = k ** 2 / (8 * np.pi * n0) * (abs(first) ** 2 + abs(second) ** 2)
        out.append(val / (np.sqrt(EPS0 / MU0) / 2))
    return np.array(out)

"""NumPy restatement of the batched checkerboard Monte Carlo (TEST INFRASTRUCTURE ONLY: the
checker of csrc/batch.cu's proposals, features and decisions on small boxes, never the
product).

The scheme is this project's (the reference visits molecules in cell order with one ran1
stream); what it shares with the reference is the pair energy of molfit.py:1251-1279, which
the checks evaluate with the C oracle's FP64 restatement, and the Metropolis rule.  Every
float32 step below follows the device's operation order (round-to-nearest, no fused
multiply-add), and sin/cos are evaluated in double and rounded once, as the device does.
"""

from __future__ import annotations

import numpy as np

f32 = np.float32
M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85
P_BIN, P_MOVE, P_DECIDE = 0xB1, 1, 2
FEAT_BINS, FEAT_HALF = 64, 640


def philox(c, k0, k1):
    """Philox4x32-10 of one counter (four uint32) and key; returns four uint32."""
    x, y, z, w = (int(v) & 0xFFFFFFFF for v in c)
    k0 &= 0xFFFFFFFF
    k1 &= 0xFFFFFFFF
    for _ in range(10):
        p0 = M0 * x
        p1 = M1 * z
        h0, l0 = p0 >> 32, p0 & 0xFFFFFFFF
        h1, l1 = p1 >> 32, p1 & 0xFFFFFFFF
        x, y, z, w = (h1 ^ y ^ k0) & 0xFFFFFFFF, l1, (h0 ^ w ^ k1) & 0xFFFFFFFF, l0
        k0 = (k0 + W0) & 0xFFFFFFFF
        k1 = (k1 + W1) & 0xFFFFFFFF
    return x, y, z, w


def u01(v):
    return f32(f32(v >> 8) * f32(1.0 / 16777216.0))


def nint(x):
    t = f32(np.trunc(x))
    fr = f32(x - t)
    if fr >= f32(0.5):
        t = f32(t + f32(1.0))
    elif fr <= f32(-0.5):
        t = f32(t - f32(1.0))
    return t


def wrap(c):
    return f32(c - nint(c))


def cell_coord(x, shift, n):
    i = int(np.floor(f32(f32(f32(x + f32(0.5)) + shift) * f32(n))))
    return i % n


def cosr(x):
    return f32(np.cos(np.float64(x)))


def sinr(x):
    return f32(np.sin(np.float64(x)))


def begin(desc, sweep):
    """(shift[3], colour_off) of a box for a sweep."""
    r = philox((sweep & 0xFFFFFFFF, sweep >> 32, P_BIN, 0), desc["key0"], desc["key1"])
    a = f32(f32(1.0) / f32(desc["ncell"]))
    shift = [f32(u01(r[i]) * a) for i in range(3)]
    ncol = desc["stride"] ** 3
    return shift, r[3] % ncol


def bin_cells(desc, shift, xadd, yadd, zadd):
    """Members of every cell of one box (local molecule indices, ascending)."""
    n = desc["ncell"]
    cells = [[] for _ in range(n ** 3)]
    for m in range(xadd.shape[0]):
        c = (cell_coord(xadd[m], shift[0], n) * n + cell_coord(yadd[m], shift[1], n)) * n + \
            cell_coord(zadd[m], shift[2], n)
        cells[c].append(m)
    return cells


def slot_cell(desc, colour_off, step, j):
    n, s = desc["ncell"], desc["stride"]
    na = n // s
    colour = (colour_off + step) % (s ** 3)
    cx, cy, cz = colour // (s * s), (colour // s) % s, colour % s
    return cx + s * (j // (na * na)), cy + s * ((j // na) % na), cz + s * (j % na)


def propose(desc, sweep, step, k_global, cell_members, box):
    """The move of slot k (global slot index k_global) of one box: None if its cell is empty,
    else dict(mol, left, centre (3,), off (n,3), new (n,3)) -- float32, device order.  ``box``
    holds the box's arrays: xa, ya, za, xadd, yadd, zadd, naf, nato (local indices)."""
    cnt = len(cell_members)
    if cnt == 0:
        return None
    k0, k1 = desc["key0"], desc["key1"]
    r0 = philox((sweep & 0xFFFFFFFF, step, k_global, P_MOVE), k0, k1)
    r1 = philox((sweep & 0xFFFFFFFF, step, k_global, P_MOVE + 16), k0, k1)
    pick = min(int(u01(r0[0]) * f32(cnt)), cnt - 1)
    mol = cell_members[pick]
    ct = f32(f32(f32(2.0) * u01(r0[1])) - f32(1.0))
    st = f32(np.sqrt(f32(max(f32(f32(1.0) - f32(ct * ct)), f32(0.0)))))
    ph = f32(f32(6.2831853071795864769) * u01(r0[2]))
    ax, ay, az = f32(st * cosr(ph)), f32(st * sinr(ph)), ct
    al = f32(f32(desc["rotmax"]) * f32(f32(f32(2.0) * u01(r0[3])) - f32(1.0)))
    ca, sa = cosr(al), sinr(al)
    oc = f32(f32(1.0) - ca)
    tm = f32(desc["transmax"])
    cx, cy, cz = box["xadd"][mol], box["yadd"][mol], box["zadd"][mol]
    nx = wrap(f32(cx + f32(tm * f32(f32(f32(2.0) * u01(r1[0])) - f32(1.0)))))
    ny = wrap(f32(cy + f32(tm * f32(f32(f32(2.0) * u01(r1[1])) - f32(1.0)))))
    nz = wrap(f32(cz + f32(tm * f32(f32(f32(2.0) * u01(r1[2])) - f32(1.0)))))
    a0, na = int(box["naf"][mol]), int(box["nato"][mol])
    off = np.zeros((na, 3), f32)
    new = np.zeros((na, 3), f32)
    for q in range(na):
        vx, vy, vz = box["xa"][a0 + q], box["ya"][a0 + q], box["za"][a0 + q]
        dot = f32(f32(f32(ax * vx) + f32(ay * vy)) + f32(az * vz))
        cxv = f32(f32(ay * vz) - f32(az * vy))
        cyv = f32(f32(az * vx) - f32(ax * vz))
        czv = f32(f32(ax * vy) - f32(ay * vx))
        dd = f32(dot * oc)
        rx = f32(f32(f32(vx * ca) + f32(cxv * sa)) + f32(ax * dd))
        ry = f32(f32(f32(vy * ca) + f32(cyv * sa)) + f32(ay * dd))
        rz = f32(f32(f32(vz * ca) + f32(czv * sa)) + f32(az * dd))
        off[q] = (rx, ry, rz)
        new[q] = (f32(rx + nx), f32(ry + ny), f32(rz + nz))
    return dict(mol=mol, centre=np.array([nx, ny, nz], f32), off=off, new=new)


def left_cell(desc, shift, prop, cell):
    n = desc["ncell"]
    c = prop["centre"]
    return (cell_coord(c[0], shift[0], n), cell_coord(c[1], shift[1], n), cell_coord(c[2], shift[2], n)) != cell


def dist(a, b):
    d = [f32(b[i] - a[i]) for i in range(3)]
    d = [f32(v - nint(v)) for v in d]
    return f32(np.sqrt(f32(f32(f32(d[0] * d[0]) + f32(d[1] * d[1])) + f32(d[2] * d[2]))))


def features(desc, prop, box, pos, fclass, partners):
    """Radial histograms (before, after) of the moved molecule against ``partners`` (local
    molecule indices), as integer counts [1280]."""
    hist = np.zeros(2 * FEAT_HALF, np.int64)
    mol = prop["mol"]
    a0, na = int(box["naf"][mol]), int(box["nato"][mol])
    rf = f32(desc["rfeat"])
    binf = f32(f32(f32(FEAT_BINS) / f32(8.0)) * f32(desc["dmax"]))
    for jm in partners:
        if jm == mol:
            continue
        b0, nb = int(box["naf"][jm]), int(box["nato"][jm])
        for q in range(nb):
            pb = pos[b0 + q]
            for a in range(na):
                c1, c2 = sorted((int(fclass[a0 + a]), int(fclass[b0 + q])))
                fc = ((c1 * (7 - c1)) // 2 + c2) * FEAT_BINS
                d0 = dist(pos[a0 + a], pb)
                d1 = dist(prop["new"][a], pb)
                if d0 < rf:
                    hist[fc + min(int(f32(d0 * binf)), FEAT_BINS - 1)] += 1
                if d1 < rf:
                    hist[FEAT_HALF + fc + min(int(f32(d1 * binf)), FEAT_BINS - 1)] += 1
    return hist


def decide_draw(desc, sweep, step, k_global):
    """(u1, u2): the first- and second-stage uniforms of slot k."""
    r = philox((sweep & 0xFFFFFFFF, step, k_global, P_DECIDE), desc["key0"], desc["key1"])
    return u01(r[0]), u01(r[1])

"""Linear-optics design of the synthetic RHIC-like ring (design-time tool).

The benchmark ring is synthetic: 6 arcs of 36 FODO cells (thick sector
dipoles, thick quadrupoles, thin chromatic sextupoles), two low-beta
interaction regions with thick triplets, and four utility straights.  This
module computes the quadrupole and sextupole strengths with a plain 4x4 /
3x3 transfer-matrix model (hard-edge thick quadrupoles, sector bends,
drifts) and a least-squares fit: beta* at both interaction points,
alpha = 0 at every straight's centre, the working-point tunes and the
linear chromaticities.  The fitted numbers are frozen into
simtrack_b200.lattices (RHIC_LIKE_STRENGTHS), so the ring itself needs no
optimiser; run this module to reproduce them:

    python -m simtrack_b200.lattice_design
"""
from __future__ import annotations

import math

import numpy as np

# Geometry (metres)
N_ARC = 6
CELLS_PER_ARC = 36
LQ = 1.1          # arc quadrupole length
LB = 5.8          # arc dipole length
LD = 0.5          # arc drift between sextupole and dipole
L_STAR = 10.0     # IP to first triplet quadrupole
LQ1, LQ2, LQ3 = 1.5, 3.0, 1.5
LQ4 = 1.5
LQU = 1.1         # utility straight quadrupoles
ANGLE = 2 * math.pi / (2 * N_ARC * CELLS_PER_ARC)
CIRC = 3834.0


def cell_length():
    return 2 * LQ + 2 * LB + 2 * LD


def ins_length():
    return (CIRC - N_ARC * CELLS_PER_ARC * cell_length()) / N_ARC


def ir_drifts():
    """Drifts of the half interaction region: [a, Q4, b, Q3, c, Q2, d, Q1, L*]."""
    half = ins_length() / 2
    quads = LQ4 + LQ3 + LQ2 + LQ1
    free = half - quads - L_STAR
    # split the remaining length: a (towards the arc) takes the most
    c = 0.8
    d = 0.8
    b = 8.0
    a = free - b - c - d
    assert a > 1.0, a
    return a, b, c, d


def util_drifts():
    half = ins_length() / 2
    # [a, Qa, b, Qb, c] with c to the centre
    b = 20.0
    c = 5.0
    a = half - 2 * LQU - b - c
    assert a > 1.0, a
    return a, b, c


def drift(L):
    m = np.eye(4)
    m[0, 1] = L
    m[2, 3] = L
    return m


def quad(L, k1l):
    m = np.eye(4)
    if L == 0:
        m[1, 0] = -k1l
        m[3, 2] = k1l
        return m
    k = k1l / L
    for (i, kk) in ((0, k), (2, -k)):
        if kk > 0:
            s = math.sqrt(kk)
            m[i:i + 2, i:i + 2] = [[math.cos(s * L), math.sin(s * L) / s], [-s * math.sin(s * L), math.cos(s * L)]]
        elif kk < 0:
            s = math.sqrt(-kk)
            m[i:i + 2, i:i + 2] = [[math.cosh(s * L), math.sinh(s * L) / s], [s * math.sinh(s * L), math.cosh(s * L)]]
        else:
            m[i:i + 2, i:i + 2] = [[1, L], [0, 1]]
    return m


def sbend(L, ang):
    m = np.eye(4)
    rho = L / ang
    c, s = math.cos(ang), math.sin(ang)
    m[0:2, 0:2] = [[c, rho * s], [-s / rho, c]]
    m[2, 3] = L
    return m


def disp3(L, kind, val=0.0):
    """3x3 horizontal matrix with dispersion column."""
    m = np.eye(3)
    if kind == "drift":
        m[0, 1] = L
    elif kind == "quad":
        m[0:2, 0:2] = quad(L, val)[0:2, 0:2]
    elif kind == "bend":
        rho = L / val
        c, s = math.cos(val), math.sin(val)
        m[0:2, 0:2] = [[c, rho * s], [-s / rho, c]]
        m[0, 2] = rho * (1 - c)
        m[1, 2] = s
    return m


def build_sequence(p):
    """Sequence of (kind, L, value, tag) for the whole ring starting at IP1.
    p = dict of strengths."""
    seq = []
    a, b, c, d = ir_drifts()
    ua, ub, uc = util_drifts()

    def half_ir(reverse):
        h = [("drift", L_STAR, 0, "ds"), ("quad", LQ1, p["q1"], "q1"), ("drift", d, 0, ""),
             ("quad", LQ2, p["q2"], "q2"), ("drift", c, 0, ""), ("quad", LQ3, p["q3"], "q3"),
             ("drift", b, 0, ""), ("quad", LQ4, p["q4"], "q4"), ("drift", a, 0, "")]
        return h if not reverse else h[::-1]

    def half_util(reverse):
        h = [("drift", uc, 0, ""), ("quad", LQU, p["ub"], "ub"), ("drift", ub, 0, ""),
             ("quad", LQU, p["ua"], "ua"), ("drift", ua, 0, "")]
        return h if not reverse else h[::-1]

    def arc():
        s = [("quad", LQ / 2, p["kf"] / 2, "qf")]
        for i in range(CELLS_PER_ARC):
            s += [("sext", 0, 0, "sf"), ("drift", LD, 0, ""), ("bend", LB, ANGLE, "b"),
                  ("quad", LQ, p["kd"], "qd"), ("sext", 0, 0, "sd"), ("drift", LD, 0, ""), ("bend", LB, ANGLE, "b")]
            s += [("quad", LQ / 2 if i == CELLS_PER_ARC - 1 else LQ, p["kf"] / 2 if i == CELLS_PER_ARC - 1 else p["kf"],
                   "qf")]
        return s

    # insertions: 0 and 3 are IRs (IP at their centre), others utility
    for k in range(N_ARC):
        is_ir = k in (0, 3)
        if k == 0:
            seq += [("marker", 0, 0, "ip1")] + half_ir(False)
        elif is_ir:
            seq += half_ir(True) + [("marker", 0, 0, "ip2")] + half_ir(False)
        else:
            seq += half_util(True) + [("marker", 0, 0, f"u{k}")] + half_util(False)
        seq += arc()
    seq += half_ir(True)
    return seq


def one_turn(seq):
    m = np.eye(4)
    for kind, L, v, _ in seq:
        if kind == "drift":
            m = drift(L) @ m
        elif kind == "quad":
            m = quad(L, v) @ m
        elif kind == "bend":
            m = sbend(L, v) @ m
    return m


def twiss_from(m):
    out = []
    for i in (0, 2):
        a, b, c, d = m[i, i], m[i, i + 1], m[i + 1, i], m[i + 1, i + 1]
        cosmu = (a + d) / 2
        if abs(cosmu) >= 1:
            return None
        sinmu = math.copysign(math.sqrt(1 - cosmu * cosmu), b)
        beta = b / sinmu
        alpha = (a - d) / (2 * sinmu)
        out.append((beta, alpha, math.acos(cosmu) / (2 * math.pi) if b > 0 else 1 - math.acos(cosmu) / (2 * math.pi)))
    return out


def propagate(seq, tw0):
    """Twiss and phase along seq from (bx, ax, by, ay) at its start."""
    bx, ax, by, ay = tw0
    gx, gy = (1 + ax * ax) / bx, (1 + ay * ay) / by
    mux = muy = 0.0
    rows = []
    for kind, L, v, tag in seq:
        if kind == "drift":
            m = drift(L)
        elif kind == "quad":
            m = quad(L, v)
        elif kind == "bend":
            m = sbend(L, v)
        else:
            m = np.eye(4)
        for i, (b, a, g) in enumerate(((bx, ax, gx), (by, ay, gy))):
            j = 2 * i
            C, S, Cp, Sp = m[j, j], m[j, j + 1], m[j + 1, j], m[j + 1, j + 1]
            nb = C * C * b - 2 * C * S * a + S * S * g
            na = -C * Cp * b + (C * Sp + S * Cp) * a - S * Sp * g
            dmu = math.atan2(S, C * b - S * a) / (2 * math.pi)
            if i == 0:
                bx, ax, gx, mux = nb, na, (1 + na * na) / nb, mux + dmu
            else:
                by, ay, gy, muy = nb, na, (1 + na * na) / nb, muy + dmu
        rows.append((tag, kind, L, v, bx, ax, by, ay, mux, muy))
    return rows


def dispersion(seq, d0):
    D = np.array(d0 + [1.0])
    out = []
    for kind, L, v, tag in seq:
        if kind in ("drift", "quad", "bend"):
            D = disp3(L, kind, v) @ D
        out.append(D[0])
    return out


def periodic_dispersion(seq):
    M = np.eye(3)
    for kind, L, v, _ in seq:
        if kind in ("drift", "quad", "bend"):
            M = disp3(L, kind, v) @ M
    A = np.eye(2) - M[0:2, 0:2]
    return list(np.linalg.solve(A, M[0:2, 2]))


def ring_optics(p):
    seq = build_sequence(p)
    tw = twiss_from(one_turn(seq))
    return seq, tw


def chromaticity(seq, rows, Dx, k2f, k2d):
    """Linear chromaticity from thick quads (slice-integrated beta) and thin sextupoles."""
    xi_x = xi_y = 0.0
    prev = None
    for (tag, kind, L, v, bx, ax, by, ay, mx, my), D in zip(rows, Dx):
        if kind == "quad":
            # use average of entrance/exit beta (entrance from previous row)
            pbx, pby = (prev[4], prev[6]) if prev else (bx, by)
            xi_x -= v * (bx + pbx) / 2
            xi_y += v * (by + pby) / 2
        elif kind == "sext":
            k2 = k2f if tag == "sf" else k2d
            xi_x += k2 * D * bx
            xi_y -= k2 * D * by
        prev = (tag, kind, L, v, bx, ax, by, ay, mx, my)
    return xi_x / (4 * math.pi), xi_y / (4 * math.pi)


def cell_matrix(kf, kd):
    m = np.eye(4)
    for kind, L, v in (("quad", LQ / 2, kf / 2), ("drift", LD, 0), ("bend", LB, ANGLE), ("quad", LQ, kd),
                       ("drift", LD, 0), ("bend", LB, ANGLE), ("quad", LQ / 2, kf / 2)):
        m = (drift(L) if kind == "drift" else quad(L, v) if kind == "quad" else sbend(L, v)) @ m
    return m


def transport(elems, tw0):
    rows = propagate([(k, L, v, "") for k, L, v in elems], tw0)
    r = rows[-1]
    return r[4], r[5], r[6], r[7], r[8], r[9]


def fit(beta_star=0.6, qx_frac=0.31, qy_frac=0.32, chrom=(1.0, 1.0), seed=1):
    """Staged fit: arc cell phase advances -> triplet match to beta* -> utility
    straight match -> outer loop on the cell phase advance for the tunes."""
    from scipy.optimize import least_squares

    rng = np.random.default_rng(seed)
    a, b, c, d = ir_drifts()
    ua, ub, uc = util_drifts()

    def arc_k(mux, muy, guess):
        def r(v):
            tw = twiss_from(cell_matrix(*v))
            if tw is None:
                return [10.0, 10.0]
            return [tw[0][2] - mux, tw[1][2] - muy]
        sol = least_squares(r, guess)
        return sol.x

    def match_ir(tw0, guess):
        def r(v):
            q1, q2, q3, q4 = v
            el = [("drift", a, 0), ("quad", LQ4, q4), ("drift", b, 0), ("quad", LQ3, q3), ("drift", c, 0),
                  ("quad", LQ2, q2), ("drift", d, 0), ("quad", LQ1, q1), ("drift", L_STAR, 0)]
            bx, ax, by, ay, _, _ = transport(el, tw0)
            if bx <= 0 or by <= 0:
                return [10, 10, 10, 10]
            return [math.log(bx / beta_star), math.log(by / beta_star), ax, ay]
        best = None
        starts = [guess] + [list(rng.normal(0, 0.12, 4)) for _ in range(400)]
        for s0 in starts:
            if s0 is None:
                continue
            try:
                sol = least_squares(r, s0, bounds=([-0.4] * 4, [0.4] * 4))
            except ValueError:
                continue
            if best is None or sol.cost < best.cost:
                best = sol
            if best.cost < 1e-20:
                break
        return best.x, best.cost

    def match_util(tw0, guess):
        def r(v):
            qa, qb = v
            el = [("drift", ua, 0), ("quad", LQU, qa), ("drift", ub, 0), ("quad", LQU, qb), ("drift", uc, 0)]
            bx, ax, by, ay, _, _ = transport(el, tw0)
            return [ax, ay]
        best = None
        for s0 in [guess] + [list(rng.normal(0, 0.1, 2)) for _ in range(200)]:
            if s0 is None:
                continue
            sol = least_squares(r, s0, bounds=([-0.4] * 2, [0.4] * 2))
            if best is None or sol.cost < best.cost:
                best = sol
            if best.cost < 1e-22:
                break
        return best.x, best.cost

    def design(mux, muy, gk=(0.16, -0.16), gir=None, gu=None):
        kf, kd = arc_k(mux, muy, list(gk))
        tw = twiss_from(cell_matrix(kf, kd))
        tw0 = (tw[0][0], tw[0][1], tw[1][0], tw[1][1])
        qir, cir = match_ir(tw0, gir)
        qu, cu = match_util(tw0, gu)
        p = dict(kf=kf, kd=kd, q1=qir[0], q2=qir[1], q3=qir[2], q4=qir[3], ua=qu[0], ub=qu[1])
        return p, cir, cu

    mux, muy = 0.21, 0.205
    p, cir, cu = design(mux, muy)
    for _ in range(6):
        seq = build_sequence(p)
        tw = twiss_from(one_turn(seq))
        (bx, ax, qx), (by, ay, qy) = tw
        rows = propagate(seq, (bx, ax, by, ay))
        Qx, Qy = rows[-1][8], rows[-1][9]
        dqx = ((qx_frac - Qx) + 0.5) % 1 - 0.5
        dqy = ((qy_frac - Qy) + 0.5) % 1 - 0.5
        if abs(dqx) < 1e-7 and abs(dqy) < 1e-7:
            break
        n_cells = N_ARC * CELLS_PER_ARC
        mux += dqx / n_cells
        muy += dqy / n_cells
        p, cir, cu = design(mux, muy, (p["kf"], p["kd"]), [p["q1"], p["q2"], p["q3"], p["q4"]], [p["ua"], p["ub"]])
    seq = build_sequence(p)
    (bx, ax, qx), (by, ay, qy) = twiss_from(one_turn(seq))
    rows = propagate(seq, (bx, ax, by, ay))
    Dx = dispersion(seq, periodic_dispersion(seq))
    x0 = chromaticity(seq, rows, Dx, 0.0, 0.0)
    ca = chromaticity(seq, rows, Dx, 1.0, 0.0)
    cb = chromaticity(seq, rows, Dx, 0.0, 1.0)
    A = np.array([[ca[0] - x0[0], cb[0] - x0[0]], [ca[1] - x0[1], cb[1] - x0[1]]])
    k2 = np.linalg.solve(A, np.array(chrom) - np.array(x0))
    info = dict(match_cost=(float(cir), float(cu)), tunes=(rows[-1][8], rows[-1][9]), beta_ip=(bx, by),
                alpha_ip=(ax, ay), natural_chrom=x0, beta_max=(max(r[4] for r in rows), max(r[6] for r in rows)),
                dmax=max(abs(v) for v in Dx), d_ip=Dx[0], cell_mu=(mux, muy))
    return p, dict(k2f=float(k2[0]), k2d=float(k2[1])), info


if __name__ == "__main__":
    p, k2, info = fit()
    print("strengths (K1L):", {k: float(repr_v) for k, repr_v in p.items()})
    print("sextupoles (K2L):", k2)
    print(info)

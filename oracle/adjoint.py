"""Test infrastructure: FP64 restatement of the PRP objective over a fixed support and of its
derivatives, the checker of the CUDA adjoint (u26_prp_adjoint) and of the finite-difference
tests. Not used by the product path.

A hit (HIT_DTYPE record) has the distance delta(x, r) = (w . n) / (r . n):
  VF  vertex p = sv[0] along +r onto face a b c = dv:   w = a - p,   n = (b - a) x (c - a)
  FV  vertex q = dv[0] along -r onto face a b c = sv:   w = q - a,   n = (b - a) x (c - a)
  EE  edge p0 p1 = sv[0:2] swept along r onto q0 q1 = dv[0:2]:  w = q0 - p0, n = (p1 - p0) x (q1 - q0)
(the closed forms of the reference's ray-triangle and swept-edge tests,
intersection_resolver_helper.cpp:319-514, cached_bvh.cpp:321-555). Per contour:
  J = (sum of source rest areas) * max(delta)^2      (prp_eval_penetration_v2, resolver2.cpp:1883-1954)
  E = sum (delta + 3e-3)^2 / kappa                    (its displacement cost; kappa: helper.cpp:611-645)
"""
import numpy as np


def hit_vertices(h):
    """The four vertex ids of a hit in the order (p, a, b, c) / (q, a, b, c) / (p0, p1, q0, q1)."""
    t = int(h["type"])
    sv, dv = [int(v) for v in h["sv"]], [int(v) for v in h["dv"]]
    if t == 0:
        return [sv[0], dv[0], dv[1], dv[2]]
    if t == 2:
        return [dv[0], sv[0], sv[1], sv[2]]
    return [sv[0], sv[1], dv[0], dv[1]]


def delta(h, P, r):
    """delta of hit h from its four vertex positions P [4, 3] (float64) and direction r."""
    t = int(h["type"])
    if t == 1:
        n = np.cross(P[1] - P[0], P[3] - P[2])
        w = P[2] - P[0]
    else:
        n = np.cross(P[2] - P[1], P[3] - P[1])
        w = P[1] - P[0] if t == 0 else P[0] - P[1]
    return float(np.dot(w, n) / np.dot(r, n))


def delta_grads(h, P, r):
    """(d delta / d P [4, 3], d delta / d r [3]) in closed form."""
    t = int(h["type"])
    if t == 1:
        e1, e2 = P[1] - P[0], P[3] - P[2]
        n, w = np.cross(e1, e2), P[2] - P[0]
    else:
        n = np.cross(P[2] - P[1], P[3] - P[1])
        w = P[1] - P[0] if t == 0 else P[0] - P[1]
    rn = np.dot(r, n)
    d = np.dot(w, n) / rn
    u = w - d * r
    g = np.zeros((4, 3))
    if t == 1:
        g[0] = -n - np.cross(e2, u)
        g[1] = np.cross(e2, u)
        g[2] = n - np.cross(u, e1)
        g[3] = np.cross(u, e1)
    else:
        A, B, C = P[1], P[2], P[3]
        g[0] = -n if t == 0 else n
        g[1] = (n if t == 0 else -n) + np.cross(u, C - B)
        g[2] = np.cross(C - A, u)
        g[3] = np.cross(u, B - A)
    return g / rn, -d * n / rn


def kappa(h, vert_mass):
    im = lambda v: 1.0 / max(float(vert_mass[v]), 1e-8)
    t = int(h["type"])
    b0, b1 = float(h["bary"][0]), float(h["bary"][1])
    sv, dv = [int(v) for v in h["sv"]], [int(v) for v in h["dv"]]
    if t == 0:
        bz = 1.0 - b0 - b1
        return im(sv[0]) + b0 * b0 * im(dv[0]) + b1 * b1 * im(dv[1]) + bz * bz * im(dv[2])
    if t == 2:
        bz = 1.0 - b0 - b1
        return b0 * b0 * im(sv[0]) + b1 * b1 * im(sv[1]) + bz * bz * im(sv[2]) + im(dv[0])
    return b0 * b0 * im(sv[0]) + (1 - b0) ** 2 * im(sv[1]) + b1 * b1 * im(dv[0]) + (1 - b1) ** 2 * im(dv[1])


def source_area(h, vert_area, edge_area, face_area):
    t = int(h["type"])
    return float((vert_area, edge_area, face_area)[t][int(h["src_id"])])


def objective(hits, x, r, vert_area, edge_area, face_area, vert_mass):
    """(J, E, index of the first maximal hit) of one contour's support in FP64."""
    x = np.asarray(x, np.float64)
    r = np.asarray(r, np.float64)
    A, E, D, imax = 0.0, 0.0, -np.inf, -1
    for i, h in enumerate(hits):
        d = delta(h, x[hit_vertices(h)], r)
        A += source_area(h, vert_area, edge_area, face_area)
        k = kappa(h, vert_mass)
        E += (d + 3e-3) ** 2 / k if k > 1e-8 else 0.0
        if d > D:
            D, imax = d, i
    if not len(hits):
        D = 0.0
    return A * D * D, E, imax


def gradients(hits, x, r, vert_area, edge_area, face_area, vert_mass):
    """(dJ/dx [V, 3], dJ/dr, dE/dx [V, 3], dE/dr) in FP64, J through its first maximal hit."""
    x = np.asarray(x, np.float64)
    r = np.asarray(r, np.float64)
    J, E, imax = objective(hits, x, r, vert_area, edge_area, face_area, vert_mass)
    A = sum(source_area(h, vert_area, edge_area, face_area) for h in hits)
    gJx, gEx = np.zeros_like(x), np.zeros_like(x)
    gJr, gEr = np.zeros(3), np.zeros(3)
    for i, h in enumerate(hits):
        V = hit_vertices(h)
        d = delta(h, x[V], r)
        gP, gr = delta_grads(h, x[V], r)
        k = kappa(h, vert_mass)
        if k > 1e-8:
            c = 2.0 * (d + 3e-3) / k
            gEr += c * gr
            np.add.at(gEx, V, c * gP)
        if i == imax:
            c = 2.0 * A * d
            gJr += c * gr
            np.add.at(gJx, V, c * gP)
    return gJx, gJr, gEx, gEr


def refine_gradient(hits, x, r, vert_mass):
    """The gradient of the reference's direction refinement with the stored hit distances:
    sum 2 w (dist + 3e-3) (-dist n / (n . r)), n the unit characteristic normal, w = 1 / kappa
    (prp_compute_direction_optimization_step, intersection_resolver2.cpp:1268-1320), FP64."""
    x = np.asarray(x, np.float64)
    r = np.asarray(r, np.float64)
    g = np.zeros(3)
    for h in hits:
        P = x[hit_vertices(h)]
        t = int(h["type"])
        n = np.cross(P[1] - P[0], P[3] - P[2]) if t == 1 else np.cross(P[2] - P[1], P[3] - P[1])
        n = n / np.linalg.norm(n)
        k = kappa(h, vert_mass)
        if k <= 1e-8 or abs(np.dot(n, r)) < 1e-6:
            continue
        d = float(h["dist"])
        g += 2.0 / k * (d + 3e-3) * (-d * n / np.dot(n, r))
    return g

"""Test infrastructure only (the checker): a numpy restatement of the
primitive contact generation of sap_warp_b200/csrc/sapb_contacts.cu -- the
same closed-form pair tests, the same pair and contact order, the output in
the format of the reference's contact writer (sim/collision/pipeline.py:52-118:
witness points in the body frames of their shapes, normal from shape0 to
shape1, margins; a sphere's centre with its radius in the margin)."""

from __future__ import annotations

import numpy as np

from oracle.boundary import qrot

PLANE, SPHERE, BOX = 0, 1, 2


def _conj(q):
    return np.array([-q[0], -q[1], -q[2], q[3]])


def _qmul(a, b):
    ax, ay, az, aw = a
    bx, by, bz, bw = b
    return np.array([aw * bx + ax * bw + ay * bz - az * by, aw * by - ax * bz + ay * bw + az * bx,
                     aw * bz + ax * by - ay * bx + az * bw, aw * bw - ax * bx - ay * by - az * bz])


def generate(shapes, body_q, gap=1.0e-3):
    """shapes: collision.ShapeSet; body_q [B][7].  Returns a dict of lists."""
    E, Sw, G = shapes.num_worlds, shapes.shapes_per_world, shapes.num_global_shapes
    out = dict(shape0=[], shape1=[], point0=[], point1=[], normal=[], margin0=[], margin1=[])
    margin = shapes.shape_margin if shapes.shape_margin is not None else np.zeros(len(shapes.shape_type))

    def world(sh):
        X = shapes.shape_X_bs[sh]
        b = shapes.shape_body[sh]
        if b < 0:
            return X[:3], X[3:]
        bq = body_q[b]
        return bq[:3] + qrot(bq[3:], X[:3]), _qmul(bq[3:], X[3:])

    def local(sh, pw):
        b = shapes.shape_body[sh]
        if b < 0:
            return pw
        return qrot(_conj(body_q[b, 3:]), pw - body_q[b, :3])

    def emit(a, b, xa, xb, n, ma, mb):
        out["shape0"].append(a)
        out["shape1"].append(b)
        out["point0"].append(local(a, xa))
        out["point1"].append(local(b, xb))
        out["normal"].append(n)
        out["margin0"].append(ma)
        out["margin1"].append(mb)

    def corners(h):
        return [np.array([h[0] if c & 1 else -h[0], h[1] if c & 2 else -h[1], h[2] if c & 4 else -h[2]])
                for c in range(8)]

    def box_vs_box(a, b, Xa, ha, Xb, hb, g, ma, mb):
        for vl in corners(hb):
            vw = Xb[0] + qrot(Xb[1], vl)
            p = qrot(_conj(Xa[1]), vw - Xa[0])
            e = np.abs(p) - ha
            if np.any(e > g):
                continue
            k = int(np.argmax(e))  # first maximum, as the kernel's strict comparisons
            s = 1.0 if p[k] >= 0 else -1.0
            nl = np.zeros(3)
            nl[k] = s
            face = p.copy()
            face[k] = s * ha[k]
            emit(a, b, Xa[0] + qrot(Xa[1], face), vw, qrot(Xa[1], nl), ma, mb)

    def box_edge(a, b, Xa, ha, Xb, hb, g, ma, mb):
        """The edge-edge contact of two boxes: separating axes over the 6
        face and 9 edge-pair axes; the best edge axis, if it beats every face
        axis by a relative 1e-6 and lies within g, gives one contact at the
        closest points of its two supporting edges when both lie inside the
        edges (as sap_collide_box_box's edge case,
        sim/collision/primitive.py:692-1148)."""
        A = [qrot(Xa[1], e) for e in np.eye(3)]
        B = [qrot(Xb[1], e) for e in np.eye(3)]
        d = Xb[0] - Xa[0]

        def radius(E, h, L):
            return h[0] * abs(np.dot(E[0], L)) + h[1] * abs(np.dot(E[1], L)) + h[2] * abs(np.dot(E[2], L))

        best_face = -1.0e300
        for k in range(3):
            sa = abs(np.dot(d, A[k])) - (ha[k] + radius(B, hb, A[k]))
            sb = abs(np.dot(d, B[k])) - (radius(A, ha, B[k]) + hb[k])
            best_face = max(best_face, max(sa, sb))
        best_edge, bi, bj, bL = -1.0e300, -1, -1, None
        for i in range(3):
            for j in range(3):
                L = np.cross(A[i], B[j])
                ln = np.sqrt(np.dot(L, L))
                if ln < 1.0e-6:
                    continue
                L = (1.0 / ln) * L
                if np.dot(d, L) < 0.0:
                    L = -L
                sep = np.dot(d, L) - radius(A, ha, L) - radius(B, hb, L)
                if sep > best_edge:
                    best_edge, bi, bj, bL = sep, i, j, L
        scale = max(max(ha), max(hb))
        if bi < 0 or not best_edge > best_face + 1.0e-6 * scale or not best_edge < g:
            return
        cA, cB = Xa[0].copy(), Xb[0].copy()
        for m in range(3):
            if m != bi:
                cA = cA + (ha[m] if np.dot(A[m], bL) >= 0.0 else -ha[m]) * A[m]
            if m != bj:
                cB = cB - (hb[m] if np.dot(B[m], bL) >= 0.0 else -hb[m]) * B[m]
        u, v, w = A[bi], B[bj], cA - cB
        uv, uw, vw = np.dot(u, v), np.dot(u, w), np.dot(v, w)
        den = 1.0 - uv * uv
        if den < 1.0e-12:
            return
        s_, t_ = (uv * vw - uw) / den, (vw - uv * uw) / den
        if abs(s_) > ha[bi] or abs(t_) > hb[bj]:
            return
        emit(a, b, cA + s_ * u, cB + t_ * v, bL, ma, mb)

    groups = getattr(shapes, "shape_collision_group", None)

    def groups_meet(ga, gb):  # sim/collision/broad_phase_common.py:133-150
        if ga == 0 or gb == 0:
            return False
        if ga > 0:
            return ga == gb or gb < 0
        return ga != gb

    def pair(sa, sb):
        if groups is not None and not groups_meet(int(groups[sa]), int(groups[sb])):
            return
        a, b = sa, sb
        if shapes.shape_type[a] > shapes.shape_type[b]:
            a, b = b, a
        t1, t2 = shapes.shape_type[a], shapes.shape_type[b]
        m1, m2 = margin[a], margin[b]
        Xa, Xb = world(a), world(b)
        s1, s2 = shapes.shape_scale[a], shapes.shape_scale[b]
        if t1 == PLANE and t2 == PLANE:
            return
        if t1 != PLANE:
            # the kernel's conservative bounding-sphere cut
            ra = s1[0] if t1 == SPHERE else np.sqrt(np.dot(s1, s1))
            rb = s2[0] if t2 == SPHERE else np.sqrt(np.dot(s2, s2))
            dd = Xb[0] - Xa[0]
            reach = (ra + rb + 1.7320508075688772 * (abs(m1) + abs(m2) + abs(gap))) * (1.0 + 1.0e-12) + 1.0e-12
            if np.dot(dd, dd) > reach * reach:
                return
        if t1 == PLANE:
            n = qrot(Xa[1], np.array([0.0, 0.0, 1.0]))
            if t2 == SPHERE:
                h = np.dot(Xb[0] - Xa[0], n)
                if h - s2[0] - m1 - m2 < gap:
                    emit(a, b, Xb[0] - h * n, Xb[0], n, m1, s2[0] + m2)
            elif t2 == BOX:
                # at most four corners, the deepest, in the slots of
                # sap_collide_plane_box (sim/collision/primitive.py:354-428)
                kept = []  # [distance, world corner]
                worst = 0
                for vl in corners(s2):
                    vw = Xb[0] + qrot(Xb[1], vl)
                    d = np.dot(vw - Xa[0], n)
                    if not d - m1 - m2 < gap:
                        continue
                    if len(kept) < 4:
                        kept.append([d, vw])
                        if len(kept) == 1 or d > kept[worst][0]:
                            worst = len(kept) - 1
                    elif d < kept[worst][0]:
                        kept[worst] = [d, vw]
                        worst = int(np.argmax([k[0] for k in kept]))
                for d, vw in kept:
                    emit(a, b, vw - d * n, vw, n, m1, m2)
            return
        if t1 == SPHERE and t2 == SPHERE:
            dl = Xb[0] - Xa[0]
            dist = np.linalg.norm(dl)
            if dist - s1[0] - s2[0] - m1 - m2 >= gap:
                return
            n = dl / dist if dist > 1e-12 else np.array([0.0, 0.0, 1.0])
            emit(a, b, Xa[0], Xb[0], n, s1[0] + m1, s2[0] + m2)
            return
        if t1 == SPHERE and t2 == BOX:
            c = qrot(_conj(Xb[1]), Xa[0] - Xb[0])
            p = np.clip(c, -s2, s2)
            dl = c - p
            dd = np.linalg.norm(dl)
            if dd > 1e-12:
                nl, d = dl / dd, dd
            else:
                e = np.abs(c) - s2
                k = int(np.argmax(e))
                s = 1.0 if c[k] >= 0 else -1.0
                nl = np.zeros(3)
                nl[k] = s
                p = p.copy()
                p[k] = s * s2[k]
                d = e[k]
            if d - s1[0] - m1 - m2 >= gap:
                return
            emit(b, a, Xb[0] + qrot(Xb[1], p), Xa[0], qrot(Xb[1], nl), m2, s1[0] + m1)
            return
        if t1 == BOX and t2 == BOX:
            box_vs_box(a, b, Xa, s1, Xb, s2, gap + m1 + m2, m1, m2)
            box_vs_box(b, a, Xb, s2, Xa, s1, gap + m1 + m2, m2, m1)
            box_edge(a, b, Xa, s1, Xb, s2, gap + m1 + m2, m1, m2)

    for w in range(E):
        base, gbase = w * Sw, E * Sw
        for i in range(Sw):
            for g in range(G):
                pair(gbase + g, base + i)
        for i in range(Sw):
            for j in range(i + 1, Sw):
                pair(base + i, base + j)
    return {k: np.array(v) for k, v in out.items()}

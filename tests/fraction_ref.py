"""Independent exact triangle-triangle intersection with Python Fractions.

Test infrastructure.  This is a second, deliberately different restatement of
the pair semantics used to pin the C oracle (oracle/gi_oracle.c):

  * the oracle decides with exact orient3d/orient2d signs and symbolic points;
  * this module clips one closed convex set by the half-spaces that describe
    the other (Sutherland-Hodgman with rational arithmetic), then classifies
    the clipped point set with an exact convex hull.

Semantics restated (reference project paths):
  src/CPU/YellowFilter.h:80-137 -- CGAL::do_intersect(Triangle_3, Triangle_3)
      on closed triangles (here: the exact closed point sets);
  src/CPU/MeshIntersectionCurves.cpp:63-78 -- CGAL::intersection result kinds:
      point, segment, triangle (coplanar, 3 corners), polygon (>= 4 corners).
Degenerate (collinear) triangles are treated as the segment or point they span.
"""
from fractions import Fraction

NONE, POINT, SEGMENT, TRIANGLE, POLYGON = 0, 1, 2, 3, 4


def _F(p):
    return tuple(Fraction(x) for x in p)


def _sub(a, b):
    return (a[0] - b[0], a[1] - b[1], a[2] - b[2])


def _add(a, b):
    return (a[0] + b[0], a[1] + b[1], a[2] + b[2])


def _mul(a, s):
    return (a[0] * s, a[1] * s, a[2] * s)


def _dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def _is_zero(v):
    return v[0] == 0 and v[1] == 0 and v[2] == 0


def _dedupe(pts):
    out = []
    for p in pts:
        if p not in out:
            out.append(p)
    return out


def orient3d(a, b, c, d):
    """Exact sign of det[a - d; b - d; c - d] (the orient3d convention of the
    device predicates and the oracle), from the doubles as exact rationals."""
    a, b, c, d = _F(a), _F(b), _F(c), _F(d)
    v = _dot(_sub(a, d), _cross(_sub(b, d), _sub(c, d)))
    return (v > 0) - (v < 0)


def orient2d(a, b, c, drop):
    """Exact sign of (a_u - c_u)(b_v - c_v) - (a_v - c_v)(b_u - c_u) with
    (u, v) = ((drop + 1) % 3, (drop + 2) % 3)."""
    u, v = (drop + 1) % 3, (drop + 2) % 3
    a, b, c = _F(a), _F(b), _F(c)
    x = (a[u] - c[u]) * (b[v] - c[v]) - (a[v] - c[v]) * (b[u] - c[u])
    return (x > 0) - (x < 0)


def _shape(tri):
    """Return ('tri', pts) / ('seg', (e0, e1)) / ('pt', (p,))."""
    p, q, r = tri
    n = _cross(_sub(q, p), _sub(r, p))
    if not _is_zero(n):
        return "tri", tri
    d = _dedupe([p, q, r])
    if len(d) == 1:
        return "pt", (p,)
    # collinear: extreme points along the direction
    base = d[0]
    direction = _sub(d[1], d[0])
    ts = [(_dot(_sub(x, base), direction), x) for x in d]
    ts.sort(key=lambda z: z[0])
    return "seg", (ts[0][1], ts[-1][1])


def _constraints(shape, pts):
    """Half-space constraints h(x) = dot(n, x) - c >= 0 describing the set."""
    cons = []
    if shape == "tri":
        p, q, r = pts
        n = _cross(_sub(q, p), _sub(r, p))
        cons.append((n, _dot(n, p)))
        cons.append((_mul(n, -1), -_dot(n, p)))
        for a, b in ((p, q), (q, r), (r, p)):
            m = _cross(n, _sub(b, a))  # inward for a counter-clockwise triangle about n
            cons.append((m, _dot(m, a)))
    elif shape == "seg":
        e0, e1 = pts
        d = _sub(e1, e0)
        axes = [(1, 0, 0), (0, 1, 0), (0, 0, 1)]
        na = None
        for ax in axes:
            c = _cross(d, _F(ax))
            if not _is_zero(c):
                na = c
                break
        nb = _cross(d, na)
        for n in (na, nb):
            cons.append((n, _dot(n, e0)))
            cons.append((_mul(n, -1), -_dot(n, e0)))
        cons.append((d, _dot(d, e0)))
        cons.append((_mul(d, -1), -_dot(d, e1)))
    else:
        (p,) = pts
        for ax in ((1, 0, 0), (0, 1, 0), (0, 0, 1)):
            n = _F(ax)
            cons.append((n, _dot(n, p)))
            cons.append((_mul(n, -1), -_dot(n, p)))
    return cons


def _clip(poly, n, c):
    """Sutherland-Hodgman clip of a cyclic vertex list by dot(n,x) >= c."""
    if not poly:
        return []
    out = []
    k = len(poly)
    for i in range(k):
        cur, nxt = poly[i], poly[(i + 1) % k]
        hc = _dot(n, cur) - c
        hn = _dot(n, nxt) - c
        if hc >= 0:
            out.append(cur)
        if (hc > 0 and hn < 0) or (hc < 0 and hn > 0):
            t = hc / (hc - hn)
            out.append(_add(cur, _mul(_sub(nxt, cur), t)))
    return out


def _hull_corners(pts):
    """Number of strict convex-hull corners of coplanar points, and the corners."""
    pts = _dedupe(pts)
    if len(pts) <= 2:
        return pts
    # find a normal from a non-collinear triple
    n = None
    for i in range(len(pts)):
        for j in range(i + 1, len(pts)):
            for k in range(j + 1, len(pts)):
                c = _cross(_sub(pts[j], pts[i]), _sub(pts[k], pts[i]))
                if not _is_zero(c):
                    n = c
                    break
            if n:
                break
        if n:
            break
    if n is None:
        # collinear: extremes
        d = _sub(pts[1], pts[0])
        ts = sorted(pts, key=lambda x: _dot(_sub(x, pts[0]), d))
        return [ts[0], ts[-1]]
    drop = max(range(3), key=lambda i: abs(n[i]))
    u, v = [i for i in range(3) if i != drop]
    idx = sorted(range(len(pts)), key=lambda i: (pts[i][u], pts[i][v]))

    def cr(o, a, b):
        return (a[u] - o[u]) * (b[v] - o[v]) - (a[v] - o[v]) * (b[u] - o[u])

    lower, upper = [], []
    for i in idx:
        while len(lower) >= 2 and cr(pts[lower[-2]], pts[lower[-1]], pts[i]) <= 0:
            lower.pop()
        lower.append(i)
    for i in reversed(idx):
        while len(upper) >= 2 and cr(pts[upper[-2]], pts[upper[-1]], pts[i]) <= 0:
            upper.pop()
        upper.append(i)
    hull = lower[:-1] + upper[:-1]
    return [pts[i] for i in hull]


def tri_tri(t1, t2):
    """Exact intersection of two closed triangles given as 3 points each.

    Returns (kind, points) with points as tuples of Fractions."""
    P = [_F(p) for p in t1]
    Q = [_F(p) for p in t2]
    sp, pp = _shape(P)
    sq, qp = _shape(Q)
    rank = {"tri": 2, "seg": 1, "pt": 0}
    # clip the lower-dimensional set by the constraints of the other one
    if rank[sp] < rank[sq]:
        poly, cons = list(pp), _constraints(sq, qp)
    else:
        poly, cons = list(qp), _constraints(sp, pp)
    for n, c in cons:
        poly = _clip(poly, n, c)
        if not poly:
            break
    pts = _dedupe(poly)
    if not pts:
        return NONE, []
    if len(pts) == 1:
        return POINT, pts
    corners = _hull_corners(pts)
    if len(corners) == 1:
        return POINT, corners
    if len(corners) == 2:
        return SEGMENT, corners
    if len(corners) == 3:
        return TRIANGLE, corners
    return POLYGON, corners


def tri_tri_float(t1, t2):
    """As tri_tri, with points correctly rounded to floats."""
    kind, pts = tri_tri(t1, t2)
    return kind, [tuple(float(x) for x in p) for p in pts]

"""Derive the minimax polynomial coefficients used by sbx_math.h.

The Remez exchange algorithm (E. Ya. Remez, 1934; see e.g. Cheney, "Introduction to
Approximation Theory", ch. 3) finds the polynomial of a given degree whose weighted error
against a function equioscillates on an interval, i.e. the minimax polynomial. Each
function of sbx_math.h keeps its argument reduction and its evaluation shape; only the
polynomial on the reduced range is the minimax one instead of a truncated Taylor series,
which reaches the same accuracy with fewer terms:

    sin r = r + r^3 P(r^2)              |r| <= pi/4     P degree 5   (Taylor: degree 9)
    cos r = 1 + r^2 (-1/2 + r^2 Q(r^2))  |r| <= pi/4     Q degree 5   (Taylor: degree 9)
    log m = 2s + 2s s^2 R(s^2), s = (m-1)/(m+1), |s| <= 3 - 2 sqrt 2   R degree 6   (Taylor: 10)
    e^r = 1 + r + r^2 E(r)              |r| <= ln2 / 2  E degree 10  (Taylor: degree 13)

Weights: the error of P, Q and R is weighted by the factor that carries it into the
relative error of the result (r^2, r^4, s^2); E is fitted in absolute error (its error
reaches e^r scaled by r^2 <= 0.121). The intervals are widened by 1e-4 relative to cover
the reduction's rounding. Coefficients are printed as C99 hex doubles.

Needs mpmath (not needed to build or run the library).

    python softbox_b200/csrc/gen_math_polys.py
"""
import mpmath as mp

mp.mp.dps = 60


def remez(f, w, a, b, deg, iters=40, npts=6000):
    """Weighted minimax polynomial c[0] + c[1] x + ... for f on [a, b] (weight w)."""
    n = deg + 2
    xs = [(a + b) / 2 - (b - a) / 2 * mp.cos(mp.pi * i / (n - 1)) for i in range(n)]
    mx = None
    for _ in range(iters):
        A = mp.matrix(n, n)
        y = mp.matrix(n, 1)
        for i, x in enumerate(xs):
            for j in range(deg + 1):
                A[i, j] = x ** j
            A[i, deg + 1] = (-1) ** i / w(x)
            y[i] = f(x)
        sol = mp.lu_solve(A, y)
        c = [sol[j] for j in range(deg + 1)]

        def err(x):
            return w(x) * (f(x) - mp.polyval(c[::-1], x))

        grid = [a + (b - a) * k / npts for k in range(npts + 1)]
        ev = [err(x) for x in grid]
        ext = [0] + [k for k in range(1, npts) if (ev[k] - ev[k - 1]) * (ev[k + 1] - ev[k]) <= 0] + [npts]
        alt = []
        for k in ext:
            p = (grid[k], ev[k])
            if alt and (alt[-1][1] > 0) == (p[1] > 0):
                if abs(p[1]) > abs(alt[-1][1]):
                    alt[-1] = p
            else:
                alt.append(p)
        while len(alt) > n:
            alt.pop(0 if abs(alt[0][1]) < abs(alt[-1][1]) else -1)
        mx = max(abs(p[1]) for p in alt)
        if len(alt) < n:
            raise RuntimeError("Remez: lost the alternation")
        xs = [p[0] for p in alt]
        if mx / min(abs(p[1]) for p in alt) - 1 < mp.mpf("1e-4"):
            break
    return c, mx


def main():
    tiny = mp.mpf("1e-40")
    R = mp.pi / 4 * mp.mpf("1.0001")
    T = R * R
    S = (mp.sqrt(2) - 1) / (mp.sqrt(2) + 1) * mp.mpf("1.0001")
    X = mp.log(2) / 2 * mp.mpf("1.0002")
    jobs = [
        ("SBXM_SIN", lambda t: (mp.sin(mp.sqrt(t)) - mp.sqrt(t)) / mp.sqrt(t) ** 3 if t > 0 else mp.mpf(-1) / 6,
         lambda t: max(t, tiny), mp.mpf(0), T, 5),
        ("SBXM_COS", lambda t: (mp.cos(mp.sqrt(t)) - 1 + t / 2) / (t * t) if t > 0 else mp.mpf(1) / 24,
         lambda t: max(t * t, tiny), mp.mpf(0), T, 5),
        ("SBXM_LOG", lambda u: (mp.atanh(mp.sqrt(u)) / mp.sqrt(u) - 1) / u if u > 0 else mp.mpf(1) / 3,
         lambda u: max(u, tiny), mp.mpf(0), S * S, 6),
        ("SBXM_EXP", lambda r: (mp.exp(r) - 1 - r) / (r * r) if r != 0 else mp.mpf(1) / 2,
         lambda r: mp.mpf(1), -X, X, 10),
    ]
    for name, f, w, a, b, deg in jobs:
        c, mx = remez(f, w, a, b, deg)
        print(f"// {name}: weighted minimax error 2^{float(mp.log(mx, 2)):.1f}")
        for j, v in enumerate(c):
            print(f"#define {name}{j} {float(v).hex()}")


if __name__ == "__main__":
    main()

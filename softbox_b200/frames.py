"""Headless frame output in FrameWriter's JSON schema (FrameWriter.java:16-150).

    fw = FrameWriter("out/run", x_dim, y_dim, z_dim)      # creates out/run or out/run.001, ...
    fw.write_frame(fil, t)                                  # every slot, the viewer's schema
    fw.write_frame(fil, t, nuc_frac=nf)                     # ACTIVE slots, coloured by aging

One file per frame, frame_%06d.json:
    {"frame":N,"t":T,"bounds":{"xDim":..,"yDim":..,"zDim":..},
     "segments":[{"id":I,"end1":[x,y,z],"end2":[x,y,z],"r":R,"notADPRatio":..,
                  "cofilinCount":0,"isBarbedEnd":..}, ...]}
end1/end2 are derived as the reference does, in double from the float pose: end = c -/+
(segLength * 0.5) u; r is Constants.radius; a barbed terminal has no end2 neighbour. The
aging form emits notADPRatio = f_ATP + f_ADPPi and the three fractions. Numbers use
java.util.Formatter's %g layout (significant digits from the shortest decimal
representation rounded half-up, trailing zeros kept, exponent with sign and two digits).
Arrays may be host numpy or device tensors (pulled once per frame).
"""
import math
import os
from decimal import ROUND_HALF_UP, Decimal

import numpy as np

from . import scenes

RADIUS = scenes.ACTIN_RADIUS            # Constants.radius = actinWidth / 2


def java_g(x, prec):
    """Java's String.format(Locale.US, "%.<prec>g", x) for a finite double."""
    x = float(x)
    prec = max(prec, 1)
    sign = "-" if math.copysign(1.0, x) < 0 else ""          # -0.0 prints with its sign too
    if x == 0.0:
        return sign + "0." + "0" * (prec - 1) if prec > 1 else sign + "0"
    d = Decimal(repr(abs(x)))                  # the shortest round-trip decimal
    exp10 = d.adjusted()
    q = d.scaleb(-exp10).quantize(Decimal(1).scaleb(1 - prec), rounding=ROUND_HALF_UP)
    if q >= 10:                                # rounding carried into a new digit
        exp10 += 1
        q = (q / 10).quantize(Decimal(1).scaleb(1 - prec), rounding=ROUND_HALF_UP)
    digits = str(q).replace(".", "")
    if -4 <= exp10 < prec:                     # plain decimal, prec significant digits
        if exp10 >= 0:
            ip, fp = digits[:exp10 + 1], digits[exp10 + 1:]
        else:
            ip, fp = "0", "0" * (-exp10 - 1) + digits
        return sign + ip + ("." + fp if fp else "")
    body = digits[0] + ("." + digits[1:] if prec > 1 else "")
    return f"{sign}{body}e{'-' if exp10 < 0 else '+'}{abs(exp10):02d}"


def _host(a):
    if a is None:
        return None
    if hasattr(a, "detach"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


class FrameWriter:
    def __init__(self, requested_dir, x_dim, y_dim, z_dim):
        self.dir = self._resolve(requested_dir)
        self.x_dim, self.y_dim, self.z_dim = x_dim, y_dim, z_dim
        self.frame = 0

    @staticmethod
    def _resolve(d):
        """Creates `d`, or the first free `d.NNN` (FrameWriter.resolveOutputDir)."""
        if not os.path.exists(d):
            os.makedirs(d)
            return d
        for n in range(1, 1000):
            c = f"{d}.{n:03d}"
            if not os.path.exists(c):
                os.makedirs(c)
                return c
        raise RuntimeError(f"no free output directory for {d}")

    def write_frame(self, fil, t, nuc_frac=None):
        b = fil["body"]
        n = int(b["n"]) if "n" in b else int(_host(b["segLength"]).size)
        c = _host(b["coord"]).reshape(3, n).astype(np.float64)
        u = _host(b["uVec"]).reshape(3, n).astype(np.float64)
        half = _host(b["segLength"]).astype(np.float64) * 0.5
        e1 = c - half * u
        e2 = c + half * u
        barbed = _host(fil["end2NbrSlot"]) < 0
        if nuc_frac is not None:
            state = _host(fil["filState"])
            nf = _host(nuc_frac).reshape(3, n).astype(np.float64)
            slots = np.flatnonzero(state >= 0)
        else:
            nf = None
            slots = np.arange(n)
        g5 = lambda v: java_g(v, 5)          # noqa: E731
        parts = []
        for i in slots:
            s = (f'{{"id":{i},"end1":[{g5(e1[0, i])},{g5(e1[1, i])},{g5(e1[2, i])}],'
                 f'"end2":[{g5(e2[0, i])},{g5(e2[1, i])},{g5(e2[2, i])}],"r":{g5(RADIUS)},')
            if nf is None:
                s += f'"notADPRatio":{java_g(1.0, 3)},"cofilinCount":0,"isBarbedEnd":{"true" if barbed[i] else "false"}}}'
            else:
                fa, fp, fd = nf[0, i], nf[1, i], nf[2, i]
                s += (f'"notADPRatio":{java_g(fa + fp, 3)},"cofilinCount":0,'
                      f'"isBarbedEnd":{"true" if barbed[i] else "false"},"fATP":{java_g(fa, 3)},'
                      f'"fADPPi":{java_g(fp, 3)},"fADP":{java_g(fd, 3)}}}')
            parts.append(s)
        text = (f'{{"frame":{self.frame},"t":{java_g(t, 6)},"bounds":{{"xDim":{g5(self.x_dim)},'
                f'"yDim":{g5(self.y_dim)},"zDim":{g5(self.z_dim)}}},"segments":[' + ",".join(parts) + "]}")
        path = os.path.join(self.dir, f"frame_{self.frame:06d}.json")
        with open(path, "w") as fh:
            fh.write(text)
        self.frame += 1
        return path

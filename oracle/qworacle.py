"""CPU restatement (numpy) of QWalk's per-configuration Slater-Jastrow
evaluation for molecular systems.

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg import this module, and only as the checker.
The product path (mainline_b200 + its CUDA library) never imports it.

Parity is pinned: tests/test_oracle_golden.py checks every quantity below
against golden vectors written by the reference itself (oracle/_ref harness,
tests/golden/make_golden.py).

Reference files cited as path:line inside QWalk/mainline ``src/``.
"""
from __future__ import annotations

import math
import os

import numpy as np

# ----------------------------------------------------------------------------
# input grammar (program_utils/qmc_io.cpp:280-345 parsefile, :168-230 readsection)


def tokenize(path: str) -> list[str]:
    words: list[str] = []
    base = os.path.dirname(os.path.abspath(path))
    with open(path) as fh:
        for line in fh:
            line = line.split("#", 1)[0]
            for tok in line.split():
                # '{' and '}' become words of their own
                buf = ""
                for ch in tok:
                    if ch in "{}":
                        if buf:
                            words.append(buf)
                        words.append(ch)
                        buf = ""
                    else:
                        buf += ch
                if buf:
                    words.append(buf)
    out: list[str] = []
    i = 0
    while i < len(words):
        if words[i].upper() == "INCLUDE":
            inc = words[i + 1]
            if not os.path.isabs(inc):
                inc = os.path.join(base, inc)
            out.extend(tokenize(inc))
            i += 2
        else:
            out.append(words[i])
            i += 1
    return out


def sections(words: list[str], name: str) -> list[list[str]]:
    """All level-0 sections ``name { ... }`` (contents without the braces)."""
    res, level, i = [], 0, 0
    while i < len(words):
        w = words[i]
        if w == "{":
            level += 1
        elif w == "}":
            level -= 1
        elif level == 0 and w.upper() == name.upper() and i + 1 < len(words) and words[i + 1] == "{":
            depth, j = 0, i + 2
            while j < len(words):
                if words[j] == "{":
                    depth += 1
                elif words[j] == "}":
                    if depth == 0:
                        break
                    depth -= 1
                j += 1
            res.append(words[i + 2:j])
            i = j
        i += 1
    return res


def section(words, name):
    s = sections(words, name)
    return s[0] if s else None


def value(words, name, default=None, conv=float):
    level = 0
    for i, w in enumerate(words):
        if w == "{":
            level += 1
        elif w == "}":
            level -= 1
        elif level == 0 and w.upper() == name.upper():
            return conv(words[i + 1])
    return default


def haskey(words, name):
    level = 0
    for w in words:
        if w == "{":
            level += 1
        elif w == "}":
            level -= 1
        elif level == 0 and w.upper() == name.upper():
            return True
    return False


# ----------------------------------------------------------------------------
# cubic spline radial functions (basis_function/Cubic_spline_build.cpp:396-660,
# Spline_fitter.cpp:153-293)

LVAL = {"S": 0, "P": 1, "5D": 2, "6D": 2, "D": 2, "7F": 3, "10F": 3, "F": 3, "7F_CRYSTAL": 3,
        "9G": 4, "15G": 4, "G": 4}
NFUNC = {"S": 1, "P": 3, "5D": 5, "6D": 6, "D": 6, "10F": 10, "F": 10, "7F": 7, "7F_CRYSTAL": 7,
         "9G": 9, "15G": 15, "G": 15}


def spline_fit(x, y, yp1, ypn):
    """Natural/clamped cubic spline (Spline_fitter.cpp:208-293)."""
    n = len(x)
    y2 = np.zeros(n)
    u = np.zeros(n)
    if yp1 > 0.99e30:
        y2[0] = 0.0
        u[0] = 0.0
    else:
        y2[0] = -0.5
        u[0] = (3.0 / (x[1] - x[0])) * ((y[1] - y[0]) / (x[1] - x[0]) - yp1)
    for i in range(1, n - 1):
        sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1])
        p = sig * y2[i - 1] + 2.0
        y2[i] = (sig - 1.0) / p
        u[i] = (6.0 * ((y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1]))
                / (x[i + 1] - x[i - 1]) - sig * u[i - 1]) / p
    if ypn > 0.99e30:
        qn = un = 0.0
    else:
        qn = 0.5
        un = (3.0 / (x[n - 1] - x[n - 2])) * (ypn - (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]))
    y2[n - 1] = (un - qn * u[n - 2]) / (qn * y2[n - 2] + 1.0)
    for k in range(n - 2, -1, -1):
        y2[k] = y2[k] * y2[k + 1] + u[k]
    c = np.zeros((n, 4))
    h = x[1:] - x[:-1]
    c[:-1, 0] = y[:-1]
    c[:-1, 1] = (y[1:] - y[:-1]) / h - h * (2.0 * y2[:-1] + y2[1:]) / 6.0
    c[:-1, 2] = y2[:-1] / 2.0
    c[:-1, 3] = (y2[1:] - y2[:-1]) / (6.0 * h)
    c[-1, 0] = y[-1]
    return c


def spline_findcutoff(c, spacing, threshold):
    """Spline_fitter::findCutoff (Spline_fitter.cpp:153-184)."""
    mx = min(float(np.max(np.abs(c[:, 0]))), 1.0)
    thr = 1e-10 * mx
    x = threshold - 0.5
    inv = 1.0 / spacing
    while x >= 0:
        i = int(x * inv)
        h = x - i * spacing
        t = c[i, 0] + h * (c[i, 1] + h * (c[i, 2] + h * c[i, 3]))
        if abs(t) > thr:
            return x + 0.5
        x -= 0.5
    return 0.0


class SplineBasis:
    """One AOSPLINE basis object (Cubic_spline)."""

    def __init__(self, words):
        self.label = words[0]
        assert words[1].upper() == "AOSPLINE", words[1]
        spacing, n = 0.02, 2500
        self.norm_type = value(words, "NORMTYPE", "GAMESSNORM", str)
        self.renorm = not haskey(words, "NORENORMALIZE")
        req_cut = value(words, "CUTOFF", -1.0)
        sp = value(words, "SPACING", None)
        if sp is not None:
            spacing, n = sp, int(50.0 / sp)
        g = section(words, "GAMESS")
        shells = []
        p = 0
        while p < len(g):
            sym = g[p].upper()
            sym = {"D": "6D", "F": "10F", "G": "15G"}.get(sym, sym)
            ng = int(g[p + 1])
            ex, co = [], []
            for i in range(ng):
                ex.append(float(g[p + 3 + 3 * i]))
                co.append(float(g[p + 4 + 3 * i]))
            p += 2 + 3 * ng
            shells.append((sym, ex, co))
        x = np.arange(n) * spacing
        self.spacing = spacing
        self.syms = []
        coeffs = []
        for sym, ex, co in shells:
            y = np.zeros(n)
            for e, cc in zip(ex, co):
                fac = math.sqrt(2.0 * e / math.pi)
                feg = 4.0 * e
                feg2 = feg * feg
                L = LVAL[sym]
                nt = self.norm_type.upper()
                if nt == "GAMESSNORM":
                    norm = [math.sqrt(2.0 * feg * fac), math.sqrt(2.0 * feg2 * fac / 3.0),
                            math.sqrt(2.0 * feg * feg2 * fac / 15.0),
                            math.sqrt(2.0 * feg2 * feg2 * fac / 105.0),
                            math.sqrt(2.0 * feg2 * feg2 * feg * fac / 945.0)][L]
                elif nt == "CRYSTAL":
                    norm = 1.0 / math.sqrt(2 * L + 1)
                else:
                    assert nt == "NONE", nt
                    norm = 1.0
                y += norm * cc * np.exp(-e * x * x)
            if self.renorm:
                pw = LVAL[sym] + 1
                s = float(np.sum(spacing * x ** (2 * pw) * y * y))
                if abs(s - 1.0) > 1e-5:
                    y = y / math.sqrt(s)
            if req_cut > 0:
                cutmax = req_cut - 1e-6
                cutmin = cutmax - 1.2
                zz = (x - cutmin) / 1.2
                y = np.where(x > cutmax, 0.0, np.where(x > cutmin, y * (1 - zz ** 3 * (6 * zz * zz - 15 * zz + 10)), y))
            yp1 = (y[1] - y[0]) / spacing
            ypn = (y[n - 1] - y[n - 2]) / spacing
            coeffs.append(spline_fit(x, y, yp1, ypn))
            self.syms.append(sym)
        thr0 = x[n - 1]
        cuts = [spline_findcutoff(c, spacing, thr0) for c in coeffs]
        self.cuts = cuts                  # per spline (CUTOFF_MO evaluates inside each)
        self.threshold = max(cuts)
        # pad each table out to the common threshold (Spline_fitter::pad)
        self.coeffs = []
        for c in coeffs:
            if thr0 < self.threshold:
                extra = int((self.threshold - thr0) / spacing) + 1
                c = np.vstack([c, np.zeros((extra, 4))])
            self.coeffs.append(c)
        self.nfunc = sum(NFUNC[s] for s in self.syms)

    def eval_lap(self, d, per_function=False):
        """Values [..., nfunc, 5] = (f, df/dx, df/dy, df/dz, lap) at
        displacement d [..., 3] from the center (Cubic_spline_calc.cpp:353-).
        per_function: zero each function outside its own spline's cutoff (the
        CUTOFF_MO evaluator, MO_matrix_cutoff.h:480-569)."""
        d = np.asarray(d, dtype=float)
        r2 = np.sum(d * d, axis=-1)
        r = np.sqrt(r2)
        inside = r < self.threshold
        rr = np.where(inside, r, 0.0)
        out = np.zeros(d.shape[:-1] + (self.nfunc, 5))
        x, y, z = d[..., 0], d[..., 1], d[..., 2]
        inv = 1.0 / self.spacing
        k = 0
        with np.errstate(divide="ignore", invalid="ignore"):
            for sym, c, cut in zip(self.syms, self.coeffs, self.cuts):
                i = (rr * inv).astype(np.int64)
                h = rr - i * self.spacing
                c0, c1, c2, c3 = c[i, 0], c[i, 1], c[i, 2], c[i, 3]
                f = c0 + h * (c1 + h * (c2 + h * c3))
                fd = (c1 + h * (2 * c2 + h * (3 * c3))) / rr
                f2 = 2 * c2 + 6 * h * c3
                for (ang, ax, ay, az, lapA, L) in _angular(sym, x, y, z):
                    val = ang * f
                    h1 = ang * fd
                    out[..., k, 0] = val
                    out[..., k, 1] = h1 * x + ax * f
                    out[..., k, 2] = h1 * y + ay * f
                    out[..., k, 3] = h1 * z + az * f
                    out[..., k, 4] = ang * f2 + (2 * L + 2) * h1 + lapA * f
                    if per_function:
                        out[..., k, :] = np.where((r < cut)[..., None], out[..., k, :], 0.0)
                    k += 1
        out[~inside] = 0.0
        return out


def _angular(sym, x, y, z):
    """Cartesian angular factors A, dA/dx, dA/dy, dA/dz, lap A, l (the
    GAMESS orderings of Cubic_spline_build.cpp:660-760)."""
    o, zr = np.ones_like(x), np.zeros_like(x)
    if sym == "S":
        return [(o, zr, zr, zr, zr, 0)]
    if sym == "P":
        return [(x, o, zr, zr, zr, 1), (y, zr, o, zr, zr, 1), (z, zr, zr, o, zr, 1)]
    if sym in ("6D", "D"):
        return [(x * x, 2 * x, zr, zr, 2 * o, 2), (y * y, zr, 2 * y, zr, 2 * o, 2),
                (z * z, zr, zr, 2 * z, 2 * o, 2), (x * y, y, x, zr, zr, 2),
                (x * z, z, zr, x, zr, 2), (y * z, zr, z, y, zr, 2)]
    if sym == "5D":
        return [(2 * z * z - x * x - y * y, -2 * x, -2 * y, 4 * z, zr, 2), (x * z, z, zr, x, zr, 2),
                (y * z, zr, z, y, zr, 2), (x * x - y * y, 2 * x, -2 * y, zr, zr, 2), (x * y, y, x, zr, zr, 2)]
    # F and G shells: polynomials of Cubic_spline_calc.cpp:106-296 in the orders of
    # Cubic_spline_build.cpp:702-776 (gradients and Laplacians by differentiation)
    x2, y2, z2 = x * x, y * y, z * z
    F = {
        "xxx": (x2 * x, 3 * x2, zr, zr, 6 * x), "yyy": (y2 * y, zr, 3 * y2, zr, 6 * y),
        "zzz": (z2 * z, zr, zr, 3 * z2, 6 * z), "xxy": (x2 * y, 2 * x * y, x2, zr, 2 * y),
        "xxz": (x2 * z, 2 * x * z, zr, x2, 2 * z), "yyx": (y2 * x, y2, 2 * x * y, zr, 2 * x),
        "yyz": (y2 * z, zr, 2 * y * z, y2, 2 * z), "zzx": (z2 * x, z2, zr, 2 * x * z, 2 * x),
        "zzy": (z2 * y, zr, z2, 2 * y * z, 2 * y), "xyz": (x * y * z, y * z, x * z, x * y, zr),
        "m3": (y * (3 * x2 - y2), 6 * x * y, 3 * (x2 - y2), zr, zr),
        "m1": (y * (4 * z2 - x2 - y2), -2 * x * y, 4 * z2 - x2 - 3 * y2, 8 * y * z, zr),
        "0": (z * (2 * z2 - 3 * (x2 + y2)), -6 * x * z, -6 * y * z, 6 * z2 - 3 * (x2 + y2), zr),
        "p1": (x * (4 * z2 - x2 - y2), 4 * z2 - 3 * x2 - y2, -2 * x * y, 8 * x * z, zr),
        "p2": (z * (x2 - y2), 2 * x * z, -2 * y * z, x2 - y2, zr),
        "p3mod": (x * (x2 - 3 * y2), 3 * (x2 - y2), -6 * x * y, zr, zr),
    }
    order = {"10F": ["xxx", "yyy", "zzz", "xxy", "xxz", "yyx", "yyz", "zzx", "zzy", "xyz"],
             "7F": ["0", "m3", "p3mod", "p2", "xyz", "m1", "p1"],
             "7F_CRYSTAL": ["0", "p1", "m1", "p2", "xyz", "p3mod", "m3"]}
    if sym in order:
        return [F[k] + (3,) for k in order[sym]]
    if sym == "15G":
        return [(x2 * x2, 4 * x2 * x, zr, zr, 12 * x2, 4), (y2 * y2, zr, 4 * y2 * y, zr, 12 * y2, 4),
                (z2 * z2, zr, zr, 4 * z2 * z, 12 * z2, 4), (x2 * x * y, 3 * x2 * y, x2 * x, zr, 6 * x * y, 4),
                (x2 * x * z, 3 * x2 * z, zr, x2 * x, 6 * x * z, 4), (y2 * y * x, y2 * y, 3 * y2 * x, zr, 6 * x * y, 4),
                (y2 * y * z, zr, 3 * y2 * z, y2 * y, 6 * y * z, 4), (z2 * z * x, z2 * z, zr, 3 * z2 * x, 6 * x * z, 4),
                (z2 * z * y, zr, z2 * z, 3 * z2 * y, 6 * y * z, 4),
                (x2 * y2, 2 * x * y2, 2 * x2 * y, zr, 2 * (x2 + y2), 4),
                (x2 * z2, 2 * x * z2, zr, 2 * x2 * z, 2 * (x2 + z2), 4),
                (y2 * z2, zr, 2 * y * z2, 2 * y2 * z, 2 * (y2 + z2), 4),
                (x2 * y * z, 2 * x * y * z, x2 * z, x2 * y, 2 * y * z, 4),
                (y2 * x * z, y2 * z, 2 * x * y * z, x * y2, 2 * x * z, 4),
                (z2 * x * y, y * z2, x * z2, 2 * x * y * z, 2 * x * y, 4)]
    if sym == "9G":
        r2 = x2 + y2 + z2
        return [(35 * z2 * z2 - 30 * z2 * r2 + 3 * r2 * r2, 12 * (x2 + y2 - 4 * z2) * x, 12 * (x2 + y2 - 4 * z2) * y,
                 -48 * r2 * z + 80 * z2 * z, zr, 4),
                (x * z * (7 * z2 - 3 * r2), (-9 * x2 - 3 * y2 + 4 * z2) * z, -6 * x * y * z,
                 (-3 * x2 - 3 * y2 + 12 * z2) * x, zr, 4),
                (y * z * (7 * z2 - 3 * r2), -6 * x * y * z, (-3 * x2 - 9 * y2 + 4 * z2) * z,
                 (-3 * x2 - 3 * y2 + 12 * z2) * y, zr, 4),
                ((x2 - y2) * (7 * z2 - r2), 4 * x * (3 * z2 - x2), -4 * y * (3 * z2 - y2), 12 * z * (x2 - y2), zr, 4),
                (x * y * (7 * z2 - r2), y * (6 * z2 - 3 * x2 - y2), x * (6 * z2 - x2 - 3 * y2), 12 * x * y * z, zr, 4),
                ((x2 - 3 * y2) * x * z, 3 * (x2 - y2) * z, -6 * x * y * z, (x2 - 3 * y2) * x, zr, 4),
                ((3 * x2 - y2) * y * z, 6 * x * y * z, 3 * (x2 - y2) * z, (3 * x2 - y2) * y, zr, 4),
                ((x2 - 3 * y2) * x2 - (3 * x2 - y2) * y2, 4 * x * (x2 - 3 * y2), 4 * y * (y2 - 3 * x2), zr, zr, 4),
                ((x2 - y2) * x * y, (3 * x2 - y2) * y, (x2 - 3 * y2) * x, zr, zr, 4)]
    raise NotImplementedError(sym)


# ----------------------------------------------------------------------------
# Jastrow radial functions


def cutoff_cusp(r, cusp, gamma, rcut):
    """Cutoff_cusp::calcLap (Cutoff_cusp.cpp:122-154): returns (f, f'/r, lap)."""
    inside = r < rcut
    with np.errstate(divide="ignore", invalid="ignore"):
        zz = r / rcut
        zz2 = zz * zz
        pp = zz - zz2 + zz * zz2 / 3
        pade = 1.0 / (1 + gamma * pp)
        pade0 = 1.0 / (3.0 + gamma)
        f = cusp * rcut * (pp * pade - pade0)
        pade2 = pade * pade
        ppd = 1.0 - 2.0 * zz + zz2
        ppdd = -2.0 + 2.0 * zz
        dadr = ppd * pade2 / r
        lap = ppdd * pade2 / rcut - 2.0 * gamma * ppd * ppd * pade2 * pade / rcut + 2.0 * dadr
    return (np.where(inside, f, 0.0), np.where(inside, cusp * dadr, 0.0), np.where(inside, cusp * lap, 0.0))


def pade(r, alpha):
    """Pade_function::calcLap (Pade_function.cpp:128-184): f = (a r/(1+a r))^2,
    f'/r = 2 a^2/(1+a r)^3, lap = 6 a^2/(1+a r)^4."""
    p = 1.0 / (1.0 + alpha * r)
    app = alpha * alpha * p * p
    return app * r * r, 2.0 * app * p, 6.0 * app * p * p


def poly_pade(r, beta, rcut):
    """Poly_pade_function::calcLap (Poly_pade_function.cpp:183-237) for one
    beta: returns (f, f'/r, lap)."""
    inside = r < rcut
    with np.errstate(divide="ignore", invalid="ignore"):
        zz = r / rcut
        zz2 = zz * zz
        zpp = zz2 * (6.0 - 8.0 * zz + 3.0 * zz2)
        zpp1 = 1 - zpp
        zppd = 12.0 * zz * (1.0 - 2.0 * zz + zz2)
        zppdd2 = 6.0 - 24.0 * zz + 18 * zz2
        zpade = 1.0 / (1 + beta * zpp)
        zpade2 = zpade * zpade
        crs = zpp1 * zpade
        crsd = -zppd * zpade2 * (beta + 1) / (r * rcut)
        crsdd2 = -zpade2 * (zppdd2 - beta * zppd * zppd * zpade) * (beta + 1) / (rcut * rcut)
        lap = 2 * (crsdd2 + crsd)
    return (np.where(inside, crs, 0.0), np.where(inside, crsd, 0.0), np.where(inside, lap, 0.0))


class RadialSet:
    """A Jastrow EIBASIS/EEBASIS object: list of scalar radial functions."""

    def __init__(self, words):
        self.label = words[0]
        t = words[1].upper()
        self.kind = t
        if t == "CUTOFF_CUSP":
            self.cusp = value(words, "CUSP")
            self.gamma = value(words, "GAMMA")
            self.rcut = value(words, "CUTOFF")
            self.n = 1
        elif t == "POLYPADE":
            self.rcut = value(words, "RCUT")
            b0 = value(words, "BETA0")
            self.n = int(value(words, "NFUNC", conv=int))
            b1 = math.log(b0 + 1.00001)
            self.beta = [b0] + [math.exp(b1 + 1.6 * i) - 1 for i in range(1, self.n)]
        elif t == "PADE":
            # Pade_function::read (Pade_function.cpp:21-45): alpha_i = ALPHA0 / 2^i, no cutoff
            a0 = value(words, "ALPHA0")
            self.n = int(value(words, "NFUNC", conv=int))
            self.alpha = [a0 / 2.0 ** i for i in range(self.n)]
            self.rcut = 1e99
        else:
            raise NotImplementedError(t)

    def eval(self, r):
        """[..., n, 3] = (f, f'/r, lap)."""
        if self.kind == "CUTOFF_CUSP":
            return np.stack(cutoff_cusp(r, self.cusp, self.gamma, self.rcut), axis=-1)[..., None, :]
        if self.kind == "PADE":
            return np.stack([np.stack(pade(r, a), axis=-1) for a in self.alpha], axis=-2)
        return np.stack([np.stack(poly_pade(r, b, self.rcut), axis=-1) for b in self.beta], axis=-2)


# ----------------------------------------------------------------------------
# the system


class System:
    """Molecule + Slater-Jastrow wave function + pseudopotential, built from a
    QWalk deck with the reference's rules."""

    def __init__(self, deck_path: str):
        self.deck_path = deck_path
        words = tokenize(deck_path)
        sysw = section(words, "SYSTEM")
        self.periodic = sysw[0].upper() == "PERIODIC"
        assert self.periodic or sysw[0].upper() in ("MOLECULE", "MOLECULAR"), sysw[0]
        ns = section(sysw, "NSPIN")
        self.nup, self.ndn = int(ns[0]), int(ns[1])
        self.nelec = self.nup + self.ndn
        self.labels, self.charges, pos = [], [], []
        for a in sections(sysw, "ATOM"):
            self.labels.append(a[0])
            self.charges.append(float(a[1]))
            i = [k for k, w in enumerate(a) if w.upper() == "COOR"][0]
            pos.append([float(a[i + 1]), float(a[i + 2]), float(a[i + 3])])
        self.atoms = np.array(pos)
        self.charges = np.array(self.charges)
        # KPOINT (units of pi per lattice vector; Periodic_system.cpp:106-413)
        kp = section(sysw, "KPOINT")
        self.kpt = np.array([float(x) for x in kp[:3]]) if kp else np.zeros(3)
        # all k components integer: the overall sign of a wrap is tracked
        # (Periodic_sample.cpp:201-209)
        self.kint = bool(np.all(self.kpt == np.floor(self.kpt)))
        if self.periodic:
            self._read_cell(sysw)
        tf = section(words, "TRIALFUNC")
        if tf[0].upper() == "SLATER":        # Slater wave function alone: U = 0
            wf1, wf2 = tf, ["JASTROW2"]
        else:
            wf1 = section(tf, "WF1")
            wf2 = section(tf, "WF2")
        self._read_slater(wf1, os.path.dirname(os.path.abspath(deck_path)))
        self._read_jastrow(wf2)
        self._read_pseudo(sections(words, "PSEUDO"))

    # Slater determinant (wavefunction/Slat_wf_data.cpp:34-303, MO_matrix.h:383-462,
    # MO_matrix_blas.h:101-190)
    def _read_slater(self, w, base):
        # CORBITALS: complex orbitals, Slat_wf<dcomplex> (Slat_wf_data.cpp:130-147)
        self.cplx = bool(section(w, "CORBITALS"))
        orbw = section(w, "CORBITALS") if self.cplx else section(w, "ORBITALS")
        self.mo_kind = orbw[0].upper()
        self.cutoff_mo = self.mo_kind == "CUTOFF_MO"
        self.magnify = value(orbw, "MAGNIFY", 1.0)
        self.nmo = int(value(orbw, "NMO", conv=int))
        self.basis = [SplineBasis(b) for b in sections(orbw, "BASIS")]
        # centers = atoms (USEATOMS / USEGLOBAL for molecules); a periodic cell
        # sums each atom's functions over its image centers
        self.center_basis = []
        for lab in self.labels:
            self.center_basis.append([b for b in self.basis if b.label == lab])
        if not self.periodic:
            self.images = [self.atoms[a:a + 1] for a in range(len(self.atoms))]
            self.image_shifts = [np.zeros((1, 3)) for _ in range(len(self.atoms))]
        # k-point factor of every image center (eval_kpoint_fac, MO_matrix.h:333-342;
        # MO_matrix_blas.h:179-188): e^{i pi k.n} for complex orbitals, cos(pi k.n)
        # for real ones, n the image's lattice translation
        self.kfac = []
        for sh in self.image_shifts:
            dot = np.asarray(sh, dtype=float) @ self.kpt
            self.kfac.append(np.exp(1j * math.pi * dot) if self.cplx else np.cos(math.pi * dot))
        self.nfunc_center = [sum(b.nfunc for b in bl) for bl in self.center_basis]
        self.totbasis = sum(self.nfunc_center)
        orbfile = value(orbw, "ORBFILE", conv=str)
        if not os.path.isabs(orbfile) and not os.path.exists(orbfile):
            orbfile = os.path.join(base, orbfile)
        self.moc = self._read_orb(orbfile)
        if self.cutoff_mo:
            # MO_matrix_cutoff::init (MO_matrix_cutoff.h:198-235): |c| <= 1e-12 dropped, MAGNIFY applied
            self.moc = np.where(np.abs(self.moc) > 1e-12, self.moc * self.magnify, 0.0)
        states = [int(s) - 1 for s in section(w, "STATES")]
        self.occ = [states[:self.nup], states[self.nup:]]

    def _read_orb(self, path):
        toks = open(path).read().split()
        k = toks.index("COEFFICIENTS")
        ent = np.array(toks[:k], dtype=np.int64).reshape(-1, 4) - 1
        if self.cplx:
            # "(re,im)" (or a plain real), the stream format of a complex number
            def cnum(t):
                if t.startswith("("):
                    parts = t.strip("()").split(",")
                    return complex(float(parts[0]), float(parts[1]) if len(parts) > 1 else 0.0)
                return complex(float(t), 0.0)
            coef = np.array([cnum(t) for t in toks[k + 1:]])
        else:
            coef = np.array(toks[k + 1:], dtype=float)
        maxbasis = max(self.nfunc_center)
        cm = -np.ones((self.nmo, len(self.labels), maxbasis), dtype=np.int64)
        for mo, b, c, lab in ent:
            if mo <= self.nmo:
                if mo < self.nmo:
                    cm[mo, c, b] = lab
        moc = np.zeros((self.totbasis, self.nmo), dtype=complex if self.cplx else float)
        row = 0
        for c, nf in enumerate(self.nfunc_center):
            for f in range(nf):
                for mo in range(self.nmo):
                    moc[row, mo] = coef[cm[mo, c, f]] if cm[mo, c, f] >= 0 else 0.0
                row += 1
        return moc

    def _read_jastrow(self, w):
        assert w[0].upper() == "JASTROW2", w[0]
        self.groups = []
        self._has3 = self._has3s = False
        for g in sections(w, "GROUP"):
            grp = {"ee": [RadialSet(b) for b in sections(g, "EEBASIS")],
                   "ei": [RadialSet(b) for b in sections(g, "EIBASIS")]}
            ob = section(g, "ONEBODY")
            if ob is not None:
                grp["onebody"] = {c[0]: [float(x) for x in c[1:]] for c in sections(ob, "COEFFICIENTS")}
            tb = section(g, "TWOBODY_SPIN")
            if tb is not None:
                grp["twobody_spin"] = ([float(x) for x in section(tb, "LIKE_COEFFICIENTS")],
                                       [float(x) for x in section(tb, "UNLIKE_COEFFICIENTS")])
            tb = section(g, "TWOBODY")
            if tb is not None:
                grp["twobody"] = [float(x) for x in section(tb, "COEFFICIENTS")]
            # THREEBODY, or THREEBODY_SPIN with like/unlike coefficients
            # (Jastrow2_three_diffspin.cpp:130-186); SM_TERMS replaces the default list
            th = section(g, "THREEBODY")
            ths = section(g, "THREEBODY_SPIN")
            self._has3 = getattr(self, "_has3", False) or th is not None
            self._has3s = getattr(self, "_has3s", False) or ths is not None
            if th is not None or ths is not None:
                t = th if th is not None else ths
                sc = float(value(t, "SCALE", 1.0))
                like = sections(t, "COEFFICIENTS" if th is not None else "LIKE_COEFFICIENTS")
                unlike = like if th is not None else sections(t, "UNLIKE_COEFFICIENTS")
                grp["threebody"] = {c[0]: ([sc * float(x) for x in c[1:]], [sc * float(x) for x in u[1:]])
                                    for c, u in zip(like, unlike)}
                sm = section(t, "SM_TERMS")
                if sm is not None:
                    grp["klm"] = [(int(sm[i]), int(sm[i + 1]), int(sm[i + 2])) for i in range(0, len(sm), 3)]
            self.groups.append(grp)
        self.tb_stale_ei = self._has3s and not self._has3

    # Pseudopotential (system/Pseudopotential.cpp:874-1033, Rgaussian_function.cpp)
    @staticmethod
    def _read_rgaussian(bw):
        """OLDQMC channels of an RGAUSSIAN basis (Rgaussian_function.cpp:24-107)."""
        oq = section(bw, "OLDQMC")
        it = 1  # zeff
        nl = int(oq[it]); it += 1
        nper = [int(oq[it + l]) for l in range(nl)]
        it += nl
        chans = []
        for l in range(nl):
            terms = []
            for _ in range(nper[l]):
                terms.append((float(oq[it]) - 2.0, float(oq[it + 1]), float(oq[it + 2])))
                it += 3
            chans.append(terms)
        return chans

    def _read_pseudo(self, pstexts):
        """SPIN_DEP: BASIS_UP / BASIS_DN radial sets per electron spin;
        ADD_ZEFF: +Z_ion/r in the local channel (Pseudopotential.cpp:305-336,
        874-1033)."""
        self.pp = {}
        for t in pstexts:
            lab = t[0]
            aip = int(value(t, "AIP", 6, int))
            if haskey(t, "SPIN_DEP"):
                up = self._read_rgaussian(section(t, "BASIS_UP"))
                dn = self._read_rgaussian(section(t, "BASIS_DN"))
            else:
                up = dn = self._read_rgaussian(section(t, "BASIS"))
            self.pp[lab] = {"aip": aip, "chans": up, "chans_dn": dn, "add_zeff": haskey(t, "ADD_ZEFF")}
        for lab, p in self.pp.items():
            p["quad"], p["w"] = gesqua(p["aip"])
            p["cutoff"] = self._pp_cutoff_pair(p["chans"], p["chans_dn"])

    def _pp_cutoff_pair(self, up, dn):
        """The cutoff scan over both spins' channels."""
        nl = len(up)
        cutL = [20.0] * (nl - 1)
        found = [False] * (nl - 1)
        r = 20.0
        while r > 0:
            vu, vd = self._vl(up, r), self._vl(dn, r)
            for l in range(nl - 1):
                if (abs(float(vu[l])) > 1e-5 or abs(float(vd[l])) > 1e-5) and not found[l]:
                    cutL[l] = r - 0.05
                    found[l] = True
            r -= 0.05
        return max(cutL) if cutL else 0.0

    def _vl_spin(self, p, r, a):
        """Channel radials [nl][nc, N] for every electron with its spin's
        basis; the local channel with ADD_ZEFF's Z_ion / r."""
        vu, vd = self._vl(p["chans"], r), self._vl(p["chans_dn"], r)
        up = np.arange(r.shape[-1]) < self.nup
        vl = [np.where(up, u, d) for u, d in zip(vu, vd)]
        if p["add_zeff"]:
            vl[-1] = vl[-1] + self.charges[a] / r
        return vl

    @staticmethod
    def _vl(chans, r):
        r = np.asarray(r, dtype=float)
        out = []
        for terms in chans:
            v = np.zeros_like(r)
            for n, a, c in terms:
                v = v + c * r ** n * np.exp(-np.minimum(a * r * r, 60.0))
            out.append(v)
        return out

    def _pp_cutoff(self, chans):
        """Cutoff scan from 20 bohr down in 0.05 steps (Pseudopotential.cpp:985-1026)."""
        nl = len(chans)
        cutL = [20.0] * (nl - 1)
        found = [False] * (nl - 1)
        r = 20.0
        while r > 0:
            vl = self._vl(chans, r)
            for l in range(nl - 1):
                if abs(float(vl[l])) > 1e-5 and not found[l]:
                    cutL[l] = r - 0.05
                    found[l] = True
            r -= 0.05
        return max(cutL) if cutL else 0.0

    # ------------------------------------------------------------------
    # evaluation

    def mo_lap(self, P):
        """MO values for positions P [..., 3]: [..., nmo, 5] (MO_matrix_blas::updateLap,
        MO_matrix_blas.h:411-491, including its |value| > 1e-8 basis skip)."""
        P = np.asarray(P, dtype=float)
        vals = []
        for c, bl in enumerate(self.center_basis):
            for b in bl:
                v = 0.0
                for img, kf in zip(self.images[c], self.kfac[c]):
                    d = P - img
                    v = v + kf * b.eval_lap(d, per_function=self.cutoff_mo)
                keep = np.abs(v[..., 0]) > 1e-8          # modulus for complex sums
                if self.cutoff_mo:                       # no skip of small values
                    keep = np.ones_like(keep)
                vals.append(np.where(keep[..., None], v, 0.0))
        B = np.concatenate(vals, axis=-2)          # [..., totbasis, 5]
        return np.einsum("...bk,bm->...mk", B, self.moc)

    def slater(self, R):
        """log|D|, sign, grad ratios [nc,N,3], lap ratios [nc,N] from the
        transpose-inverse convention of Slat_wf::calcLap/getDetLap.  Complex
        orbitals: sign is the unit phase factor of D, and the grad / lap ratios
        are the real parts that enter the drift and -1/2 Re(lap psi / psi)
        (Wf_return.cpp:129-152, System.cpp:105-140)."""
        nc = R.shape[0]
        mo = self.mo_lap(R)                           # [nc, N, nmo, 5]
        logd = np.zeros(nc)
        sign = np.ones(nc, dtype=mo.dtype)
        g = np.zeros((nc, self.nelec, 3))
        l = np.zeros((nc, self.nelec))
        inv_all = []
        for s, (e0, ns) in enumerate([(0, self.nup), (self.nup, self.ndn)]):
            if ns == 0:
                inv_all.append(None)
                continue
            occ = self.occ[s]
            M = mo[:, e0:e0 + ns][:, :, occ, :]      # [nc, e, i, 5]
            A = M[..., 0]
            sgn, ld = np.linalg.slogdet(A)
            logd += ld
            sign *= sgn
            Ainv = np.linalg.inv(A)                  # Ainv[i, e]
            # ratio_k(e) = sum_i dphi_i(r_e) Ainv[i, e]
            r = np.einsum("ceik,cie->cek", M[..., 1:], Ainv).real
            g[:, e0:e0 + ns] = r[..., :3]
            l[:, e0:e0 + ns] = r[..., 3]
            inv_all.append(Ainv)
        return logd, sign, g, l, inv_all, mo

    def jastrow(self, R, ei_stale=None):
        """U, per-electron grad U [nc,N,3], lap U [nc,N] (Jastrow2_wf.cpp:988-1221).
        ei_stale = (e, Re): the e-e-n terms take electron e's e-n basis values at
        Re [nc,3] instead of at R[:, e] (the value-only update of the reference
        with THREEBODY_SPIN; see nonlocal_pp)."""
        nc, N, _ = R.shape
        U = np.zeros(nc)
        G = np.zeros((nc, N, 3))
        L = np.zeros((nc, N))
        spin = np.array([0] * self.nup + [1] * self.ndn)
        for grp in self.groups:
            # e-n one-body
            if "onebody" in grp or "threebody" in grp:
                ei = {}
                for a, lab in enumerate(self.labels):
                    d = self.min_image(R - self.atoms[a])         # [nc,N,3]
                    r = np.sqrt(np.sum(d * d, axis=-1))
                    fs = [b.eval(r) for b in grp["ei"] if b.label == lab]
                    F = np.concatenate(fs, axis=-2) if fs else np.zeros((nc, N, 0, 3))
                    ei[a] = (F, d)
                ei3 = ei
                if ei_stale is not None and "threebody" in grp:
                    e, Re = ei_stale
                    ei3 = {}
                    for a, lab in enumerate(self.labels):
                        F, d = ei[a]
                        F, d = F.copy(), d.copy()
                        de = self.min_image(Re - self.atoms[a])    # [nc,3]
                        re = np.sqrt(np.sum(de * de, axis=-1))
                        fs = [b.eval(re) for b in grp["ei"] if b.label == lab]
                        if fs:
                            F[:, e] = np.concatenate(fs, axis=-2)
                        d[:, e] = de
                        ei3[a] = (F, d)
            if "onebody" in grp:
                for a, lab in enumerate(self.labels):
                    cf = np.array(grp["onebody"][lab])
                    F, d = ei[a]
                    k = len(cf)
                    U += np.einsum("cnk,k->c", F[..., :k, 0], cf)
                    fd = np.einsum("cnk,k->cn", F[..., :k, 1], cf)
                    G += fd[..., None] * d
                    L += np.einsum("cnk,k->cn", F[..., :k, 2], cf)
            # e-e
            if "twobody_spin" in grp or "twobody" in grp or "threebody" in grp:
                eef = []
                iu, ju = np.triu_indices(N, 1)
                d = self.min_image(R[:, iu] - R[:, ju])            # r_i - r_j
                r = np.sqrt(np.sum(d * d, axis=-1))
                E = np.concatenate([b.eval(r) for b in grp["ee"]], axis=-2)   # [nc,P,k,3]
                if "twobody_spin" in grp or "twobody" in grp:
                    if "twobody_spin" in grp:
                        like, unlike = grp["twobody_spin"]
                        same = (spin[iu] == spin[ju])
                        cf = np.where(same[:, None], np.array(like)[None, :], np.array(unlike)[None, :])
                    else:
                        cf = np.broadcast_to(np.array(grp["twobody"])[None, :], (len(iu), len(grp["twobody"])))
                    k = cf.shape[1]
                    u = np.einsum("cpk,pk->cp", E[..., :k, 0], cf)
                    fd = np.einsum("cpk,pk->cp", E[..., :k, 1], cf)
                    lp = np.einsum("cpk,pk->cp", E[..., :k, 2], cf)
                    U += u.sum(axis=1)
                    gi = fd[..., None] * d
                    np.add.at(G, (slice(None), iu), gi)
                    np.add.at(G, (slice(None), ju), -gi)
                    np.add.at(L, (slice(None), iu), lp)
                    np.add.at(L, (slice(None), ju), lp)
                if "threebody" in grp:
                    self._threebody(grp, R, ei3, E, d, iu, ju, spin[iu] == spin[ju], U, G, L)
        return U, G, L

    def _threebody(self, grp, R, ei, E, dij, iu, ju, same, U, G, L):
        """e-e-n term sum_at sum_{i<j} sum_p c_p (a_k(i)a_l(j)+a_l(i)a_k(j)) b_m(ij)
        (Jastrow2_three.cpp:138-404, default klm table :30-46); c_p is the like
        or unlike coefficient by the pair's spins (THREEBODY_SPIN)."""
        klm = grp.get("klm") or [(1, 1, 0), (1, 0, 1), (1, 1, 1), (2, 2, 0), (2, 0, 1), (2, 0, 2), (2, 2, 2),
                                 (3, 3, 0), (3, 0, 2), (3, 3, 2), (1, 2, 2), (2, 3, 2)]
        for a, lab in enumerate(self.labels):
            cl, cu = grp["threebody"][lab]
            F, dia = ei[a]                         # F [nc,N,k,3], dia [nc,N,3]
            for p in range(len(cl)):
                c = np.where(same, cl[p], cu[p])   # [P]
                k, l, m = klm[p]
                ak = F[..., k, :]                  # [nc,N,3] (f, f'/r, lap)
                al = F[..., l, :]
                b = E[..., m, :]                   # [nc,P,3]
                # values
                aki, akj = ak[:, iu, 0], ak[:, ju, 0]
                ali, alj = al[:, iu, 0], al[:, ju, 0]
                s = aki * alj + ali * akj          # [nc,P]
                U += np.sum(c * s * b[..., 0], axis=1)
                # gradients of a at i and j (vectors)
                gki = ak[:, iu, 1:2] * dia[:, iu]
                gkj = ak[:, ju, 1:2] * dia[:, ju]
                gli = al[:, iu, 1:2] * dia[:, iu]
                glj = al[:, ju, 1:2] * dia[:, ju]
                gs_i = gki * alj[..., None] + gli * akj[..., None]     # d s / d r_i
                gs_j = aki[..., None] * glj + ali[..., None] * gkj     # d s / d r_j
                gb = b[..., 1:2] * dij                                  # d b / d r_i (= -d b/ d r_j)
                gi = c[:, None] * (gs_i * b[..., 0:1] + s[..., None] * gb)
                gj = c[:, None] * (gs_j * b[..., 0:1] - s[..., None] * gb)
                lsi = ak[:, iu, 2] * alj + al[:, iu, 2] * akj
                lsj = aki * al[:, ju, 2] + ali * ak[:, ju, 2]
                li = c * (lsi * b[..., 0] + s * b[..., 2] + 2 * np.sum(gs_i * gb, axis=-1))
                lj = c * (lsj * b[..., 0] + s * b[..., 2] - 2 * np.sum(gs_j * gb, axis=-1))
                np.add.at(G, (slice(None), iu), gi)
                np.add.at(G, (slice(None), ju), gj)
                np.add.at(L, (slice(None), iu), li)
                np.add.at(L, (slice(None), ju), lj)

    def evaluate(self, R):
        """Full evaluation of configurations R [nc, N, 3]."""
        R = self.wrap(np.asarray(R, dtype=float))
        logd, sign, gD, lD, inv, mo = self.slater(R)
        U, gU, lU = self.jastrow(R)
        grad = gD + gU
        lap = lD + lU + np.sum(gU * gU, axis=-1) + 2 * np.sum(gD * gU, axis=-1)
        out = {"logpsi": logd + U, "sign": np.angle(sign) if self.cplx else sign, "grad": grad, "lap": lap,
               "kinetic": -0.5 * lap.sum(axis=1),
               "potential": self.ewald(R) if self.periodic else self.coulomb(R)}
        return out

    def logpsi(self, R, ei_stale=None):
        R = self.wrap(np.asarray(R, dtype=float))
        logd, sign, *_ = self.slater(R)
        U, _, _ = self.jastrow(R, ei_stale)
        return logd + U, sign

    def coulomb(self, R):
        """Molecular_system::calcLoc (Molecular_system.cpp:209-287), no field."""
        nc, N, _ = R.shape
        pot = np.zeros(nc)
        for a in range(len(self.atoms)):
            r = np.sqrt(np.sum((R - self.atoms[a]) ** 2, axis=-1))
            pot -= self.charges[a] * np.sum(1.0 / r, axis=1)
        for i in range(len(self.atoms)):
            for j in range(i):
                pot += self.charges[i] * self.charges[j] / np.linalg.norm(self.atoms[i] - self.atoms[j])
        iu, ju = np.triu_indices(N, 1)
        pot += np.sum(1.0 / np.sqrt(np.sum((R[:, iu] - R[:, ju]) ** 2, axis=-1)), axis=1)
        return pot

    def nonlocal_pp(self, R, rot):
        """Deterministic semilocal PP (Pseudopotential.cpp:596-815): local
        channel plus Q-point quadrature of the nonlocal channels for every
        (electron, atom) pair with |r| < cutoff.  rot [nc,3,3] rows x,y,z."""
        R = self.wrap(np.asarray(R, dtype=float))
        nc, N, _ = R.shape
        tot = np.zeros(nc)
        lp0, sg0 = self.logpsi(R)
        for a, lab in enumerate(self.labels):
            p = self.pp.get(lab)
            if p is None:
                continue
            d = self.min_image(R - self.atoms[a])
            r = np.sqrt(np.sum(d * d, axis=-1))
            vl = self._vl_spin(p, r, a)
            nl = len(p["chans"])
            tot += np.sum(vl[nl - 1], axis=1)
            q = np.einsum("qk,ckj->cqj", p["quad"], rot)     # rotated points [nc,Q,3]
            for e in range(N):
                acc = r[:, e] < p["cutoff"]
                if not np.any(acc):
                    continue
                for iq in range(len(p["w"])):
                    Rn = R.copy()
                    # move relative to the nearest image of the atom
                    Rn[:, e] = R[:, e] + q[:, iq] * r[:, e:e + 1] - d[:, e]
                    kd = self._wrap_kphase(Rn[:, e])
                    # with THREEBODY_SPIN and no plain THREEBODY group, the
                    # reference's value-only Jastrow update (Jastrow2_wf::updateVal,
                    # Jastrow2_wf.cpp:877-882, 931-936) does not refresh the moved
                    # electron's saved e-n basis, so its e-e-n terms see electron
                    # e's e-n values at its current position
                    lp, sg = self.logpsi(Rn, (e, R[:, e]) if self.tb_stale_ei else None)
                    ratio = np.exp(lp - lp0) * self._point_sign(sg, sg0, kd) * p["w"][iq]
                    cosq = np.sum(q[:, iq] * d[:, e], axis=-1) / r[:, e]
                    ts = np.zeros(nc)
                    for l in range(nl - 1):
                        ts += (2 * l + 1) * vl[l][:, e] * legendre(cosq, l)
                    tot += np.where(acc, ts * ratio, 0.0)
        return tot

    def tmove_terms(self, R, rot):
        """Per quadrature point terms of the deterministic nonlocal PP for one
        configuration R [N,3] and rotation rot [3,3]: list of (electron,
        target position, v_xx) with v_xx = sum_l (2l+1) v_l(r) P_l(cos) *
        psi(target)/psi(R) * w_q, the T-move matrix elements of
        Pseudopotential::calcNonlocWithAllvariables (Pseudopotential.cpp:740-763)."""
        R = self.wrap(np.asarray(R, dtype=float)[None])
        N = R.shape[1]
        lp0, sg0 = self.logpsi(R)
        out = []
        for a, lab in enumerate(self.labels):
            p = self.pp.get(lab)
            if p is None:
                continue
            d = self.min_image(R - self.atoms[a])
            r = np.sqrt(np.sum(d * d, axis=-1))
            vl = self._vl_spin(p, r, a)
            nl = len(p["chans"])
            q = p["quad"] @ np.asarray(rot, dtype=float)
            for e in range(N):
                if not r[0, e] < p["cutoff"]:
                    continue
                for iq in range(len(p["w"])):
                    Rn = R.copy()
                    Rn[:, e] = R[:, e] + q[iq] * r[:, e:e + 1] - d[:, e]
                    kd = self._wrap_kphase(Rn[:, e])
                    Rn = self.wrap(Rn)
                    lp, sg = self.logpsi(Rn)
                    ratio = np.exp(lp - lp0) * self._point_sign(sg, sg0, kd) * p["w"][iq]
                    cosq = np.sum(q[iq] * d[0, e]) / r[0, e]
                    ts = sum((2 * l + 1) * vl[l][0, e] * legendre(cosq, l) for l in range(nl - 1))
                    out.append((e, Rn[0, e].copy(), float(ts * ratio[0])))
        return out

    def _wrap_kphase(self, P):
        """k-point phase pi k.n of putting positions P [nc, 3] into the cell,
        n the lattice translations applied (+1 per +L_i; Periodic_system::
        enforcePbc, Periodic_sample::translateElectron, Periodic_sample.cpp:388-420)."""
        if not self.periodic:
            return np.zeros(len(P))
        out = np.zeros(len(P))
        for c, p in enumerate(np.asarray(P, dtype=float)):
            n = np.zeros(3)
            for i in range(3):
                while True:
                    if float(np.dot(self.normvec[i], p - self.origin)) < -1e-12:
                        p = p + self.lat[i]
                        n[i] += 1
                    elif float(np.dot(self.normvec[i], p - self.corners[i])) > 1e-12:
                        p = p - self.lat[i]
                        n[i] -= 1
                    else:
                        break
            out[c] = math.pi * float(n @ self.kpt)
        return out

    def _point_sign(self, sg, sg0, kd):
        """Sign (phase) factor of a quadrature point (Pseudopotential.cpp:727-745):
        cos(phase' - phase - pi k.n) for complex orbitals; sign' sign cos(pi k.n)
        for real ones when every k component is an integer (else sign' sign)."""
        if self.cplx:
            return np.real(sg / sg0 * np.exp(-1j * kd))
        return sg * sg0 * (np.cos(kd) if self.kint else 1.0)

    def move_ratio(self, R, e, rnew):
        """ln|psi(R')| - ln|psi(R)|, sign ratio (complex orbitals: the phase
        change), grad and lap of electron e at R'."""
        R = np.asarray(R, dtype=float)
        lp0, s0 = self.logpsi(R)
        Rn = R.copy()
        Rn[np.arange(len(R)), e] = rnew
        ev = self.evaluate(Rn)
        _, s1 = self.logpsi(Rn)
        idx = np.arange(len(R))
        sr = np.angle(s1 / s0) if self.cplx else s1 * s0
        return ev["logpsi"] - lp0, sr, ev["grad"][idx, e], ev["lap"][idx, e]


def _erfcm(x):
    """Polynomial erfc approximation used by the Ewald sum (A&S 7.1.26,
    system/Periodic_system.h:221-227)."""
    p, a, b, c, d, e = .3275911, .254829592, -.284496736, 1.421413741, -1.453152027, 1.061405429
    y = 1. / (1. + p * x)
    return y * (a + y * (b + y * (c + y * (d + y * e)))) * np.exp(-x * x)


def _cell_setup(self, sysw):
    """Periodic_system::read (system/Periodic_system.cpp:106-413)."""
    lv = np.array([float(x) for x in section(sysw, "LATTICEVEC")]).reshape(3, 3)
    og = section(sysw, "ORIGIN")
    self.origin = np.array([float(x) for x in og[:3]]) if og else np.zeros(3)
    self.lat = lv
    cross = np.array([np.cross(lv[1], lv[2]), np.cross(lv[2], lv[0]), np.cross(lv[0], lv[1])])
    det = abs(np.linalg.det(lv))
    self.volume = det
    self.recip = cross / det
    nv = cross.copy()
    for i in range(3):
        if np.dot(nv[i], lv[i]) < 0:
            nv[i] = -nv[i]
    self.normvec = nv
    self.corners = self.origin[None, :] + lv
    heights = [abs(np.dot(cross[i], lv[i])) / np.linalg.norm(cross[i]) for i in range(3)]
    self.smallest = min(heights)
    self.alpha = 5.0 / self.smallest
    self.atoms = np.array([self._wrap1(a) for a in self.atoms])
    self.lattice_basis = np.array([aa * lv[0] + bb * lv[1] + cc * lv[2]
                                   for aa in (-1, 0, 1) for bb in (-1, 0, 1) for cc in (-1, 0, 1)])
    div = value(sysw, "CUTOFF_DIVIDER", 2.000001)
    gmax = int(value(sysw, "EWALD_GMAX", 200, int))
    self._find_centers(div)
    # G vectors: half space, weight 4 pi exp(-G^2 / 4 alpha^2) / (V G^2) > 1e-10
    gs, ws = [], []
    for ig in range(0, gmax + 1):
        for jg in range(0 if ig == 0 else -gmax, gmax + 1):
            for kg in range(0 if (ig == 0 and jg == 0) else -gmax, gmax + 1):
                g = 2 * math.pi * (ig * self.recip[0] + jg * self.recip[1] + kg * self.recip[2])
                g2 = float(np.dot(g, g))
                if g2 > 1e-8:
                    w = 4.0 * math.pi * math.exp(-g2 / (4 * self.alpha ** 2)) / (self.volume * g2)
                    if w > 1e-10:
                        gs.append(g)
                        ws.append(w)
    self.gvec = np.array(gs)
    self.gw = np.array(ws)
    # constant terms (constEwald, ewaldIon, Periodic_system.cpp:620-749)
    N = self.nelec
    q = self.charges
    nion = len(q)
    ionion = sum(q[i] * q[j] for i in range(nion) for j in range(i + 1, nion))
    ionelec = float(np.sum(q)) * (-N)
    sq = -.5 * (2 * self.alpha / math.sqrt(math.pi) + math.pi / (self.volume * self.alpha ** 2))
    ij = -math.pi / (self.volume * self.alpha ** 2)
    self.self_ii = ionion * ij + float(np.sum(q * q)) * sq
    self.self_ei = ionelec * ij
    self.self_ee = .5 * N * (N - 1) * ij + N * sq
    real = 0.0
    im5 = [aa * lv[0] + bb * lv[1] + cc * lv[2] for aa in range(-2, 3) for bb in range(-2, 3) for cc in range(-2, 3)]
    for i in range(nion):
        for j in range(i):
            r1 = self.atoms[i] - self.atoms[j]
            for v in im5:
                r = float(np.linalg.norm(r1 + v))
                real += q[i] * q[j] * _erfcm(self.alpha * r) / r
    ph = self.atoms @ self.gvec.T                       # [nion, G]
    self.ion_sin = (q[:, None] * np.sin(ph)).sum(0)
    self.ion_cos = (q[:, None] * np.cos(ph)).sum(0)
    self.ion_ewald = real + float(np.sum(self.gw * (self.ion_sin ** 2 + self.ion_cos ** 2) / 2)) * 2


def _wrap1(self, p):
    """Periodic_system::enforcePbc (system/Periodic_system.cpp:521-570)."""
    p = np.array(p, dtype=float)
    for i in range(3):
        while True:
            tooshort = float(np.dot(self.normvec[i], p - self.origin))
            toofar = float(np.dot(self.normvec[i], p - self.corners[i]))
            if tooshort < -1e-12:
                p = p + self.lat[i]
            elif toofar > 1e-12:
                p = p - self.lat[i]
            else:
                break
    return p


def _find_centers(self, divider):
    """Image centers of every atom (find_centers, system/Pbc_enforcer.cpp:205-420)."""
    lv = self.lat
    h = [abs(np.dot(lv[0], np.cross(lv[1], lv[2]))) / np.linalg.norm(np.cross(lv[1], lv[2])),
         abs(np.dot(lv[1], np.cross(lv[0], lv[2]))) / np.linalg.norm(np.cross(lv[0], lv[2])),
         abs(np.dot(lv[2], np.cross(lv[0], lv[1]))) / np.linalg.norm(np.cross(lv[0], lv[1]))]
    cutoff = min(h) / divider
    org = self.origin.copy()
    piped = np.zeros((3, 3))
    for i in range(3):
        org = org - cutoff * lv[i] / h[i]
        piped[i] = lv[i] * (1 + 2 * cutoff / h[i])
    cm = self.origin + 0.5 * lv.sum(0)
    diag1 = lv.sum(0)
    radius = float(np.linalg.norm(diag1))
    for j in range(3):
        rad2 = float(np.linalg.norm(diag1 - 2 * lv[j]))
        radius = max(radius, rad2)
    radius = 0.5 * radius + cutoff
    pc = np.array([np.cross(piped[1], piped[2]), np.cross(piped[2], piped[0]), np.cross(piped[0], piped[1])])
    for i in range(3):
        if np.dot(pc[i], piped[i]) < 0:
            pc[i] = -pc[i]
    corners = org[None, :] + piped
    images = [[] for _ in range(len(self.atoms))]
    shifts = [[] for _ in range(len(self.atoms))]
    n = 4
    for ii in range(-n, n + 1):
        for jj in range(-n, n + 1):
            for kk in range(-n, n + 1):
                for at in range(len(self.atoms)):
                    pos = self.atoms[at] + lv[0] * ii + lv[1] * jj + lv[2] * kk
                    inside = all(np.dot(pc[i], pos - org) >= 0 and np.dot(pc[i], pos - corners[i]) <= 0
                                 for i in range(3))
                    if inside and np.linalg.norm(pos - cm) < radius:
                        images[at].append(pos)
                        shifts[at].append((ii, jj, kk))
    self.images = [np.array(im) for im in images]
    self.image_shifts = [np.array(sh) for sh in shifts]


def _min_image(self, dr):
    """Periodic_sample::minimum_image (system/Periodic_sample.cpp:259-287),
    vectorised over leading axes."""
    if not self.periodic:
        return dr
    dr = np.asarray(dr, dtype=float)
    h2 = self.smallest * self.smallest * .25
    d2 = np.sum(dr * dr, axis=-1)
    out = dr.copy()
    flat = dr.reshape(-1, 3)
    of = out.reshape(-1, 3)
    for n, (v, dd) in enumerate(zip(flat, d2.reshape(-1))):
        if dd < h2:
            continue
        best, bd = None, 1e99
        for lb in self.lattice_basis:
            t = v + lb
            td = float(np.dot(t, t))
            if td < bd:
                best, bd = t, td
                if td < h2:
                    break
            if td < h2:
                break
        of[n] = best
    return out


def _wrap(self, R):
    if not self.periodic:
        return R
    R = np.array(R, dtype=float)
    flat = R.reshape(-1, 3)
    for n in range(len(flat)):
        flat[n] = self._wrap1(flat[n])
    return R


def _ewald(self, R):
    """Periodic_system::ewaldElectron + constants (Periodic_system.cpp:586-973)."""
    nc, N, _ = R.shape
    out = np.full(nc, self.ion_ewald + self.self_ii + self.self_ee + self.self_ei)
    im3 = np.array([aa * self.lat[0] + bb * self.lat[1] + cc * self.lat[2]
                    for aa in (-1, 0, 1) for bb in (-1, 0, 1) for cc in (-1, 0, 1)])
    for a in range(len(self.atoms)):
        d = self.min_image(R - self.atoms[a])                     # [nc,N,3]
        r = np.linalg.norm(d[:, :, None, :] + im3[None, None], axis=-1)
        out -= self.charges[a] * np.sum(_erfcm(self.alpha * r) / r, axis=(1, 2))
    iu, ju = np.triu_indices(N, 1)
    d = self.min_image(R[:, iu] - R[:, ju])
    r = np.linalg.norm(d[:, :, None, :] + im3[None, None], axis=-1)
    out += np.sum(_erfcm(self.alpha * r) / r, axis=(1, 2))
    ph = R @ self.gvec.T                                          # [nc,N,G]
    ss = np.sin(ph).sum(1)
    cs = np.cos(ph).sum(1)
    out += 2 * np.sum(-(self.ion_cos * cs + self.ion_sin * ss) * self.gw, axis=1)
    out += 2 * np.sum((cs * cs + ss * ss) * self.gw / 2, axis=1)
    return out


System._read_cell = _cell_setup
System._wrap1 = _wrap1
System._find_centers = _find_centers
System.min_image = _min_image
System.wrap = _wrap
System.ewald = _ewald


def legendre(x, l):
    """Pseudopotential.cpp:35-55."""
    return [np.ones_like(x), x, 0.5 * (3 * x * x - 1), 0.5 * (5 * x ** 3 - 3 * x)][l]


def gesqua(aip):
    """Quadrature points/weights (system/gesqua.cpp:32-320) for AIP 4, 6, 12, 18, 26, 32."""
    if aip < 6:
        q = 1.0 / math.sqrt(3.0)
        pts = np.array([[q, q, q], [q, -q, -q], [-q, q, -q], [-q, -q, q]])
        return pts, np.full(4, 0.25)
    if aip < 12:
        pts = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], dtype=float)
        return pts, np.full(6, 1.0 / 6.0)
    if aip < 18:
        fi0 = math.pi / 5.0
        c, s = 1.0 / math.sqrt(5.0), 2.0 / math.sqrt(5.0)
        pts = np.zeros((12, 3))
        pts[0, 2], pts[1, 2] = 1.0, -1.0
        for i in range(5):
            rk2 = 2 * i
            pts[i + 2] = [s * math.cos(rk2 * fi0), s * math.sin(rk2 * fi0), c]
            pts[i + 7] = [s * math.cos((rk2 + 1) * fi0), s * math.sin((rk2 + 1) * fi0), -c]
        return pts, np.full(12, 1.0 / 12.0)
    if aip < 32:
        # gesqua.cpp:121-273: octahedron vertices, edge midpoints, (26) cube vertices
        h, b = 1.0 / math.sqrt(2.0), 1.0 / math.sqrt(3.0)
        pts = [[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
               [h, h, 0], [-h, h, 0], [h, -h, 0], [-h, -h, 0],
               [h, 0, h], [-h, 0, h], [h, 0, -h], [-h, 0, -h],
               [0, h, h], [0, h, -h], [0, -h, h], [0, -h, -h]]
        if aip < 26:
            return np.array(pts, float), np.array([1.0 / 30.0] * 6 + [1.0 / 15.0] * 12)
        pts += [[sx * b, sy * b, sz * b] for sx in (1, -1) for sz in (1, -1) for sy in (1, -1)]
        return np.array(pts, float), np.array([40.0 / 840.0] * 6 + [32.0 / 840.0] * 12 + [27.0 / 840.0] * 8)
    assert aip == 32, aip
    # gesqua.cpp:274-320: icosahedron + dodecahedron vertices
    t5 = math.sqrt(15.0 + 6.0 * math.sqrt(5.0))
    th1, th2 = math.acos((2.0 + math.sqrt(5.0)) / t5), math.acos(1.0 / t5)
    pts = np.zeros((32, 3))
    pts[0, 2], pts[1, 2] = 1.0, -1.0

    def sph(th, ph):
        return [math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)]
    for i in range(5):
        ev, od = 2 * i * math.pi / 5, (2 * i + 1) * math.pi / 5
        pts[i + 2], pts[i + 7] = sph(math.atan(2.0), ev), sph(math.pi - math.atan(2.0), od)
        pts[i + 12], pts[i + 17] = sph(th1, od), sph(th2, od)
        pts[i + 22], pts[i + 27] = sph(math.pi - th1, ev), sph(math.pi - th2, ev)
    return pts, np.array([5.0 / 168.0] * 12 + [27.0 / 840.0] * 20)

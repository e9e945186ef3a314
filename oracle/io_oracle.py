"""Python restatement of the reference's output formats -- TEST
INFRASTRUCTURE ONLY.

Used by tests/ as the checker of the library's file writers
(evora_b200/csrc/io.cu) and of the command-line drivers; the product never
imports it.  Each function follows the reference routine it names:

  fort_e / fort_f / fort_i      Fortran Ew.d / Fw.d / Iw output, with the
                                decimal rounding done in exact Decimal
                                arithmetic (round half even on the exact
                                binary value), independent of the C library
  dump_bytes                    writedata, write.f90:47-65
  units_noncomoving, units_text compunits units.f90:26-73, writeunits 76-113
  parameter_text                writeparameter, parameter.f90:267-337
  snapshot_files                snapshot, snapshot.f90:196-360
  cuts_and_slices_files         post.f90:85-246, compstate comp.f90:201-239,
                                writecut/writeslice write.f90:106-164
"""
from __future__ import annotations

import math
import struct
from decimal import Decimal, ROUND_HALF_EVEN, localcontext

import numpy as np


def f32(x: float) -> float:
    """A default-real (single precision) literal as the reference stores it."""
    return float(np.float32(x))


# ------------------------------------------------------------- edit descriptors
def fort_e(x: float, w: int, d: int) -> str:
    x = float(x)
    if math.isnan(x):
        s = "NaN"
    elif math.isinf(x):
        s = ("-" if x < 0 else "") + ("Infinity" if w >= 9 else "Inf")
    else:
        neg = math.copysign(1.0, x) < 0
        if x == 0.0:
            digits, e = "0" * d, 0
        else:
            with localcontext() as ctx:
                ctx.prec = d
                ctx.rounding = ROUND_HALF_EVEN
                r = ctx.plus(Decimal(abs(x)))
            t = r.as_tuple()
            dg = "".join(map(str, t.digits))
            e = t.exponent + len(dg)             # abs(x) ~ 0.dg * 10^e
            digits = (dg + "0" * d)[:d]
        if abs(e) <= 99:
            exp = "E%s%02d" % ("-" if e < 0 else "+", abs(e))
        elif abs(e) <= 999:
            exp = "%s%03d" % ("-" if e < 0 else "+", abs(e))
        else:
            return "*" * w
        s = ("-" if neg else "") + "0." + digits + exp
        if len(s) > w:
            s = s.replace("0.", ".", 1)
    if len(s) > w:
        return "*" * w
    return s.rjust(w)


def fort_f(x: float, w: int, d: int) -> str:
    with localcontext() as ctx:
        ctx.rounding = ROUND_HALF_EVEN
        ctx.prec = 60
        r = Decimal(float(x)).quantize(Decimal(1).scaleb(-d))
    s = format(r, "f")
    if math.copysign(1.0, float(x)) < 0 and not s.startswith("-"):
        s = "-" + s
    if len(s) > w:
        return "*" * w
    return s.rjust(w)


def fort_i(v: int, w: int) -> str:
    s = str(int(v))
    return "*" * w if len(s) > w else s.rjust(w)


def fort_a(s: str, w: int) -> str:
    return s[:w] if len(s) >= w else s.rjust(w)


def line_e(values, w=16, d=6) -> str:
    return "".join(fort_e(v, w, d) for v in values) + "\n"


# ------------------------------------------------------------------- dumps
def dump_bytes(q: np.ndarray, nz: int | None = None, lz: int = 1) -> bytes:
    """q of C shape (slab z, ny, nx, nn) -> the two records of writedata."""
    q = np.ascontiguousarray(q, dtype="<f8")
    nzs, ny, nx, nn = q.shape
    mz = lz + nzs - 1
    nz = mz if nz is None else nz
    head = struct.pack("<6i", nn, nx, ny, nz, lz, mz)
    body = q.tobytes()
    rec = lambda b: struct.pack("<i", len(b)) + b + struct.pack("<i", len(b))
    return rec(head) + rec(body)


# ------------------------------------------------------------------- units
UNIT_NAMES = ("t", "cosmo", "redshift", "length0", "time0", "density0", "velocity0", "temp0",
              "press0", "number0", "chem0", "photo0", "cool0", "heat0", "jeans0", "jeansfloor0",
              "kappa0", "meanfreepath0")


def units_noncomoving(t: float, g: float, fb: float = 1.0) -> dict:
    kb, megapc, pi = 1.3806200e-16, 3.08568025e24, f32(3.1415927)
    cosmo, d0, t0, l0, m0 = 1.0, 1.0, 1.0, 1.0, kb
    g1 = g - 1.0
    u = dict(t=t, cosmo=cosmo, redshift=0.0)
    u["density0"] = d0 / cosmo ** 3.0
    u["length0"] = l0 * cosmo
    u["time0"] = t0 * cosmo ** 2.0
    u["velocity0"] = l0 / cosmo / t0
    u["temp0"] = l0 ** 2.0 / cosmo ** 2.0 / t0 ** 2.0 * m0 / kb
    u["press0"] = d0 * l0 * l0 / (t0 * t0) / cosmo ** 5.0
    u["number0"] = d0 / cosmo ** 3.0 / m0
    u["chem0"] = d0 * t0 / cosmo / m0
    u["photo0"] = t0 * cosmo ** 2.0
    u["cool0"] = g1 * t0 ** 3.0 * cosmo * d0 / l0 ** 2.0 / m0 ** 2.0
    u["heat0"] = g1 * t0 ** 3.0 * cosmo ** 4.0 / l0 ** 2.0 / m0
    kappa_coef = 4.6e13 * 1e-20 / float(np.float32(37.8) / np.float32(40.0))
    u["kappa0"] = cosmo ** 5.0 * t0 ** 3.0 / d0 / l0 ** 4.0 * 0.5 * kappa_coef
    mfp_coef = f32(0.023) * megapc * 1e-16 * 1e-3
    u["meanfreepath0"] = cosmo ** 2.0 * m0 / l0 / d0 * 0.5 * f32(4.2) * mfp_coef
    u["jeans0"] = math.sqrt(pi * g * fb)
    u["jeansfloor0"] = 0.0
    return u


def units_text(u: dict) -> str:
    return "".join((k + " =").ljust(16) + fort_e(u[k], 16, 8) + "\n" for k in UNIT_NAMES)


# --------------------------------------------------------------- parameter
PARA = [  # writeparameter order and readparameter defaults (parameter.f90:41-82, 279-333)
    ("iconly", "L", False), ("hydro", "L", True), ("secondorder", "L", True), ("solver", "I", 2),
    ("limiter", "I", 1), ("cfl", "E", f32(0.5)), ("g", "E", f32(1.4)), ("atomic", "L", False),
    ("nx", "I", 32), ("ny", "I", 32), ("nz", "I", 32), ("xmin", "E", 0.0), ("xmax", "E", 1.0),
    ("ymin", "E", 0.0), ("ymax", "E", 1.0), ("zmin", "E", 0.0), ("zmax", "E", 1.0),
    ("boundtype", "I", 2), ("cut", "L", False), ("slice", "L", False), ("bov", "L", False),
    ("nsnap", "I", 100), ("gravity", "L", False), ("tstart", "E", 0.0), ("tend", "E", 1.0),
    ("supercomoving", "L", False), ("c_cosmo", "E", f32(0.1)), ("omega0", "E", 1.0),
    ("lambda0", "E", 0.0), ("fb", "E", 1.0), ("hubble0", "E", 50.0), ("box", "E", 1.0),
    ("zstart", "E", 99.0), ("zend", "E", 0.0), ("chemistry", "L", False), ("noncie", "L", False),
    ("cooling", "L", False), ("background", "L", False), ("bg", "I", 0), ("j0", "E", 1e-21),
    ("c_chem", "E", f32(0.1)), ("substep", "E", f32(0.1)), ("rhoH", "E", f32(0.76)),
    ("rhoHe", "E", f32(0.24)), ("cooldt", "L", False), ("c_cooldt", "E", 0.0),
    ("tempfloor", "L", False), ("temp_fl", "E", 0.0), ("jeansfloor", "L", False),
    ("c_jeans", "E", 0.0), ("conduction", "L", False), ("c_cond", "E", f32(0.1)),
    ("simplekappa", "L", False), ("dualenergy", "L", False), ("de_thresh", "E", 0.0),
]


def parameter_text(**values) -> str:
    out = []
    for name, kind, default in PARA:
        v = values.get(name, values.get(name.lower(), default))
        lab = (name + " =").ljust(16)
        if kind == "L":
            out.append(lab + ("T" if v else "F").rjust(16))
        elif kind == "I":
            out.append(lab + fort_i(v, 16))
        else:
            out.append(lab + fort_e(v, 16, 8))
    return "\n".join(out) + "\n"


# ----------------------------------------------------------------- physics
class Gas:
    """The constants of compparameter that pressure() reads."""

    def __init__(self, g: float, dualenergy: bool = False, de_thresh: float = 0.0, atomic: bool = False):
        self.g = f32(5.0 / 3.0) if atomic else g
        self.g1 = self.g - 1.0
        self.g1inv = 1.0 / self.g1
        self.de = bool(dualenergy)
        self.de_thresh1 = 1.0 - de_thresh if dualenergy else 1.0


def pressure(q: np.ndarray, c: Gas) -> float:
    """comp.f90:45-85 on one cell (a length-6 float64 array, in place)."""
    q1, q2, q3, q4, q5, q6 = (float(v) for v in q[:6])
    m2 = (q2 * q2) + (q3 * q3) + (q4 * q4)
    kin = 0.5 * m2 / q1
    if c.de:
        ratio = kin / q5
        if ratio > c.de_thresh1:
            press = q6 * (q1 ** c.g1)
            q[4] = kin + press * c.g1inv
        else:
            press = c.g1 * (q5 - kin)
            q[5] = press / (q1 ** c.g1)
    else:
        press = c.g1 * (q5 - kin)
    if press <= 0.0:
        raise ValueError("negative pressure")
    return press


class Geometry:
    """compparameter's grid constants, including its resetting of the y and
    z bounds of 1D and 2D runs (parameter.f90:164-265)."""

    def __init__(self, nx, ny, nz, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.one = ny == 1 and nz == 1
        self.two = nz == 1
        self.dx = (xmax - xmin) / nx
        self.dy = (ymax - ymin) / ny
        self.dz = (zmax - zmin) / nz
        if self.one:
            self.dy = self.dz = self.dx
            ymin, ymax, zmin, zmax = 0.0, self.dy, 0.0, self.dz
            self.dy = (ymax - ymin) / ny
            self.dz = (zmax - zmin) / nz
        if self.two:
            self.dz = self.dx
            zmin, zmax = 0.0, self.dz
            self.dz = (zmax - zmin) / nz
        self.xmin, self.xmax, self.ymin, self.ymax, self.zmin, self.zmax = xmin, xmax, ymin, ymax, zmin, zmax
        self.x0 = xmin + self.dx / 2
        self.y0 = ymin + self.dy / 2
        self.z0 = zmin + self.dz / 2


# ---------------------------------------------------------------- snapshot
def snapshot_files(geo: Geometry, c: Gas, q: np.ndarray, u: dict, k3: int, cut=True, slice_=True,
                   bov=False) -> dict:
    """snapshot.f90:196-360 -> {file name: bytes}; q (C shape (nz, ny, nx,
    nq)) is updated in place like the reference's.  nq = 12 is the chemistry
    build: T = p / sum(q(7:12)) temp0, summed in element order (press2temp,
    comp.f90:87-102)."""
    nx, ny, nz = geo.nx, geo.ny, geo.nz
    y1, z1 = max(ny // 2, 1), max(nz // 2, 1)
    name = "%03d" % k3
    files = {}

    chem = q.shape[-1] == 12

    def cell(ix, iy, iz):
        qq = q[iz - 1, iy - 1, ix - 1]
        press = pressure(qq, c)
        if chem:
            ns = qq[6] + qq[7] + qq[8] + qq[9] + qq[10] + qq[11]
            return qq, press, press / ns * u["temp0"]
        return qq, press, press / qq[0] * u["temp0"]

    X = lambda ix: geo.x0 + (ix - 1) * geo.dx
    Y = lambda iy: geo.y0 + (iy - 1) * geo.dy
    Z = lambda iz: geo.z0 + (iz - 1) * geo.dz
    if cut:
        s = ""
        for ix in range(1, nx + 1):
            qq, p, T = cell(ix, y1, z1)
            s += line_e([X(ix), qq[0], T, qq[1] / qq[0] * u["velocity0"], p * u["press0"]])
        files[name + ".x"] = s.encode()
        if not geo.one:
            s = ""
            for ix in range(1, nx + 1):
                qq, p, T = cell(ix, 1, z1)
                s += line_e([X(ix), qq[0], T, qq[1] / qq[0] * u["velocity0"], p * u["press0"]])
            files[name + ".x0"] = s.encode()
    if slice_:
        s = ""
        for ix in range(1, nx + 1):
            for iy in range(1, ny + 1):
                qq, p, T = cell(ix, iy, z1)
                s += line_e([X(ix), Y(iy), qq[0], T, p * u["press0"]])
            s += "\n"
        files[name + ".xy"] = s.encode()
        s = ""
        for iz in range(1, nz + 1):
            for ix in range(1, nx + 1):
                qq, p, T = cell(ix, y1, iz)
                s += line_e([X(ix), Z(iz), qq[0], T, p * u["press0"]])
            s += "\n"
        files[name + ".xz"] = s.encode()
    if bov:
        f2 = lambda var: (name + "." + var + ".bovdata").ljust(127)[:20]
        for var, vname in (("dens", "Density"), ("temp", "Temperature")):
            s = "TIME: " + fort_e(u["t"], 10, 2) + "\n"
            s += "DATA_FILE: " + f2(var) + "\n"
            s += "DATA_SIZE: " + fort_i(nx, 5) + fort_i(ny, 5) + fort_i(nz, 5) + "\n"
            s += "DATA_FORMAT: FLOAT\n"
            s += "VARIABLE:" + fort_a(vname, 20) + "\n"
            s += "DATA_ENDIAN: LITTLE\nCENTERING: ZONAL\n"
            s += "BRICK_ORIGIN: " + "".join(fort_e(v, 12, 2) for v in (geo.xmin, geo.ymin, geo.zmin)) + "\n"
            s += "BRICK_SIZE: " + "".join(fort_e(v, 12, 2) for v in (geo.xmax - geo.xmin, geo.ymax - geo.ymin,
                                                                       geo.zmax - geo.zmin)) + "\n"
            files[name + "." + var + ".bov"] = s.encode()
        dens = np.empty((nz, ny, nx), np.float32)
        temp = np.empty((nz, ny, nx), np.float32)
        for iz in range(1, nz + 1):
            for iy in range(1, ny + 1):
                for ix in range(1, nx + 1):
                    qq, p, T = cell(ix, iy, iz)
                    dens[iz - 1, iy - 1, ix - 1] = np.float32(qq[0])
                    temp[iz - 1, iy - 1, ix - 1] = np.float32(T)
        files[name + ".dens.bovdata"] = dens.tobytes()
        files[name + ".temp.bovdata"] = temp.tobytes()
    return files


# ----------------------------------------------------------- post: cs mode
STATE_NAMES = ["rho", "rho u", "rho v", "rho w", "E", "S", "rho_phys", "u", "v", "w", "p", "T", "xi_HI",
               "xi_HII", "xi_HeI", "xi_HeII", "xi_HeIII", "xi_e", "n_HI", "n_HII", "n_HeI", "n_HeII",
               "n_HeIII", "n_e", "lambda", "gamma"]


# -------------------------------------- post: the chemistry's state vector
# The CIE build's rates as post-processing evaluates them (rates.f90:26-189,
# cie.f90:58-217, chemistry.f90:123-176), restated from the reference with
# its own powers; default-real literals are single precision.
NFLOOR, RATEFLOOR, CIE_TOL, CIE_NIT = 1.0e-40, 1.0e-40, 1e-10, 1000
M_H, M_HE = f32(1.00794), f32(4.002602)


def compbackground(background, bg, j0, z, cosmo, uv=0.0):
    if not background:
        return uv
    if bg == 1:
        return j0
    if bg == 2:
        if 3 < z < 6:
            return j0 * 4.0 * cosmo
        return j0 if 1 < z <= 3 else 0.0
    if bg == 3:
        if z > 8.0:
            return 1e-5 * j0
        if 6.0 < z <= 8.0:
            return 0.5 * j0 * 10.0 ** ((-z + 6.0) * f32(0.35))
        if 3.0 < z <= 6.0:
            return j0 * 10.0 ** ((-z + 3.0) * f32(0.1))
        if 1.0 < z <= 3.0:
            return j0
        return j0 * f32(0.1) * 10.0 ** z
    return uv


def compcoef(u: dict, uv: float):
    """coef(13, 2) of rates.f90:26-78 from the unit file's chem0, photo0,
    cool0, heat0."""
    k = [[0.0, 0.0] for _ in range(13)]
    c0, p0, k0, h0 = u["chem0"], u["photo0"], u["cool0"], u["heat0"]
    k[0] = [c0 * 5.85e-11, k0 * 1.27e-21]
    k[1] = [c0 * 2.38e-11, k0 * 9.38e-22]
    k[2] = [c0 * 5.68e-12, k0 * 4.95e-22]
    k[3] = [c0 * 8.4e-11, k0 * 8.7e-27]
    k[4] = [c0 * 1.5e-10, k0 * 1.55e-26]
    k[5] = [c0 * 3.36e-10, k0 * 3.48e-26]
    k[6] = [c0 * 1.9e-3, k0 * 1.24e-13]
    k[7] = [0.0, k0 * 7.5e-19]
    k[8] = [0.0, k0 * 5.54e-17]
    k[9] = [0.0, k0 * 1.42e-27 * 1.5]
    k[10] = [p0 * 2.54e8 * uv, h0 * 2.54e8 * 7.75e-12 * uv]
    k[11] = [p0 * 2.49e8 * uv, h0 * 2.49e8 * 2.19e-11 * uv]
    k[12] = [p0 * 1.60e7 * uv, h0 * 1.60e7 * 3.10e-11 * uv]
    return k


def comprates(temp, k, background, cooling):
    """rates.f90:80-158: chemical rates r[9], cooling rates cr[13]."""
    troot, tinv, t15 = math.sqrt(temp), 1.0 / temp, temp ** -1.5
    fec = 1.0 / (1.0 + math.sqrt(temp * 1e-5))
    fc1 = troot * fec
    e1 = math.exp(-(f32(157809.1) * tinv))
    e2 = math.exp(-(f32(286335.4) * tinv))
    e3 = math.exp(-(f32(631515.0) * tinv))
    fr = (temp * 1e-3) ** f32(-0.2) / (1.0 + (temp * 1e-6) ** f32(0.7))
    fr1, fr2 = fr / troot, fr * troot
    c3 = f32(f32(0.3) * f32(-94000.0))
    edr = math.exp(f32(-470000.0) * tinv) * (1.0 + c3 * tinv)
    r = [k[0][0] * fc1 * e1, k[1][0] * fc1 * e2, k[2][0] * fc1 * e3, k[3][0] * fr1,
         k[4][0] * temp ** f32(-0.6353) + k[6][0] * t15 * edr, k[5][0] * fr1]
    r += [k[10][0], k[11][0], k[12][0]] if background else [0.0, 0.0, 0.0]
    cr = None
    if cooling:
        cr = [k[0][1] * fc1 * e1, k[1][1] * fc1 * e2, k[2][1] * fc1 * e3, k[3][1] * fr2,
              k[4][1] * temp ** f32(0.3647), k[5][1] * fr2, k[6][1] * t15 * edr,
              k[7][1] * fec * math.exp(f32(-118348.0) * tinv),
              k[8][1] * temp ** f32(-0.397) * fec * math.exp(f32(-473638.0) * tinv), k[9][1] * troot]
        cr += [k[10][1], k[11][1], k[12][1]] if background else [0.0, 0.0, 0.0]
    return r, cr


def _cieions(nH, nHe, ne, r):
    ion1, ion2, ion3 = r[0] * ne + r[6], r[1] * ne + r[7], r[2] * ne + r[8]
    nHII = NFLOOR if ion1 < RATEFLOOR else nH / (1.0 + r[3] * ne / ion1)
    if ion2 < RATEFLOOR:
        return nHII, NFLOOR, NFLOOR
    xi2 = r[4] * ne / ion2
    if ion3 < RATEFLOOR:
        return nHII, nHe / (1.0 + xi2), NFLOOR
    xi3 = r[5] * ne / ion3
    return nHII, nHe / (1.0 + xi2 + 1.0 / xi3), nHe / (1.0 + (xi2 + 1.0) * xi3)


def _fne(nH, nHe, ne, r):
    a, b, c = _cieions(nH, nHe, ne, r)
    return a + b + 2 * c - ne


def _rf_cie(nH, nHe, l, rr, r):
    fl, fr, m = _fne(nH, nHe, l, r), _fne(nH, nHe, rr, r), 0.0
    if fl * fr > 0.0:
        raise ValueError("rf_cie: no root")
    s = 0
    for _ in range(CIE_NIT):
        m = (fr * l - fl * rr) / (fr - fl)
        if abs(rr - l) < CIE_TOL * abs(rr + l):
            break
        fm = _fne(nH, nHe, m, r)
        if fm * fr > 0.0:
            rr, fr = m, fm
            if s == -1:
                fl = fl * 0.5
            s = -1
        elif fl * fm > 0.0:
            l, fl = m, fm
            if s == 1:
                fr = fr * 0.5
            s = 1
        else:
            break
    return m


def cieabundance(nH, nHe, n, r, background, uv):
    """cie.f90:58-112 with ncheck (chemistry.f90:159-176), n in place."""
    if background and uv > 0.0:
        ne = _rf_cie(nH, nHe, NFLOOR, nH + 2 * nHe, r)
        a, b, c = _cieions(nH, nHe, ne, r)
        n[:] = [nH - a, a, nHe - b - c, b, c, ne]
        n[:] = [NFLOOR if NFLOOR > v else v for v in n]
    else:
        fH, fHe1, fHe2 = r[0] / r[3], r[1] / r[4], r[2] / r[5]
        n0 = nH / (1.0 + fH)
        n2 = nHe / (1.0 + fHe1 * (1.0 + fHe2))
        n3 = n2 * fHe1
        n4 = n3 * fHe2
        n1 = n0 * fH
        n[:] = [n0, n1, n2, n3, n4, n1 + n3 + 2 * n4]
    for v in n[:5]:
        if not (0.0 <= v <= 1e20):
            raise ValueError("ncheck: abundance out of range")
    n[:] = [NFLOOR if NFLOOR > v else v for v in n]


def cool(n, cr, background):
    """rates.f90:160-189: (Lambda, Gamma)."""
    lam = (cr[0] * n[0] + cr[1] * n[2] + cr[2] * n[3] + cr[3] * n[1] + cr[4] * n[3] + cr[5] * n[4]
           + cr[6] * n[3] + cr[7] * n[0] + cr[8] * n[3] + cr[9] * (n[1] + n[3] + 4.0 * n[4]))
    gam = n[0] * cr[10] + n[2] * cr[11] + n[3] * cr[12] if background else 0.0
    return lam * n[5], gam


def post_chem(u: dict, cooling=True, background=0, bg=0, j0=1e-21, rhoh=None, rhohe=None) -> dict:
    """post.f90:58-62: chiH, chiHe, compbackground and compcoef at the dump's
    units."""
    rhoh = f32(0.76) if rhoh is None else rhoh
    rhohe = f32(0.24) if rhohe is None else rhohe
    uv = compbackground(background, bg, j0, u["redshift"], u["cosmo"], 0.0)
    return dict(cooling=cooling, background=background, chiH=rhoh / M_H, chiHe=rhohe / M_HE, k=compcoef(u, uv),
                uv=uv)


def compstate(qq: np.ndarray, c: Gas, fb: float, u: dict, chem: dict | None = None) -> list:
    """comp.f90:201-239; with chem (the CIE build, qq of 12 values) the 26
    entries, cieabundance leaving qq's species in equilibrium."""
    press = pressure(qq, c)
    if chem is None:
        temp = press / qq[0] * u["temp0"]
    else:
        ns = qq[6] + qq[7] + qq[8] + qq[9] + qq[10] + qq[11]
        temp = press / ns * u["temp0"]
    s1 = qq[0] / fb
    st = [s1] + [float(v) for v in qq[1:6]] + [s1 * u["density0"]]
    st += [qq[i] / s1 * u["velocity0"] for i in (1, 2, 3)]
    st += [press * u["press0"], temp]
    if chem is None:
        return st
    st += [qq[i] / s1 for i in range(6, 12)] + [qq[i] * u["number0"] for i in range(6, 12)]
    lam = gam = 0.0
    if chem["cooling"]:
        nH, nHe = chem["chiH"] * qq[0], chem["chiHe"] * qq[0]
        r, cr = comprates(temp, chem["k"], chem["background"], True)
        n = [float(v) for v in qq[6:12]]
        cieabundance(nH, nHe, n, r, chem["background"], chem["uv"])
        qq[6:12] = n
        lam, gam = cool(n, cr, chem["background"])
    return st + [lam, gam]


def cuts_and_slices_files(geo: Geometry, c: Gas, fb: float, u: dict, slabs, infile: str, chem=None) -> dict:
    """post cs: slabs = [(lz, q slab of C shape (mz-lz+1, ny, nx, nq)), ...];
    chem (post_chem) for the CIE build's q(12)."""
    nx, ny, nz = geo.nx, geo.ny, geo.nz
    xm, ym, zm = max(nx // 2, 1), max(ny // 2, 1), max(nz // 2, 1)
    one, two = geo.one, geo.two
    cut_y = slice_xy = not one
    cut_xy = (not one) and nx == ny
    cut_z = slice_xz = slice_yz = (not one) and not two
    cut_xyz = cut_z and nx == ny == nz
    hc = lambda k: float(np.float32(k) - np.float32(0.5))
    s2, s3 = float(np.sqrt(np.float32(2.0))), float(np.sqrt(np.float32(3.0)))
    cx = [[geo.xmin + hc(k) * geo.dx] for k in range(1, nx + 1)]
    cy = [[geo.ymin + hc(k) * geo.dy] for k in range(1, ny + 1)] if cut_y else None
    cz = [[geo.zmin + hc(k) * geo.dz] for k in range(1, nz + 1)] if cut_z else None
    cxy = [[s2 * (geo.xmin + hc(k) * geo.dx)] for k in range(1, nx + 1)] if cut_xy else None
    sl = lambda n1, n2, m1, d1, m2, d2: {(i1, i2): [m1 + hc(i1) * d1, m2 + hc(i2) * d2]
                                         for i2 in range(1, n2 + 1) for i1 in range(1, n1 + 1)}
    sxy = sl(nx, ny, geo.xmin, geo.dx, geo.ymin, geo.dy) if slice_xy else None
    sxz = sl(nx, nz, geo.xmin, geo.dx, geo.zmin, geo.dz) if slice_xz else None
    syz = sl(ny, nz, geo.ymin, geo.dy, geo.zmin, geo.dz) if slice_yz else None
    for lz, q in slabs:
        q = np.array(q, dtype=np.float64, copy=True)
        for iz in range(lz, lz + q.shape[0]):
            for iy in range(1, ny + 1):
                for ix in range(1, nx + 1):
                    qq = q[iz - lz, iy - 1, ix - 1]
                    if iy == ym and iz == zm:
                        cx[ix - 1][1:] = compstate(qq, c, fb, u, chem)
                    if cut_y and ix == xm and iz == zm:
                        cy[iy - 1][1:] = compstate(qq, c, fb, u, chem)
                    if cut_z and ix == xm and iy == ym:
                        cz[iz - 1][1:] = compstate(qq, c, fb, u, chem)
                    if cut_xy and iz == zm and ix == iy:
                        cxy[ix - 1][1:] = compstate(qq, c, fb, u, chem)
                    if cut_xyz and ix == iy == iz:
                        compstate(qq, c, fb, u, chem)      # computed, then never written (post.f90:228)
                    if slice_xy and iz == zm:
                        sxy[(ix, iy)][2:] = compstate(qq, c, fb, u, chem)
                    if slice_xz and iy == ym:
                        sxz[(ix, iz)][2:] = compstate(qq, c, fb, u, chem)
                    if slice_yz and ix == xm:
                        syz[(iy, iz)][2:] = compstate(qq, c, fb, u, chem)
    files = {}
    head_cut = "#" + "x".rjust(15) + "".join(h.rjust(16) for h in STATE_NAMES) + "\n"
    head_slice = "#" + "x".rjust(15) + "y".rjust(16) + "".join(h.rjust(16) for h in STATE_NAMES) + "\n"

    def cut(rows, name):
        files[f"{infile}.{name}.cut"] = (head_cut + "".join(line_e(r) for r in rows)).encode()

    def slc(d, n1, n2, name):
        s = head_slice
        for i1 in range(1, n1 + 1):
            for i2 in range(1, n2 + 1):
                s += line_e(d[(i1, i2)])
            s += "  \n"
        files[f"{infile}.{name}.slice"] = s.encode()

    cut(cx, "x")
    if cut_y:
        cut(cy, "y")
    if cut_z:
        cut(cz, "z")
    if cut_xy:
        cut(cxy, "xy")
    if cut_xyz:
        cut(cxy, "xyz")
    if slice_xy:
        slc(sxy, nx, ny, "xy")
    if slice_xz:
        slc(sxz, nx, nz, "xz")
    if slice_yz:
        slc(syz, ny, nz, "yz")
    return files

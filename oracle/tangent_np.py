"""Vectorised numpy restatement of one RK3 step, usable with complex arrays (test infrastructure).

This is a checker for the discrete adjoint, not a product path.  It restates the same step as
r3d_oracle.c (src/step.cpp:114-257, src/fluxes.cpp:87-533, src/bcon.cpp:12-141 and, with
--lmag, golden/fortran/3dmhdsub.f:2146-2650) as whole-array numpy statements that keep the C
evaluation order, so that

* with float64 arrays it reproduces the oracle's step to rounding (tests pin it against
  r3d_oracle.c), and
* with complex128 arrays, X + i*h*V with h = 1e-30, the imaginary part of the result divided by
  h is the exact directional derivative (tangent) of the step along V ("complex step").  Every
  operation on the path is analytic except the dt minimum, which follows the real part, so the
  tangent is that of the branch the real run takes - the same branch a hand-written adjoint
  differentiates.

A dot-product test <lambda, J V> = <J^T lambda, V> then checks any adjoint of the step to rounding
without finite-difference truncation error.  Arrays are the oracle's global (NZ, NY, NX) layout
(x fastest) with one ghost layer; x and y are periodic; the two z ghost planes are constants.
"""
from __future__ import annotations

from typing import Dict

import numpy as np

HYDRO = ["ru", "rv", "rw", "ro", "tt"]
MAG = ["bx", "by", "bz"]


def _f4(x: float) -> float:
    return float(np.float32(x))


class NumpyStep:
    """The step of an initialised Oracle (grid lines, constants and boundary data read from it)."""

    def __init__(self, o):
        self.NX, self.NY, self.NZ = o.NX, o.NY, o.NZ
        P = o.param
        self.lmag = bool(P("--lmag"))
        self.lrot = bool(P("--lrot"))
        self.fields = HYDRO + (MAG if self.lmag else [])
        for n in ["c13", "c23", "c43", "gam1", "gam2", "gam3", "zeta1", "zeta2", "hx", "h2x", "hy",
                  "h2y", "hz", "h2z", "repr", "ore", "cv", "ocv", "orm", "obeta", "omx", "omz"]:
            setattr(self, n, P(n))
        self.grav = P("--grav")
        self.gamma = P("--gamma")
        self.re = P("--re")
        self.rm = P("--rm")
        self.sff = P("--sff")
        self.theta = P("--theta")
        self.tp, self.tc, self.hh = P("--tp"), P("--tc"), P("--hh")
        self.xp, self.yp = P("--xp"), P("--yp")
        self.itcon, self.izcon = int(P("--itcon")), int(P("--izcon"))
        self.ibcon = int(P("--ibcon"))
        self.npz = int(P("--npz"))
        self.tb = o.scalars()["tb"]
        L = {n: np.array(o.line(n), dtype=np.float64) for n in
             ["exx", "dxxdx", "d2xxdx2", "ddx", "wyy", "dyydy", "d2yydy2", "ddy", "dzzdz",
              "d2zzdz2", "ddz", "rkapa", "dkapa"]}
        self.L = L
        self.timi = o.scalars()["timi"]
        # z slab held (the whole domain by default): one-sided z stencils and BCON only on the
        # domain's faces; hooks for the multi-rank form (the reduction of the dt minimum over
        # the slabs and the ghost-plane exchange after every stage)
        self.top = self.bot = True
        self.z0 = 0
        self.reduce_min = None
        self.exchange = None

    def slab(self, z0: int, nloc: int) -> "NumpyStep":
        """The same step on global planes z0+1 .. z0+nloc, with the neighbours' planes as
        ghost planes (the decomposition of src/communicate.cpp over npez ranks)."""
        import copy
        s = copy.copy(self)
        s.L = dict(self.L)
        for n in ("dzzdz", "d2zzdz2", "ddz", "rkapa", "dkapa"):
            s.L[n] = self.L[n][z0:z0 + nloc + 2].copy()
        s.NZ = nloc + 2
        s.z0 = z0
        s.top = z0 == 0
        s.bot = z0 + nloc == self.npz
        return s

    # ------------------------------------------------------------------ helpers ------------
    def _box(self, kr, jr, ir):
        NX, NY, NZ = self.NX, self.NY, self.NZ
        kr = kr or (1, NZ - 2)
        jr = jr or (1, NY - 2)
        ir = ir or (1, NX - 2)
        return kr, jr, ir

    def v(self, a, di=0, dj=0, dk=0, kr=None, jr=None, ir=None):
        """a over the box kr x jr x ir (inclusive, default interior) shifted by (di, dj, dk)."""
        kr, jr, ir = self._box(kr, jr, ir)
        return a[kr[0] + dk:kr[1] + 1 + dk, jr[0] + dj:jr[1] + 1 + dj, ir[0] + di:ir[1] + 1 + di]

    def lx(self, name, ir=None):
        ir = ir or (1, self.NX - 2)
        return self.L[name][ir[0]:ir[1] + 1][None, None, :]

    def ly(self, name, jr=None):
        jr = jr or (1, self.NY - 2)
        return self.L[name][jr[0]:jr[1] + 1][None, :, None]

    def lz(self, name, kr=None):
        kr = kr or (1, self.NZ - 2)
        return self.L[name][kr[0]:kr[1] + 1][:, None, None]

    def DX(self, f, kr=None, jr=None, ir=None):
        return (self.v(f, 1, 0, 0, kr, jr, ir) - self.v(f, -1, 0, 0, kr, jr, ir)) * self.hx * self.lx("dxxdx", ir)

    def DY(self, f, kr=None, jr=None, ir=None):
        return (self.v(f, 0, 1, 0, kr, jr, ir) - self.v(f, 0, -1, 0, kr, jr, ir)) * self.hy * self.ly("dyydy", jr)

    def DZ(self, f, kr=None, jr=None, ir=None):
        return (self.v(f, 0, 0, 1, kr, jr, ir) - self.v(f, 0, 0, -1, kr, jr, ir)) * self.hz * self.lz("dzzdz", kr)

    def D2X(self, f):
        v = self.v
        d = self.lx("dxxdx")
        return ((v(f, 1) - v(f, -1)) * self.hx * self.lx("d2xxdx2") +
                (v(f, 1) - 2.0 * v(f) + v(f, -1)) * self.h2x * d * d)

    def D2Y(self, f):
        v = self.v
        d = self.ly("dyydy")
        return ((v(f, 0, 1) - v(f, 0, -1)) * self.hy * self.ly("d2yydy2") +
                (v(f, 0, 1) - 2.0 * v(f) + v(f, 0, -1)) * self.h2y * d * d)

    def D2Z(self, f):
        v = self.v
        d = self.lz("dzzdz")
        return ((v(f, 0, 0, 1) - v(f, 0, 0, -1)) * self.hz * self.lz("d2zzdz2") +
                (v(f, 0, 0, 1) - 2.0 * v(f) + v(f, 0, 0, -1)) * self.h2z * d * d)

    def _edge_z(self, out, f, second: bool):
        """One-sided z stencils on the planes k1 = 1 and k2 = npz (3dmhdsub.f 1125/1126, 1391/1392)."""
        NZ = self.NZ
        k1, k2 = 1, NZ - 2
        J = slice(1, self.NY - 1)
        I = slice(1, self.NX - 1)
        dz1, dz2 = self.L["dzzdz"][k1], self.L["dzzdz"][k2]
        if not second:
            if self.top:
                out[0] = (4.0 * f[k1 + 1, J, I] - f[k1 + 2, J, I]) * (self.hz * dz1)
            if self.bot:
                out[-1] = (f[k2 - 2, J, I] - 4.0 * f[k2 - 1, J, I]) * (self.hz * dz2)
        else:
            d21, d22 = self.L["d2zzdz2"][k1], self.L["d2zzdz2"][k2]
            top = ((-3.0 * f[k1, J, I] + 4.0 * f[k1 + 1, J, I] - f[k1 + 2, J, I]) * self.hz * d21 +
                      (2.0 * f[k1, J, I] - 5.0 * f[k1 + 1, J, I] + 4.0 * f[k1 + 2, J, I] - f[k1 + 3, J, I]) *
                      self.h2z * dz1 * dz1)
            if self.top:
                out[0] = top
            bot = ((3.0 * f[k2, J, I] - 4.0 * f[k2 - 1, J, I] + f[k2 - 2, J, I]) * self.hz * d22 +
                       (2.0 * f[k2, J, I] - 5.0 * f[k2 - 1, J, I] + 4.0 * f[k2 - 2, J, I] - f[k2 - 3, J, I]) *
                       self.h2z * dz2 * dz2)
            if self.bot:
                out[-1] = bot
        return out

    # ------------------------------------------------------------------ FLUXES -------------
    def fluxes(self, X: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
        """Right-hand sides on the interior: fu fv fw fr ft (+ w1 w2 w3 = dBx/dt, dBy/dt, dBz/dt)."""
        v, DX, DY, DZ = self.v, self.DX, self.DY, self.DZ
        NX, NY = self.NX, self.NY
        RU, RV, RW, RO, TT = (X[n] for n in HYDRO)
        hx, hy, hz = self.hx, self.hy, self.hz
        dxx = self.lx("dxxdx")
        tmpy = hy * self.ly("dyydy")
        tmpz = hz * self.lz("dzzdz")
        c13, c43, ore, ocv = self.c13, self.c43, self.ore, self.ocv
        # FR (src/fluxes.cpp:87-121)
        FR = (v(RU, -1) - v(RU, 1)) * hx * dxx
        FR = FR - (v(RV, 0, 1) - v(RV, 0, -1)) * tmpy
        W1z = (v(RW, 0, 0, 1) - v(RW, 0, 0, -1)) * tmpz
        W1z = self._edge_z(W1z, RW, False)
        FR = FR - W1z
        # pressure, buoyancy, 1/rho, velocities (src/fluxes.cpp:126-166)
        FW = self.grav * v(RO)
        P = RO * TT
        r = 1.0 / RO
        FW = FW - (v(P, 0, 0, 1) - v(P, 0, 0, -1)) * tmpz
        FV = (v(P, 0, -1) - v(P, 0, 1)) * tmpy
        FU = (v(P, -1) - v(P, 1)) * hx * dxx
        UU, VV, WW = RU * r, RV * r, RW * r
        # momentum advection (src/fluxes.cpp:171-224)
        F = [FU, FV, FW]
        for c, R in enumerate((RU, RV, RW)):
            F[c] = F[c] - (v(R, 1) * v(UU, 1) - v(R, -1) * v(UU, -1)) * hx * dxx
            F[c] = F[c] - (v(R, 0, 1) * v(VV, 0, 1) - v(R, 0, -1) * v(VV, 0, -1)) * tmpy
            F[c] = F[c] - (v(R, 0, 0, 1) * v(WW, 0, 0, 1) - v(R, 0, 0, -1) * v(WW, 0, 0, -1)) * tmpz
        FU, FV, FW = F
        rc, Tc = v(r), v(TT)
        # energy advection (src/fluxes.cpp:229-243)
        FT = -1.0 * v(UU) * (v(TT, 1) - v(TT, -1)) * hx * dxx
        FT = FT - v(VV) * (v(TT, 0, 1) - v(TT, 0, -1)) * tmpy
        FT = FT - v(WW) * (v(TT, 0, 0, 1) - v(TT, 0, 0, -1)) * tmpz
        # thermal diffusion (src/fluxes.cpp:246-276)
        tmp = ocv / self.repr
        rk, dk = self.lz("rkapa"), self.lz("dkapa")
        tmpz1 = hz * self.lz("d2zzdz2")
        tmpz2 = self.h2z * self.lz("dzzdz") * self.lz("dzzdz")
        tmpy1 = hy * self.ly("d2yydy2")
        tmpy2 = self.h2y * self.ly("dyydy") * self.ly("dyydy")
        FT = FT + ((v(TT, 1) - v(TT, -1)) * hx * self.lx("d2xxdx2") +
                   (v(TT, 1) - 2.0 * Tc + v(TT, -1)) * self.h2x * dxx * dxx) * rc * tmp * rk
        FT = FT + ((v(TT, 0, 1) - v(TT, 0, -1)) * tmpy1 + (v(TT, 0, 1) - 2.0 * Tc + v(TT, 0, -1)) * tmpy2) * rc * tmp * rk
        FT = FT + ((v(TT, 0, 0, 1) - v(TT, 0, 0, -1)) * tmpz1 +
                   (v(TT, 0, 0, 1) - 2.0 * Tc + v(TT, 0, 0, -1)) * tmpz2) * rc * tmp * rk
        FT = FT + (v(TT, 0, 0, 1) - v(TT, 0, 0, -1)) * hz * self.lz("dzzdz") * rc * tmp * dk

        # viscous momentum (src/fluxes.cpp:281-320)
        def sxy(f):
            return ((v(f, 1) - v(f, -1)) * hx * self.lx("d2xxdx2") + (v(f, 1) - 2.0 * v(f) + v(f, -1)) * self.h2x * dxx * dxx,
                    (v(f, 0, 1) - v(f, 0, -1)) * tmpy1, (v(f, 0, 1) - 2.0 * v(f) + v(f, 0, -1)) * tmpy2,
                    (v(f, 0, 0, 1) - v(f, 0, 0, -1)) * tmpz1, (v(f, 0, 0, 1) - 2.0 * v(f) + v(f, 0, 0, -1)) * tmpz2)
        a, b1, b2, e1, e2 = sxy(UU)
        FU = FU + ore * (c43 * a + b1 + b2 + e1 + e2)
        a, b1, b2, e1, e2 = sxy(VV)
        FV = FV + ore * (a + c43 * (b1 + b2) + e1 + e2)
        a, b1, b2, e1, e2 = sxy(WW)
        FW = FW + ore * (a + b1 + b2 + c43 * (e1 + e2))
        # viscous heating, p dV, cross terms (src/fluxes.cpp:327-514)
        allj, alli = (0, NY - 1), (0, NX - 1)
        ux_e = DX(UU, jr=allj)             # j over the whole y range
        vx_e = DX(VV, jr=allj)
        wx = DX(WW)
        ux, vx = ux_e[:, 1:-1, :], vx_e[:, 1:-1, :]
        tA = ocv * ore
        FT = FT + (c43 * ux * ux + vx * vx + wx * wx) * rc * tA
        FT = FT - ocv * ux * Tc
        tB = c13 * ore
        FU = FU + tB * (vx_e[:, 2:, :] - vx_e[:, :-2, :]) * hy * self.ly("dyydy")
        FV = FV + tB * (ux_e[:, 2:, :] - ux_e[:, :-2, :]) * hy * self.ly("dyydy")
        uy = DY(UU)
        FT = FT + (uy * uy + 2.0 * uy * vx) * rc * tA
        vy = DY(VV)
        tC = c43 * ocv * ore
        FT = FT + vy * vy * rc * tC
        FT = FT - ocv * vy * Tc
        wz_e = DZ(WW, jr=allj, ir=alli)    # the whole x-y plane
        wz = wz_e[:, 1:-1, 1:-1]
        FT = FT + (wz * wz - ux * wz - ux * vy - vy * wz) * rc * tC
        FT = FT - ocv * wz * Tc
        FU = FU + tB * (wz_e[:, 1:-1, 2:] - wz_e[:, 1:-1, :-2]) * hx * dxx
        FV = FV + tB * (wz_e[:, 2:, 1:-1] - wz_e[:, :-2, 1:-1]) * hy * self.ly("dyydy")
        uz_e = DZ(UU, ir=alli)
        vz_e = DZ(VV, jr=allj)
        wy = DY(WW)
        uz, vz = uz_e[:, :, 1:-1], vz_e[:, 1:-1, :]
        FT = FT + (uz * uz + vz * vz + wy * wy + 2.0 * vz * wy) * rc * tA
        FW = FW + tB * ((uz_e[:, :, 2:] - uz_e[:, :, :-2]) * hx * dxx +
                        (vz_e[:, 2:, :] - vz_e[:, :-2, :]) * hy * self.ly("dyydy"))
        FT = FT + 2.0 * uz * wx * rc * tA
        # rotation (src/fluxes.cpp:519-533)
        if self.lrot:
            FU = FU + self.omz * v(RV)
            FV = FV + (-self.omz * v(RU) + self.omx * v(RW))
            FW = FW + -self.omx * v(RV)
        out = {"fu": FU, "fv": FV, "fw": FW, "fr": FR, "ft": FT}
        if not self.lmag:
            return out
        # MHD (golden/fortran/3dmhdsub.f:2146-2650, statement labels in the comments)
        BX, BY, BZ = X["bx"], X["by"], X["bz"]
        bx, by, bz = v(BX), v(BY), v(BZ)
        uc, vc, wc = v(UU), v(VV), v(WW)
        obeta, orm = self.obeta, self.orm
        W2 = bx * vx - by * ux                                   # 1030
        W3 = bx * wx - bz * ux                                   # 1040
        W1 = by * uy - bx * vy                                   # 1080
        W3 = W3 + by * wy - bz * vy                              # 1090
        wzm = self._edge_z(wz.copy(), WW, False)                 # 1120-1126
        W1 = W1 + bz * uz - bx * wzm                             # 1130
        W2 = W2 + bz * vz - by * wzm                             # 1140
        bxx, byx, bzx, bxy = DX(BX), DX(BY), DX(BZ), DY(BX)      # 1150-1180
        FU = FU + obeta * by * (bxy - byx) - obeta * bz * bzx    # 1190
        FV = FV + obeta * bx * (byx - bxy)                       # 1200
        FW = FW + obeta * bx * bzx                               # 1210
        tM = obeta * orm * ocv
        FT = FT + (bxy * bxy + byx * byx + bzx * bzx - 2.0 * byx * bxy) * rc * tM   # 1220
        W1 = W1 - uc * bxx - vc * bxy                            # 1230
        W2 = W2 - uc * byx                                       # 1240
        W3 = W3 - uc * bzx                                       # 1250
        W1 = W1 + orm * (self.D2X(BX) + self.D2Y(BX))            # 1260-1280
        W2 = W2 + orm * self.D2X(BY)                             # 1265, 1290
        W3 = W3 + orm * self.D2X(BZ)                             # 1300, 1310
        bxz, byy = DZ(BX), DY(BY)                                # 1320, 1330
        FU = FU + obeta * bz * bxz                               # 1340
        FW = FW - obeta * bx * bxz                               # 1350
        FT = FT + (bxz * bxz - 2.0 * bxz * bzx) * rc * tM        # 1360
        W1 = W1 - wc * bxz                                       # 1370
        W2 = W2 - vc * byy                                       # 1380
        d2 = self._edge_z(self.D2Z(BX), BX, True)                # 1390-1392
        W1 = W1 + orm * d2                                       # 1410
        W2 = W2 + orm * self.D2Y(BY)                             # 1400, 1420
        byz, bzy = DZ(BY), DY(BZ)                                # 1430, 1440
        xu = byz - bzy                                           # 1450
        FV = FV + obeta * bz * xu                                # 1460
        FW = FW - obeta * by * xu                                # 1470
        FT = FT + (byz * byz + bzy * bzy - 2.0 * byz * bzy) * rc * tM   # 1480
        W2 = W2 - wc * byz                                       # 1490
        W3 = W3 - vc * bzy                                       # 1500
        d2 = self._edge_z(self.D2Z(BY), BY, True)                # 1510-1513
        W2 = W2 + orm * d2                                       # 1530
        W3 = W3 + orm * self.D2Y(BZ)                             # 1520, 1540
        W3 = W3 - wc * DZ(BZ)                                    # 1550, 1560
        W3 = W3 + orm * self.D2Z(BZ)                             # 1570, 1580
        out.update({"fu": FU, "fv": FV, "fw": FW, "ft": FT, "w1": W1, "w2": W2, "w3": W3})
        return out

    # --------------------------------------------------------------- BCON, ghosts ----------
    def ghost_fill(self, f):
        """Periodic x/y ghost images on every plane (src/communicate.cpp on one domain)."""
        f[:, 0, :] = f[:, -2, :]
        f[:, -1, :] = f[:, 1, :]
        f[:, :, 0] = f[:, :, -2]
        f[:, :, -1] = f[:, :, 1]

    def bcon(self, X):
        """src/bcon.cpp:12-141 on the global top (k=1) and bottom (k=npz) planes."""
        c13, c23, c43 = self.c13, self.c23, self.c43
        J, I = slice(1, self.NY - 1), slice(1, self.NX - 1)
        ru, rv, rw, ro, tt = (X[n] for n in HYDRO)
        k1, k2 = 1, self.NZ - 2
        for k, d in ((k1, 1), (k2, -1)):
            if (k == k1 and not self.top) or (k == k2 and not self.bot):
                continue  # a neighbour's plane, not a face of the domain
            ru[k, J, I] = ro[k, J, I] * (c43 * ru[k + d, J, I] / ro[k + d, J, I] - c13 * ru[k + 2 * d, J, I] / ro[k + 2 * d, J, I])
            rv[k, J, I] = ro[k, J, I] * (c43 * rv[k + d, J, I] / ro[k + d, J, I] - c13 * rv[k + 2 * d, J, I] / ro[k + 2 * d, J, I])
            rw[k, J, I] = 0.0
            if k == k1:
                self._top_t(tt, J, I)
            else:
                if self.izcon == 0:
                    tt[k2, J, I] = self.tb
                else:
                    dz = _f4(np.float32(1.0) / np.float32(self.npz - 1)) / self.L["dzzdz"][k2]
                    tt[k2, J, I] = (c43 * tt[k2 - 1, J, I] - c13 * tt[k2 - 2, J, I] +
                                    c23 * dz * self.theta / self.L["rkapa"][k2])
            if self.lmag and self.ibcon == 0:
                X["bz"][k, J, I] = 0.0

    def _top_t(self, tt, J, I):
        c13, c23, c43 = self.c13, self.c23, self.c43
        k1 = 1
        exx = self.L["exx"][1:-1][None, :]
        wyy = self.L["wyy"][1:-1][:, None]
        if self.tp != 0.0 and self.itcon in (0, 1):
            if self.tc != 0.0:
                raise NotImplementedError("time-dependent top temperature")
            tpr = self.tp
            cln = _f4(np.float32(-4.0) * np.log(np.float32(2.0))) / (self.hh * self.hh)
            g = (np.exp(cln * (exx - self.xp) * (exx - self.xp)) / self.hh *
                 np.exp(cln * ((wyy - self.yp) * (wyy - self.yp))) / self.hh)
            if self.itcon == 0:
                tt[k1, J, I] = 1.0 - (1.0 - tpr) * g
            else:
                dz = _f4(np.float32(1.0) / np.float32(self.npz - 1)) / self.L["dzzdz"][k1]
                tt[k1, J, I] = (c43 * tt[k1 + 1, J, I] - c13 * tt[k1 + 2, J, I] -
                                c23 * dz * (self.theta - (self.theta - tpr) * g))
        else:
            if self.itcon in (0, 2, 4):
                tt[k1, J, I] = 1.0
                if self.itcon == 4:
                    tt[k1, J, 1:self.NX // 2 + 1] = 1.0 - self.tp
            if self.itcon == 1:
                dz = _f4(np.float32(1.0) / np.float32(self.npz - 1)) / self.L["dzzdz"][k1]
                tt[k1, J, I] = c43 * tt[k1 + 1, J, I] - c13 * tt[k1 + 2, J, I] - c23 * dz * self.theta

    # ------------------------------------------------------------------- dt, STEP ----------
    def dt(self, X):
        """src/step.cpp:122-229: sff x the minimum of the CFL, diffusion (and magnetic) limits.

        As in the C fold, a NaN limit (a cell with T < 0 makes sqrt(uu*gamma*T) NaN) never
        becomes the minimum.  The minimum is chosen on the real run; complex arrays carry the
        tangent of the chosen (cell, limit)."""
        wc = self._limits(X)
        wr = self._limits({n: np.real(a) for n, a in X.items()}) if np.iscomplexobj(X["tt"]) else wc
        best, bq, bi = None, -1, -1
        with np.errstate(invalid="ignore"):
            for q, w in enumerate(wr):
                flat = w.reshape(-1)
                if np.all(np.isnan(flat)):
                    continue
                i = int(np.nanargmin(flat))
                if best is None or flat[i] < best:
                    best, bq, bi = flat[i], q, i
        if self.reduce_min is not None:  # a slab: the minimum over every slab (real runs only)
            return self.sff * self.reduce_min(float(best) if best is not None else 1e300)
        return self.sff * wc[bq].reshape(-1)[bi]

    def _limits(self, X):
        v = self.v
        ru, rv, rw, ro, tt = (v(X[n]) for n in HYDRO)
        with np.errstate(invalid="ignore"):
            uu = (ru * ru + rv * rv + rw * rw) * (1.0 / ro) * (1.0 / ro)
            if self.lmag:
                bx, by, bz = (v(X[n]) for n in MAG)
                b2 = (bx * bx + by * by + bz * bz) * self.obeta / ro
                uu = uu + self.gamma * tt + b2 + 2.0 * np.sqrt(uu * (self.gamma * tt + b2))
            else:
                uu = uu + self.gamma * tt + 2.0 * np.sqrt(uu * self.gamma * tt)
            a = self.lx("ddx")
            b = self.ly("ddy")
            c = self.lz("ddz")
            m = np.where(b < a, b, a)
            dd = np.where(c < m, c, m)
            w = [dd / np.sqrt(uu),
                 0.5 * dd * dd * self.repr * self.cv * ro / self.lz("rkapa"),
                 0.375 * dd * dd * self.re * ro]
            if self.lmag:
                w.append(0.5 * dd * dd * self.rm + 0.0 * ro)
        return w

    def step(self, X: Dict[str, np.ndarray]):
        """One full RK3 step (src/step.cpp:114-257); returns (new state, dt).  X is not modified."""
        X = {n: a.copy() for n, a in X.items()}
        dt = self.dt(X)
        names = self.fields
        fmap = {"ru": "fu", "rv": "fv", "rw": "fw", "ro": "fr", "tt": "ft", "bx": "w1", "by": "w2", "bz": "w3"}
        I = (slice(1, self.NZ - 1), slice(1, self.NY - 1), slice(1, self.NX - 1))
        Z = {n: X[n][I].copy() for n in names}
        gam = [self.gam1, self.gam2, self.gam3]
        zeta = [0.0, self.zeta1, self.zeta2]
        F = None
        for st in range(3):
            if st > 0:
                coef = zeta[st] * dt
                Z = {n: X[n][I] + coef * F[fmap[n]] for n in names}
            F = self.fluxes(X)
            coef = gam[st] * dt
            for n in names:
                X[n][I] = Z[n] + coef * F[fmap[n]]
            self.bcon(X)
            for n in names:
                self.ghost_fill(X[n])
            if self.exchange is not None:
                self.exchange(X)
        return X, dt

    def run(self, X, nsteps: int):
        dts = []
        for _ in range(nsteps):
            X, dt = self.step(X)
            dts.append(dt)
        return X, dts

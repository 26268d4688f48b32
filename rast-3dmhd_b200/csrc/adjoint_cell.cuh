// adjoint_cell.cuh - per-cell arithmetic of the discrete adjoint of one FP64 RK3 step.
//
// The forward step (src/step.cpp:114-257 with src/fluxes.cpp:87-533, src/bcon.cpp:12-141 and,
// with LMAG, golden/fortran/3dmhdsub.f:2146-2650) is, per stage s,
//     Y = Z_s + gam_s dt F(X_s),  X_{s+1} = BCON(Y),  Z_{s+1} = X_{s+1} + zeta_{s+1} dt F(X_s),
// with dt = sff * min over cells of the CFL / diffusion limits of X_0.  Its adjoint runs the
// stages backwards; the one non-trivial piece is the transpose of the flux Jacobian, F'(X)^T.
// Every flux term is a product of point values at the output cell (u, v, w, 1/rho, T, B) and
// first/second differences of u, v, w, T, P = rho*T, B and the momenta, plus the cross
// differences d/dy(du/dx)-type terms of the viscous stress.  F'^T is therefore evaluated in
// two gather passes, with no atomics:
//
//   pass 1 (per output cell c): from the flux adjoint a = lambda_F(c) and the forward values
//     at c, the adjoints of every difference quantity evaluated at c (the "Lambda" arrays:
//     du/dx .. dw/dz, the conduction stencils of T, dB/dx ..) and the pointwise partials
//     w.r.t. u, v, w, 1/rho, T, B at c.  The cross-difference terms (FU += c13/Re d/dy(dv/dx)
//     ...) add the transposed outer difference of a's neighbours to the Lambda of the inner
//     difference, so pass 1 reads a at the x/y neighbours of c.
//   pass 2 (per input cell m): the transposed difference stencils, gathered from Lambda and a
//     at the neighbours of m (a central difference coef(c)*(f(c+e) - f(c-e)) contributes
//     coef(m-e)*Lambda(m-e) - coef(m+e)*Lambda(m+e) to f's adjoint at m), then the chain rule
//     through u = RU/rho, P = rho*T, 1/rho back to RU RV RW RO TT (BX BY BZ).
//
// x and y are periodic: the forward reads ghost cells that are exact images of interior cells,
// so the adjoint works on the npx x npy torus with wrapped neighbour indices and never stores an
// adjoint in a ghost cell.  The z ghost planes are constants of the forward map (zero momenta
// and field there), so adjoints that would land on them are dropped.  The one-sided z stencils
// of the planes k = 1 and k = npz (the continuity flux, src/fluxes.cpp:106-117, and the LMAG
// terms of 3dmhdsub.f 1125/1126, 1391/1392, 1511/1513) transpose to the extra edge terms of
// gzos() and d2zos().
#pragma once

#include "r3d_device.cuh"

#ifdef __CUDACC__
#define R3D_HD __host__ __device__ __forceinline__
#else
#define R3D_HD inline
#endif

namespace r3dk {

// Lambda arrays written by pass 1 and read by pass 2 (the last 13 only with LMAG).
enum {
    L_UX, L_VX, L_WX, L_UY, L_VY, L_WY, L_UZ, L_VZ, L_WZ,   // adjoints of du/dx .. dw/dz (central)
    L_TSX, L_TLX, L_TSY, L_TLY, L_TSZ, L_TLZ,               // T stencils: coefficient * lambda_FT
    P_U, P_V, P_W, P_R, P_T,                                // pointwise partials at the cell
    kLamHydro,
    L_WZM = kLamHydro,                                      // one-sided-at-edges dw/dz (LMAG)
    L_BXX, L_BYX, L_BZX, L_BXY, L_BYY, L_BZY, L_BXZ, L_BYZ, L_BZZ,
    P_BX, P_BY, P_BZ,
    kLamMax
};

enum { F_RU, F_RV, F_RW, F_RO, F_TT, F_BX, F_BY, F_BZ };

// Everything the adjoint passes read or write.  Field pointers use the padded device layout.
struct AdjArgs {
    Geometry g;
    Physics ph;
    Lines L;
    const double* x[kMaxFields];     // forward state X_s
    const double* a[kMaxFields];     // lambda_F: adjoint of F(X_s) = (FU FV FW FR FT W1 W2 W3)
    double* lam[kMaxFields];         // pass 2: in lambda_Y (the Z path), out lambda_X_s
    double* Lam[kLamMax];            // pass 1 out, pass 2 in
    double* fnext[kMaxFields];       // pass 2, stage s > 0: lambda_F of the previous stage
    const double* fprev[kMaxFields]; // pass 2, stage s > 0: F(X_{s-1}) for d/d(dt)
    const Scalars* sc;               // dt of the step
    double zeta;                     // zeta_s
    int nf;                          // 5 or 8
};

struct Nbr {  // neighbour offsets of an interior cell on the x/y torus
    int n, xp, xm, yp, ym, ip, im, jp, jm;
};

R3D_HD Nbr neighbours(const Geometry& g, int i, int j, int k) {
    Nbr b;
    const int P = (int)g.pitch, PL = (int)g.plane;
    b.ip = (i == g.npx) ? 1 : i + 1;
    b.im = (i == 1) ? g.npx : i - 1;
    b.jp = (j == g.npy) ? 1 : j + 1;
    b.jm = (j == 1) ? g.npy : j - 1;
    b.n = k * PL + j * P + i;
    b.xp = k * PL + j * P + b.ip;
    b.xm = k * PL + j * P + b.im;
    b.yp = k * PL + b.jp * P + i;
    b.ym = k * PL + b.jm * P + i;
    return b;
}

// ------------------------------------------------------------------------ pass 1 --------
R3D_HD void adj_pass1_cell(const AdjArgs& A, int i, int j, int k) {
    const Geometry& g = A.g;
    const Physics& ph = A.ph;
    const Lines& L = A.L;
    const Nbr b = neighbours(g, i, j, k);
    const int PL = (int)g.plane;
    const int n = b.n, zp = n + PL, zm = n - PL;
    const double* const* x = A.x;
    const double* const* a = A.a;
    const bool mhd = A.nf == 8;

    auto vel = [&](int q, int m) { return x[q][m] / x[F_RO][m]; };  // u = RU/rho etc.
    const double r = 1.0 / x[F_RO][n];
    const double u = x[F_RU][n] * r, v = x[F_RV][n] * r, w = x[F_RW][n] * r;
    const double T = x[F_TT][n];

    const double X1 = ph.hx * L.dxxdx[i], Y1 = L.tmpy[j], Z1 = L.tmpz[k];
    const double X2s = ph.hx * L.d2xxdx2[i], X2l = ph.h2x * L.dxxdx[i] * L.dxxdx[i];
    const double Y2s = L.tmpy1[j], Y2l = L.tmpy2[j], Z2s = L.tmpz1[k], Z2l = L.tmpz2[k];

    // first differences of the velocities at c (central on every plane; planes 1 and npz
    // read the constant z ghost planes, where the momenta vanish)
    const double ux = (vel(F_RU, b.xp) - vel(F_RU, b.xm)) * X1;
    const double vx = (vel(F_RV, b.xp) - vel(F_RV, b.xm)) * X1;
    const double wx = (vel(F_RW, b.xp) - vel(F_RW, b.xm)) * X1;
    const double uy = (vel(F_RU, b.yp) - vel(F_RU, b.ym)) * Y1;
    const double vy = (vel(F_RV, b.yp) - vel(F_RV, b.ym)) * Y1;
    const double wy = (vel(F_RW, b.yp) - vel(F_RW, b.ym)) * Y1;
    const double uz = (vel(F_RU, zp) - vel(F_RU, zm)) * Z1;
    const double vz = (vel(F_RV, zp) - vel(F_RV, zm)) * Z1;
    const double wz = (vel(F_RW, zp) - vel(F_RW, zm)) * Z1;
    // T stencils
    const double* tt = x[F_TT];
    const double sxT = tt[b.xp] - tt[b.xm], lxT = tt[b.xp] - 2.0 * T + tt[b.xm];
    const double syT = tt[b.yp] - tt[b.ym], lyT = tt[b.yp] - 2.0 * T + tt[b.ym];
    const double szT = tt[zp] - tt[zm], lzT = tt[zp] - 2.0 * T + tt[zm];

    const double aU = a[F_RU][n], aV = a[F_RV][n], aW = a[F_RW][n], aT = a[F_TT][n];
    // transposed outer differences of the cross terms, read at c's x/y neighbours
    const double Y1m = L.tmpy[b.jm], Y1p = L.tmpy[b.jp];
    const double X1m = ph.hx * L.dxxdx[b.im], X1p = ph.hx * L.dxxdx[b.ip];
    const double GUy = Y1m * a[F_RU][b.ym] - Y1p * a[F_RU][b.yp];
    const double GVy = Y1m * a[F_RV][b.ym] - Y1p * a[F_RV][b.yp];
    const double GWy = Y1m * a[F_RW][b.ym] - Y1p * a[F_RW][b.yp];
    const double GUx = X1m * a[F_RU][b.xm] - X1p * a[F_RU][b.xp];
    const double GWx = X1m * a[F_RW][b.xm] - X1p * a[F_RW][b.xp];

    const double tA = ph.theat, tC = ph.theat43, tB = ph.t13, ocv = ph.ocv, c43 = ph.c43;
    const double tk = ph.tdiff, rk = L.rkapa[k], dk = L.dkapa[k];

    // energy advection and conduction (src/fluxes.cpp:229-276)
    double Pu = -aT * X1 * sxT, Pv = -aT * Y1 * syT, Pw = -aT * Z1 * szT;
    double Pr = aT * tk * (rk * (sxT * X2s + lxT * X2l + syT * Y2s + lyT * Y2l + szT * Z2s + lzT * Z2l) +
                           dk * Z1 * szT);
    double* const* Lm = A.Lam;
    Lm[L_TSX][n] = aT * (-u * X1 + r * tk * rk * X2s);
    Lm[L_TLX][n] = aT * r * tk * rk * X2l;
    Lm[L_TSY][n] = aT * (-v * Y1 + r * tk * rk * Y2s);
    Lm[L_TLY][n] = aT * r * tk * rk * Y2l;
    Lm[L_TSZ][n] = aT * (-w * Z1 + r * tk * rk * Z2s + r * tk * dk * Z1);
    Lm[L_TLZ][n] = aT * r * tk * rk * Z2l;

    // viscous heating, p dV and the cross terms (src/fluxes.cpp:327-514)
    double Lux = aT * (tA * r * 2.0 * c43 * ux - ocv * T + tC * r * (-wz - vy)) + tB * GVy;
    double Lvx = aT * tA * r * (2.0 * vx + 2.0 * uy) + tB * GUy;
    double Lwx = aT * tA * r * (2.0 * wx + 2.0 * uz);
    double Luy = aT * tA * r * (2.0 * uy + 2.0 * vx);
    double Lvy = aT * (tC * r * (2.0 * vy - ux - wz) - ocv * T);
    double Lwy = aT * tA * r * (2.0 * wy + 2.0 * vz);
    double Luz = aT * tA * r * (2.0 * uz + 2.0 * wx) + tB * GWx;
    double Lvz = aT * tA * r * (2.0 * vz + 2.0 * wy) + tB * GWy;
    double Lwz = aT * (tC * r * (2.0 * wz - ux - vy) - ocv * T) + tB * (GUx + GVy);
    Pr += aT * (tA * (c43 * ux * ux + vx * vx + wx * wx + uy * uy + 2.0 * uy * vx + uz * uz + vz * vz +
                      wy * wy + 2.0 * vz * wy + 2.0 * uz * wx) +
                tC * (vy * vy + wz * wz - ux * wz - ux * vy - vy * wz));
    double PT = -aT * ocv * (ux + vy + wz);

    if (mhd) {
        // golden/fortran/3dmhdsub.f:2146-2650
        const double BX = x[F_BX][n], BY = x[F_BY][n], BZ = x[F_BZ][n];
        const double a1 = a[F_BX][n], a2 = a[F_BY][n], a3 = a[F_BZ][n];
        const double ob = ph.obeta, tM = ph.tmag;
        const double* bx = x[F_BX];
        const double* by = x[F_BY];
        const double* bz = x[F_BZ];
        const double bxx = (bx[b.xp] - bx[b.xm]) * X1, byx = (by[b.xp] - by[b.xm]) * X1,
                     bzx = (bz[b.xp] - bz[b.xm]) * X1;
        const double bxy = (bx[b.yp] - bx[b.ym]) * Y1, byy = (by[b.yp] - by[b.ym]) * Y1,
                     bzy = (bz[b.yp] - bz[b.ym]) * Y1;
        const double bxz = (bx[zp] - bx[zm]) * Z1, byz = (by[zp] - by[zm]) * Z1, bzz = (bz[zp] - bz[zm]) * Z1;
        double wzm = wz;  // 3dmhdsub.f 1125/1126: one-sided on the edge planes
        if (k == 1) wzm = (4.0 * vel(F_RW, zp) - vel(F_RW, zp + PL)) * Z1;
        if (k == g.npz) wzm = (vel(F_RW, zm - PL) - 4.0 * vel(F_RW, zm)) * Z1;
        // induction: W1 = BY uy - BX vy + BZ uz - BX wzm ..., W2, W3
        Luy += a1 * BY;
        Lvy += -a1 * BX - a3 * BZ;
        Luz += a1 * BZ;
        Lvx += a2 * BX;
        Lux += -a2 * BY - a3 * BZ;
        Lvz += a2 * BZ;
        Lwx += a3 * BX;
        Lwy += a3 * BY;
        Lm[L_WZM][n] = -a1 * BX - a2 * BY;
        // field differences: advection of B, Lorentz force and ohmic heating
        Lm[L_BXX][n] = -a1 * u;
        Lm[L_BXY][n] = -a1 * v + ob * (aU * BY - aV * BX) + aT * tM * r * (2.0 * bxy - 2.0 * byx);
        Lm[L_BXZ][n] = -a1 * w + ob * (aU * BZ - aW * BX) + aT * tM * r * (2.0 * bxz - 2.0 * bzx);
        Lm[L_BYX][n] = -a2 * u + ob * (-aU * BY + aV * BX) + aT * tM * r * (2.0 * byx - 2.0 * bxy);
        Lm[L_BYY][n] = -a2 * v;
        Lm[L_BYZ][n] = -a2 * w + ob * (aV * BZ - aW * BY) + aT * tM * r * (2.0 * byz - 2.0 * bzy);
        Lm[L_BZX][n] = -a3 * u + ob * (-aU * BZ + aW * BX) + aT * tM * r * (2.0 * bzx - 2.0 * bxz);
        Lm[L_BZY][n] = -a3 * v + ob * (-aV * BZ + aW * BY) + aT * tM * r * (2.0 * bzy - 2.0 * byz);
        Lm[L_BZZ][n] = -a3 * w;
        Lm[P_BX][n] = a1 * (-vy - wzm) + a2 * vx + a3 * wx + aV * ob * (byx - bxy) + aW * ob * (bzx - bxz);
        Lm[P_BY][n] = a1 * uy + a2 * (-ux - wzm) + a3 * wy + aU * ob * (bxy - byx) - aW * ob * (byz - bzy);
        Lm[P_BZ][n] = a1 * uz + a2 * vz + a3 * (-ux - vy) + aU * ob * (bxz - bzx) + aV * ob * (byz - bzy);
        Pu += -a1 * bxx - a2 * byx - a3 * bzx;
        Pv += -a1 * bxy - a2 * byy - a3 * bzy;
        Pw += -a1 * bxz - a2 * byz - a3 * bzz;
        Pr += aT * tM * (bxy * bxy + byx * byx + bzx * bzx - 2.0 * byx * bxy + bxz * bxz - 2.0 * bxz * bzx +
                         byz * byz + bzy * bzy - 2.0 * byz * bzy);
    }
    Lm[L_UX][n] = Lux;
    Lm[L_VX][n] = Lvx;
    Lm[L_WX][n] = Lwx;
    Lm[L_UY][n] = Luy;
    Lm[L_VY][n] = Lvy;
    Lm[L_WY][n] = Lwy;
    Lm[L_UZ][n] = Luz;
    Lm[L_VZ][n] = Lvz;
    Lm[L_WZ][n] = Lwz;
    Lm[P_U][n] = Pu;
    Lm[P_V][n] = Pv;
    Lm[P_W][n] = Pw;
    Lm[P_R][n] = Pr;
    Lm[P_T][n] = PT;
}

// ------------------------------------------------------------------------ pass 2 --------
// Returns this cell's contribution to sum_f F_{s-1} * lambda_Y (the d/d(dt) dot of the Z path),
// zero for stage 0.
R3D_HD double adj_pass2_cell(const AdjArgs& A, int i, int j, int k) {
    const Geometry& g = A.g;
    const Physics& ph = A.ph;
    const Lines& L = A.L;
    const Nbr b = neighbours(g, i, j, k);
    const int PL = (int)g.plane, npz = g.npz;
    const int n = b.n, zp = n + PL, zm = n - PL;
    const int c1 = n - (k - 1) * PL, c2 = n + (npz - k) * PL;  // (i, j, 1) and (i, j, npz)
    const bool lo = k > 1, hi = k < npz;
    const double* const* a = A.a;
    double* const* Lm = A.Lam;
    const bool mhd = A.nf == 8;

    const double X1m = ph.hx * L.dxxdx[b.im], X1p = ph.hx * L.dxxdx[b.ip];
    const double Y1m = L.tmpy[b.jm], Y1p = L.tmpy[b.jp];
    const double Z1m = lo ? L.tmpz[k - 1] : 0.0, Z1p = hi ? L.tmpz[k + 1] : 0.0;
    // transposed central first differences (coefficients live at the output cell)
    auto gx = [&](const double* F) { return X1m * F[b.xm] - X1p * F[b.xp]; };
    auto gy = [&](const double* F) { return Y1m * F[b.ym] - Y1p * F[b.yp]; };
    auto gz = [&](const double* F) { return (lo ? Z1m * F[zm] : 0.0) - (hi ? Z1p * F[zp] : 0.0); };
    // same, for a difference that is one-sided on the planes 1 and npz
    auto gzos = [&](const double* F) {
        double s = 0.0;
        if (k - 1 >= 2 && k - 1 <= npz - 1) s += L.tmpz[k - 1] * F[zm];
        if (k + 1 >= 2 && k + 1 <= npz - 1) s -= L.tmpz[k + 1] * F[zp];
        if (k == 2) s += 4.0 * L.tmpz[1] * F[c1];      // (4 f(2) - f(3)) tmpz(1)
        if (k == 3) s -= L.tmpz[1] * F[c1];
        if (k == npz - 1) s -= 4.0 * L.tmpz[npz] * F[c2];  // (f(npz-2) - 4 f(npz-1)) tmpz(npz)
        if (k == npz - 2) s += L.tmpz[npz] * F[c2];
        return s;
    };
    // transposed second differences Sx f * X2s + Lx f * X2l (and y, z)
    const double X2sm = ph.hx * L.d2xxdx2[b.im], X2sp = ph.hx * L.d2xxdx2[b.ip];
    const double X2lm = ph.h2x * L.dxxdx[b.im] * L.dxxdx[b.im], X2lp = ph.h2x * L.dxxdx[b.ip] * L.dxxdx[b.ip];
    const double X2l0 = ph.h2x * L.dxxdx[i] * L.dxxdx[i];
    auto d2x = [&](const double* F) {
        return (X2sm + X2lm) * F[b.xm] + (-X2sp + X2lp) * F[b.xp] - 2.0 * X2l0 * F[n];
    };
    auto d2y = [&](const double* F) {
        return (L.tmpy1[b.jm] + L.tmpy2[b.jm]) * F[b.ym] + (-L.tmpy1[b.jp] + L.tmpy2[b.jp]) * F[b.yp] -
               2.0 * L.tmpy2[j] * F[n];
    };
    auto d2z = [&](const double* F) {
        double s = -2.0 * L.tmpz2[k] * F[n];
        if (lo) s += (L.tmpz1[k - 1] + L.tmpz2[k - 1]) * F[zm];
        if (hi) s += (-L.tmpz1[k + 1] + L.tmpz2[k + 1]) * F[zp];
        return s;
    };
    auto d2zos = [&](const double* F) {  // 3dmhdsub.f 1391/1392, 1511/1513 on the edge planes
        double s = 0.0;
        if (k >= 2 && k <= npz - 1) s -= 2.0 * L.tmpz2[k] * F[n];
        if (k - 1 >= 2 && k - 1 <= npz - 1) s += (L.tmpz1[k - 1] + L.tmpz2[k - 1]) * F[zm];
        if (k + 1 >= 2 && k + 1 <= npz - 1) s += (-L.tmpz1[k + 1] + L.tmpz2[k + 1]) * F[zp];
        // coefficients of f(1+o) (top) / f(npz-o) (bottom), o = 0..3, in the one-sided first
        // (s) and second (l) differences; selected, not indexed, so that no local array is made
        auto l4 = [](int o) { return o == 0 ? 2.0 : (o == 1 ? -5.0 : (o == 2 ? 4.0 : -1.0)); };
        auto s4 = [](int o) { return o == 0 ? -3.0 : (o == 1 ? 4.0 : (o == 2 ? -1.0 : 0.0)); };
        const int o1 = k - 1, o2 = npz - k;
        if (o1 <= 3) s += (L.tmpz1[1] * s4(o1) + L.tmpz2[1] * l4(o1)) * F[c1];
        if (o2 <= 3) s += (L.tmpz1[npz] * -s4(o2) + L.tmpz2[npz] * l4(o2)) * F[c2];
        return s;
    };
    // transposed T stencils (the Lambda already carry their coefficients)
    auto sx = [&](const double* F) { return F[b.xm] - F[b.xp]; };
    auto sy = [&](const double* F) { return F[b.ym] - F[b.yp]; };
    auto sz = [&](const double* F) { return (lo ? F[zm] : 0.0) - (hi ? F[zp] : 0.0); };
    auto lx = [&](const double* F) { return F[b.xm] + F[b.xp] - 2.0 * F[n]; };
    auto ly = [&](const double* F) { return F[b.ym] + F[b.yp] - 2.0 * F[n]; };
    auto lz = [&](const double* F) { return (lo ? F[zm] : 0.0) + (hi ? F[zp] : 0.0) - 2.0 * F[n]; };

    const double* aU = a[F_RU];
    const double* aV = a[F_RV];
    const double* aW = a[F_RW];
    const double* aR = a[F_RO];
    const double RU = A.x[F_RU][n], RV = A.x[F_RV][n], RW = A.x[F_RW][n], RO = A.x[F_RO][n], TT = A.x[F_TT][n];
    const double r = 1.0 / RO, u = RU * r, v = RV * r, w = RW * r;
    const double gUx = gx(aU), gVx = gx(aV), gWx = gx(aW);
    const double gUy = gy(aU), gVy = gy(aV), gWy = gy(aW);
    const double gUz = gz(aU), gVz = gz(aV), gWz = gz(aW);
    const double ore = ph.ore, c43 = ph.c43;

    double lu = Lm[P_U][n] + gx(Lm[L_UX]) + gy(Lm[L_UY]) + gz(Lm[L_UZ]) +
                ore * (c43 * d2x(aU) + d2y(aU) + d2z(aU)) - (RU * gUx + RV * gVx + RW * gWx);
    double lv = Lm[P_V][n] + gx(Lm[L_VX]) + gy(Lm[L_VY]) + gz(Lm[L_VZ]) +
                ore * (d2x(aV) + c43 * d2y(aV) + d2z(aV)) - (RU * gUy + RV * gVy + RW * gWy);
    double lw = Lm[P_W][n] + gx(Lm[L_WX]) + gy(Lm[L_WY]) + gz(Lm[L_WZ]) +
                ore * (d2x(aW) + d2y(aW) + c43 * d2z(aW)) - (RU * gUz + RV * gVz + RW * gWz);
    if (mhd) lw += gzos(Lm[L_WZM]);
    const double lP = -(gUx + gVy + gWz);
    const double lT = Lm[P_T][n] + sx(Lm[L_TSX]) + lx(Lm[L_TLX]) + sy(Lm[L_TSY]) + ly(Lm[L_TLY]) +
                      sz(Lm[L_TSZ]) + lz(Lm[L_TLZ]);
    double out[kMaxFields];
    // momenta: advection (R_a * u_b), continuity, rotation, then the chain rule through u = RU/rho
    out[F_RU] = -(u * gUx + v * gUy + w * gUz) - gx(aR) - ph.omz * aV[n] + r * lu;
    out[F_RV] = -(u * gVx + v * gVy + w * gVz) - gy(aR) + ph.omz * aU[n] - ph.omx * aW[n] + r * lv;
    out[F_RW] = -(u * gWx + v * gWy + w * gWz) - gzos(aR) + ph.omx * aV[n] + r * lw;
    out[F_RO] = ph.grav * aW[n] - r * r * (Lm[P_R][n] + RU * lu + RV * lv + RW * lw) + TT * lP;
    out[F_TT] = lT + RO * lP;
    if (mhd) {
        const double orm = ph.orm;
        out[F_BX] = Lm[P_BX][n] + gx(Lm[L_BXX]) + gy(Lm[L_BXY]) + gz(Lm[L_BXZ]) +
                    orm * (d2x(a[F_BX]) + d2y(a[F_BX]) + d2zos(a[F_BX]));
        out[F_BY] = Lm[P_BY][n] + gx(Lm[L_BYX]) + gy(Lm[L_BYY]) + gz(Lm[L_BYZ]) +
                    orm * (d2x(a[F_BY]) + d2y(a[F_BY]) + d2zos(a[F_BY]));
        out[F_BZ] = Lm[P_BZ][n] + gx(Lm[L_BZX]) + gy(Lm[L_BZY]) + gz(Lm[L_BZZ]) +
                    orm * (d2x(a[F_BZ]) + d2y(a[F_BZ]) + d2z(a[F_BZ]));
    }
    // + the Z path: lambda_X_s = F'^T lambda_F + lambda_Y; the previous stage's flux adjoint
    // receives zeta_s dt lambda_Y
    double dot = 0.0;
    const double zdt = A.zeta * A.sc->dt;
#pragma unroll
    for (int f = 0; f < kMaxFields; ++f) {  // unrolled over the largest field count: out[] stays in registers
        if (f < A.nf) {
            const double ly_ = A.lam[f][n];
            A.lam[f][n] = out[f] + ly_;
            if (A.fnext[0]) {
                A.fnext[f][n] = zdt * ly_;
                dot += A.fprev[f][n] * ly_;
            }
        }
    }
    return dot;
}

// ------------------------------------------------------------------- BCON^T -------------
// src/bcon.cpp:27-140 on one (i, j) column: the written values (momenta, T, Bz on the planes
// 1 and npz) pass their adjoint to what they were computed from, and their own pre-BCON
// values get none.  x holds the post-BCON state (equal to the pre-BCON state on every value
// BCON reads).
R3D_HD void adj_bcon_column(const Geometry& g, const Physics& ph, const Boundary& bd, const double* const* x,
                            double* const* lam, int nf, int i, int j) {
    const int PL = (int)g.plane;
    const double c13 = ph.c13, c43 = ph.c43;
    for (int side = 0; side < 2; ++side) {
        const int k = side == 0 ? 1 : g.npz;
        const int d = side == 0 ? PL : -PL;
        const int n = k * PL + j * (int)g.pitch + i, n1 = n + d, n2 = n + 2 * d;
        const double ro0 = x[F_RO][n], ro1 = x[F_RO][n1], ro2 = x[F_RO][n2];
        for (int q = F_RU; q <= F_RV; ++q) {  // ru = ro0 (c43 ru1/ro1 - c13 ru2/ro2), same for rv
            const double A = lam[q][n];
            const double m1 = x[q][n1], m2 = x[q][n2];
            lam[F_RO][n] += A * (c43 * m1 / ro1 - c13 * m2 / ro2);
            lam[q][n1] += A * ro0 * c43 / ro1;
            lam[q][n2] -= A * ro0 * c13 / ro2;
            lam[F_RO][n1] -= A * ro0 * c43 * m1 / (ro1 * ro1);
            lam[F_RO][n2] += A * ro0 * c13 * m2 / (ro2 * ro2);
            lam[q][n] = 0.0;
        }
        lam[F_RW][n] = 0.0;
        const bool linear = side == 0 ? (bd.top_mode == 1 || bd.top_mode == 3) : (bd.bottom_mode == 1);
        if (linear) {  // T = c43 T1 - c13 T2 + const
            const double C = lam[F_TT][n];
            lam[F_TT][n1] += c43 * C;
            lam[F_TT][n2] -= c13 * C;
        }
        lam[F_TT][n] = 0.0;
        if (nf == 8) lam[F_BZ][n] = 0.0;  // Bz = 0 at both boundaries (ibcon 0)
    }
}

// ------------------------------------------------------------------- dt^T ---------------
// Partial derivatives of the winning time-step limit at one cell (src/step.cpp:122-229):
// ww1 = dd/sqrt(c2) with c2 = q + s + 2 sqrt(q s), q = |rho u|^2/rho^2, s = gamma T (+ B^2
// obeta/rho); ww2 ~ rho; ww3 ~ rho; vv constant.  At q = 0 (a cell at rest) sqrt(q s) has no
// derivative along the momenta; its symmetric subgradient 0 is used.
R3D_HD void adj_dt_cell(const Physics& ph, int term, double dd, double rkap, const double* xv, int nf,
                        double L, double* gout) {
    for (int f = 0; f < nf; ++f) gout[f] = 0.0;
    const double ro = xv[F_RO], r = 1.0 / ro;
    if (term == 1) {  // 0.5 dd^2 repr cv rho / rkapa
        gout[F_RO] = L * (0.5 * dd * dd * ph.repr * ph.cv / rkap);
        return;
    }
    if (term == 2) {  // 0.375 dd^2 re rho
        gout[F_RO] = L * (0.375 * dd * dd * ph.re);
        return;
    }
    if (term != 0) return;
    const double ru = xv[F_RU], rv = xv[F_RV], rw = xv[F_RW], tt = xv[F_TT];
    const double q = (ru * ru + rv * rv + rw * rw) * r * r;
    double b2 = 0.0, bx = 0.0, by = 0.0, bz = 0.0;
    if (nf == 8) {
        bx = xv[F_BX];
        by = xv[F_BY];
        bz = xv[F_BZ];
        b2 = (bx * bx + by * by + bz * bz) * ph.obeta * r;
    }
    const double s = ph.gamma * tt + b2;
    const double c2 = q + s + 2.0 * sqrt(q * s);
    const double w1 = dd / sqrt(c2);
    const double dw_dc2 = -0.5 * w1 / c2;
    const double dc2_dq = 1.0 + (q > 0.0 ? sqrt(s / q) : 0.0);
    const double dc2_ds = 1.0 + (s > 0.0 ? sqrt(q / s) : 0.0);
    const double gq = L * dw_dc2 * dc2_dq, gs = L * dw_dc2 * dc2_ds;
    gout[F_RU] = gq * 2.0 * ru * r * r;
    gout[F_RV] = gq * 2.0 * rv * r * r;
    gout[F_RW] = gq * 2.0 * rw * r * r;
    gout[F_RO] = gq * (-2.0 * q * r) + gs * (-b2 * r);
    gout[F_TT] = gs * ph.gamma;
    if (nf == 8) {
        gout[F_BX] = gs * 2.0 * bx * ph.obeta * r;
        gout[F_BY] = gs * 2.0 * by * ph.obeta * r;
        gout[F_BZ] = gs * 2.0 * bz * ph.obeta * r;
    }
}

}  // namespace r3dk

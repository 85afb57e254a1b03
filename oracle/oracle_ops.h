// FP64 CPU restatement of the reference's per-node operators (test
// infrastructure: only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline use it).  Every function works in the reference's SI units and
// keeps the reference's floating-point evaluation order, so that single-level
// runs agree bit-for-bit with the reference built from its own sources.
#pragma once
#include <cmath>

namespace orc {

constexpr int Q = 19;
// D3Q19 direction order of Control.cpp:58-116 (0:+x 1:+y 2:-x 3:-y 4:+z 5:-z
// 6:(+x+z) 7:(+x-z) 8:(+y+z) 9:(+y-z) 10:(-x+z) 11:(-x-z) 12:(-y+z)
// 13:(-y-z) 14:(-x+y) 15:(+x-y) 16:(+x+y) 17:(-x-y) 18:rest)
constexpr int EX[Q] = {1, 0, -1, 0, 0, 0, 1, 1, 0, 0, -1, -1, 0, 0, -1, 1, 1, -1, 0};
constexpr int EY[Q] = {0, 1, 0, -1, 0, 0, 0, 0, 1, 1, 0, 0, -1, -1, 1, -1, 1, -1, 0};
constexpr int EZ[Q] = {0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 0};
// opposite directions (FluidNode.h:43-62)
constexpr int OPP[Q] = {2, 3, 0, 1, 5, 4, 11, 10, 13, 12, 7, 6, 9, 8, 15, 14, 17, 16, 18};

// Lattice constants derived by Control (Control.cpp:51-131) and per level by
// Lattice::initialization (Lattice.cpp:1404).
struct Consts {
    double cs, cs2, c, dt0, spacing, nu, rho0, mach, k1, sigma;
    double xsi[3][Q];
    double w[Q];
    int order;
    bool cubic;
    bool transverse;
    void setup(double speedOfSound, double spacing_, double nu_, double rho0_, double mach_, double k1_,
               double sigma_, int order_, bool cubic_, bool transverse_) {
        cs = speedOfSound;
        cs2 = std::pow(cs, 2.);
        c = cs * std::sqrt(3.);
        spacing = spacing_;
        dt0 = spacing / c;
        nu = nu_;
        rho0 = rho0_;
        mach = mach_;
        k1 = k1_;
        sigma = sigma_;
        order = order_;
        cubic = cubic_;
        transverse = transverse_;
        for (int d = 0; d < Q; ++d) {
            xsi[0][d] = EX[d] == 0 ? 0. : (EX[d] > 0 ? c : -c);
            xsi[1][d] = EY[d] == 0 ? 0. : (EY[d] > 0 ? c : -c);
            xsi[2][d] = EZ[d] == 0 ? 0. : (EZ[d] > 0 ? c : -c);
            w[d] = d < 6 ? 1. / 18. : (d < 18 ? 1. / 36. : 1. / 3.);
        }
    }
    double dt(int level) const { return dt0 / std::pow(2., level); }
    double omega(int level) const {
        double dtl = dt0 / std::pow(2., level);
        return (std::pow(cs, 2.) * dtl) / (nu + 0.5 * std::pow(cs, 2.) * dtl);
    }
};

// Node::calcDensity (Node.cpp:11-30)
inline double density(const Consts& k, const double* f, const double* psi, double dt) {
    double r = 0;
    if (!k.cubic) {
        for (int d = 0; d < Q; ++d) r += f[d];
    } else {
        for (int d = 0; d < Q; ++d) r += f[d] + 0.5 * dt * psi[d];
    }
    return r;
}

// Node::calcVelocity (Node.cpp:85-118)
inline void velocity(const Consts& k, const double* f, const double* psi, double dt, double rho, double* u) {
    u[0] = u[1] = u[2] = 0.;
    if (!k.cubic) {
        for (int d = 0; d < Q; ++d) {
            u[0] += k.xsi[0][d] * f[d];
            u[1] += k.xsi[1][d] * f[d];
            u[2] += k.xsi[2][d] * f[d];
        }
    } else {
        for (int d = 0; d < Q; ++d) {
            u[0] += k.xsi[0][d] * f[d] + 0.5 * dt * k.xsi[0][d] * psi[d];
            u[1] += k.xsi[1][d] * f[d] + 0.5 * dt * k.xsi[1][d] * psi[d];
            u[2] += k.xsi[2][d] * f[d] + 0.5 * dt * k.xsi[2][d] * psi[d];
        }
    }
    u[0] /= rho;
    u[1] /= rho;
    u[2] /= rho;
}

// Plain moments of an array without cubic-Mach terms (calcDensityPreCol /
// calcVelocityPreCol with psiPreCol = 0, Node.cpp:32-51,121-154).
inline void plainMoments(const Consts& k, const double* f, double& rho, double* u) {
    rho = 0;
    for (int d = 0; d < Q; ++d) rho += f[d];
    u[0] = u[1] = u[2] = 0.;
    for (int d = 0; d < Q; ++d) {
        u[0] += k.xsi[0][d] * f[d];
        u[1] += k.xsi[1][d] * f[d];
        u[2] += k.xsi[2][d] * f[d];
    }
    u[0] /= rho;
    u[1] /= rho;
    u[2] /= rho;
}

// Second-order Hermite tensor of direction d (xsi xsi - cs^2 I), as the
// operator functions form it (Node.cpp:795-800, 1781-1788).
struct Herm2 {
    double xx, yy, zz, xy, xz, yz;
};
inline Herm2 herm2(const Consts& k, int d) {
    Herm2 h;
    h.xx = k.xsi[0][d] * k.xsi[0][d] - k.cs2;
    h.yy = k.xsi[1][d] * k.xsi[1][d] - k.cs2;
    h.zz = k.xsi[2][d] * k.xsi[2][d] - k.cs2;
    h.xy = k.xsi[0][d] * k.xsi[1][d];
    h.xz = k.xsi[0][d] * k.xsi[2][d];
    h.yz = k.xsi[1][d] * k.xsi[2][d];
    return h;
}

// The six orthogonal third-order Hermite combinations (Node.cpp:904-917).
struct Herm3 {
    double c[6];  // XXY+YZZ, XXZ+YYZ, XYY+XZZ, YZZ-XXY, YYZ-XXZ, XZZ-XYY
};
inline Herm3 herm3(const Consts& k, const Herm2& h, int d) {
    double hx = k.xsi[0][d], hy = k.xsi[1][d], hz = k.xsi[2][d];
    double xxy = h.xx * hy, xyy = h.yy * hx, xxz = h.xx * hz, xzz = h.zz * hx, yyz = h.yy * hz, yzz = h.zz * hy;
    Herm3 r;
    r.c[0] = xxy + yzz;
    r.c[1] = xxz + yyz;
    r.c[2] = xyy + xzz;
    r.c[3] = yzz - xxy;
    r.c[4] = yyz - xxz;
    r.c[5] = xzz - xyy;
    return r;
}

// Fully orthogonalised fourth-order Hermite combinations (Node.cpp:1082-1094).
inline void orth4(double xxyy, double xxzz, double yyzz, double sxx, double syy, double szz, double* fo) {
    const double oneOver6 = 1. / 6., twoOver7 = 2. / 7., twoOver5 = 2. / 5.;
    double a = xxyy + oneOver6 * szz;
    double b = xxzz + oneOver6 * syy;
    double c = yyzz + oneOver6 * sxx;
    fo[0] = a;
    fo[1] = b + twoOver7 * fo[0];
    fo[2] = c + twoOver7 * fo[0] + twoOver5 * fo[1];
}

// Node::calcEquilibrium{2,3,4}_GHbasis (Node.cpp:739-1132)
inline void equilibrium(const Consts& k, int order, double dens, const double* u, double* eq) {
    const double oneOver2 = 1. / 2., oneOver4 = 1. / 4., oneOver6 = 1. / 6.;
    const double eightOver7 = 8. / 7., fiftysixOver45 = 56. / 45., fortyOver27 = 40. / 27.;
    double cs2 = std::pow(k.cs, 2.), cs4 = std::pow(k.cs, 4.), cs6 = std::pow(k.cs, 6.), cs8 = std::pow(k.cs, 8.);
    double r2 = 1. / cs2, r4 = 1. / cs4, r6 = 1. / cs6, r8 = 1. / cs8;
    double ax = u[0], ay = u[1], az = u[2];
    double axx, ayy, azz, axy, axz, ayz;
    if (order == 2) {
        axx = u[0] * ax; ayy = u[1] * ay; azz = u[2] * az;
        axy = u[0] * ay; axz = u[0] * az; ayz = u[1] * az;
    } else {
        axx = ax * ax; ayy = ay * ay; azz = az * az;
        axy = ax * ay; axz = ax * az; ayz = ay * az;
    }
    double a3[6] = {0, 0, 0, 0, 0, 0}, a4[3] = {0, 0, 0};
    if (order >= 3) {
        double xxy = ay * axx, xyy = ax * ayy, xxz = az * axx, xzz = ax * azz, yyz = az * ayy, yzz = ay * azz;
        a3[0] = xxy + yzz; a3[1] = xxz + yyz; a3[2] = xyy + xzz;
        a3[3] = yzz - xxy; a3[4] = yyz - xxz; a3[5] = xzz - xyy;
        if (order == 4) orth4(ay * xxy, az * xxz, ay * yzz, axx, ayy, azz, a4);
    }
    for (int d = 0; d < Q; ++d) {
        Herm2 h = herm2(k, d);
        double hx = k.xsi[0][d], hy = k.xsi[1][d], hz = k.xsi[2][d];
        double s = 1. * 1. + r2 * (hx * ax + hy * ay + hz * az) +
                   oneOver2 * r4 * (h.xx * axx + h.yy * ayy + h.zz * azz + h.xy * axy * 2. + h.xz * axz * 2. + h.yz * ayz * 2.);
        if (order >= 3) {
            Herm3 t = herm3(k, h, d);
            s = s + oneOver6 * r6 * (t.c[0] * a3[0] * 3. + t.c[1] * a3[1] * 3. + t.c[2] * a3[2] * 3. + t.c[3] * a3[3] +
                                     t.c[4] * a3[4] + t.c[5] * a3[5]);
            if (order == 4) {
                double h4[3];
                orth4(h.xx * h.yy, h.xx * h.zz, h.yy * h.zz, h.xx, h.yy, h.zz, h4);
                s = s + oneOver4 * r8 * (eightOver7 * h4[0] * a4[0] + fiftysixOver45 * h4[1] * a4[1] + fortyOver27 * h4[2] * a4[2]);
            }
        }
        eq[d] = dens * k.w[d] * s;
    }
}

// Node::calcPi1Tensor (Node.cpp:2493-2558): P = {xx, yy, zz, xy, xz, yz}
inline void pi1(const Consts& k, const double* f, const double* eq, const double* psi, double dt, double* P) {
    for (int a = 0; a < 6; ++a) P[a] = 0.;
    for (int d = 0; d < Q; ++d) {
        double hxx = std::pow(k.xsi[0][d], 2.) - k.cs2, hyy = std::pow(k.xsi[1][d], 2.) - k.cs2,
               hzz = std::pow(k.xsi[2][d], 2.) - k.cs2;
        double hxy = k.xsi[0][d] * k.xsi[1][d], hxz = k.xsi[0][d] * k.xsi[2][d], hyz = k.xsi[1][d] * k.xsi[2][d];
        double g = k.cubic ? (f[d] - eq[d] + 0.5 * dt * psi[d]) : (f[d] - eq[d]);
        P[0] += hxx * g;
        P[1] += hyy * g;
        P[2] += hzz * g;
        P[3] += hxy * g;
        P[4] += hxz * g;
        P[5] += hyz * g;
    }
}

// Recursive off-equilibrium of Node::calcRRoffEquilibrium{2,3,4}_GHbasis
// (Node.cpp:1136-1427) and the hybrid version of calcHRRoffEquilibrium*
// (Node.cpp:1430-1747): a = second-order coefficients {xx,yy,zz,xy,xz,yz}.
inline void recursiveNeq(const Consts& k, int order, const double* a, const double* u, double* neq) {
    const double oneOver2 = 1. / 2., oneOver4 = 1. / 4., oneOver6 = 1. / 6.;
    const double eightOver7 = 8. / 7., fiftysixOver45 = 56. / 45., fortyOver27 = 40. / 27.;
    double cs4 = std::pow(k.cs, 4.), cs6 = std::pow(k.cs, 6.), cs8 = std::pow(k.cs, 8.);
    double r4 = 1. / cs4, r6 = 1. / cs6, r8 = 1. / cs8;
    double Pxx = a[0], Pyy = a[1], Pzz = a[2], Pxy = a[3], Pxz = a[4], Pyz = a[5];
    double a3[6] = {0, 0, 0, 0, 0, 0}, a4[3] = {0, 0, 0};
    if (order >= 3) {
        double xxy = 2. * u[0] * Pxy + u[1] * Pxx;
        double xyy = 2. * u[1] * Pxy + u[0] * Pyy;
        double xxz = 2. * u[0] * Pxz + u[2] * Pxx;
        double xzz = 2. * u[2] * Pxz + u[0] * Pzz;
        double yyz = 2. * u[1] * Pyz + u[2] * Pyy;
        double yzz = 2. * u[2] * Pyz + u[1] * Pzz;
        a3[0] = xxy + yzz; a3[1] = xxz + yyz; a3[2] = xyy + xzz;
        a3[3] = yzz - xxy; a3[4] = yyz - xxz; a3[5] = xzz - xyy;
        if (order == 4) {
            double xxyy = u[1] * u[1] * Pxx + u[0] * u[0] * Pyy + 4. * u[0] * u[1] * Pxy;
            double xxzz = u[2] * u[2] * Pxx + u[0] * u[0] * Pzz + 4. * u[0] * u[2] * Pxz;
            double yyzz = u[1] * u[1] * Pzz + u[2] * u[2] * Pyy + 4. * u[1] * u[2] * Pyz;
            orth4(xxyy, xxzz, yyzz, Pxx, Pyy, Pzz, a4);
        }
    }
    for (int d = 0; d < Q; ++d) {
        Herm2 h = herm2(k, d);
        double s = oneOver2 * r4 * (h.xx * Pxx + h.yy * Pyy + h.zz * Pzz + h.xy * Pxy * 2. + h.xz * Pxz * 2. + h.yz * Pyz * 2.);
        if (order >= 3) {
            Herm3 t = herm3(k, h, d);
            s = s + oneOver6 * r6 * (t.c[0] * a3[0] * 3. + t.c[1] * a3[1] * 3. + t.c[2] * a3[2] * 3. + t.c[3] * a3[3] +
                                     t.c[4] * a3[4] + t.c[5] * a3[5]);
            if (order == 4) {
                double h4[3];
                orth4(h.xx * h.yy, h.xx * h.zz, h.yy * h.zz, h.xx, h.yy, h.zz, h4);
                s = s + oneOver4 * r8 * (eightOver7 * h4[0] * a4[0] + fiftysixOver45 * h4[1] * a4[1] + fortyOver27 * h4[2] * a4[2]);
            }
        }
        neq[d] = k.w[d] * s;
    }
}

// Central-difference strain rate and cubic-Mach correction from the six
// axis neighbours' (rho, u) (Node.cpp:1750-1889); nb[dir] for dir 0..5 =
// +x,+y,-x,-y,+z,-z neighbour, dist[dir] its distance.  S = {xx,yy,zz,xy,xz,yz}.
inline void strainAndPsi(const Consts& k, const double nbRho[6], const double nbU[6][3], const double dist[6],
                         double* S, double* psi) {
    double cs2 = std::pow(k.cs, 2.);
    double rec_cs4 = 1. / (cs2 * cs2);
    double XXX[6], XXY[6], XXZ[6], XYY[6], YYY[6], YYZ[6], XZZ[6], YZZ[6], ZZZ[6], XYZ[6];
    for (int n = 0; n < 6; ++n) {
        double r = nbRho[n];
        const double* v = nbU[n];
        XXX[n] = r * v[0] * v[0] * v[0];
        XXY[n] = 0.5 * r * v[1] * v[2] * v[2];
        XXZ[n] = 0.5 * r * v[2] * v[1] * v[1];
        XYY[n] = 0.5 * r * v[0] * v[2] * v[2];
        YYY[n] = r * v[1] * v[1] * v[1];
        YYZ[n] = 0.5 * r * v[2] * v[0] * v[0];
        XZZ[n] = 0.5 * r * v[0] * v[1] * v[1];
        YZZ[n] = 0.5 * r * v[1] * v[0] * v[0];
        ZZZ[n] = r * v[2] * v[2] * v[2];
        XYZ[n] = r * v[0] * v[1] * v[2];
    }
    double dx = dist[0] + dist[2], dy = dist[1] + dist[3], dz = dist[4] + dist[5];
    double XXX_dx = (XXX[0] - XXX[2]) / dx, XYY_dx = (XYY[0] - XYY[2]) / dx, XZZ_dx = (XZZ[0] - XZZ[2]) / dx;
    double XXY_dx = (XXY[0] - XXY[2]) / dx, XXZ_dx = (XXZ[0] - XXZ[2]) / dx, XYZ_dx = (XYZ[0] - XYZ[2]) / dx;
    double XXY_dy = (XXY[1] - XXY[3]) / dy, YYY_dy = (YYY[1] - YYY[3]) / dy, YZZ_dy = (YZZ[1] - YZZ[3]) / dy;
    double XYY_dy = (XYY[1] - XYY[3]) / dy, XYZ_dy = (XYZ[1] - XYZ[3]) / dy, YYZ_dy = (YYZ[1] - YYZ[3]) / dy;
    double XXZ_dz = (XXZ[4] - XXZ[5]) / dz, YYZ_dz = (YYZ[4] - YYZ[5]) / dz, ZZZ_dz = (ZZZ[4] - ZZZ[5]) / dz;
    double XYZ_dz = (XYZ[4] - XYZ[5]) / dz, XZZ_dz = (XZZ[4] - XZZ[5]) / dz, YZZ_dz = (YZZ[4] - YZZ[5]) / dz;
    for (int d = 0; d < Q; ++d) {
        double hxx = std::pow(k.xsi[0][d], 2.) - cs2, hyy = std::pow(k.xsi[1][d], 2.) - cs2,
               hzz = std::pow(k.xsi[2][d], 2.) - cs2;
        double hxy = k.xsi[0][d] * k.xsi[1][d], hxz = k.xsi[0][d] * k.xsi[2][d], hyz = k.xsi[1][d] * k.xsi[2][d];
        psi[d] = 0.5 * k.w[d] * rec_cs4 *
                 (hxx * (XXX_dx + XXY_dy + XXZ_dz) + hyy * (XYY_dx + YYY_dy + YYZ_dz) + hzz * (XZZ_dx + YZZ_dy + ZZZ_dz) +
                  hxy * (XXY_dx + XYY_dy + XYZ_dz) * 2. + hxz * (XXZ_dx + XYZ_dy + XZZ_dz) * 2. +
                  hyz * (XYZ_dx + YYZ_dy + YZZ_dz) * 2.);
    }
    S[0] = (nbU[0][0] - nbU[2][0]) / dx;
    S[1] = (nbU[1][1] - nbU[3][1]) / dy;
    S[2] = (nbU[4][2] - nbU[5][2]) / dz;
    S[3] = 0.5 * ((nbU[0][1] - nbU[2][1]) / dx + (nbU[1][0] - nbU[3][0]) / dy);
    S[4] = 0.5 * ((nbU[0][2] - nbU[2][2]) / dx + (nbU[4][0] - nbU[5][0]) / dz);
    S[5] = 0.5 * ((nbU[1][2] - nbU[3][2]) / dy + (nbU[4][1] - nbU[5][1]) / dz);
}

// Node::LODIpressureCalcVelocity (Node.cpp:447-504), in the boundary-normal
// frame: index 0 is the normal component.
inline void lodiIntegrate(const Consts& k, double dt, double domainLength, double& density, double densB,
                          double densGrad, const double* veloGrad, const double* veloB, double* velocity, bool negNormal,
                          const double* densGradT, const double veloGradT[2][3]) {
    double speedOfSound = k.cs;
    double speedOfSoundSq = std::pow(speedOfSound, 2.);
    double csDivL = speedOfSound / domainLength;
    double Ma = k.mach;
    double MaSq = Ma * Ma;
    double K1 = k.k1;
    double K2 = Ma;
    double densityOutlet = k.rho0;
    double L1, L5, T1, T5;
    double Texact = 0.;
    T1 = -(speedOfSoundSq * (densB * (veloGradT[0][1] + veloGradT[1][2]) + veloB[1] * densGradT[0] + veloB[2] * densGradT[1]) -
           densB * speedOfSound * (veloB[1] * veloGradT[0][0] + veloB[2] * veloGradT[1][0]));
    T5 = -(speedOfSoundSq * (densB * (veloGradT[0][1] + veloGradT[1][2]) + veloB[1] * densGradT[0] + veloB[2] * densGradT[1]) +
           densB * speedOfSound * (veloB[1] * veloGradT[0][0] + veloB[2] * veloGradT[1][0]));
    if (negNormal) {
        L5 = K1 * (1 - MaSq) * csDivL * speedOfSoundSq * (densB - densityOutlet) - K2 * (T5 - Texact) + T5;
        L1 = (veloB[0] - speedOfSound) * speedOfSound * (speedOfSound * densGrad - densB * veloGrad[0]);
    } else {
        L1 = K1 * (1 - MaSq) * csDivL * speedOfSoundSq * (densB - densityOutlet) - K2 * (T1 - Texact) + T1;
        L5 = (veloB[0] + speedOfSound) * speedOfSound * (speedOfSound * densGrad + densB * veloGrad[0]);
    }
    double L3 = veloB[0] * veloGrad[1];
    double L4 = veloB[0] * veloGrad[2];
    double T3 = -(veloB[1] * veloGradT[0][1] + veloB[2] * veloGradT[1][1]) - (speedOfSoundSq / densB) * densGradT[0];
    double T4 = -(veloB[1] * veloGradT[0][2] + veloB[2] * veloGradT[1][2]) - (speedOfSoundSq / densB) * densGradT[1];
    density = densB - dt / (2. * speedOfSoundSq) * (L5 + L1) + dt / (2. * speedOfSoundSq) * (T5 + T1);
    velocity[0] = veloB[0] - dt / (2. * densB * speedOfSound) * (L5 - L1) + dt / (2. * densB * speedOfSound) * (T5 - T1);
    velocity[1] = veloB[1] - dt * L3 + dt * T3;
    velocity[2] = veloB[2] - dt * L4 + dt * T4;
}

}  // namespace orc

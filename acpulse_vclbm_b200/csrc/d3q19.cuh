// D3Q19 lattice and the per-node collision operators of the acPulse_vcLBM hot
// path, written for registers: everything is in lattice units (velocities
// divided by the molecular velocity c = sqrt(3) cs, time in level steps), and
// populations are handled as deviations g_i = f_i - w_i * shift, where shift
// is the reference density for the deviation storage forms and 0 for the
// plain FP64 form.  Every direction loop is unrolled so the Hermite tensors of
// each direction become compile-time constants.
//
// Reference operators restated here (Node.cpp): calcEquilibrium{2,3,4}_GHbasis
// 739-1132, calcPi1Tensor 2493-2558, calcRRoffEquilibrium{2,3,4} 1136-1427,
// calcHRRoffEquilibrium{2,3,4} 1430-1747, the strain-rate / cubic-Mach
// correction 1750-1889, collideSRT/RR/HRR 511-736, collideMRT_GSbasis
// 2798-2835 and collideMRT_RMbasis 2565-2605.  The SI formulas of the
// reference map to lattice units exactly except for the orthogonalisation of
// the fourth-order Hermite terms, which adds a second-order tensor with the
// dimensional factor 1/6 (Node.cpp:1087-1089); in lattice units that factor
// becomes kappa = 1 / (6 c^2), carried as a per-case constant.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>

#include <type_traits>
#include <utility>

namespace acp {

constexpr int Q = 19;
// direction order of Control.cpp:58-116
__host__ __device__ constexpr int ex(int q) {
    return q == 0 || q == 6 || q == 7 || q == 15 || q == 16 ? 1 : (q == 2 || q == 10 || q == 11 || q == 14 || q == 17 ? -1 : 0);
}
__host__ __device__ constexpr int ey(int q) {
    return q == 1 || q == 8 || q == 9 || q == 14 || q == 16 ? 1 : (q == 3 || q == 12 || q == 13 || q == 15 || q == 17 ? -1 : 0);
}
__host__ __device__ constexpr int ez(int q) {
    return q == 4 || q == 6 || q == 8 || q == 10 || q == 12 ? 1 : (q == 5 || q == 7 || q == 9 || q == 11 || q == 13 ? -1 : 0);
}
__host__ __device__ constexpr double wq(int q) { return q < 6 ? 1.0 / 18.0 : (q < 18 ? 1.0 / 36.0 : 1.0 / 3.0); }

// correctly rounded reciprocal (the same value as 1 / x under IEEE division)
__device__ __forceinline__ float rcpRN(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double rcpRN(double x) { return __drcp_rn(x); }

// operator ids (enum acp_op)
enum { OP_SRT = 0, OP_MRT_GS = 1, OP_MRT_RM = 2, OP_RR = 3, OP_HRR = 4 };

// second-order Hermite tensor components (lattice): e_a e_b - delta_ab / 3
template <typename R>
__host__ __device__ constexpr R h2xx(int q) { return R(ex(q) * ex(q)) - R(1) / R(3); }
template <typename R>
__host__ __device__ constexpr R h2yy(int q) { return R(ey(q) * ey(q)) - R(1) / R(3); }
template <typename R>
__host__ __device__ constexpr R h2zz(int q) { return R(ez(q) * ez(q)) - R(1) / R(3); }

// s += c * x for a coefficient c that is a constant once the direction loops
// are unrolled; zero coefficients drop the term.  Sums start from -0, the
// additive identity of IEEE arithmetic, so the first term is not added to a
// zero: leaving the zero terms out changes no result, while 0 * x cannot be
// folded away by the compiler (x may be infinite or NaN).
template <typename R>
__device__ __forceinline__ void acc(R& s, R c, R x) {
    if (c != R(0)) s += c * x;
}

// H2 : A for a symmetric tensor A = {xx, yy, zz, xy, xz, yz}
template <typename R>
__device__ __forceinline__ R h2dot(int q, const R* A) {
    R d = R(-0.0), o = R(-0.0);
    acc(d, h2xx<R>(q), A[0]);
    acc(d, h2yy<R>(q), A[1]);
    acc(d, h2zz<R>(q), A[2]);
    acc(o, R(ex(q) * ey(q)), A[3]);
    acc(o, R(ex(q) * ez(q)), A[4]);
    acc(o, R(ey(q) * ez(q)), A[5]);
    return d + R(2) * o;
}

// sum of the six orthogonal third-order Hermite terms, weighted as the
// reference weights them (x3 for the symmetric combinations, x1 for the
// antisymmetric ones, Node.cpp:942-947):  a = {xxy+yzz, xxz+yyz, xyy+xzz,
// yzz-xxy, yyz-xxz, xzz-xyy}
template <typename R>
__device__ __forceinline__ R h3dot(int q, const R* a) {
    const R hx = R(ex(q)), hy = R(ey(q)), hz = R(ez(q));
    const R xxy = h2xx<R>(q) * hy, xyy = h2yy<R>(q) * hx, xxz = h2xx<R>(q) * hz;
    const R xzz = h2zz<R>(q) * hx, yyz = h2yy<R>(q) * hz, yzz = h2zz<R>(q) * hy;
    R sym = R(-0.0);
    acc(sym, xxy + yzz, a[0]);
    acc(sym, xxz + yyz, a[1]);
    acc(sym, xyy + xzz, a[2]);
    R t = R(3) * sym;
    acc(t, yzz - xxy, a[3]);
    acc(t, yyz - xxz, a[4]);
    acc(t, xzz - xyy, a[5]);
    return t;
}

// e_q . v
template <typename R>
__device__ __forceinline__ R edot(int q, const R* v) {
    R t = R(-0.0);
    acc(t, R(ex(q)), v[0]);
    acc(t, R(ey(q)), v[1]);
    acc(t, R(ez(q)), v[2]);
    return t;
}

// fully orthogonalised fourth-order combination (Node.cpp:1082-1094, 1130):
// orth(p, s) with p = {xxyy, xxzz, yyzz} products and s = {xx, yy, zz}
template <typename R>
__device__ __forceinline__ void orth4(R pxxyy, R pxxzz, R pyyzz, R sxx, R syy, R szz, R kappa, R* fo) {
    fo[0] = pxxyy + kappa * szz;
    fo[1] = pxxzz + kappa * syy + R(2.0 / 7.0) * fo[0];
    fo[2] = pyyzz + kappa * sxx + R(2.0 / 7.0) * fo[0] + R(2.0 / 5.0) * fo[1];
}
template <typename R>
__device__ __forceinline__ R h4dot(int q, const R* a4, R kappa) {
    R h[3];
    orth4<R>(h2xx<R>(q) * h2yy<R>(q), h2xx<R>(q) * h2zz<R>(q), h2yy<R>(q) * h2zz<R>(q), h2xx<R>(q), h2yy<R>(q),
             h2zz<R>(q), kappa, h);
    R t = R(-0.0);
    acc(t, R(8.0 / 7.0) * h[0], a4[0]);
    acc(t, R(56.0 / 45.0) * h[1], a4[1]);
    acc(t, R(40.0 / 27.0) * h[2], a4[2]);
    return t;
}

// Velocity coefficients of the Hermite equilibrium up to `ORDER`.
template <typename R, int ORDER>
struct EqCoef {
    R u[3];
    R uu[6];  // xx yy zz xy xz yz
    R a3[6];
    R a4[3];
    __device__ __forceinline__ void set(const R* v, R kappa) {
        u[0] = v[0]; u[1] = v[1]; u[2] = v[2];
        uu[0] = v[0] * v[0]; uu[1] = v[1] * v[1]; uu[2] = v[2] * v[2];
        uu[3] = v[0] * v[1]; uu[4] = v[0] * v[2]; uu[5] = v[1] * v[2];
        if (ORDER >= 3) {
            const R xxy = v[1] * uu[0], xyy = v[0] * uu[1], xxz = v[2] * uu[0];
            const R xzz = v[0] * uu[2], yyz = v[2] * uu[1], yzz = v[1] * uu[2];
            a3[0] = xxy + yzz; a3[1] = xxz + yyz; a3[2] = xyy + xzz;
            a3[3] = yzz - xxy; a3[4] = yyz - xxz; a3[5] = xzz - xyy;
            if (ORDER == 4) orth4<R>(uu[0] * uu[1], uu[0] * uu[2], uu[1] * uu[2], uu[0], uu[1], uu[2], kappa, a4);
        }
    }
    // feq_q / (rho w_q) - 1
    __device__ __forceinline__ R poly(int q, R kappa) const {
        R p = R(3) * edot<R>(q, u) + R(4.5) * h2dot<R>(q, uu);
        if (ORDER >= 3) p += R(4.5) * h3dot<R>(q, a3);
        if (ORDER == 4) p += R(20.25) * h4dot<R>(q, a4, kappa);
        return p;
    }
    // w_q times the even and odd parts below, w_q folded into the constant
    // coefficients: adds to `even` (which carries w_q drho on entry) and `odd`
    __device__ __forceinline__ void weightedTerms(int q, R kappa, R& even, R& odd) const {
        const R w = R(wq(q));
        const R c2 = w * R(4.5), c3 = w * R(4.5);
        acc(odd, w * R(3 * ex(q)), u[0]);
        acc(odd, w * R(3 * ey(q)), u[1]);
        acc(odd, w * R(3 * ez(q)), u[2]);
        acc(even, c2 * h2xx<R>(q), uu[0]);
        acc(even, c2 * h2yy<R>(q), uu[1]);
        acc(even, c2 * h2zz<R>(q), uu[2]);
        acc(even, c2 * R(2 * ex(q) * ey(q)), uu[3]);
        acc(even, c2 * R(2 * ex(q) * ez(q)), uu[4]);
        acc(even, c2 * R(2 * ey(q) * ez(q)), uu[5]);
        if (ORDER >= 3) {
            const R hx = R(ex(q)), hy = R(ey(q)), hz = R(ez(q));
            const R xxy = h2xx<R>(q) * hy, xyy = h2yy<R>(q) * hx, xxz = h2xx<R>(q) * hz;
            const R xzz = h2zz<R>(q) * hx, yyz = h2yy<R>(q) * hz, yzz = h2zz<R>(q) * hy;
            acc(odd, c3 * R(3) * (xxy + yzz), a3[0]);
            acc(odd, c3 * R(3) * (xxz + yyz), a3[1]);
            acc(odd, c3 * R(3) * (xyy + xzz), a3[2]);
            acc(odd, c3 * (yzz - xxy), a3[3]);
            acc(odd, c3 * (yyz - xxz), a3[4]);
            acc(odd, c3 * (xzz - xyy), a3[5]);
        }
        if (ORDER == 4) even += (w * R(20.25)) * h4dot<R>(q, a4, kappa);
    }
    // the same polynomial split into its even (second and fourth order) and
    // odd (first and third order) parts: direction q gives even + odd, its
    // opposite even - odd
    __device__ __forceinline__ void evenOdd(int q, R kappa, R& even, R& odd) const {
        odd = R(3) * edot<R>(q, u);
        if (ORDER >= 3) odd += R(4.5) * h3dot<R>(q, a3);
        even = R(4.5) * h2dot<R>(q, uu);
        if (ORDER == 4) even += R(20.25) * h4dot<R>(q, a4, kappa);
    }
};

// the nine pairs of opposite directions (FluidNode.h:43-62); the rest
// direction 18 is its own opposite
__host__ __device__ constexpr int pairA(int p) { return p == 0 ? 0 : p == 1 ? 1 : p == 2 ? 4 : p == 3 ? 6 : p == 4 ? 7 : p == 5 ? 8 : p == 6 ? 9 : p == 7 ? 14 : 16; }
__host__ __device__ constexpr int pairB(int p) { return p == 0 ? 2 : p == 1 ? 3 : p == 2 ? 5 : p == 3 ? 11 : p == 4 ? 10 : p == 5 ? 13 : p == 6 ? 12 : p == 7 ? 15 : 17; }

// visit (q, value) for every direction of a polynomial given per pair as
// even +- odd: f(q, even + odd), f(opposite, even - odd), then the rest
template <typename R, int ORDER, typename F>
__device__ __forceinline__ void forEachDirection(const EqCoef<R, ORDER>& c, R kappa, F&& f) {
#pragma unroll
    for (int p = 0; p < 9; ++p) {
        R even, odd;
        c.evenOdd(pairA(p), kappa, even, odd);
        f(pairA(p), even + odd);
        f(pairB(p), even - odd);
    }
    f(18, c.poly(18, kappa));
}

// visit (q, w_q (drho + p_q)) for every direction of the polynomial p of the
// coefficients c: per pair the weighted even sum, started from w_q drho, and
// the weighted odd sum give w_q (drho + p) = even + odd and, for the opposite
// direction, even - odd, so no direction needs its own add and multiply
template <typename R, int ORDER, typename F>
__device__ __forceinline__ void forEachWeighted(const EqCoef<R, ORDER>& c, R drho, R kappa, F&& f) {
    const R axis = R(wq(0)) * drho, diag = R(wq(6)) * drho;
#pragma unroll
    for (int p = 0; p < 9; ++p) {
        const int q = pairA(p);
        R even = q < 6 ? axis : diag, odd = R(-0.0);
        c.weightedTerms(q, kappa, even, odd);
        f(q, even + odd);
        f(pairB(p), even - odd);
    }
    R even = R(wq(18)) * drho, odd = R(-0.0);
    c.weightedTerms(18, kappa, even, odd);
    f(18, even);
}

// Recursive off-equilibrium of a second-order coefficient tensor A
// (RR: A = Pi1; HRR: A = hybrid of Pi1 and the finite-difference strain).
template <typename R, int ORDER>
struct NeqCoef {
    R A[6];
    R a3[6];
    R a4[3];
    __device__ __forceinline__ void set(const R* Ain, const R* u, R kappa) {
        for (int c = 0; c < 6; ++c) A[c] = Ain[c];
        if (ORDER >= 3) {
            const R Pxx = A[0], Pyy = A[1], Pzz = A[2], Pxy = A[3], Pxz = A[4], Pyz = A[5];
            const R xxy = R(2) * u[0] * Pxy + u[1] * Pxx;
            const R xyy = R(2) * u[1] * Pxy + u[0] * Pyy;
            const R xxz = R(2) * u[0] * Pxz + u[2] * Pxx;
            const R xzz = R(2) * u[2] * Pxz + u[0] * Pzz;
            const R yyz = R(2) * u[1] * Pyz + u[2] * Pyy;
            const R yzz = R(2) * u[2] * Pyz + u[1] * Pzz;
            a3[0] = xxy + yzz; a3[1] = xxz + yyz; a3[2] = xyy + xzz;
            a3[3] = yzz - xxy; a3[4] = yyz - xxz; a3[5] = xzz - xyy;
            if (ORDER == 4) {
                const R xxyy = u[1] * u[1] * Pxx + u[0] * u[0] * Pyy + R(4) * u[0] * u[1] * Pxy;
                const R xxzz = u[2] * u[2] * Pxx + u[0] * u[0] * Pzz + R(4) * u[0] * u[2] * Pxz;
                const R yyzz = u[1] * u[1] * Pzz + u[2] * u[2] * Pyy + R(4) * u[1] * u[2] * Pyz;
                orth4<R>(xxyy, xxzz, yyzz, Pxx, Pyy, Pzz, kappa, a4);
            }
        }
    }
    // neq_q / w_q
    __device__ __forceinline__ R poly(int q, R kappa) const {
        R p = R(4.5) * h2dot<R>(q, A);
        if (ORDER >= 3) p += R(4.5) * h3dot<R>(q, a3);
        if (ORDER == 4) p += R(20.25) * h4dot<R>(q, a4, kappa);
        return p;
    }
};

// moment rows (integer coefficients) of the two MRT bases, in lattice units
// Gram-Schmidt basis (Node.cpp:2934-3004)
__host__ __device__ constexpr int gsRow(int m, int q) {
    const int x = ex(q), y = ey(q), z = ez(q), e2 = x * x + y * y + z * z;
    const bool axis = e2 == 1;
    switch (m) {
        case 0: return 1;
        case 1: return q == 18 ? -1 : (e2 == 2 ? 1 : 0);
        case 2: return axis ? -2 : 1;
        case 3: return x;
        case 4: return x * (axis ? -2 : 1);
        case 5: return y;
        case 6: return y * (axis ? -2 : 1);
        case 7: return z;
        case 8: return z * (axis ? -2 : 1);
        case 9: return 3 * x * x - e2;
        case 10: return (3 * x * x - e2) * (axis ? -1 : 1);
        case 11: return y * y - z * z;
        case 12: return (y * y - z * z) * (axis ? -1 : 1);
        case 13: return x * y;
        case 14: return y * z;
        case 15: return x * z;
        case 16: return x * (y * y - z * z);
        case 17: return y * (z * z - x * x);
        default: return z * (x * x - y * y);
    }
}
// Inverse of the Gram-Schmidt basis, evaluated by the compiler (Gauss-Jordan
// with partial pivoting on the integer rows above); GsInv<q, m>::v is a
// compile-time constant, so the back transforms skip its zero entries
// (154 of 361) and fold the others into the instructions.
struct Mat19 {
    double a[19][19];
};
constexpr double cabs(double x) { return x < 0 ? -x : x; }
// inverse of the 19 x 19 integer basis row(m, q) by Gauss-Jordan elimination
// with partial pivoting, evaluated by the compiler
constexpr Mat19 basisInverse(int (*row)(int, int)) {
    double m[19][38] = {};
    for (int r = 0; r < 19; ++r)
        for (int c = 0; c < 19; ++c) {
            m[r][c] = row(r, c);
            m[r][19 + c] = r == c ? 1.0 : 0.0;
        }
    for (int c = 0; c < 19; ++c) {
        int p = c;
        for (int r = c + 1; r < 19; ++r)
            if (cabs(m[r][c]) > cabs(m[p][c])) p = r;
        for (int k = 0; k < 38; ++k) {
            const double t = m[p][k];
            m[p][k] = m[c][k];
            m[c][k] = t;
        }
        const double piv = m[c][c];
        for (int k = 0; k < 38; ++k) m[c][k] /= piv;
        for (int r = 0; r < 19; ++r) {
            if (r == c) continue;
            const double f = m[r][c];
            if (f == 0) continue;
            for (int k = 0; k < 38; ++k) m[r][k] -= f * m[c][k];
        }
    }
    Mat19 out = {};
    for (int r = 0; r < 19; ++r)
        for (int c = 0; c < 19; ++c) out.a[r][c] = m[r][19 + c];
    return out;
}
constexpr Mat19 gsInverse() { return basisInverse(gsRow); }
constexpr Mat19 kGsInverse = gsInverse();
template <int q, int m>
struct GsInv {
    static constexpr double v = kGsInverse.a[q][m];
};
__host__ __device__ constexpr bool gsConserved(int m) { return m == 0 || m == 3 || m == 5 || m == 7; }

// raw-moment basis (Node.cpp:2607-2795): 1, x, y, z, |e|^2, x^2-z^2, y^2-z^2,
// xy, xz, yz, x^2 z, x z^2, y^2 z, y z^2, x^2 y, x y^2, x^2 z^2, x^2 y^2, y^2 z^2
__host__ __device__ constexpr int rmRow(int m, int q) {
    const int x = ex(q), y = ey(q), z = ez(q);
    switch (m) {
        case 0: return 1;
        case 1: return x;
        case 2: return y;
        case 3: return z;
        case 4: return x * x + y * y + z * z;
        case 5: return x * x - z * z;
        case 6: return y * y - z * z;
        case 7: return x * y;
        case 8: return x * z;
        case 9: return y * z;
        case 10: return x * x * z;
        case 11: return x * z * z;
        case 12: return y * y * z;
        case 13: return y * z * z;
        case 14: return x * x * y;
        case 15: return x * y * y;
        case 16: return x * x * z * z;
        case 17: return x * x * y * y;
        default: return y * y * z * z;
    }
}
constexpr Mat19 kRmInverse = basisInverse(rmRow);
template <int q, int m>
struct RmInv {
    static constexpr double v = kRmInverse.a[q][m];
};


// sum_m Minv[q][m] * x[m] over the moments (the conserved ones skipped when
// `skipConserved`), zero coefficients dropped at compile time
template <typename R, int q, bool skipConserved, int... m>
__device__ __forceinline__ R gsBackRow(const R* x, std::integer_sequence<int, m...>) {
    R acc = 0;
    ((GsInv<q, m>::v != 0.0 && !(skipConserved && gsConserved(m)) ? (void)(acc += R(GsInv<q, m>::v) * x[m])
                                                                     : (void)0),
     ...);
    return acc;
}
// f(q, back-transformed value) for every direction q
template <typename R, bool skipConserved, typename F, int... q>
__device__ __forceinline__ void gsBackAll(const R* x, F&& f, std::integer_sequence<int, q...>) {
    (f(q, gsBackRow<R, q, skipConserved>(x, std::make_integer_sequence<int, 19>{})), ...);
}

// sum_m Minv[q][m] * x[m] over the moments m in the bit set `mask`, zero
// coefficients dropped at compile time
template <typename R, int q, unsigned mask, int... m>
__device__ __forceinline__ R gsBackRowMasked(const R* x, std::integer_sequence<int, m...>) {
    R acc = R(-0.0);
    ((GsInv<q, m>::v != 0.0 && ((mask >> m) & 1u) ? (void)(acc += R(GsInv<q, m>::v) * x[m]) : (void)0), ...);
    return acc;
}
template <typename R, unsigned mask, typename F, int... q>
__device__ __forceinline__ void gsBackAllMasked(const R* x, F&& f, std::integer_sequence<int, q...>) {
    (f(q, gsBackRowMasked<R, q, mask>(x, std::make_integer_sequence<int, 19>{})), ...);
}

// raw-moment basis rows 5..9: the deviatoric second-order moments relaxed with
// omega (Node.cpp:2720-2733, 2580-2584)
__host__ __device__ constexpr int rmRow2(int m, int q) {
    const int x = ex(q), y = ey(q), z = ez(q);
    switch (m) {
        case 0: return x * x - z * z;
        case 1: return y * y - z * z;
        case 2: return x * y;
        case 3: return x * z;
        default: return y * z;
    }
}

// storage conversion: populations are stored as S and computed as R
template <typename S>
struct Store;
template <>
struct Store<double> {
    __device__ __forceinline__ static double load(const double* p, float) { return *p; }
    __device__ __forceinline__ static void store(double* p, double v, float) { *p = v; }
};
template <>
struct Store<float> {
    __device__ __forceinline__ static float load(const float* p, float) { return *p; }
    __device__ __forceinline__ static void store(float* p, float v, float) { *p = v; }
};
template <>
struct Store<__half> {
    __device__ __forceinline__ static float load(const __half* p, float scale) { return __half2float(*p) * scale; }
    // the scales are powers of two: their correctly rounded reciprocal is
    // exact, so the multiply equals the division v / scale
    __device__ __forceinline__ static void store(__half* p, float v, float scale) {
        *p = __float2half_rn(v * __frcp_rn(scale));
    }
};

}  // namespace acp

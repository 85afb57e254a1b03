// Kernels of one level's step.  Data layout (HBM): populations in
// structure-of-arrays form, g[q][k][j][i] with i fastest, two ping-pong
// arrays per level (the reference's distr_[2][19], Node.h:190); one byte per
// node for the node class; a 32-byte moment record per node only where the
// operator needs the neighbours' pre-collision (rho, u).
//
// One coarse step of a single level (Lattice::timeSteppingX,
// Lattice.cpp:1496-2156) is:
//   k_moments        (HRR, and RR with cubic-Mach) neighbours' pre-collision rho,u
//   k_collide_push   collide every fluid node and push to the 18 neighbours
//                    (FluidNode::transport); boundary nodes push their
//                    uncollided populations inward (BoundaryNode::transport)
//   k_lodi (x faces) LODI on the x faces, which at the corners read edge nodes
//                    of the z faces before those are updated (Lattice.cpp:1582-1596)
//   k_lodi (z, y)    LODI on the remaining faces; no node of this pass reads
//                    another node's new array within the pass
#pragma once
#include "d3q19.cuh"
#include <stdint.h>

namespace acp {

// node classes: 0..26 LODI boundary node of face class
// (fx+1)*9+(fy+1)*3+(fz+1) (13 = none: fluid); 27 + c a coupling node (fine
// C2F target on the box faces of class c, or coarse F2C target with c = 13),
// which collides like fluid but pushes only inside its level; 255 covered by
// the other level
constexpr uint8_t CODE_FLUID = 13;
constexpr uint8_t CODE_IFACE0 = 27;
constexpr uint8_t CODE_DEAD = 255;
__host__ __device__ constexpr bool collides(uint8_t c) { return c == CODE_FLUID || (c >= CODE_IFACE0 && c < CODE_IFACE0 + 27); }

// pushed-direction mask of each node class
__constant__ uint32_t c_pushMask[54];

// host copy of that table.  Without relocatable device code every
// translation unit that includes this header owns its own __constant__
// copy, so each one uploads it (uploadTables is static per unit), once per
// device.  (The MRT bases' inverses are compile-time constants: GsInv, RmInv.)
struct ConstTables {
    uint32_t masks[54];
};
int makeConstTables(ConstTables& t);
static inline int uploadTables(const ConstTables& t) {
    if (cudaMemcpyToSymbol(c_pushMask, t.masks, sizeof t.masks) != cudaSuccess) return -2;
    return 0;
}

// pre-collision moments of a node
template <typename R>
struct MomR {
    R drho, ux, uy, uz;  // deviation density and lattice velocity
};

template <typename S>
struct LevelArgs {
    int nx, ny, nz;
    long long N;
    int Ni;      // N as int: 19 * N < 2^31, so population element indices are 32-bit
    int per[3];  // periodic axes
    const S* A;  // array read this step
    S* B;        // array written this step
    const S* Aq[Q];  // population q's part of A (A + q N): one address operand per load
    S* Bq[Q];        // population q's part of B
    const uint8_t* code;
    double shift;   // w_q * shift is subtracted in storage (0 for the FP64 form)
    double omega;   // collision frequency of the level
    double kappa;   // 1/(6 c^2): fourth-order orthogonalisation constant
    double sigma;   // HRR hybrid parameter
    float hscale[Q];  // FP16 per-population scales (1 otherwise)
    double m4[18];    // sum_q w_q H2_q,ab H4_q,k(kappa), ab in {xx,yy,zz,xy,xz,yz}, k in 0..2
    const int* slot;  // coupling node -> record of its partner strain (null: none kept)
    const double* sg; // partner strain S and cubic-Mach gradient G, [12][nSlots], level lattice units
    int nSlots;
};

__device__ __forceinline__ int wrapc(int c, int n, int per) {
    if (c < 0) return per ? c + n : -1;
    if (c >= n) return per ? c - n : -1;
    return c;
}
// any distance: periodic axes wrap modulo n, others report -1 outside [0, n)
__device__ __forceinline__ int wrapm(int c, int n, int per) {
    if (c >= 0 && c < n) return c;
    return per ? ((c % n) + n) % n : -1;
}

template <typename S>
__device__ __forceinline__ float scaleOf(const LevelArgs<S>& a, int q) {
    return a.hscale[q];
}

// ---------------------------------------------------------------------------
// collision of one fluid node in registers (deviation form).  The
// post-collision populations are handed to `emit(q, value)` as they are
// formed, so the regularised operators never hold the old populations and
// the equilibrium at the same time (the equilibrium is formed twice instead).

// second-order sums {xx, yy, zz, xy, xz, yz} of a node's deviations g:
// sum over the directions with a nonzero component (diagonal) or of the
// signed products (off-diagonal)
template <typename R>
__device__ __forceinline__ void secondSums(const R* g, R* s2) {
    R sxx = R(-0.0), syy = R(-0.0), szz = R(-0.0), sxy = R(-0.0), sxz = R(-0.0), syz = R(-0.0);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        if (ex(q)) sxx += g[q];
        if (ey(q)) syy += g[q];
        if (ez(q)) szz += g[q];
        if (ex(q) * ey(q)) sxy += R(ex(q) * ey(q)) * g[q];
        if (ex(q) * ez(q)) sxz += R(ex(q) * ez(q)) * g[q];
        if (ey(q) * ez(q)) syz += R(ey(q) * ez(q)) * g[q];
    }
    s2[0] = sxx; s2[1] = syy; s2[2] = szz; s2[3] = sxy; s2[4] = sxz; s2[5] = syz;
}

// drho, momentum j and the six second-order sums of a node's 19 deviations,
// summed per pair of opposite directions: g_a + g_b carries the even
// moments (drho, second order), g_a - g_b the odd ones (momentum)
template <typename R>
__device__ __forceinline__ void pairMoments(const R* g, R& drho, R* j, R* s2) {
    R sp[9], dp[9];
#pragma unroll
    for (int p = 0; p < 9; ++p) {
        sp[p] = g[pairA(p)] + g[pairB(p)];
        dp[p] = g[pairA(p)] - g[pairB(p)];
    }
    const R z0 = R(-0.0);  // additive identity: the first term is not added to a zero
    R d = g[18], jx = z0, jy = z0, jz = z0, sxx = z0, syy = z0, szz = z0, sxy = z0, sxz = z0, syz = z0;
#pragma unroll
    for (int p = 0; p < 9; ++p) {
        const int q = pairA(p);
        d += sp[p];
        if (ex(q)) jx += R(ex(q)) * dp[p];
        if (ey(q)) jy += R(ey(q)) * dp[p];
        if (ez(q)) jz += R(ez(q)) * dp[p];
        if (ex(q)) sxx += sp[p];
        if (ey(q)) syy += sp[p];
        if (ez(q)) szz += sp[p];
        if (ex(q) * ey(q)) sxy += R(ex(q) * ey(q)) * sp[p];
        if (ex(q) * ez(q)) sxz += R(ex(q) * ez(q)) * sp[p];
        if (ey(q) * ez(q)) syz += R(ey(q) * ez(q)) * sp[p];
    }
    drho = d;
    j[0] = jx; j[1] = jy; j[2] = jz;
    if (s2) {
        s2[0] = sxx; s2[1] = syy; s2[2] = szz; s2[3] = sxy; s2[4] = sxz; s2[5] = syz;
    }
}

// Regularised collision (RR, Node.cpp:560-650; HRR, Node.cpp:653-736) of one
// node from its moments: drho, lattice velocity u and the second-order sums
// s2 of its deviations.  nb: strain S and cubic-Mach gradient G of the node
// (12 values), or null for a coupling node, whose neighbours are not all on
// its level: there the hybrid operator falls back to the population-based Pi1
// (sigma = 1) and the cubic-Mach correction is dropped.
template <typename R, int OP, int ORDER, bool CUBIC, typename ST, typename Emit>
__device__ __forceinline__ void regularisedEmit(R drho, const R* u, const R* s2, const LevelArgs<ST>& a, const R* nb,
                                                Emit& emit) {
    const R rho = R(a.shift) + drho;
    const R omega = R(a.omega);
    const R kappa = R(a.kappa);
    EqCoef<R, ORDER> ec;
    ec.set(u, kappa);
    R S[6] = {0, 0, 0, 0, 0, 0};
    R G[6] = {0, 0, 0, 0, 0, 0};
    if ((OP == OP_HRR || CUBIC) && nb) {
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            S[c] = nb[c];
            G[c] = nb[6 + c];
        }
    }
    // Pi1 = sum_q H2_q (g_q - geq_q [+ dt/2 psi_q]) (Node.cpp:2493-2558), with
    // the equilibrium and correction parts summed in closed form by the
    // fourth-order isotropy of D3Q19 (sum_q w_q H2_q,ab H2_q,cd =
    // (d_ac d_bd + d_ad d_bc) / 9, odd moments vanish): sum_q H2_q geq_q =
    // rho (u u + 20.25 M a4), M = sum_q w_q H2_q (x) H4_q(kappa) per case
    // (zero unless ORDER == 4), and sum_q H2_q dt/2 psi_q = G / 2.
    R P[6];
    {
        const R sxx = s2[0], syy = s2[1], szz = s2[2], sxy = s2[3], sxz = s2[4], syz = s2[5];
        const R third = drho * R(1.0 / 3.0);  // within an ulp of drho / 3, without a division per node
        P[0] = sxx - third - rho * ec.uu[0];
        P[1] = syy - third - rho * ec.uu[1];
        P[2] = szz - third - rho * ec.uu[2];
        P[3] = sxy - rho * ec.uu[3];
        P[4] = sxz - rho * ec.uu[4];
        P[5] = syz - rho * ec.uu[5];
        if (ORDER == 4) {
#pragma unroll
            for (int c = 0; c < 6; ++c)
                P[c] -= rho * R(20.25) *
                        (R(a.m4[c * 3 + 0]) * ec.a4[0] + R(a.m4[c * 3 + 1]) * ec.a4[1] + R(a.m4[c * 3 + 2]) * ec.a4[2]);
        }
        if (CUBIC) {
#pragma unroll
            for (int c = 0; c < 6; ++c) P[c] += R(0.5) * G[c];
        }
    }
    R A2[6];
    if (OP == OP_HRR) {
        const R sg = nb ? R(a.sigma) : R(1);
        const R fd = (R(1) - sg) * (rho * (R(-2) / (R(3) * omega)));  // the quotient is the same for every node
#pragma unroll
        for (int c = 0; c < 6; ++c) A2[c] = sg * P[c] + fd * S[c];
    } else {
#pragma unroll
        for (int c = 0; c < 6; ++c) A2[c] = P[c];
    }
    NeqCoef<R, ORDER> nc;
    nc.set(A2, u, kappa);
    // post-collision f_q = feq_q + (1 - omega) neq_q [+ dt/2 psi_q]: one
    // Hermite polynomial per direction with the merged coefficients
    // rho * (equilibrium) + (1 - omega) * (recursive non-equilibrium)
    // [+ G / 2 in the second order for the cubic-Mach correction]
    const R om1 = R(1) - omega;
    EqCoef<R, ORDER> mc;
#pragma unroll
    for (int c = 0; c < 3; ++c) mc.u[c] = rho * u[c];
#pragma unroll
    for (int c = 0; c < 6; ++c) mc.uu[c] = rho * ec.uu[c] + om1 * nc.A[c] + (CUBIC ? R(0.5) * G[c] : R(0));
    if (ORDER >= 3) {
#pragma unroll
        for (int c = 0; c < 6; ++c) mc.a3[c] = rho * ec.a3[c] + om1 * nc.a3[c];
    }
    if (ORDER == 4) {
#pragma unroll
        for (int c = 0; c < 3; ++c) mc.a4[c] = rho * ec.a4[c] + om1 * nc.a4[c];
    }
    forEachWeighted<R, ORDER>(mc, drho, kappa, [&](int q, R v) { emit(q, v); });
}

// acc + Minv_RM[q][m] * d[m - 5], the term left out when the coefficient is zero
template <typename R, int q, int m>
__device__ __forceinline__ R rmBack(R acc, const R* d) {
    if constexpr (RmInv<q, m>::v != 0.0) return acc + R(RmInv<q, m>::v) * d[m - 5];
    else return acc;
}
// f(std::integral_constant<int, q>) for q = 0 .. 18
template <typename F, int... q>
__device__ __forceinline__ void forEachQ(F&& f, std::integer_sequence<int, q...>) {
    (f(std::integral_constant<int, q>{}), ...);
}

template <typename R, int OP, int ORDER, bool CUBIC, bool MRTWB>
struct Collider {
    // nb: as for regularisedEmit
    template <typename ST, typename Emit>
    __device__ __forceinline__ static void run(R* g, const LevelArgs<ST>& a, const R* nb, Emit& emit) {
        if ((OP == OP_MRT_GS || OP == OP_MRT_RM) && !MRTWB) {
            // the reference discards the MRT back transform (Node.cpp:2603,2833)
#pragma unroll
            for (int q = 0; q < Q; ++q) emit(q, g[q]);
            return;
        }
        R drho, jj[3];
        pairMoments<R>(g, drho, jj, (R*)nullptr);
        const R jx = jj[0], jy = jj[1], jz = jj[2];
        const R rho = R(a.shift) + drho;
        const R inv = rcpRN(rho);
        R u[3] = {jx * inv, jy * inv, jz * inv};
        const R omega = R(a.omega);
        const R kappa = R(a.kappa);

        if (OP == OP_MRT_GS) {
            // post-collision moments, back-transformed at once: the conserved
            // ones (drho, j), the six viscous ones relaxed at omega towards
            // their equilibria, every other one at its equilibrium, which is
            // zero (Node.cpp:2838-2931).  The moments of the rest state
            // w_q rho0 vanish except the density's, so in the deviation form
            // only moment 0 carries drho instead of rho.
            R mp[Q];
            const R om1 = R(1) - omega;
#pragma unroll
            for (int mm = 0; mm < Q; ++mm) {
                const bool visc = mm == 1 || mm == 9 || mm == 11 || mm == 13 || mm == 14 || mm == 15;
                if (!visc) continue;
                R m = R(-0.0);
#pragma unroll
                for (int q = 0; q < Q; ++q)
                    if (gsRow(mm, q) != 0) m += R(gsRow(mm, q)) * g[q];
                R meq;
                switch (mm) {
                    case 1: meq = (jx * jx + jy * jy + jz * jz) * inv; break;
                    case 9: meq = (R(2) * jx * jx - jy * jy - jz * jz) * inv; break;
                    case 11: meq = (jy * jy - jz * jz) * inv; break;
                    case 13: meq = jx * jy * inv; break;
                    case 14: meq = jy * jz * inv; break;
                    default: meq = jx * jz * inv; break;
                }
                mp[mm] = meq + om1 * (m - meq);
            }
            mp[0] = drho;
            mp[3] = jx;
            mp[5] = jy;
            mp[7] = jz;
            constexpr unsigned kPost = (1u << 0) | (1u << 1) | (1u << 3) | (1u << 5) | (1u << 7) | (1u << 9) |
                                       (1u << 11) | (1u << 13) | (1u << 14) | (1u << 15);
            gsBackAllMasked<R, kPost>(mp, [&](int q, R back) { emit(q, back); }, std::make_integer_sequence<int, Q>{});
            return;
        }

        if (OP == OP_MRT_RM) {
            // extended raw-moment equilibrium (Node.cpp:2627-2645)
            const R u2[3] = {u[0] * u[0], u[1] * u[1], u[2] * u[2]};
            auto geqRM = [&](int q) -> R {
                const int e[3] = {ex(q), ey(q), ez(q)};
                const int nzc = (e[0] != 0) + (e[1] != 0) + (e[2] != 0);
                R p;
                if (nzc == 0) {
                    p = -(u2[0] + u2[1] + u2[2]) + R(3) * (u2[0] * u2[1] + u2[0] * u2[2] + u2[1] * u2[2]);
                } else if (nzc == 1) {
                    const int aa = e[0] ? 0 : (e[1] ? 1 : 2);
                    const int bb = (aa + 1) % 3, cc = (aa + 2) % 3;
                    const R sg = R(e[aa]);
                    p = R(3) * sg * u[aa] + R(3) * (u2[aa] - u2[bb] - u2[cc]) - R(9) * sg * u[aa] * (u2[bb] + u2[cc]) -
                        R(9) * u2[aa] * (u2[bb] + u2[cc]);
                } else {
                    const int aa = e[0] ? 0 : 1;
                    const int bb = e[2] ? 2 : 1;
                    const R sa = R(e[aa]), sb = R(e[bb]);
                    p = R(3) * (sa * u[aa] + sb * u[bb]) + R(3) * (u2[aa] + u2[bb]) + R(9) * sa * sb * u[aa] * u[bb] +
                        R(9) * (sb * u2[aa] * u[bb] + sa * u[aa] * u2[bb]) + R(9) * u2[aa] * u2[bb];
                }
                return R(wq(q)) * (drho + rho * p);
            };
            R d[5] = {0, 0, 0, 0, 0};
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const R gn = g[q] - geqRM(q);
#pragma unroll
                for (int mm = 0; mm < 5; ++mm)
                    if (rmRow2(mm, q) != 0) d[mm] += R(rmRow2(mm, q)) * gn;
            }
            const R om1 = R(1) - omega;
            // back transform of the five relaxed moments (raw-moment basis rows
            // 5..9), its inverse's coefficients compile-time constants
            auto back = [&](auto qc) {
                constexpr int q = decltype(qc)::value;
                R acc = R(-0.0);
                acc = rmBack<R, q, 5>(acc, d);
                acc = rmBack<R, q, 6>(acc, d);
                acc = rmBack<R, q, 7>(acc, d);
                acc = rmBack<R, q, 8>(acc, d);
                acc = rmBack<R, q, 9>(acc, d);
                emit(q, geqRM(q) + om1 * acc);
            };
            forEachQ(back, std::make_integer_sequence<int, Q>{});
            return;
        }

        if (OP == OP_SRT) {
            EqCoef<R, ORDER> ec;
            ec.set(u, kappa);
            forEachDirection<R, ORDER>(ec, kappa, [&](int q, R poly) {
                const R geq = R(wq(q)) * (drho + rho * poly);
                emit(q, g[q] + omega * (geq - g[q]));
            });
            return;
        }

        // RR / HRR: the post-collision state depends on the populations only
        // through drho, u and the six second-order sums
        R s2[6];
        secondSums<R>(g, s2);
        regularisedEmit<R, OP, ORDER, CUBIC>(drho, u, s2, a, nb, emit);
    }
};

// ---------------------------------------------------------------------------
// push of a node's 18 moving populations and the rest population.  Element
// offsets of the neighbours are formed once per thread (wrapped on periodic
// axes); fluid nodes push everywhere, boundary nodes along their class mask.
struct NbOffsets {
    int dx[3], dy[3], dz[3];  // offsets for e = -1, 0, +1 along each axis
};

template <typename S>
__device__ __forceinline__ NbOffsets nbOffsets(const LevelArgs<S>& a, int i, int j, int k) {
    NbOffsets o;
    const int row = a.nx, pl = a.nx * a.ny;
    o.dx[0] = (i == 0) ? (a.nx - 1) : -1;
    o.dx[1] = 0;
    o.dx[2] = (i == a.nx - 1) ? -(a.nx - 1) : 1;
    o.dy[0] = (j == 0) ? (a.ny - 1) * row : -row;
    o.dy[1] = 0;
    o.dy[2] = (j == a.ny - 1) ? -(a.ny - 1) * row : row;
    o.dz[0] = (k == 0) ? (a.nz - 1) * pl : -pl;
    o.dz[1] = 0;
    o.dz[2] = (k == a.nz - 1) ? -(a.nz - 1) * pl : pl;
    return o;
}

// stores population q of node n into its push target (direction q's
// neighbour; the rest population stays), skipping directions off the mask
template <typename S>
struct Pusher {
    const LevelArgs<S>& a;
    int n;
    uint32_t mask;
    NbOffsets o;
    template <typename V>
    __device__ __forceinline__ void operator()(int q, V v) const {
        if (q == 18) {
            Store<S>::store(a.Bq[18] + n, v, scaleOf(a, 18));
        } else if (mask >> q & 1u) {
            const int t = n + o.dx[ex(q) + 1] + o.dy[ey(q) + 1] + o.dz[ez(q) + 1];
            Store<S>::store(a.Bq[q] + t, v, scaleOf(a, q));
        }
    }
};

// collide + push for operators without neighbour data (SRT, RR, MRT): one
// thread per node, x fastest so each direction's loads and stores coalesce
template <typename S, typename R, int OP, int ORDER, bool CUBIC, bool MRTWB>
__device__ __forceinline__ void collidePushBody(const LevelArgs<S>& a, int bx, int by, int bz) {
    const int i = bx * blockDim.x + threadIdx.x;
    const int j = by, k = bz;
    if (i >= a.nx) return;
    const int n = (k * a.ny + j) * a.nx + i;
    const uint8_t code = a.code[n];
    if (code == CODE_DEAD) return;
    R g[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) g[q] = R(Store<S>::load(a.Aq[q] + n, scaleOf(a, q)));
    if (collides(code)) {
        Pusher<S> emit{a, n, c_pushMask[code], nbOffsets(a, i, j, k)};
        Collider<R, OP, ORDER, CUBIC, MRTWB>::run(g, a, (const R*)nullptr, emit);
    } else {
        Pusher<S> emit{a, n, c_pushMask[code], nbOffsets(a, i, j, k)};
#pragma unroll
        for (int q = 0; q < Q; ++q) emit(q, g[q]);
    }
}
template <typename S, typename R, int OP, int ORDER, bool CUBIC, bool MRTWB>
__global__ void __launch_bounds__(128) k_collide_push(LevelArgs<S> a) {
    collidePushBody<S, R, OP, ORDER, CUBIC, MRTWB>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}


// ---------------------------------------------------------------------------
// collide + push for the operators that read the six axis neighbours'
// pre-collision (rho, u): HRR (finite-difference strain rate, Node.cpp:1750-1889)
// and RR with the cubic-Mach correction.  A block owns a TX x TY column of
// nodes and marches through z.  One pass over a plane loads each node's 19
// populations once and forms everything the regularised collision needs:
// drho and u of the tile and of its one-node ring go to shared memory (the
// neighbours' strain stencil), the six second-order sums of the thread's own
// node stay in registers until that plane collides.  The populations are not
// loaded a second time: the post-collision state of RR / HRR depends on them
// only through these ten moments.  Planes of a periodic z axis of at most
// three nodes are all resident at once.
#ifndef ACP_TILE_Y
#define ACP_TILE_Y 8
#endif
constexpr int TX = 32, TY = ACP_TILE_Y;

// drho, jx, jy, jz of a node's deviations
template <typename S, typename R>
__device__ __forceinline__ MomR<R> nodeMoments(const LevelArgs<S>& a, int n) {
    R g[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) g[q] = R(Store<S>::load(a.Aq[q] + n, scaleOf(a, q)));
    R d, jj[3];
    pairMoments<R>(g, d, jj, (R*)nullptr);
    MomR<R> m;
    m.drho = d;
    const R inv = rcpRN(R(a.shift) + d);
    m.ux = jj[0] * inv;
    m.uy = jj[1] * inv;
    m.uz = jj[2] * inv;
    return m;
}

// one plane of the tile: moments of the own node (with its second-order
// sums into s2) and of the one-node ring into `slot`
template <typename S, typename R>
__device__ __forceinline__ void planePass(const LevelArgs<S>& a, MomR<R> (*slot)[TX + 2], int x0, int y0, int z, R* s2) {
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    // own node (on a periodic axis a thread past the end holds the wrapped
    // node, which is the neighbour of the last node of a partial tile)
    {
        const int i = wrapm(x0 + tx, a.nx, a.per[0]), j = wrapm(y0 + ty, a.ny, a.per[1]);
        if (i >= 0 && j >= 0) {
            const int n = (z * a.ny + j) * a.nx + i;
            if (a.code[n] != CODE_DEAD) {
                R g[Q];
#pragma unroll
                for (int q = 0; q < Q; ++q) g[q] = R(Store<S>::load(a.Aq[q] + n, scaleOf(a, q)));
                R d, jj[3];
                pairMoments<R>(g, d, jj, s2);
                MomR<R> m;
                m.drho = d;
                const R inv = rcpRN(R(a.shift) + d);
                m.ux = jj[0] * inv;
                m.uy = jj[1] * inv;
                m.uz = jj[2] * inv;
                slot[ty + 1][tx + 1] = m;
            }
        }
    }
    // one-node ring (axis neighbours only): bottom row, top row, left column, right column
    if (tid < 2 * TX + 2 * TY) {
        int i, j, si, sj;
        if (tid < TX) { i = x0 + tid; j = y0 - 1; si = tid + 1; sj = 0; }
        else if (tid < 2 * TX) { i = x0 + tid - TX; j = y0 + TY; si = tid - TX + 1; sj = TY + 1; }
        else if (tid < 2 * TX + TY) { i = x0 - 1; j = y0 + tid - 2 * TX; si = 0; sj = tid - 2 * TX + 1; }
        else { i = x0 + TX; j = y0 + tid - 2 * TX - TY; si = TX + 1; sj = tid - 2 * TX - TY + 1; }
        i = wrapm(i, a.nx, a.per[0]);
        j = wrapm(j, a.ny, a.per[1]);
        if (i >= 0 && j >= 0) {
            const int n = (z * a.ny + j) * a.nx + i;
            if (a.code[n] != CODE_DEAD) slot[sj][si] = nodeMoments<S, R>(a, n);
        }
    }
}

// strain rate S = {xx,yy,zz,xy,xz,yz} (central differences of the
// neighbours' velocities, Node.cpp:1882-1888) and the cubic-Mach gradient
// G of the Psi terms (Node.cpp:1832-1878), both in lattice units, from the
// six axis neighbours' moments (+x, -x, +y, -y, +z, -z)
// (inv2h: 1 / (2 h) for neighbours h level cells away; 1/2 on the level's own lattice)
template <typename R, bool STRAIN, bool CUBIC>
__device__ __forceinline__ void neighbourTerms(const MomR<R>& mxp, const MomR<R>& mxm, const MomR<R>& myp,
                                               const MomR<R>& mym, const MomR<R>& mzp, const MomR<R>& mzm, R shift,
                                               R* SG, R inv2h = R(0.5)) {
#pragma unroll
    for (int c = 0; c < 12; ++c) SG[c] = 0;
    if (STRAIN) {
        const R half = R(0.5) * inv2h;
        SG[0] = inv2h * (mxp.ux - mxm.ux);
        SG[1] = inv2h * (myp.uy - mym.uy);
        SG[2] = inv2h * (mzp.uz - mzm.uz);
        SG[3] = half * ((mxp.uy - mxm.uy) + (myp.ux - mym.ux));
        SG[4] = half * ((mxp.uz - mxm.uz) + (mzp.ux - mzm.ux));
        SG[5] = half * ((myp.uz - mym.uz) + (mzp.uy - mzm.uy));
    }
    if (CUBIC) {
        auto psiT = [shift](const MomR<R>& m, R* P) {
            const R r = shift + m.drho, x = m.ux, y = m.uy, z = m.uz;
            P[0] = r * x * x * x;           // XXX
            P[1] = R(0.5) * r * y * z * z;  // XXY
            P[2] = R(0.5) * r * z * y * y;  // XXZ
            P[3] = R(0.5) * r * x * z * z;  // XYY
            P[4] = r * y * y * y;           // YYY
            P[5] = R(0.5) * r * z * x * x;  // YYZ
            P[6] = R(0.5) * r * x * y * y;  // XZZ
            P[7] = R(0.5) * r * y * x * x;  // YZZ
            P[8] = r * z * z * z;           // ZZZ
            P[9] = r * x * y * z;           // XYZ
        };
        R* G = SG + 6;
        R Pp[10], Pm[10];
        const R h = inv2h;
        psiT(mxp, Pp); psiT(mxm, Pm);
        G[0] += h * (Pp[0] - Pm[0]); G[1] += h * (Pp[3] - Pm[3]); G[2] += h * (Pp[6] - Pm[6]);
        G[3] += h * (Pp[1] - Pm[1]); G[4] += h * (Pp[2] - Pm[2]); G[5] += h * (Pp[9] - Pm[9]);
        psiT(myp, Pp); psiT(mym, Pm);
        G[0] += h * (Pp[1] - Pm[1]); G[1] += h * (Pp[4] - Pm[4]); G[2] += h * (Pp[7] - Pm[7]);
        G[3] += h * (Pp[3] - Pm[3]); G[4] += h * (Pp[9] - Pm[9]); G[5] += h * (Pp[5] - Pm[5]);
        psiT(mzp, Pp); psiT(mzm, Pm);
        G[0] += h * (Pp[2] - Pm[2]); G[1] += h * (Pp[5] - Pm[5]); G[2] += h * (Pp[8] - Pm[8]);
        G[3] += h * (Pp[9] - Pm[9]); G[4] += h * (Pp[6] - Pm[6]); G[5] += h * (Pp[7] - Pm[7]);
    }
}

// Register cap of the tiled kernel: blocks of 256 threads per SM for FP64 /
// FP32 compute.
#ifndef ACP_TILED_MINB_F64
#define ACP_TILED_MINB_F64 2
#endif
#ifndef ACP_TILED_MINB_F32
#define ACP_TILED_MINB_F32 4
#endif
template <typename R>
struct TiledMinBlocks {
    static constexpr int value = sizeof(R) == 8 ? ACP_TILED_MINB_F64 : ACP_TILED_MINB_F32;
};

// collide + push of node n = (i, j, z) of class `code` from its own moments
// `me`, its six axis neighbours' moments (+x, -x, +y, -y, +z, -z) and its
// second-order sums s2
template <typename S, typename R, int OP, int ORDER, bool CUBIC>
__device__ __forceinline__ void tiledCollide(const LevelArgs<S>& a, int n, int i, int j, int z, uint8_t code,
                                             const MomR<R>& me, const MomR<R>& xp, const MomR<R>& xm,
                                             const MomR<R>& yp, const MomR<R>& ym, const MomR<R>& zp,
                                             const MomR<R>& zm, const R* s2) {
    if (code == CODE_DEAD) return;
    if (collides(code)) {
        const R u[3] = {me.ux, me.uy, me.uz};
        if (code >= CODE_IFACE0) {
            // coupling node: partner strain from the other level when kept, else Pi1 alone
            Pusher<S> emit{a, n, c_pushMask[code], nbOffsets(a, i, j, z)};
            if (a.slot) {
                const int sl = a.slot[n];
                R SG[12];
#pragma unroll
                for (int c = 0; c < 12; ++c) SG[c] = R(a.sg[c * a.nSlots + sl]);
                regularisedEmit<R, OP, ORDER, CUBIC>(me.drho, u, s2, a, SG, emit);
            } else {
                regularisedEmit<R, OP, ORDER, CUBIC>(me.drho, u, s2, a, (const R*)nullptr, emit);
            }
        } else {
            // fluid nodes are interior or on periodic axes: every axis neighbour exists
            R SG[12];
            neighbourTerms<R, OP == OP_HRR, CUBIC>(xp, xm, yp, ym, zp, zm, R(a.shift), SG);
            Pusher<S> emit{a, n, 0x3FFFFu, nbOffsets(a, i, j, z)};
            regularisedEmit<R, OP, ORDER, CUBIC>(me.drho, u, s2, a, SG, emit);
        }
    } else {
        // LODI boundary node: pushes its uncollided populations inward
        Pusher<S> emit{a, n, c_pushMask[code], nbOffsets(a, i, j, z)};
#pragma unroll
        for (int q = 0; q < Q; ++q) emit(q, R(Store<S>::load(a.Aq[q] + n, scaleOf(a, q))));
    }
}

// collide + push of the thread's node of plane z: slots sc / sp / sn hold the
// moments of planes z, z+1, z-1; s2 the node's second-order sums (null: form
// them from the populations again)
template <typename S, typename R, int OP, int ORDER, bool CUBIC>
__device__ __forceinline__ void tiledNode(const LevelArgs<S>& a, MomR<R> (*sm)[TY + 2][TX + 2], int i, int j, int z,
                                          int sc, int sp, int sn, const R* s2own) {
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int n = (z * a.ny + j) * a.nx + i;
    const uint8_t code = a.code[n];
    if (code == CODE_DEAD) return;
    R s2buf[6];
    const R* s2 = s2own;
    if (!s2 && collides(code)) {
        R g[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) g[q] = R(Store<S>::load(a.Aq[q] + n, scaleOf(a, q)));
        secondSums<R>(g, s2buf);
        s2 = s2buf;
    }
    tiledCollide<S, R, OP, ORDER, CUBIC>(a, n, i, j, z, code, sm[sc][ty + 1][tx + 1], sm[sc][ty + 1][tx + 2],
                                         sm[sc][ty + 1][tx], sm[sc][ty + 2][tx + 1], sm[sc][ty][tx + 1],
                                         sm[sp][ty + 1][tx + 1], sm[sn][ty + 1][tx + 1], s2);
}

// plane slots of the tiled kernel: four rolling ones (the pass over plane
// z+2 never overwrites a plane that a slower warp still reads for plane z,
// so one barrier per plane suffices), plus (FP32 compute) two that keep the
// first and last plane of a periodic column resident, so a block that owns a
// whole periodic z column passes over each plane once
template <typename R>
struct TiledSlots {
    static constexpr int value = sizeof(R) == 4 ? 6 : 4;
};

template <typename S, typename R, int OP, int ORDER, bool CUBIC>
__device__ __forceinline__ void tiledBody(const LevelArgs<S>& a, int zChunk, int bx, int by, int bz) {
    __shared__ MomR<R> sm[TiledSlots<R>::value][TY + 2][TX + 2];
    const int x0 = bx * TX, y0 = by * TY;
    const int i = x0 + threadIdx.x, j = y0 + threadIdx.y;
    const bool mine = i < a.nx && j < a.ny;
    if (a.per[2] && a.nz <= 3) {
        // every plane resident: one pass per plane, then the collisions; the
        // second-order sums of all planes stay in registers in the FP32 form,
        // the FP64 form forms them again at the collision (register budget)
        constexpr bool keep = sizeof(R) == 4;
        R s2[3][6];
#pragma unroll
        for (int z = 0; z < 3; ++z)
            if (z < a.nz) planePass<S, R>(a, sm[z], x0, y0, z, s2[z]);
        __syncthreads();
        if (mine) {
#pragma unroll
            for (int z = 0; z < 3; ++z)
                if (z < a.nz)
                    tiledNode<S, R, OP, ORDER, CUBIC>(a, sm, i, j, z, z, wrapm(z + 1, a.nz, 1), wrapm(z - 1, a.nz, 1),
                                                      keep ? s2[z] : (const R*)nullptr);
        }
        return;
    }
    R cur[6], nxt[6];
    if (TiledSlots<R>::value == 6 && a.per[2] && zChunk >= a.nz) {
        // whole periodic column: planes 0 and nz-1 in slots 4 and 5, planes
        // 1..nz-2 rolling through slots p mod 4; the last plane's own sums
        // wait in shared memory
        __shared__ R lastS2[6][TY][TX];
        const int nz = a.nz;
        const int tx = threadIdx.x, ty = threadIdx.y;
        auto slot = [nz](int p) { return p == 0 ? 4 : (p == nz - 1 ? 5 : (p & 3)); };
        planePass<S, R>(a, sm[5], x0, y0, nz - 1, nxt);
#pragma unroll
        for (int c = 0; c < 6; ++c) lastS2[c][ty][tx] = nxt[c];
        planePass<S, R>(a, sm[4], x0, y0, 0, cur);
        for (int z = 0; z < nz; ++z) {
            if (z + 1 <= nz - 2) planePass<S, R>(a, sm[slot(z + 1)], x0, y0, z + 1, nxt);
            __syncthreads();
            if (mine)
                tiledNode<S, R, OP, ORDER, CUBIC>(a, sm, i, j, z, slot(z), slot(z + 1 == nz ? 0 : z + 1),
                                                  slot(z == 0 ? nz - 1 : z - 1), cur);
            if (z + 1 == nz - 1) {
#pragma unroll
                for (int c = 0; c < 6; ++c) cur[c] = lastS2[c][ty][tx];
            } else {
#pragma unroll
                for (int c = 0; c < 6; ++c) cur[c] = nxt[c];
            }
        }
        return;
    }
    const int zBeg = bz * zChunk;
    const int zEnd = min(a.nz, zBeg + zChunk);
    // rolling planes: slot of the unwrapped plane u in [zBeg-1, zEnd] is (u - zBeg + 1) mod 4
    auto key = [&](int u) { return (u - zBeg + 1) & 3; };
    {
        const int zm = wrapc(zBeg - 1, a.nz, a.per[2]);
        if (zm >= 0) planePass<S, R>(a, sm[key(zBeg - 1)], x0, y0, zm, (R*)nullptr);  // ring and moments only
        planePass<S, R>(a, sm[key(zBeg)], x0, y0, zBeg, cur);
    }
    for (int z = zBeg; z < zEnd; ++z) {
        const int zp = wrapc(z + 1, a.nz, a.per[2]);
        // the plane past the chunk's end gives moments only
        if (zp >= 0) planePass<S, R>(a, sm[key(z + 1)], x0, y0, zp, z + 1 < zEnd ? nxt : (R*)nullptr);
        __syncthreads();
        if (mine) tiledNode<S, R, OP, ORDER, CUBIC>(a, sm, i, j, z, key(z), key(z + 1), key(z - 1), cur);
#pragma unroll
        for (int c = 0; c < 6; ++c) cur[c] = nxt[c];
    }
}
template <typename S, typename R, int OP, int ORDER, bool CUBIC>
__global__ void __launch_bounds__(TX * TY, TiledMinBlocks<R>::value) k_collide_push_tiled(LevelArgs<S> a, int zChunk) {
    tiledBody<S, R, OP, ORDER, CUBIC>(a, zChunk, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------------------
// The same collide + push for lattices whose z axis is periodic and at most
// MARCH_MAX_NZ planes deep (the quasi-2D pulse cases): a block holds MARCH_TX
// x-nodes by the whole periodic z column and marches along y.  The moments of
// a row (every x and z of the block) are formed once and roll through four
// shared-memory row slots, so the y neighbours cost no extra loads and the z
// neighbours wrap inside the block; the first and last x lane of the block are
// halo lanes that only form moments (the x neighbours of the block's edge
// nodes), so x tiles advance by MARCH_TX - 2 nodes.  Per collided node the
// loads are 19 x (MARCH_TX / (MARCH_TX - 2)) x (rows + 2) / rows instead of the
// 19 x (1 + ring / tile) of the x-y tile.  Thread (tx, tz) owns the node at x =
// x0 - 1 + tx, z = tz of every row.
#ifndef ACP_MARCH_TX
#define ACP_MARCH_TX 32
#endif
constexpr int MARCH_TX = ACP_MARCH_TX;
constexpr int MARCH_MAX_NZ = 8;
constexpr int MARCH_STEP = MARCH_TX - 2;  // collided x-nodes per block
#ifndef ACP_MARCH_PREFETCH_F64
#define ACP_MARCH_PREFETCH_F64 1
#endif

// dynamic shared memory of a march block: four row slots of nz x MARCH_TX moment records
template <typename R>
constexpr size_t marchSmemBytes(int nz) {
    return sizeof(MomR<R>) * 4 * (size_t)nz * MARCH_TX;
}

template <typename S, typename R, int OP, int ORDER, bool CUBIC>
__device__ __forceinline__ void marchBody(const LevelArgs<S>& a, int yChunk, int bx, int by, MomR<R>* sm) {
    const int tx = threadIdx.x, tz = threadIdx.y, nz = a.nz;
    // slot s, plane z, lane x
    auto at = [&](int s, int z, int x) -> MomR<R>& { return sm[(s * nz + z) * MARCH_TX + x]; };
    const int xu = bx * MARCH_STEP - 1 + tx;  // unwrapped x of the lane
    const int xw = wrapm(xu, a.nx, a.per[0]);
    const bool collider = tx > 0 && tx < MARCH_TX - 1 && xu < a.nx;
    const int yBeg = by * yChunk;
    const int yEnd = min(a.ny, yBeg + yChunk);
    const int zpl = tz + 1 == nz ? 0 : tz + 1, zmi = tz == 0 ? nz - 1 : tz - 1;
    // moments of row y (wrapped) into slot s; the lane's second-order sums into s2
    auto rowPass = [&](int s, int y, R* s2) {
        if (xw < 0) return;
        const int n = (tz * a.ny + y) * a.nx + xw;
        if (a.code[n] == CODE_DEAD) return;
        R g[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) g[q] = R(Store<S>::load(a.Aq[q] + n, scaleOf(a, q)));
        R d, jj[3];
        pairMoments<R>(g, d, jj, s2);
        MomR<R> m;
        m.drho = d;
        const R inv = rcpRN(R(a.shift) + d);
        m.ux = jj[0] * inv;
        m.uy = jj[1] * inv;
        m.uz = jj[2] * inv;
        at(s, tz, tx) = m;
    };
    // Odd chunks march downwards: two neighbouring chunks then reach the row
    // they both load (the one past their common end) at about the same time,
    // so the second load hits L2 instead of DRAM.  Step s visits row
    // rowAt(s); steps -1 and len load the rows beyond the chunk's ends, and
    // the row of step s sits in slot (s + 1) mod 4.
    const int len = yEnd - yBeg;
    const int dir = (by & 1) ? -1 : 1;
    auto rowAt = [&](int st) { return dir > 0 ? yBeg + st : yEnd - 1 - st; };
    auto key = [](int st) { return (st + 1) & 3; };
    R cur[6], nxt[6];
    {
        const int ym = wrapc(rowAt(-1), a.ny, a.per[1]);
        if (ym >= 0) rowPass(key(-1), ym, (R*)nullptr);  // moments only
        rowPass(key(0), rowAt(0), cur);
    }
    for (int st = 0; st < len; ++st) {
        const int y = rowAt(st);
        const int yn = wrapc(rowAt(st + 1), a.ny, a.per[1]);
        // the row past the chunk's end gives moments only
        if (yn >= 0) rowPass(key(st + 1), yn, st + 1 < len ? nxt : (R*)nullptr);
        __syncthreads();
        if (collider) {
            const int n = (tz * a.ny + y) * a.nx + xu;
            const uint8_t code = a.code[n];
            const int sc = key(st);
            const int sp = dir > 0 ? key(st + 1) : key(st - 1);  // row y + 1
            const int sn = dir > 0 ? key(st - 1) : key(st + 1);  // row y - 1
            tiledCollide<S, R, OP, ORDER, CUBIC>(a, n, xu, y, tz, code, at(sc, tz, tx), at(sc, tz, tx + 1),
                                                 at(sc, tz, tx - 1), at(sp, tz, tx), at(sn, tz, tx), at(sc, zpl, tx),
                                                 at(sc, zmi, tx), cur);
        }
#pragma unroll
        for (int c = 0; c < 6; ++c) cur[c] = nxt[c];
    }
}

// The same march with the loads of row y+2 issued before row y collides and
// reduced to moments after it, so their latency hides behind the collision;
// the node classes run one row further ahead (a dead node's populations are
// not loaded).  Row slots as above: during step st the block writes the slot
// of step st+2 while slower threads may still read those of steps st-1..st+1.
template <typename S, typename R, int OP, int ORDER, bool CUBIC>
__device__ __forceinline__ void marchBodyPrefetch(const LevelArgs<S>& a, int yChunk, int bx, int by, MomR<R>* sm) {
    const int tx = threadIdx.x, tz = threadIdx.y, nz = a.nz;
    auto at = [&](int s, int z, int x) -> MomR<R>& { return sm[(s * nz + z) * MARCH_TX + x]; };
    const int xu = bx * MARCH_STEP - 1 + tx;
    const int xw = wrapm(xu, a.nx, a.per[0]);
    const bool collider = tx > 0 && tx < MARCH_TX - 1 && xu < a.nx;
    const int yBeg = by * yChunk;
    const int yEnd = min(a.ny, yBeg + yChunk);
    const int zpl = tz + 1 == nz ? 0 : tz + 1, zmi = tz == 0 ? nz - 1 : tz - 1;
    // steps, rows and slots as in marchBody, every chunk marching upwards:
    // with the prefetch (FP64) alternating directions measured slower, 1237
    // against 1087 us per coarse step on the 1024 x 512 x 3 HRR workload
    const int len = yEnd - yBeg;
    const int dir = 1;
    auto rowAt = [&](int st) { return dir > 0 ? yBeg + st : yEnd - 1 - st; };
    auto key = [](int st) { return (st + 1) & 3; };
    // node index of the lane in the row of step st, or -1 outside a LODI y axis
    auto nodeOf = [&](int st) -> int {
        const int y = wrapc(rowAt(st), a.ny, a.per[1]);
        return (xw < 0 || y < 0) ? -1 : (tz * a.ny + y) * a.nx + xw;
    };
    auto codeOf = [&](int n) -> uint8_t { return n < 0 ? CODE_DEAD : a.code[n]; };
    auto loadRow = [&](int n, uint8_t c, R* g) {
        if (c == CODE_DEAD) return;
#pragma unroll
        for (int q = 0; q < Q; ++q) g[q] = R(Store<S>::load(a.Aq[q] + n, scaleOf(a, q)));
    };
    auto reduceRow = [&](int s, uint8_t c, const R* g, R* s2) {
        if (c == CODE_DEAD) return;
        R d, jj[3];
        pairMoments<R>(g, d, jj, s2);
        MomR<R> m;
        m.drho = d;
        const R inv = rcpRN(R(a.shift) + d);
        m.ux = jj[0] * inv;
        m.uy = jj[1] * inv;
        m.uz = jj[2] * inv;
        at(s, tz, tx) = m;
    };
    R g[Q];
    R s2c[6], s2n[6], s2p[6];
    int nC, nN, nP;
    uint8_t cC, cN, cP, cA;
    {
        const int nM = nodeOf(-1);
        const uint8_t cM = codeOf(nM);
        loadRow(nM, cM, g);
        reduceRow(key(-1), cM, g, s2p);
        nC = nodeOf(0);
        cC = codeOf(nC);
        loadRow(nC, cC, g);
        reduceRow(key(0), cC, g, s2c);
        nN = nodeOf(1);
        cN = codeOf(nN);
        loadRow(nN, cN, g);
        reduceRow(key(1), cN, g, s2n);
        nP = 2 <= len ? nodeOf(2) : -1;
        cP = codeOf(nP);
    }
    __syncthreads();
    for (int st = 0; st < len; ++st) {
        // step st+2 in flight, the class of step st+3 behind it
        loadRow(nP, cP, g);
        const int nA = st + 3 <= len ? nodeOf(st + 3) : -1;
        cA = codeOf(nA);
        if (collider) {
            const int y = rowAt(st);
            const int sc = key(st);
            const int sp = dir > 0 ? key(st + 1) : key(st - 1);  // row y + 1
            const int sn = dir > 0 ? key(st - 1) : key(st + 1);  // row y - 1
            tiledCollide<S, R, OP, ORDER, CUBIC>(a, nC, xu, y, tz, cC, at(sc, tz, tx), at(sc, tz, tx + 1),
                                                 at(sc, tz, tx - 1), at(sp, tz, tx), at(sn, tz, tx), at(sc, zpl, tx),
                                                 at(sc, zmi, tx), s2c);
        }
        reduceRow(key(st + 2), cP, g, s2p);
        __syncthreads();
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            s2c[c] = s2n[c];
            s2n[c] = s2p[c];
        }
        nC = nN;
        cC = cN;
        nN = nP;
        cN = cP;
        nP = nA;
        cP = cA;
    }
}

// Measured on the 1024 x 512 x 3 two-level HRR workload (collide time per
// coarse step): FP64 1087 us with the prefetch against 1093 us without; FP32
// 568 us without it at 64 registers (five blocks of 32 x 6 per SM) against
// 597 us with it at 80 registers (four blocks), the lost block costing more
// than the hidden latency gains.
template <typename R>
struct MarchPrefetch {
    static constexpr bool value = sizeof(R) == 8 && ACP_MARCH_PREFETCH_F64;
};

// cols: x tiles of the launch (blockIdx.x indexes this list), or null for
// every tile (blockIdx.x is the tile)
template <typename S, typename R, int OP, int ORDER, bool CUBIC>
__global__ void __launch_bounds__(MARCH_TX * MARCH_MAX_NZ, TiledMinBlocks<R>::value)
    k_collide_push_march(LevelArgs<S> a, int yChunk, const int* __restrict__ cols) {
    extern __shared__ __align__(16) unsigned char marchSmem[];
    const int bx = cols ? cols[blockIdx.x] : (int)blockIdx.x;
    if (MarchPrefetch<R>::value)
        marchBodyPrefetch<S, R, OP, ORDER, CUBIC>(a, yChunk, bx, blockIdx.y, reinterpret_cast<MomR<R>*>(marchSmem));
    else
        marchBody<S, R, OP, ORDER, CUBIC>(a, yChunk, bx, blockIdx.y, reinterpret_cast<MomR<R>*>(marchSmem));
}

// FP32 compute: the register cap set directly, so that blocks of 32 x 6
// threads fit six to an SM at 56 registers (a launch bound can only express
// caps for the 256-thread maximum block).  FP32 collide time per coarse step
// on the workload above: 528 us at 56 registers, 538 at 64, 555 at 48 (spills).
#ifndef ACP_MARCH_REGS_F32
#define ACP_MARCH_REGS_F32 56
#endif
template <typename S, typename R, int OP, int ORDER, bool CUBIC>
__global__ void __maxnreg__(ACP_MARCH_REGS_F32)
    k_collide_push_march_f32(LevelArgs<S> a, int yChunk, const int* __restrict__ cols) {
    extern __shared__ __align__(16) unsigned char marchSmem[];
    const int bx = cols ? cols[blockIdx.x] : (int)blockIdx.x;
    marchBody<S, R, OP, ORDER, CUBIC>(a, yChunk, bx, blockIdx.y, reinterpret_cast<MomR<R>*>(marchSmem));
}


// ---------------------------------------------------------------------------
// LODI characteristic pressure boundary (Node::LODIpressureOutlet and
// LODIpressureCalcVelocity, Node.cpp:229-504), FP64 in the reference's SI
// units.  One thread per boundary node.
struct BNodeDev {
    long long n, n1, n2, t[4];  // node, normal neighbours, tangent neighbours (-1: none)
    int normalDir;              // 0:-x 1:-y 2:+x 3:+y 4:-z 5:+z
    int transverse;             // face node with transverse terms enabled
};

struct LodiArgs {
    long long N;
    double shift, cs, c, mach, k1, rho0, dt, localSpacing, kappa;
    double domainLength[3];  // NumberOfNodes_axis * coarse spacing (Node.cpp:311,324,333,...)
    int order;
    int* errorFlag;
};

template <typename S>
__device__ __forceinline__ void absMoments(const S* arr, long long N, long long n, double shift, const float* hs,
                                           double c, double& rho, double* uSI) {
    double d = 0, jx = 0, jy = 0, jz = 0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const double g = (double)Store<S>::load(arr + q * N + n, hs[q]);
        d += g;
        if (ex(q)) jx += ex(q) * g;
        if (ey(q)) jy += ey(q) * g;
        if (ez(q)) jz += ez(q) * g;
    }
    rho = shift + d;
    const double cr = c / rho;  // one division for the three components
    uSI[0] = cr * jx;
    uSI[1] = cr * jy;
    uSI[2] = cr * jz;
}

// threads per LODI boundary node: lane m of a node's group forms the moments
// of its stencil member m (0 the node, 1-2 the normal neighbours, 3-6 the
// tangent neighbours), lane 0 then the characteristic update.  Without
// transverse terms (the classical LODI) no node reads its tangents, so the
// three members fit groups of four lanes and a warp serves eight nodes.
constexpr int LODI_TPN = 8;
constexpr int LODI_TPN_CLASSICAL = 4;
__host__ __device__ inline int lodiLanes(int transverse) { return transverse ? LODI_TPN : LODI_TPN_CLASSICAL; }

// tpn: lodiLanes of the case (every node of the launch without transverse
// terms when tpn is LODI_TPN_CLASSICAL)
template <typename S, int ORDER>
__device__ __forceinline__ void lodiBody(const S* __restrict__ A, S* B, const BNodeDev* __restrict__ nodes, int count,
                                         const LodiArgs& p, const LevelArgs<S>& la, int bx, int tpn) {
    const int tg = bx * blockDim.x + threadIdx.x;
    const int t = tpn == LODI_TPN ? tg >> 3 : tg >> 2, lane = tg & (tpn - 1);
    const bool valid = t < count;
    const float* hs = la.hscale;
    // every lane of the warp reaches the shuffles below
    BNodeDev b;
    double mr = 0, mu[3] = {0, 0, 0};
    if (valid) {
        b = nodes[t];
        long long src = -1;
        const S* arr = A;
        if (lane == 0) src = b.n;
        else if (lane == 1) { src = b.n1; arr = (const S*)B; }
        else if (lane == 2) { src = b.n2; arr = (const S*)B; }
        else if (lane < 7 && b.transverse) src = b.t[lane - 3];
        if (src >= 0) absMoments(arr, p.N, src, p.shift, hs, p.c, mr, mu);
    }
    double sr[7], su[7][3];
#pragma unroll
    for (int m = 0; m < 7; ++m) {
        sr[m] = __shfl_sync(0xffffffffu, mr, m, tpn);  // members past the group: read only with transverse terms
#pragma unroll
        for (int c = 0; c < 3; ++c) su[m][c] = __shfl_sync(0xffffffffu, mu[c], m, tpn);
    }
    if (!valid || lane != 0) return;
    const double densB = sr[0], dN = sr[1], d2N = sr[2];
    const double* veloB = su[0];
    const double* vN = su[1];
    const double* v2N = su[2];
    // reciprocals formed once: the gradients' 1 / (2 dx), 1 / density, and
    // the level constants dt / (2 cs^2), dt / (2 cs), 1 / c
    const double ls = p.localSpacing;
    const double inv2ls = 1. / (2. * ls);
    double dG = -(4. * dN - d2N - 3. * densB) * inv2ls;
    double vG[3];
    for (int c = 0; c < 3; ++c) vG[c] = -(4. * vN[c] - v2N[c] - 3. * veloB[c]) * inv2ls;
    double dGT[2] = {0, 0}, vGT[2][3] = {{0, 0, 0}, {0, 0, 0}};
    if (b.transverse) {
        const double* dT = sr + 3;
        const double(*vT)[3] = su + 3;
        dGT[0] = (dT[0] - dT[1]) * inv2ls;
        dGT[1] = (dT[2] - dT[3]) * inv2ls;
        for (int c = 0; c < 3; ++c) {
            vGT[0][c] = (vT[0][c] - vT[1][c]) * inv2ls;
            vGT[1][c] = (vT[2][c] - vT[3][c]) * inv2ls;
        }
    }
    const int nd = b.normalDir;
    int perm[3];
    double L0;
    if (nd == 0 || nd == 2) { perm[0] = 0; perm[1] = 1; perm[2] = 2; L0 = p.domainLength[0]; }
    else if (nd == 1 || nd == 3) { perm[0] = 1; perm[1] = 0; perm[2] = 2; L0 = p.domainLength[1]; }
    else { perm[0] = 2; perm[1] = 0; perm[2] = 1; L0 = p.domainLength[2]; }
    const bool neg = nd == 0 || nd == 1 || nd == 4;
    if (neg) {
        dG = -dG;
        for (int c = 0; c < 3; ++c) vG[c] = -vG[c];
    }
    double sVG[3], sVB[3], sT[2][3];
    for (int c = 0; c < 3; ++c) {
        sVG[c] = vG[perm[c]];
        sVB[c] = veloB[perm[c]];
        sT[0][c] = vGT[0][perm[c]];
        sT[1][c] = vGT[1][perm[c]];
    }
    // LODIpressureCalcVelocity in the boundary frame
    const double cs = p.cs, cs2 = cs * cs, csDivL = cs / L0, MaSq = p.mach * p.mach, K1 = p.k1, K2 = p.mach;
    const double T1 = -(cs2 * (densB * (sT[0][1] + sT[1][2]) + sVB[1] * dGT[0] + sVB[2] * dGT[1]) -
                        densB * cs * (sVB[1] * sT[0][0] + sVB[2] * sT[1][0]));
    const double T5 = -(cs2 * (densB * (sT[0][1] + sT[1][2]) + sVB[1] * dGT[0] + sVB[2] * dGT[1]) +
                        densB * cs * (sVB[1] * sT[0][0] + sVB[2] * sT[1][0]));
    double L1, L5;
    if (neg) {
        L5 = K1 * (1 - MaSq) * csDivL * cs2 * (densB - p.rho0) - K2 * T5 + T5;
        L1 = (sVB[0] - cs) * cs * (cs * dG - densB * sVG[0]);
    } else {
        L1 = K1 * (1 - MaSq) * csDivL * cs2 * (densB - p.rho0) - K2 * T1 + T1;
        L5 = (sVB[0] + cs) * cs * (cs * dG + densB * sVG[0]);
    }
    const double L3 = sVB[0] * sVG[1], L4 = sVB[0] * sVG[2];
    const double invDens = 1. / densB;
    const double T3 = -(sVB[1] * sT[0][1] + sVB[2] * sT[1][1]) - (cs2 * invDens) * dGT[0];
    const double T4 = -(sVB[1] * sT[0][2] + sVB[2] * sT[1][2]) - (cs2 * invDens) * dGT[1];
    const double dt = p.dt;
    const double kr = dt / (2. * cs2), kv = dt / (2. * cs) * invDens;
    const double rho = densB - kr * (L5 + L1) + kr * (T5 + T1);
    double v[3];
    v[0] = sVB[0] - kv * (L5 - L1) + kv * (T5 - T1);
    v[1] = sVB[1] - dt * L3 + dt * T3;
    v[2] = sVB[2] - dt * L4 + dt * T4;
    double u[3];
    const double invc = 1. / p.c;
    for (int c = 0; c < 3; ++c) u[perm[c]] = v[c] * invc;
    if (!(rho > 0.5 * p.rho0 && rho < 1.5 * p.rho0)) atomicOr(p.errorFlag, 1);
    EqCoef<double, ORDER> ec;
    ec.set(u, p.kappa);
    const double drho = rho - p.shift;
    forEachDirection<double, ORDER>(ec, p.kappa, [&](int q, double poly) {
        const double geq = wq(q) * (drho + rho * poly);
        Store<S>::store(B + q * p.N + b.n, (decltype(Store<S>::load(B, 1.f)))geq, hs[q]);
    });
}
template <typename S, int ORDER>
__global__ void k_lodi(const S* __restrict__ A, S* B, const BNodeDev* __restrict__ nodes, int count, LodiArgs p,
                       LevelArgs<S> la, int tpn) {
    lodiBody<S, ORDER>(A, B, nodes, count, p, la, blockIdx.x, tpn);
}


// ---------------------------------------------------------------------------
// initial condition (Lattice::initialization, Lattice.cpp:1397-1493): f is
// the equilibrium at rest of the pulse density, in both arrays
struct InitArgs {
    int ic;                 // enum acp_ic
    double spacingLevel;    // level spacing [m]
    double halfDomain[2];   // Domain-Size-X/2, Domain-Size-Y/2
    double rho0;
    double eps, b, cell;    // Gaussian: amplitude, half-width (coarse cells), level cell size in coarse cells
    double center[3];
    int dims3;
    int off[3];             // level index of the box origin (coarse-cell units * 2^level)
};

template <typename S>
__global__ void k_init(LevelArgs<S> a, InitArgs ia) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= a.nx) return;
    const long long n = ((long long)k * a.ny + j) * a.nx + i;
    const int gi = i + ia.off[0], gj = j + ia.off[1], gk = k + ia.off[2];
    double rho;
    if (ia.ic == 0) {
        const double Rc = 0.06, A = 0.01, xCenter = -8. * Rc;
        const double xNode = gi * ia.spacingLevel - ia.halfDomain[0];
        const double yNode = gj * ia.spacingLevel - ia.halfDomain[1];
        const double xRel = xNode - xCenter;
        rho = ia.rho0 * (1 + A * exp(-(xRel * xRel + yNode * yNode) / (2 * Rc * Rc)));
    } else {
        const double dx = gi * ia.cell - ia.center[0], dy = gj * ia.cell - ia.center[1];
        const double dz = ia.dims3 ? gk * ia.cell - ia.center[2] : 0.0;
        rho = ia.rho0 * (1 + ia.eps * exp(-0.69314718055994530942 * (dx * dx + dy * dy + dz * dz) / (ia.b * ia.b)));
    }
    const double drho = rho - a.shift;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const double g = wq(q) * drho;
        Store<S>::store(a.B + q * a.N + n, (decltype(Store<S>::load(a.B, 1.f)))g, a.hscale[q]);
        Store<S>::store(const_cast<S*>(a.A) + q * a.N + n, (decltype(Store<S>::load(a.B, 1.f)))g, a.hscale[q]);
    }
}

// storage <-> absolute FP64 populations
template <typename S>
__global__ void k_to_f64(const S* __restrict__ src, double* dst, long long N, double shift, LevelArgs<S> la) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N * Q) return;
    const int q = (int)(t / N);
    dst[t] = (double)Store<S>::load(src + t, la.hscale[q]) + wq(q) * shift;
}
// one macroscopic field per node from the stored populations, in FP64 with
// the arithmetic and summation order of the host read-back (absolute
// populations as k_to_f64 forms them, summed over q = 0..18): field 0 rho,
// 1-3 velocity (c * j / rho), 4 pressure (rho * cs^2)
template <typename S>
__global__ void k_field(const S* __restrict__ src, double* dst, long long N, double shift, double c, double cs,
                        int field, LevelArgs<S> la) {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    double rho = 0, jx = 0, jy = 0, jz = 0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const double v = (double)Store<S>::load(src + q * N + n, la.hscale[q]) + wq(q) * shift;
        rho += v;
        jx += ex(q) * v;
        jy += ey(q) * v;
        jz += ez(q) * v;
    }
    double r;
    switch (field) {
        case 0: r = rho; break;
        case 1: r = c * jx / rho; break;
        case 2: r = c * jy / rho; break;
        case 3: r = c * jz / rho; break;
        default: r = rho * cs * cs; break;
    }
    dst[n] = r;
}
// density and the three velocity components of every node, out[4][N], with
// the arithmetic of k_field
template <typename S>
__global__ void k_fields4(const S* __restrict__ src, double* out, long long N, double shift, double c,
                          LevelArgs<S> la) {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    double rho = 0, jx = 0, jy = 0, jz = 0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const double v = (double)Store<S>::load(src + q * N + n, la.hscale[q]) + wq(q) * shift;
        rho += v;
        jx += ex(q) * v;
        jy += ey(q) * v;
        jz += ez(q) * v;
    }
    out[n] = rho;
    out[N + n] = c * jx / rho;
    out[2 * N + n] = c * jy / rho;
    out[3 * N + n] = c * jz / rho;
}
// storage -> absolute FP64 populations of the node window [begin, begin+count)
template <typename S>
__global__ void k_to_f64_window(const S* __restrict__ src, double* dst, long long N, long long begin, int count,
                                double shift, LevelArgs<S> la) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)count * Q) return;
    const int q = (int)(t / count);
    const long long m = t - (long long)q * count;
    dst[t] = (double)Store<S>::load(src + (long long)q * N + begin + m, la.hscale[q]) + wq(q) * shift;
}
template <typename S>
__global__ void k_from_f64(const double* __restrict__ src, S* dst0, S* dst1, long long N, double shift, LevelArgs<S> la) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N * Q) return;
    const int q = (int)(t / N);
    const double g = src[t] - wq(q) * shift;
    Store<S>::store(dst0 + t, (decltype(Store<S>::load(dst0, 1.f)))g, la.hscale[q]);
    Store<S>::store(dst1 + t, (decltype(Store<S>::load(dst0, 1.f)))g, la.hscale[q]);
}

// pressure probes: p = rho cs^2 (Node::calcPressure, Node.cpp:64-83) at each
// probe after the step, appended to an FP64 series; a probe reads the coarse
// array (level 0) or the fine one (level 1)
template <typename S>
__global__ void k_probes(const S* __restrict__ coarse, long long Nc, const S* __restrict__ fine, long long Nf,
                         LevelArgs<S> la, const long long* nodes, const int* levels, int count, double shift,
                         double cs2, double* series, int* counter, int capacity) {
    const int t = threadIdx.x;
    const int s = *counter;
    for (int m = t; m < count; m += blockDim.x) {
        const S* arr = levels[m] ? fine : coarse;
        const long long N = levels[m] ? Nf : Nc;
        double d = 0;
#pragma unroll
        for (int q = 0; q < Q; ++q) d += (double)Store<S>::load(arr + q * N + nodes[m], la.hscale[q]);
        if (s < capacity) series[(long long)s * count + m] = (shift + d) * cs2;
    }
    __syncthreads();
    if (t == 0) *counter = s + 1;
}

// ---------------------------------------------------------------------------
// grid coupling (box layout, overlap of one coarse cell, 2:1 sub-cycling).
// The reference declares these operators (GridCoupling.h:28-45) but its
// GridCoupling.cpp is absent; they follow the call order of
// Lattice::nestedTimeStepping* (Lattice.cpp:4354-5771): C2F at t+1/2 with
// linear time interpolation of the coarse state and at t+1, spatial
// interpolation of the fine coupling nodes between coarse positions, F2C of
// the coarse nodes one cell inside the fine box, non-equilibrium rescaled by
// the ratio of (relaxation time x time step) of the levels.
struct C2FDev {
    int n;           // fine node
    int src;         // coarse node (coincident) or -1
    int st[4];       // interpolation stencil (fine nodes) or -1
    float w[4];
    uint32_t mask;   // populations replaced
};
struct F2CDev {
    int n;           // coarse node
    int partner;     // coincident fine node
    uint32_t mask;
    int cube[27];    // 3x3x3 fine neighbourhood, x fastest
};
// sources of a fine coincident node's partner strain: the regular coarse axis
// neighbours of its coarse node (+x +y -x -y +z -z), or where that neighbour
// is a coupling node, the regular fine node two fine cells away
struct C2FNbDev {
    int c[6];  // coarse neighbour or -1
    int f[6];  // fine node (used when c < 0)
};
struct CouplingArgs {
    long long Nc, Nf;  // node counts of the coarse and fine arrays
    double shiftC;     // storage shift (both levels)
    double kappa;
    double alphaC2F, alphaF2C;  // population-based rescaling factors
    double omegaC, omegaF;
    int mrtStyle;      // Scaling-Style MRTSTYLE
    int filter;        // F2C-Filter
    // partner strain of the coupling nodes (HRR, RR with cubic-Mach; STD)
    int partner;
    int nSlotsF, nSlotsC;
    const C2FNbDev* nb;  // per coincident node
    void* preNb;         // [24][coincident] drho, u of the coarse neighbours at t (compute type)
    double* sgF;         // [12][nSlotsF] fine coupling nodes, in C2F list order
    double* sgC;         // [12][nSlotsC] coarse coupling nodes, in F2C list order
    const int* slotF;    // fine node -> slot
};

// threads per node of the coincident C2F kernel (blocks of 128 threads)
__host__ __device__ inline int coincidentThreadsPerNode(const CouplingArgs& c) { return c.partner ? 8 : 1; }

// drho and lattice velocity of node n of an arbitrary array of a level
template <typename S, typename R>
__device__ __forceinline__ MomR<R> nodeMomentsAt(const S* arr, long long N, const LevelArgs<S>& la, long long n) {
    R g[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) g[q] = R(Store<S>::load(arr + (long long)q * N + n, la.hscale[q]));
    R d, jj[3];
    pairMoments<R>(g, d, jj, (R*)nullptr);
    MomR<R> m;
    m.drho = d;
    const R inv = rcpRN(R(la.shift) + d);
    m.ux = jj[0] * inv;
    m.uy = jj[1] * inv;
    m.uz = jj[2] * inv;
    return m;
}

// equilibrium split of one node's populations (deviation form)
template <typename R, int ORDER>
__device__ __forceinline__ void eqSplit(const R* g, R shift, R kappa, R* geq) {
    R drho, jj[3];
    pairMoments<R>(g, drho, jj, (R*)nullptr);
    const R rho = shift + drho;
    const R inv = rcpRN(rho);
    R u[3] = {jj[0] * inv, jj[1] * inv, jj[2] * inv};
    EqCoef<R, ORDER> ec;
    ec.set(u, kappa);
#pragma unroll
    for (int q = 0; q < Q; ++q) geq[q] = R(wq(q)) * (drho + rho * ec.poly(q, kappa));
}

// rescale a non-equilibrium part between levels: population based, or per
// moment of the Gram-Schmidt basis (factor of the viscous moments from the
// collision frequencies, 1/2 or 2 for the others)
template <typename R>
__device__ __forceinline__ void rescaleNeq(R* neq, const CouplingArgs& c, bool toFine) {
    if (!c.mrtStyle) {
        const R a = R(toFine ? c.alphaC2F : c.alphaF2C);
#pragma unroll
        for (int q = 0; q < Q; ++q) neq[q] *= a;
        return;
    }
    R m[Q];
#pragma unroll
    for (int mm = 0; mm < Q; ++mm) {
        R s = 0;
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (gsRow(mm, q) != 0) s += R(gsRow(mm, q)) * neq[q];
        const bool visc = mm == 1 || mm == 9 || mm == 11 || mm == 13 || mm == 14 || mm == 15;
        const R f = visc ? R(toFine ? c.alphaC2F : c.alphaF2C) : R(toFine ? 0.5 : 2.0);
        m[mm] = f * s;
    }
    gsBackAll<R, false>(m, [&](int q, R back) { neq[q] = back; }, std::make_integer_sequence<int, Q>{});
}

// populations of the coincident coupling sources before the coarse step
template <typename S, typename R>
__device__ __forceinline__ void c2fSaveBody(const S* __restrict__ Ac, const C2FDev* __restrict__ nodes, int count, R* pre,
                                            const LevelArgs<S>& la, const CouplingArgs& c, int bx) {
    // one thread per node, or (partner strain kept) eight: the first saves the
    // populations, the first six one coarse neighbour's moments each
    const int tpn = coincidentThreadsPerNode(c);
    const int tg = bx * blockDim.x + threadIdx.x;
    const int t = tg / tpn, sub = tg - t * tpn;
    if (t >= count) return;
    if (sub == 0) {
        const int src = nodes[t].src;
#pragma unroll
        for (int q = 0; q < Q; ++q)
            pre[(long long)q * count + t] = R(Store<S>::load(Ac + (long long)q * la.N + src, la.hscale[q]));
    }
    if (c.partner && sub < 6) {
        R* pn = (R*)c.preNb;
        const int m = c.nb[t].c[sub];
        if (m < 0) return;
        const MomR<R> mo = nodeMomentsAt<S, R>(Ac, la.N, la, m);
        pn[(long long)(sub * 4 + 0) * count + t] = mo.drho;
        pn[(long long)(sub * 4 + 1) * count + t] = mo.ux;
        pn[(long long)(sub * 4 + 2) * count + t] = mo.uy;
        pn[(long long)(sub * 4 + 3) * count + t] = mo.uz;
    }
}
template <typename S, typename R>
__global__ void k_c2f_save(const S* __restrict__ Ac, const C2FDev* __restrict__ nodes, int count, R* pre,
                           LevelArgs<S> la, CouplingArgs c) {
    c2fSaveBody<S, R>(Ac, nodes, count, pre, la, c, blockIdx.x);
}


// C2F on the fine nodes at coarse positions: coarse state at (1-th)*t + th*(t+1)
template <typename S, typename R, int ORDER>
__device__ __forceinline__ void c2fCoincidentBody(const S* __restrict__ Bc, S* Ff, const C2FDev* __restrict__ nodes, int count,
                                                  const R* __restrict__ pre, R th, const CouplingArgs& c,
                                                  const LevelArgs<S>& la, int bx) {
    // one thread per node, or (partner strain kept) eight: the first forms the
    // populations, the first six each gather one stencil neighbour's moments
    const int tpn = coincidentThreadsPerNode(c);
    const int tg = bx * blockDim.x + threadIdx.x;
    const int t = tg / tpn, sub = tg - t * tpn;
    const bool valid = t < count;
    if (valid && sub == 0) {
        const C2FDev nd = nodes[t];
        R g[Q], geq[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const R now = R(Store<S>::load(Bc + (long long)q * c.Nc + nd.src, la.hscale[q]));
            g[q] = (R(1) - th) * pre[(long long)q * count + t] + th * now;
        }
        eqSplit<R, ORDER>(g, R(c.shiftC), R(c.kappa), geq);
#pragma unroll
        for (int q = 0; q < Q; ++q) g[q] -= geq[q];
        rescaleNeq<R>(g, c, true);
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (nd.mask >> q & 1u) Store<S>::store(Ff + (long long)q * c.Nf + nd.n, geq[q] + g[q], la.hscale[q]);
    }
    if (!c.partner) return;  // uniform over the launch
    // partner strain on the coarse stencil (two fine cells) at the fine state's time
    // (Node.cpp:2114-2380): regular coarse neighbours blended between t and t+1,
    // the other neighbours from regular fine nodes at the current fine time
    __shared__ R mom[128 / 8][6][4];
    const int local = threadIdx.x / 8;
    if (valid && sub < 6) {
        const R* pn = (const R*)c.preNb;
        const int cn = c.nb[t].c[sub];
        MomR<R> m;
        if (cn >= 0) {
            const MomR<R> now = nodeMomentsAt<S, R>(Bc, c.Nc, la, cn);
            m.drho = (R(1) - th) * pn[(long long)(sub * 4 + 0) * count + t] + th * now.drho;
            m.ux = (R(1) - th) * pn[(long long)(sub * 4 + 1) * count + t] + th * now.ux;
            m.uy = (R(1) - th) * pn[(long long)(sub * 4 + 2) * count + t] + th * now.uy;
            m.uz = (R(1) - th) * pn[(long long)(sub * 4 + 3) * count + t] + th * now.uz;
        } else {
            m = nodeMomentsAt<S, R>((const S*)Ff, c.Nf, la, c.nb[t].f[sub]);
        }
        mom[local][sub][0] = m.drho;
        mom[local][sub][1] = m.ux;
        mom[local][sub][2] = m.uy;
        mom[local][sub][3] = m.uz;
    }
    __syncthreads();
    if (valid && sub == 0) {
        MomR<R> m[6];
        for (int d = 0; d < 6; ++d) {
            m[d].drho = mom[local][d][0];
            m[d].ux = mom[local][d][1];
            m[d].uy = mom[local][d][2];
            m[d].uz = mom[local][d][3];
        }
        R SG[12];
        neighbourTerms<R, true, true>(m[0], m[2], m[1], m[3], m[4], m[5], R(c.shiftC), SG, R(0.25));
#pragma unroll
        for (int k = 0; k < 12; ++k) c.sgF[(long long)k * c.nSlotsF + t] = double(SG[k]);
    }
}
template <typename S, typename R, int ORDER>
__global__ void k_c2f_coincident(const S* __restrict__ Bc, S* Ff, const C2FDev* __restrict__ nodes, int count,
                                 const R* __restrict__ pre, R th, CouplingArgs c, LevelArgs<S> la) {
    c2fCoincidentBody<S, R, ORDER>(Bc, Ff, nodes, count, pre, th, c, la, blockIdx.x);
}


// C2F on the other fine coupling nodes: interpolation along the face from
// the nodes written before (mid nodes from coincident ones, centre nodes from
// mid nodes); one thread per (node, population)
template <typename S, typename R>
__device__ __forceinline__ void c2fInterpBody(S* Ff, const C2FDev* __restrict__ nodes, int count, const CouplingArgs& c,
                                              const LevelArgs<S>& la, int bx) {
    const long long t = (long long)bx * blockDim.x + threadIdx.x;
    if (t >= (long long)count * (Q + (c.partner ? 12 : 0))) return;
    const int q = (int)(t / count);
    const int m = (int)(t - (long long)q * count);
    const C2FDev& nd = nodes[m];
    if (q >= Q) {
        // partner strain of the hanging node, interpolated like its populations
        const int k = q - Q;
        double acc = 0;
        for (int s = 0; s < 4; ++s)
            if (nd.st[s] >= 0) acc += double(nd.w[s]) * c.sgF[(long long)k * c.nSlotsF + c.slotF[nd.st[s]]];
        c.sgF[(long long)k * c.nSlotsF + c.slotF[nd.n]] = acc;
        return;
    }
    if (!(nd.mask >> q & 1u)) return;
    R acc = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (nd.st[k] >= 0) acc += R(nd.w[k]) * R(Store<S>::load(Ff + (long long)q * c.Nf + nd.st[k], la.hscale[q]));
    Store<S>::store(Ff + (long long)q * c.Nf + nd.n, acc, la.hscale[q]);
}
template <typename S, typename R>
__global__ void k_c2f_interp(S* Ff, const C2FDev* __restrict__ nodes, int count, CouplingArgs c, LevelArgs<S> la) {
    c2fInterpBody<S, R>(Ff, nodes, count, c, la, blockIdx.x);
}


// F2C on the coarse nodes one cell inside the fine box: one warp per coarse
// node, lane m < 27 forms the weighted non-equilibrium of fine neighbour m
template <typename S, typename R, int ORDER>
__device__ __forceinline__ void f2cBody(const S* __restrict__ Ff, S* Bc, const F2CDev* __restrict__ nodes, int count,
                                        const CouplingArgs& c, const LevelArgs<S>& la, int bx) {
    const int warp = (int)(((long long)bx * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (warp >= count) return;  // uniform per warp
    const F2CDev& nd = nodes[warp];
    R neq[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) neq[q] = 0;
    const bool filtered = c.filter != 0;
    const int member = filtered ? lane : (lane == 0 ? 13 : -1);  // NOFI: the coincident node only
    if (member >= 0 && member < 27) {
        const int dx = member % 3, dy = (member / 3) % 3, dz = member / 9;
        const R wgt = !filtered ? R(1)
                                : (c.filter == 1 ? R(1.0 / 27.0)
                                                 : R((dx == 1 ? 0.5 : 0.25) * (dy == 1 ? 0.5 : 0.25) * (dz == 1 ? 0.5 : 0.25)));
        R h[Q], heq[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) h[q] = R(Store<S>::load(Ff + (long long)q * c.Nf + nd.cube[member], la.hscale[q]));
        eqSplit<R, ORDER>(h, R(c.shiftC), R(c.kappa), heq);
#pragma unroll
        for (int q = 0; q < Q; ++q) neq[q] = wgt * (h[q] - heq[q]);
    }
#pragma unroll
    for (int q = 0; q < Q; ++q)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) neq[q] += __shfl_down_sync(0xffffffffu, neq[q], off);
    // partner strain from the fine partner's axis neighbours at t+1 (half a
    // coarse cell away, Node.cpp:2383-2490): lane d < 6 gathers neighbour d
    // (+x +y -x -y +z -z of the cube), lane 0 assembles
    R SG[12];
    if (c.partner) {
        const int face[6] = {14, 16, 12, 10, 22, 4};
        MomR<R> mine = {R(0), R(0), R(0), R(0)};
        if (lane < 6) mine = nodeMomentsAt<S, R>(Ff, c.Nf, la, nd.cube[face[lane]]);
        MomR<R> m[6];
#pragma unroll
        for (int d = 0; d < 6; ++d) {
            m[d].drho = __shfl_sync(0xffffffffu, mine.drho, d);
            m[d].ux = __shfl_sync(0xffffffffu, mine.ux, d);
            m[d].uy = __shfl_sync(0xffffffffu, mine.uy, d);
            m[d].uz = __shfl_sync(0xffffffffu, mine.uz, d);
        }
        neighbourTerms<R, true, true>(m[0], m[2], m[1], m[3], m[4], m[5], R(c.shiftC), SG, R(1));
    }
    if (lane != 0) return;
    if (c.partner) {
#pragma unroll
        for (int k = 0; k < 12; ++k) c.sgC[(long long)k * c.nSlotsC + warp] = double(SG[k]);
    }
    R g[Q], geq[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) g[q] = R(Store<S>::load(Ff + (long long)q * c.Nf + nd.partner, la.hscale[q]));
    eqSplit<R, ORDER>(g, R(c.shiftC), R(c.kappa), geq);
    rescaleNeq<R>(neq, c, false);
#pragma unroll
    for (int q = 0; q < Q; ++q)
        if (nd.mask >> q & 1u) Store<S>::store(Bc + (long long)q * c.Nc + nd.n, geq[q] + neq[q], la.hscale[q]);
}
template <typename S, typename R, int ORDER>
__global__ void k_f2c(const S* __restrict__ Ff, S* Bc, const F2CDev* __restrict__ nodes, int count, CouplingArgs c,
                      LevelArgs<S> la) {
    f2cBody<S, R, ORDER>(Ff, Bc, nodes, count, c, la, blockIdx.x);
}


// ---------------------------------------------------------------------------
// direct coupling (Coupling-Approach DC1 / DC2, Overlap 0).  The reference
// declares interpolTimeDirectCoupling / directCoupling (GridCoupling.h:28-29,
// called at Lattice.cpp:14018-14058 and 14699-14739) without bodies.  Here the
// coarse nodes on the box faces and the fine nodes at coarse positions there
// are the same points; every population is taken from the level on which its
// source node is live, the equilibrium is that of this merged set, and each
// level's replaced populations get it plus the other level's rescaled
// non-equilibrium: population-wise (DC1) or regularised onto the
// second-order Hermite tensor (DC2).
struct DCDev {
    int nf, nc;                 // the shared node on the fine and the coarse level
    uint32_t vc, vf;            // populations whose source node is live on the coarse / fine level
    uint32_t rc, rf;            // populations replaced on the coarse / fine level
    int plane[9];               // 3x3 fine stencil in the interface plane (-1: none)
    uint32_t pv[9];             // populations valid at each stencil node (source node live)
    double w[9];                // F2C filter weights over the stencil
};

// 4.5 w_q H2_q : Pi, Pi = sum_q H2_q neq_q (lattice units)
template <typename R>
__device__ __forceinline__ void regulariseNeq(const R* neq, R* out) {
    R P[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        P[0] += h2xx<R>(q) * neq[q];
        P[1] += h2yy<R>(q) * neq[q];
        P[2] += h2zz<R>(q) * neq[q];
        P[3] += R(ex(q) * ey(q)) * neq[q];
        P[4] += R(ex(q) * ez(q)) * neq[q];
        P[5] += R(ey(q) * ez(q)) * neq[q];
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) out[q] = R(4.5) * R(wq(q)) * h2dot<R>(q, P);
}

// threads per shared node of the direct coupling: lane q gathers population
// q (coarse state, time blend, the fine plane filter over up to nine
// members), shuffles give every lane all nineteen, and lane q stores q
constexpr int DC_TPN = 32;

// th < 1: the fine side at t+1/2 (coarse state blended in time with the
// saved pre-step state); th == 1: both sides at t+1.  One warp per shared node.
template <typename S, typename R, int ORDER>
__device__ __forceinline__ void dcCoupleBody(S* Bc, S* Ff, const DCDev* __restrict__ nodes, int count, const R* __restrict__ pre,
                                             R th, int dc2, const CouplingArgs& c, const LevelArgs<S>& la, int bx) {
    const int tg = bx * blockDim.x + threadIdx.x;
    const int t = tg / DC_TPN, lane = tg % DC_TPN;
    if (t >= count) return;  // whole warps: DC_TPN is the warp size
    const DCDev& nd = nodes[t];
    const bool full = th == R(1);
    // populations whose source node is live on neither level keep the coarse
    // state of t (complete after the previous exchange): no population that a
    // level leaves unwritten is read.  At t+1 the fine populations are
    // filtered over the interface plane, gathered before this warp overwrites
    // the shared node's fine populations (the stencil's other nodes are
    // hanging fine nodes, which this kernel does not write), each population's
    // weights renormalised over the stencil nodes where it is valid.
    R xm = 0, fm = 0;
    if (lane < Q) {
        const int q = lane;
        if (nd.vc >> q & 1u) {
            const R cq = R(Store<S>::load(Bc + (long long)q * c.Nc + nd.nc, la.hscale[q]));
            xm = (R(1) - th) * pre[(long long)q * count + t] + th * cq;
        } else if (full && (nd.vf >> q & 1u)) {
            xm = R(Store<S>::load(Ff + (long long)q * c.Nf + nd.nf, la.hscale[q]));
        } else {
            xm = pre[(long long)q * count + t];
        }
        if (full) {
            R acc = 0, ws = 0;
#pragma unroll
            for (int m = 0; m < 9; ++m)
                if (nd.plane[m] >= 0 && (nd.pv[m] >> q & 1u)) {
                    acc += R(nd.w[m]) * R(Store<S>::load(Ff + (long long)q * c.Nf + nd.plane[m], la.hscale[q]));
                    ws += R(nd.w[m]);
                }
            fm = ws > R(0) ? acc / ws : R(0);
        }
    }
    R X[Q], eq[Q], ff[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        X[q] = __shfl_sync(0xffffffffu, xm, q);
        ff[q] = __shfl_sync(0xffffffffu, fm, q);
    }
    eqSplit<R, ORDER>(X, R(c.shiftC), R(c.kappa), eq);
    const R aF2C = R(c.alphaF2C), aC2F = R(c.alphaC2F);
    // fine side
    {
        R neq[Q], sc[Q];
        if (dc2) {
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const bool fineScaled = full && !(nd.vc >> q & 1u) && (nd.vf >> q & 1u);
                neq[q] = (fineScaled ? aF2C : R(1)) * (X[q] - eq[q]);
            }
            regulariseNeq<R>(neq, sc);
#pragma unroll
            for (int q = 0; q < Q; ++q)
                if (q == lane && (nd.rf >> q & 1u)) Store<S>::store(Ff + (long long)q * c.Nf + nd.nf, eq[q] + aC2F * sc[q], la.hscale[q]);
        } else {
#pragma unroll
            for (int q = 0; q < Q; ++q) neq[q] = X[q] - eq[q];
            rescaleNeq<R>(neq, c, true);
#pragma unroll
            for (int q = 0; q < Q; ++q)
                if (q == lane && (nd.rf >> q & 1u))
                    Store<S>::store(Ff + (long long)q * c.Nf + nd.nf, (nd.vc >> q & 1u) ? eq[q] + neq[q] : eq[q],
                                    la.hscale[q]);
        }
    }
    if (!full) return;
    // coarse side: fine non-equilibrium; the fine-missing populations take the
    // coarse one brought to the fine scale
    R neq[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) neq[q] = (nd.vf >> q & 1u) ? ff[q] - eq[q] : aC2F * (X[q] - eq[q]);
    if (dc2) {
#pragma unroll
        for (int q = 0; q < Q; ++q) neq[q] *= aF2C;
        R sc[Q];
        regulariseNeq<R>(neq, sc);
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (q == lane && (nd.rc >> q & 1u)) Store<S>::store(Bc + (long long)q * c.Nc + nd.nc, eq[q] + sc[q], la.hscale[q]);
    } else {
        rescaleNeq<R>(neq, c, false);
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (q == lane && (nd.rc >> q & 1u))
                Store<S>::store(Bc + (long long)q * c.Nc + nd.nc, (nd.vf >> q & 1u) ? eq[q] + neq[q] : eq[q],
                                la.hscale[q]);
    }
}
template <typename S, typename R, int ORDER>
__global__ void k_dc_couple(S* Bc, S* Ff, const DCDev* __restrict__ nodes, int count, const R* __restrict__ pre,
                            R th, int dc2, CouplingArgs c, LevelArgs<S> la) {
    dcCoupleBody<S, R, ORDER>(Bc, Ff, nodes, count, pre, th, dc2, c, la, blockIdx.x);
}


}  // namespace acp

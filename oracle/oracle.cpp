// FP64 CPU oracle for the acPulse_vcLBM hot path.
//
// TEST INFRASTRUCTURE ONLY.  This is a restatement of the reference's
// algorithm that checks the engine's results: tests/, __graft_entry__.smoke()
// and the CPU baseline of bench.py call it; the engine never does.
//
// Single level (MaxLevel 0): Lattice::timeStepping{SRT,MRT_GS,MRT_RM,RR,HRR}
// (Lattice.cpp:1496-2156) with the per-node operators of Node.cpp, restated
// with the reference's floating-point evaluation order (oracle_ops.h), push
// streaming (FluidNode.h:22-32, BoundaryNode.h:22-32) and LODI boundary passes
// in the reference's order: x faces, then z faces, then y faces
// (Lattice.cpp:1582-1624).  Pinned bit-for-bit against the reference built
// from its own sources (tests/golden/).
//
// Extensions of the reference, used by the pulse configurations: periodic
// axes (no boundary nodes, wrapped neighbours), the Gaussian pulse initial
// condition in lattice cells, and the MRT write-back switch.
#include "oracle_ops.h"
#include "oracle_topology.h"
#include "../include/acp.h"

#include <omp.h>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace orc {

enum NodeType : unsigned char {
    NT_INTERIOR = 0,  // fluid, all neighbours on the level
    NT_BOUNDARY = 1,  // LODI boundary node
    NT_IFACE = 2,     // fluid coupling node: fine C2F target or coarse F2C target
    NT_DEAD = 3       // covered by the other level
};

struct BNode {
    long n;           // node index
    int cls;          // index into kBoundaryClasses
    long n1, n2;      // normal neighbours
    long t[4];        // tangent neighbours (-1: none)
    int corner;
    int pass;         // 0: x faces, 1: z faces, 2: y faces
};

struct Level {
    int nx, ny, nz;
    long N;
    int org[3] = {0, 0, 0};  // global node index (of this level) of local node 0
    int per[3] = {0, 0, 0};  // periodic axes of this level
    std::vector<double> f[2];  // [N][19] per ping-pong array (Node::distr_)
    std::vector<double> preCol;
    std::vector<double> psi;   // Node::psi_ (cubic-Mach correction, persistent)
    std::vector<double> strain;  // [N][6] finite-difference strain of coupling nodes from partners
    std::vector<unsigned char> type;
    std::vector<BNode> bnodes;
    std::vector<long> nb;      // [N][18] push targets (-1: none)
    double dt, omega, spacing;
    long idx(int i, int j, int k) const { return ((long)k * ny + j) * nx + i; }
};

struct Mat19 {
    double a[Q][Q];
};

static bool invert19(const Mat19& m, Mat19& inv) {
    double aug[Q][2 * Q];
    for (int r = 0; r < Q; ++r)
        for (int c = 0; c < Q; ++c) {
            aug[r][c] = m.a[r][c];
            aug[r][Q + c] = r == c ? 1. : 0.;
        }
    for (int c = 0; c < Q; ++c) {
        int p = c;
        for (int r = c + 1; r < Q; ++r)
            if (std::fabs(aug[r][c]) > std::fabs(aug[p][c])) p = r;
        if (std::fabs(aug[p][c]) < 1e-12) return false;
        if (p != c)
            for (int k = 0; k < 2 * Q; ++k) std::swap(aug[p][k], aug[c][k]);
        double piv = aug[c][c];
        for (int k = 0; k < 2 * Q; ++k) aug[c][k] /= piv;
        for (int r = 0; r < Q; ++r) {
            if (r == c) continue;
            double fct = aug[r][c];
            if (fct == 0.) continue;
            for (int k = 0; k < 2 * Q; ++k) aug[r][k] -= fct * aug[c][k];
        }
    }
    for (int r = 0; r < Q; ++r)
        for (int c = 0; c < Q; ++c) inv.a[r][c] = aug[r][Q + c];
    return true;
}

// Gram-Schmidt moment basis of Node::calcAllMoments_GSbasis
// (Node.cpp:2934-3004), in lattice units (the c^n factors cancel against the
// back transform of Node.cpp:2870-2931).
static void gsBasis(Mat19& M) {
    for (int d = 0; d < Q; ++d) {
        int ex = EX[d], ey = EY[d], ez = EZ[d];
        int e2 = ex * ex + ey * ey + ez * ez;
        bool axis = e2 == 1;
        double col[Q];
        col[0] = 1;
        col[1] = d == 18 ? -1 : (e2 == 2 ? 1 : 0);
        col[2] = axis ? -2 : 1;
        col[3] = ex;
        col[4] = ex * (axis ? -2 : 1);
        col[5] = ey;
        col[6] = ey * (axis ? -2 : 1);
        col[7] = ez;
        col[8] = ez * (axis ? -2 : 1);
        col[9] = 3 * ex * ex - e2;
        col[10] = (3 * ex * ex - e2) * (axis ? -1 : 1);
        col[11] = ey * ey - ez * ez;
        col[12] = (ey * ey - ez * ez) * (axis ? -1 : 1);
        col[13] = ex * ey;
        col[14] = ey * ez;
        col[15] = ex * ez;
        col[16] = ex * (ey * ey - ez * ez);
        col[17] = ey * (ez * ez - ex * ex);
        col[18] = ez * (ex * ex - ey * ey);
        for (int m = 0; m < Q; ++m) M.a[m][d] = col[m];
    }
}

// Raw-moment basis of Node::calcAllMoments_RMbasis (Node.cpp:2693-2762),
// lattice units.
static void rmBasis(Mat19& M) {
    for (int d = 0; d < Q; ++d) {
        int ex = EX[d], ey = EY[d], ez = EZ[d];
        double col[Q] = {1., (double)ex, (double)ey, (double)ez, (double)(ex * ex + ey * ey + ez * ez),
                         (double)(ex * ex - ez * ez), (double)(ey * ey - ez * ez), (double)(ex * ey),
                         (double)(ex * ez), (double)(ey * ez), (double)(ex * ex * ez), (double)(ex * ez * ez),
                         (double)(ey * ey * ez), (double)(ey * ez * ez), (double)(ex * ex * ey),
                         (double)(ex * ey * ey), (double)(ex * ex * ez * ez), (double)(ex * ex * ey * ey),
                         (double)(ey * ey * ez * ez)};
        for (int m = 0; m < Q; ++m) M.a[m][d] = col[m];
    }
}

// Node::calcEquilibrium4_RMbasis (Node.cpp:2607-2647), lattice units.
static void equilibriumRM(double rho, const double* u, double* eq) {
    const double w[Q] = {1. / 18, 1. / 18, 1. / 18, 1. / 18, 1. / 18, 1. / 18, 1. / 36, 1. / 36, 1. / 36, 1. / 36,
                         1. / 36, 1. / 36, 1. / 36, 1. / 36, 1. / 36, 1. / 36, 1. / 36, 1. / 36, 1. / 3};
    double u2[3] = {u[0] * u[0], u[1] * u[1], u[2] * u[2]};
    for (int d = 0; d < Q; ++d) {
        int e[3] = {EX[d], EY[d], EZ[d]};
        int nz = (e[0] != 0) + (e[1] != 0) + (e[2] != 0);
        double s;
        if (nz == 0) {
            s = 1 - (u2[0] + u2[1] + u2[2]) + 3 * (u2[0] * u2[1] + u2[0] * u2[2] + u2[1] * u2[2]);
        } else if (nz == 1) {
            int a = e[0] ? 0 : (e[1] ? 1 : 2);
            int b = (a + 1) % 3, c = (a + 2) % 3;
            double sg = e[a];
            s = 1 + 3 * sg * u[a] + 3 * (u2[a] - u2[b] - u2[c]) - 9 * sg * u[a] * (u2[b] + u2[c]) -
                9 * u2[a] * (u2[b] + u2[c]);
        } else {
            int a = e[0] ? 0 : 1;
            int b = e[2] ? 2 : 1;
            double sa = e[a], sb = e[b];
            s = 1 + 3 * (sa * u[a] + sb * u[b]) + 3 * (u2[a] + u2[b]) + 9 * sa * sb * u[a] * u[b] +
                9 * (sb * u2[a] * u[b] + sa * u[a] * u2[b]) + 9 * u2[a] * u2[b];
        }
        eq[d] = rho * w[d] * s;
    }
}

struct Oracle {
    acp_case_desc desc;
    Consts k;
    std::vector<Level> lev;
    int alt = 1;  // main.cpp:55: alternatingL0 = true; state is in f[alt]
    long long steps = 0;
    Mat19 gsM, gsMinv, rmM, rmMinv;
    std::string err;
    int threads = 1;
    // two-level state (box layout)
    int altf = 1;               // fine array holding the state
    struct C2FNode {            // fine coupling node
        long n;                 // fine node
        int kind;               // 0 coincident, 1 mid, 2 centre
        long src;               // coincident: coarse node; mid/centre: -
        long st[4];             // stencil fine nodes (mid/centre), -1 unused
        double w[4];
        unsigned mask;          // populations replaced
    };
    struct F2CNode {
        long n;                 // coarse node
        long partner;           // coincident fine node
        long cube[27];          // 3x3x3 fine neighbourhood (x fastest)
        unsigned mask;
    };
    std::vector<C2FNode> c2f;   // ordered: coincident, mid, centre
    std::vector<F2CNode> f2c;
    // direct coupling (Coupling-Approach DC1 / DC2, Overlap 0): the coarse
    // nodes on the box faces and the fine nodes at coarse positions there
    // are the same points; each population is taken from the level on which
    // its source node is live
    struct DCNode {
        long nf, nc;            // the shared node on the fine and the coarse level
        unsigned vc, vf;        // populations whose source node is live on the coarse / fine level
        unsigned rc, rf;        // populations replaced on the coarse / fine level
        long plane[9];          // 3x3 fine stencil in the interface plane (-1: none), [4] = nf
        unsigned pv[9];         // populations valid at each stencil node
        double w[9];            // F2C filter weights over the stencil
    };
    std::vector<DCNode> dc;     // one per coincident C2F node, same order
    bool isDC() const { return desc.coupling != ACP_COUPLING_STD; }
    // HRR partner strain (Node.cpp:2114-2490, the STD scheme's partner passes
    // of Lattice.cpp:12142-12177, 12882-12934, 13211-13246): a coupling node's
    // finite-difference strain and cubic-Mach terms come from the other
    // level's stencil; every node read is a regular node whose state is
    // complete at that time
    bool partnerStrain() const {
        return !isDC() && lev.size() == 2 && (desc.op == ACP_OP_HRR || (desc.op == ACP_OP_RR && desc.cubic_mach));
    }
    struct NbSrc {
        long c[6];  // coarse axis neighbour (regular) of the coincident coarse node, or -1
        long f[6];  // else the regular fine node two fine cells away
    };
    std::vector<NbSrc> nbsrc;   // per coincident C2F node
    std::vector<double> preNb;  // [coincident][6][4] rho, u of the coarse neighbours at t
    bool couplingOk = true;
    std::vector<double> pre;    // coarse populations before the coarse step, per coincident C2F node
    int boxLo[3], boxHi[3], loIf[3], hiIf[3], spans[3];

    bool build() {
        const acp_case_desc& d = desc;
        if (d.max_level == 1) return buildTwoLevel();
        k.setup(d.speed_of_sound, d.spacing, d.kinematic_viscosity, d.density, d.mach, d.k1, d.hybrid_sigma, d.eq_order,
                d.cubic_mach != 0 && (d.op == ACP_OP_RR || d.op == ACP_OP_HRR), d.transverse != 0);
        gsBasis(gsM);
        rmBasis(rmM);
        if (!invert19(gsM, gsMinv) || !invert19(rmM, rmMinv)) { err = "moment basis not invertible"; return false; }
        lev.resize(1);
        Level& L = lev[0];
        L.nx = d.nx; L.ny = d.ny; L.nz = d.nz;
        L.N = (long)L.nx * L.ny * L.nz;
        for (int a = 0; a < 2; ++a) L.f[a].assign(L.N * Q, 0.);
        L.preCol.assign(L.N * Q, 0.);
        L.psi.assign(L.N * Q, 0.);
        L.type.assign(L.N, NT_INTERIOR);
        L.nb.assign(L.N * 18, -1);
        L.dt = k.dt(0);
        L.omega = k.omega(0);
        L.spacing = k.spacing;
        const int dims[3] = {L.nx, L.ny, L.nz};
        for (int a = 0; a < 3; ++a) {
            if (d.bc[a] == ACP_BC_LODI && dims[a] < 4) { err = "LODI axes need at least 4 nodes"; return false; }
            if (d.bc[a] == ACP_BC_PERIODIC && dims[a] < 1) { err = "empty axis"; return false; }
        }
        auto wrapped = [&](int i, int j, int kk, long& out) {
            int c[3] = {i, j, kk};
            for (int a = 0; a < 3; ++a) {
                if (c[a] < 0 || c[a] >= dims[a]) {
                    if (d.bc[a] != ACP_BC_PERIODIC) return false;
                    c[a] = (c[a] % dims[a] + dims[a]) % dims[a];
                }
            }
            out = L.idx(c[0], c[1], c[2]);
            return true;
        };
        for (int kk = 0; kk < L.nz; ++kk)
            for (int j = 0; j < L.ny; ++j)
                for (int i = 0; i < L.nx; ++i) {
                    int c[3] = {i, j, kk};
                    int fc[3];
                    for (int a = 0; a < 3; ++a)
                        fc[a] = d.bc[a] == ACP_BC_LODI ? (c[a] == 0 ? -1 : (c[a] == dims[a] - 1 ? 1 : 0)) : 0;
                    long n = L.idx(i, j, kk);
                    if (fc[0] == 0 && fc[1] == 0 && fc[2] == 0) {
                        for (int q = 0; q < 18; ++q) {
                            long t;
                            if (!wrapped(i + EX[q], j + EY[q], kk + EZ[q], t)) { err = "interior neighbour missing"; return false; }
                            L.nb[n * 18 + q] = t;
                        }
                        continue;
                    }
                    L.type[n] = NT_BOUNDARY;
                    const BClass* bc = boundaryClass(fc[0], fc[1], fc[2]);
                    BNode b;
                    b.n = n;
                    b.cls = (int)(bc - kBoundaryClasses);
                    b.corner = bc->corner;
                    if (!wrapped(i + bc->n1[0], j + bc->n1[1], kk + bc->n1[2], b.n1) ||
                        !wrapped(i + bc->n2[0], j + bc->n2[1], kk + bc->n2[2], b.n2)) {
                        err = "normal neighbour missing"; return false;
                    }
                    for (int m = 0; m < 4; ++m) b.t[m] = -1;
                    int nface = (fc[0] != 0) + (fc[1] != 0) + (fc[2] != 0);
                    if (nface == 1) {
                        int t[4][3];
                        faceTangents(fc[0], fc[1], fc[2], t);
                        for (int m = 0; m < 4; ++m)
                            if (!wrapped(i + t[m][0], j + t[m][1], kk + t[m][2], b.t[m])) { err = "tangent missing"; return false; }
                    }
                    for (int m = 0; m < 5 && bc->push[m] >= 0; ++m) {
                        int q = bc->push[m];
                        long t;
                        if (!wrapped(i + EX[q], j + EY[q], kk + EZ[q], t)) { err = "push target missing"; return false; }
                        L.nb[n * 18 + q] = t;
                    }
                    b.pass = fc[0] != 0 ? 0 : (fc[2] != 0 ? 1 : 2);
                    L.bnodes.push_back(b);
                }
        return true;
    }

    // Lattice::initialization (Lattice.cpp:1397-1493) and the Gaussian pulse
    // of the pulse configurations.
    void init() {
        for (size_t l = 0; l < lev.size(); ++l) {
            Level& L = lev[l];
            double sp = k.spacing / std::pow(2., (double)l);
            for (int kk = 0; kk < L.nz; ++kk)
                for (int j = 0; j < L.ny; ++j)
                    for (int i = 0; i < L.nx; ++i) {
                        double rho;
                        const int gi = i + L.org[0], gj = j + L.org[1], gk = kk + L.org[2];
                        if (desc.ic == ACP_IC_REFERENCE) {
                            double Rc = 0.06, A = 0.01, xCenter = -8. * Rc;
                            double xNode = gi * sp - desc.domain_size[0] / 2.;
                            double yNode = gj * sp - desc.domain_size[1] / 2.;
                            double xRel = xNode - xCenter;
                            rho = desc.density * (1 + A * std::exp(-(xRel * xRel + yNode * yNode) / (2 * Rc * Rc)));
                        } else {
                            double s = 1. / std::pow(2., (double)l);
                            double dx = gi * s - desc.ic_center[0], dy = gj * s - desc.ic_center[1];
                            double dz = desc.ic_dims == 3 ? gk * s - desc.ic_center[2] : 0.;
                            double r2 = dx * dx + dy * dy + dz * dz;
                            rho = desc.density * (1 + desc.ic_eps * std::exp(-std::log(2.) * r2 / (desc.ic_b * desc.ic_b)));
                        }
                        double u[3] = {0., 0., 0.}, eq[Q];
                        equilibrium(k, k.order, rho, u, eq);
                        long n = L.idx(i, j, kk);
                        for (int q = 0; q < Q; ++q) {
                            L.f[0][n * Q + q] = eq[q];
                            L.f[1][n * Q + q] = eq[q];
                            L.preCol[n * Q + q] = eq[q];
                            L.psi[n * Q + q] = 0.;
                        }
                    }
        }
        alt = 1;
        altf = 1;
        steps = 0;
    }

    // Node::collide* on one node, in place (Node.cpp:511-736, 2565-2605, 2798-2835).
    void collideNode(Level& L, long n, double* f) {
        int op = desc.op;
        double dt = L.dt;
        double* psi = &L.psi[n * Q];
        if (op == ACP_OP_MRT_GS || op == ACP_OP_MRT_RM) {
            if (!desc.mrt_writeback) return;  // the reference discards the back transform (Node.cpp:2603,2833)
            double rho = 0, j[3] = {0, 0, 0};
            for (int q = 0; q < Q; ++q) {
                rho += f[q];
                j[0] += EX[q] * f[q]; j[1] += EY[q] * f[q]; j[2] += EZ[q] * f[q];
            }
            if (op == ACP_OP_MRT_GS) {
                double m[Q], meq[Q] = {0}, s[Q];
                for (int a = 0; a < Q; ++a) {
                    m[a] = 0;
                    for (int q = 0; q < Q; ++q) m[a] += gsM.a[a][q] * f[q];
                }
                double jj = j[0] * j[0] + j[1] * j[1] + j[2] * j[2];
                meq[0] = rho; meq[3] = j[0]; meq[5] = j[1]; meq[7] = j[2];
                meq[1] = jj / rho;
                meq[9] = (2 * j[0] * j[0] - j[1] * j[1] - j[2] * j[2]) / rho;
                meq[11] = (j[1] * j[1] - j[2] * j[2]) / rho;
                meq[13] = j[0] * j[1] / rho;
                meq[14] = j[1] * j[2] / rho;
                meq[15] = j[0] * j[2] / rho;
                for (int a = 0; a < Q; ++a) s[a] = 1.;
                s[0] = s[3] = s[5] = s[7] = 0.;
                s[1] = s[9] = s[11] = s[13] = s[14] = s[15] = L.omega;
                double dm[Q];
                for (int a = 0; a < Q; ++a) dm[a] = s[a] * (meq[a] - m[a]);
                for (int q = 0; q < Q; ++q) {
                    double acc = 0;
                    for (int a = 0; a < Q; ++a) acc += gsMinv.a[q][a] * dm[a];
                    f[q] += acc;
                }
            } else {
                double u[3] = {j[0] / rho, j[1] / rho, j[2] / rho}, eq[Q], m[Q], meq[Q];
                equilibriumRM(rho, u, eq);
                for (int a = 0; a < Q; ++a) {
                    m[a] = 0; meq[a] = 0;
                    for (int q = 0; q < Q; ++q) { m[a] += rmM.a[a][q] * f[q]; meq[a] += rmM.a[a][q] * eq[q]; }
                }
                for (int a = 0; a < Q; ++a) {
                    double s = (a >= 5 && a <= 9) ? L.omega : 1.;
                    m[a] += s * (meq[a] - m[a]);
                }
                for (int q = 0; q < Q; ++q) {
                    double acc = 0;
                    for (int a = 0; a < Q; ++a) acc += rmMinv.a[q][a] * m[a];
                    f[q] = acc;
                }
            }
            return;
        }
        double dens = density(k, f, psi, dt);
        double u[3];
        velocity(k, f, psi, dt, dens, u);
        double eq[Q];
        equilibrium(k, k.order, dens, u, eq);
        if (op == ACP_OP_SRT) {
            for (int q = 0; q < Q; ++q) f[q] += L.omega * (eq[q] - f[q]);
            return;
        }
        const bool iface = L.type[n] == NT_IFACE;
        const bool partner = iface && partnerStrain();
        bool needStrain = ((op == ACP_OP_HRR) || k.cubic) && !iface;
        double S[6] = {0, 0, 0, 0, 0, 0};
        if (partner) {
            // strain and cubic-Mach terms set by the coupling passes from the partner level
            for (int c = 0; c < 6; ++c) S[c] = L.strain[n * 6 + c];
        } else if (iface) {
            for (int q = 0; q < Q; ++q) psi[q] = 0.;  // no finite differences across the interface
        }
        if (needStrain) {
            // neighbours' pre-collision moments (calcDensityPreCol/VelocityPreCol)
            double nbRho[6], nbU[6][3], dist[6];
            const int axisDir[6] = {0, 1, 2, 3, 4, 5};
            for (int a = 0; a < 6; ++a) {
                long m = L.nb[n * 18 + axisDir[a]];
                plainMoments(k, &L.preCol[m * Q], nbRho[a], nbU[a]);
                dist[a] = L.spacing;
            }
            strainAndPsi(k, nbRho, nbU, dist, S, psi);
        }
        double P[6];
        pi1(k, f, eq, psi, dt, P);
        double neq[Q];
        if (op == ACP_OP_RR) {
            recursiveNeq(k, k.order, P, u, neq);
        } else {
            double densH = density(k, f, psi, dt);
            double kinVisc = k.nu;
            double dynVisc = kinVisc * densH;
            double invPreFactor = -((dt * k.cs2) / (L.omega * kinVisc));
            double sg = iface && !partner ? 1. : k.sigma, a[6];  // without partners: regularisation of Pi1
            for (int c = 0; c < 6; ++c) a[c] = sg * P[c] + (1. - sg) * invPreFactor * (2. * dynVisc * S[c]);
            recursiveNeq(k, k.order, a, u, neq);
        }
        if (k.cubic) {
            for (int q = 0; q < Q; ++q) f[q] = eq[q] + (1 - L.omega) * neq[q] + 0.5 * dt * psi[q];
        } else {
            for (int q = 0; q < Q; ++q) f[q] = eq[q] + (1 - L.omega) * neq[q];
        }
    }

    // Node::LODIpressureOutlet (Node.cpp:229-443) writing array `nw`.
    void lodiNode(Level& L, int level, const BNode& b, int nw) {
        int od = 1 - nw;
        const double* fo = L.f[od].data();
        const double* fn = L.f[nw].data();
        double dt = L.dt;
        double localSpacing = k.spacing * std::pow(2., -level);
        double densB = density(k, &fo[b.n * Q], &L.psi[b.n * Q], dt);
        double veloB[3];
        velocity(k, &fo[b.n * Q], &L.psi[b.n * Q], dt, densB, veloB);
        double dG = 0, vG[3] = {0, 0, 0}, dGT[2] = {0, 0}, vGT[2][3] = {{0, 0, 0}, {0, 0, 0}};
        {
            double dN = density(k, &fn[b.n1 * Q], &L.psi[b.n1 * Q], dt);
            double d2N = density(k, &fn[b.n2 * Q], &L.psi[b.n2 * Q], dt);
            dG = (4. * dN - d2N - 3. * densB) / (-2. * localSpacing);
            double vN[3], v2N[3];
            velocity(k, &fn[b.n1 * Q], &L.psi[b.n1 * Q], dt, dN, vN);
            velocity(k, &fn[b.n2 * Q], &L.psi[b.n2 * Q], dt, d2N, v2N);
            for (int c = 0; c < 3; ++c) vG[c] = (4. * vN[c] - v2N[c] - 3. * veloB[c]) / (-2. * localSpacing);
            if (!b.corner && k.transverse) {
                double dT[4], vT[4][3];
                for (int m = 0; m < 4; ++m) {
                    dT[m] = density(k, &fo[b.t[m] * Q], &L.psi[b.t[m] * Q], dt);
                    velocity(k, &fo[b.t[m] * Q], &L.psi[b.t[m] * Q], dt, dT[m], vT[m]);
                }
                dGT[0] = (dT[0] - dT[1]) / (2. * localSpacing);
                dGT[1] = (dT[2] - dT[3]) / (2. * localSpacing);
                for (int c = 0; c < 3; ++c) {
                    vGT[0][c] = (vT[0][c] - vT[1][c]) / (2. * localSpacing);
                    vGT[1][c] = (vT[2][c] - vT[3][c]) / (2. * localSpacing);
                }
            }
        }
        int nd = kBoundaryClasses[b.cls].normalDir;
        double density = 0., velocity[3] = {0, 0, 0};
        // axis permutation into the boundary frame (normal first), Node.cpp:305-414
        int perm[3];
        bool neg;
        double L0;
        // L = NumberOfNodes_axis * Spacing (Node.cpp:311), or the case's override
        auto lodiNodes = [&](int a, int n) { return desc.lodi_length_nodes[a] > 0 ? desc.lodi_length_nodes[a] : n; };
        if (nd == 0 || nd == 2) { perm[0] = 0; perm[1] = 1; perm[2] = 2; L0 = lodiNodes(0, desc.nx) * k.spacing; }
        else if (nd == 1 || nd == 3) { perm[0] = 1; perm[1] = 0; perm[2] = 2; L0 = lodiNodes(1, desc.ny) * k.spacing; }
        else { perm[0] = 2; perm[1] = 0; perm[2] = 1; L0 = lodiNodes(2, desc.nz) * k.spacing; }
        neg = (nd == 0 || nd == 1 || nd == 4);
        if (neg) {
            dG *= -1.;
            for (int c = 0; c < 3; ++c) vG[c] *= -1.;
        }
        double sVG[3], sVB[3], sVGT[2][3];
        for (int c = 0; c < 3; ++c) {
            sVG[c] = vG[perm[c]];
            sVB[c] = veloB[perm[c]];
            sVGT[0][c] = vGT[0][perm[c]];
            sVGT[1][c] = vGT[1][perm[c]];
        }
        double v[3];
        lodiIntegrate(k, dt, L0, density, densB, dG, sVG, sVB, v, neg, dGT, sVGT);
        for (int c = 0; c < 3; ++c) velocity[perm[c]] = v[c];
        double eq[Q];
        equilibrium(k, k.order, density, velocity, eq);
        double* out = &L.f[nw][b.n * Q];
        for (int q = 0; q < Q; ++q) out[q] = eq[q];
    }

    // one step of a level reading array `a` (Lattice::timeStepping*, and the
    // per-level phases of Lattice::nestedTimeStepping*): save pre-collision
    // populations, collide in place and push, boundary pushes, LODI passes
    void stepLevel(int l, int a) {
        Level& L = lev[l];
        int nw = 1 - a;
        double* A = L.f[a].data();
        double* B = L.f[nw].data();
        std::memcpy(L.preCol.data(), A, sizeof(double) * L.N * Q);
        const long N = L.N;
#pragma omp parallel for num_threads(threads) schedule(static)
        for (long n = 0; n < N; ++n) {
            if (L.type[n] != NT_INTERIOR && L.type[n] != NT_IFACE) continue;
            double* f = &A[n * Q];
            collideNode(L, n, f);
            for (int q = 0; q < 18; ++q) {
                const long t = L.nb[n * 18 + q];
                if (t >= 0) B[t * Q + q] = f[q];
            }
            B[n * Q + 18] = f[18];
        }
        for (const BNode& b : L.bnodes) {
            for (int q = 0; q < 18; ++q) {
                long t = L.nb[b.n * 18 + q];
                if (t >= 0) B[t * Q + q] = A[b.n * Q + q];
            }
            B[b.n * Q + 18] = A[b.n * Q + 18];
        }
        for (int pass = 0; pass < 3; ++pass) {
            const long nb = (long)L.bnodes.size();
#pragma omp parallel for num_threads(threads) schedule(static)
            for (long m = 0; m < nb; ++m)
                if (L.bnodes[m].pass == pass) lodiNode(L, l, L.bnodes[m], nw);
        }
    }

    void stepSingle() {
        stepLevel(0, alt);
        alt = 1 - alt;
        ++steps;
    }

    // ------------------------------------------------------------------
    // two levels, box layout: the refined box [lo, hi] (coarse nodes) is
    // covered by the fine level; coarse and fine overlap by one coarse cell
    // (Overlap 1, the standard scheme).  The fine nodes on the box faces that
    // are interfaces take their populations from the coarse level (C2F), the
    // coarse nodes one cell inside the box take theirs from the fine level
    // (F2C), with the coarse step, two fine sub-steps and the couplings in the
    // order of Lattice::nestedTimeStepping* (Lattice.cpp:4354-5771).
    // coupling geometry of a level: coupling nodes on the interface faces of
    // the box [cl, ch] (local indices); the level lives inside the box, or
    // outside it and on its faces (then the nodes strictly inside are dead)
    struct Geom {
        int cl[3], ch[3], loIf[3], hiIf[3];
        bool inside;
        void normal(const int* c, int* f) const {
            const int sg = inside ? 1 : -1;
            for (int a = 0; a < 3; ++a) f[a] = (loIf[a] && c[a] == cl[a]) ? -sg : ((hiIf[a] && c[a] == ch[a]) ? sg : 0);
        }
        bool dead(const int* c) const {
            if (inside) return false;
            for (int a = 0; a < 3; ++a) {
                const int lo = loIf[a] ? cl[a] + 1 : cl[a], hi = hiIf[a] ? ch[a] - 1 : ch[a];
                if (c[a] < lo || c[a] > hi) return false;
            }
            return true;
        }
        bool coupling(const int* c) const {
            bool within = true, face = false;
            for (int a = 0; a < 3; ++a) {
                if (c[a] < cl[a] || c[a] > ch[a]) within = false;
                if ((loIf[a] && c[a] == cl[a]) || (hiIf[a] && c[a] == ch[a])) face = true;
            }
            return within && face && !dead(c);
        }
    };
    Geom geom[2];

    void markLevel(Level& L, const Geom& g) {
        for (int kk = 0; kk < L.nz; ++kk)
            for (int j = 0; j < L.ny; ++j)
                for (int i = 0; i < L.nx; ++i) {
                    const int c[3] = {i, j, kk};
                    L.type[L.idx(i, j, kk)] = g.dead(c) ? NT_DEAD : (g.coupling(c) ? NT_IFACE : NT_INTERIOR);
                }
    }

    bool buildTwoLevel() {
        const acp_case_desc& d = desc;
        k.setup(d.speed_of_sound, d.spacing, d.kinematic_viscosity, d.density, d.mach, d.k1, d.hybrid_sigma, d.eq_order,
                d.cubic_mach != 0 && (d.op == ACP_OP_RR || d.op == ACP_OP_HRR), d.transverse != 0);
        gsBasis(gsM);
        rmBasis(rmM);
        if (!invert19(gsM, gsMinv) || !invert19(rmM, rmMinv)) { err = "moment basis not invertible"; return false; }
        if ((d.coupling == ACP_COUPLING_STD) != (d.overlap == 1)) { err = "STD needs Overlap 1, DC1/DC2 Overlap 0"; return false; }
        const int dims[3] = {d.nx, d.ny, d.nz};
        const int ov = isDC() ? 0 : 1;
        lev.resize(2);
        Level& C = lev[0];
        Level& F = lev[1];
        Geom& gc = geom[0];
        Geom& gf = geom[1];
        int cd[3], fd[3];
        if (d.layout == ACP_LAYOUT_BOX) {
            for (int a = 0; a < 3; ++a) {
                boxLo[a] = d.box_lo[a];
                boxHi[a] = d.box_hi[a];
                spans[a] = boxLo[a] == 0 && boxHi[a] == dims[a] - 1;
                const bool lodi = d.bc[a] == ACP_BC_LODI;
                loIf[a] = !spans[a] && !(boxLo[a] == 0 && lodi);
                hiIf[a] = !spans[a] && !(boxHi[a] == dims[a] - 1 && lodi);
                if (d.bc[a] == ACP_BC_LODI && dims[a] < 4) { err = "LODI axes need at least 4 nodes"; return false; }
                if (!(spans[a] && d.bc[a] == ACP_BC_PERIODIC) && boxHi[a] - boxLo[a] < 4) { err = "box too thin"; return false; }
                if (boxLo[a] < 0 || boxHi[a] >= dims[a] || boxLo[a] > boxHi[a]) { err = "box outside the lattice"; return false; }
            }
            // a box reaching a LODI face spans the other two axes: no coupling node on a LODI face
            for (int a = 0; a < 3; ++a)
                if (d.bc[a] == ACP_BC_LODI && (boxLo[a] == 0 || boxHi[a] == dims[a] - 1))
                    for (int b = 0; b < 3; ++b)
                        if (b != a && !spans[b]) { err = "a box touching a LODI face must span the other axes"; return false; }
            for (int a = 0; a < 3; ++a) {
                gc.loIf[a] = gf.loIf[a] = loIf[a];
                gc.hiIf[a] = gf.hiIf[a] = hiIf[a];
                C.per[a] = d.bc[a] == ACP_BC_PERIODIC;
                cd[a] = dims[a];
                gc.cl[a] = loIf[a] ? boxLo[a] + ov : boxLo[a];
                gc.ch[a] = hiIf[a] ? boxHi[a] - ov : boxHi[a];
                F.per[a] = spans[a] && d.bc[a] == ACP_BC_PERIODIC;
                fd[a] = F.per[a] ? 2 * dims[a] : 2 * (boxHi[a] - boxLo[a]) + 1;
                F.org[a] = 2 * boxLo[a];
                gf.cl[a] = 0;
                gf.ch[a] = fd[a] - 1;
            }
            gc.inside = false;
            gf.inside = true;
        } else {
            // the reference's shell layout (Lattice.cpp:17-234): a coarse core
            // inside a fine shell that reaches every (LODI) face
            const int refLo[3] = {d.ref_layer_x, d.ref_layer_yz, d.ref_layer_yz};
            for (int a = 0; a < 3; ++a) {
                if (d.bc[a] != ACP_BC_LODI) { err = "the shell layout has LODI boundaries on every face"; return false; }
                const int lo = refLo[a] - ov, hi = dims[a] - 1 - d.ref_layer_yz + ov;
                if (refLo[a] < 2 || d.ref_layer_yz < 2 || hi - lo < 4) { err = "shell layout too thin"; return false; }
                loIf[a] = hiIf[a] = 1;
                gc.loIf[a] = gf.loIf[a] = gc.hiIf[a] = gf.hiIf[a] = 1;
                cd[a] = hi - lo + 1;
                C.org[a] = lo;
                gc.cl[a] = 0;
                gc.ch[a] = cd[a] - 1;
                fd[a] = 2 * (dims[a] - 1) + 1;
                gf.cl[a] = 2 * (lo + ov);
                gf.ch[a] = 2 * (hi - ov);
            }
            gc.inside = true;
            gf.inside = false;
        }
        C.nx = cd[0]; C.ny = cd[1]; C.nz = cd[2];
        initLevelArrays(C, 0);
        markLevel(C, gc);
        if (!wireLevel(C)) return false;
        F.nx = fd[0]; F.ny = fd[1]; F.nz = fd[2];
        initLevelArrays(F, 1);
        markLevel(F, gf);
        if (!wireLevel(F)) return false;
        buildCouplings();
        if (!couplingOk) { err = "partner strain stencil missing"; return false; }
        return true;
    }

    void initLevelArrays(Level& L, int l) {
        L.N = (long)L.nx * L.ny * L.nz;
        for (int a = 0; a < 2; ++a) L.f[a].assign(L.N * Q, 0.);
        L.preCol.assign(L.N * Q, 0.);
        L.psi.assign(L.N * Q, 0.);
        L.strain.assign(L.N * 6, 0.);
        L.type.assign(L.N, NT_INTERIOR);
        L.nb.assign(L.N * 18, -1);
        L.dt = k.dt(l);
        L.omega = k.omega(l);
        L.spacing = k.spacing / std::pow(2., (double)l);
    }

    // push targets and LODI wiring of a level whose node types are set; LODI
    // faces are the domain faces the level's box reaches
    bool wireLevel(Level& L) {
        const int dims[3] = {L.nx, L.ny, L.nz};
        int lodiLo[3], lodiHi[3];
        for (int a = 0; a < 3; ++a) {
            const bool lodi = desc.bc[a] == ACP_BC_LODI;
            // the level's local index 0 / last lies on a domain face
            lodiLo[a] = lodi && L.org[a] == 0;
            const int domTop = (&desc.nx)[a] - 1;
            const int scale = &L == &lev[0] ? 1 : 2;  // level-global index of the domain's last node
            lodiHi[a] = lodi && L.org[a] + dims[a] - 1 == scale * domTop;
        }
        auto inRange = [&](int i, int j, int kk, long& out) {
            int c[3] = {i, j, kk};
            for (int a = 0; a < 3; ++a)
                if (c[a] < 0 || c[a] >= dims[a]) {
                    if (!L.per[a]) return false;
                    c[a] = (c[a] % dims[a] + dims[a]) % dims[a];
                }
            out = L.idx(c[0], c[1], c[2]);
            return true;
        };
        for (int kk = 0; kk < L.nz; ++kk)
            for (int j = 0; j < L.ny; ++j)
                for (int i = 0; i < L.nx; ++i) {
                    const long n = L.idx(i, j, kk);
                    if (L.type[n] == NT_DEAD) continue;
                    const int c[3] = {i, j, kk};
                    int fc[3];
                    for (int a = 0; a < 3; ++a)
                        fc[a] = (lodiLo[a] && c[a] == 0) ? -1 : ((lodiHi[a] && c[a] == dims[a] - 1) ? 1 : 0);
                    if (fc[0] || fc[1] || fc[2]) {
                        if (L.type[n] == NT_IFACE) { err = "a coupling node on a LODI face"; return false; }
                        L.type[n] = NT_BOUNDARY;
                        const BClass* bc = boundaryClass(fc[0], fc[1], fc[2]);
                        BNode b;
                        b.n = n;
                        b.cls = (int)(bc - kBoundaryClasses);
                        b.corner = bc->corner;
                        if (!inRange(i + bc->n1[0], j + bc->n1[1], kk + bc->n1[2], b.n1) ||
                            !inRange(i + bc->n2[0], j + bc->n2[1], kk + bc->n2[2], b.n2)) {
                            err = "normal neighbour missing"; return false;
                        }
                        for (int m = 0; m < 4; ++m) b.t[m] = -1;
                        if ((fc[0] != 0) + (fc[1] != 0) + (fc[2] != 0) == 1) {
                            int t[4][3];
                            faceTangents(fc[0], fc[1], fc[2], t);
                            for (int m = 0; m < 4; ++m)
                                if (!inRange(i + t[m][0], j + t[m][1], kk + t[m][2], b.t[m])) { err = "tangent missing"; return false; }
                        }
                        for (int m = 0; m < 5 && bc->push[m] >= 0; ++m) {
                            const int q = bc->push[m];
                            long t;
                            if (!inRange(i + EX[q], j + EY[q], kk + EZ[q], t)) { err = "push target missing"; return false; }
                            L.nb[n * 18 + q] = t;
                        }
                        b.pass = fc[0] != 0 ? 0 : (fc[2] != 0 ? 1 : 2);
                        L.bnodes.push_back(b);
                        continue;
                    }
                    for (int q = 0; q < 18; ++q) {
                        long t;
                        if (inRange(i + EX[q], j + EY[q], kk + EZ[q], t)) L.nb[n * 18 + q] = t;
                        else if (L.type[n] == NT_INTERIOR) { err = "interior neighbour missing"; return false; }
                    }
                }
        return true;
    }

    // replaced-population masks (Coarse-to-Fine / Fine-to-Coarse keywords,
    // BoundaryConditions.txt:71-83): all, missing, or missing and in-plane
    static unsigned replaceMask(int mode, const int* face) {
        unsigned m = 0;
        for (int q = 0; q < Q; ++q) {
            const int e[3] = {EX[q], EY[q], EZ[q]};
            bool missing = false, inplane = false;
            for (int a = 0; a < 3; ++a)
                if (face[a] != 0) {
                    if (e[a] == -face[a]) missing = true;
                    if (e[a] == 0) inplane = true;
                }
            if (mode == 2 || missing || (mode == 1 && inplane)) m |= 1u << q;
        }
        return m;
    }

    void buildCouplings() {
        Level& C = lev[0];
        Level& F = lev[1];
        // level-global -> local (periodic axes wrap)
        auto local = [](const Level& L, const int* g, long& out) {
            const int dd[3] = {L.nx, L.ny, L.nz};
            int c[3];
            for (int a = 0; a < 3; ++a) {
                c[a] = g[a] - L.org[a];
                if (L.per[a]) c[a] = (c[a] % dd[a] + dd[a]) % dd[a];
                if (c[a] < 0 || c[a] >= dd[a]) return false;
            }
            out = L.idx(c[0], c[1], c[2]);
            return true;
        };
        auto fineIdx = [&](const int* g, long& out) { return local(F, g, out); };
        std::vector<C2FNode> coinc, mid, cen;
        for (int kk = 0; kk < F.nz; ++kk)
            for (int j = 0; j < F.ny; ++j)
                for (int i = 0; i < F.nx; ++i) {
                    const long n = F.idx(i, j, kk);
                    if (F.type[n] != NT_IFACE) continue;
                    const int c[3] = {i, j, kk};
                    int g[3], face[3], odd[3], nodd = 0;
                    geom[1].normal(c, face);
                    for (int a = 0; a < 3; ++a) {
                        g[a] = c[a] + F.org[a];
                        odd[a] = g[a] & 1;
                        nodd += odd[a];
                    }
                    C2FNode cn;
                    cn.n = n;
                    // the direct coupling never overwrites the fine populations that only the fine level has
                    cn.mask = replaceMask(isDC() && desc.c2f_replace == ACP_C2F_FALL ? ACP_C2F_MFP : desc.c2f_replace, face);
                    for (int m = 0; m < 4; ++m) { cn.st[m] = -1; cn.w[m] = 0; }
                    cn.src = -1;
                    if (nodd == 0) {
                        cn.kind = 0;
                        int cc[3];
                        for (int a = 0; a < 3; ++a) cc[a] = g[a] / 2;
                        local(C, cc, cn.src);
                        coinc.push_back(cn);
                        continue;
                    }
                    // interpolation axis: the odd axis (mid) or the higher odd axis (centre)
                    int ax = -1;
                    for (int a = 2; a >= 0; --a)
                        if (odd[a]) { ax = a; break; }
                    cn.kind = nodd == 1 ? 1 : 2;
                    long pts[4];
                    bool ok[4];
                    const int off[4] = {-3, -1, 1, 3};
                    for (int m = 0; m < 4; ++m) {
                        int gg[3] = {g[0], g[1], g[2]};
                        gg[ax] += off[m];
                        ok[m] = fineIdx(gg, pts[m]) && F.type[pts[m]] == NT_IFACE;
                    }
                    if (ok[0] && ok[3]) {
                        const double w[4] = {-1. / 16., 9. / 16., 9. / 16., -1. / 16.};
                        for (int m = 0; m < 4; ++m) { cn.st[m] = pts[m]; cn.w[m] = w[m]; }
                    } else {
                        cn.st[0] = pts[1]; cn.w[0] = 0.5;
                        cn.st[1] = pts[2]; cn.w[1] = 0.5;
                    }
                    (nodd == 1 ? mid : cen).push_back(cn);
                }
        c2f.clear();
        c2f.insert(c2f.end(), coinc.begin(), coinc.end());
        c2f.insert(c2f.end(), mid.begin(), mid.end());
        c2f.insert(c2f.end(), cen.begin(), cen.end());
        pre.assign(coinc.size() * Q, 0.);
        nbsrc.clear();
        if (partnerStrain()) {
            auto regular = [](const Level& L, long n) { return L.type[n] == NT_INTERIOR || L.type[n] == NT_BOUNDARY; };
            for (const C2FNode& cn : coinc) {
                NbSrc nb;
                const int cc[3] = {(int)(cn.src % C.nx), (int)((cn.src / C.nx) % C.ny), (int)(cn.src / ((long)C.nx * C.ny))};
                for (int q = 0; q < 6; ++q) {
                    int g[3] = {cc[0] + C.org[0] + EX[q], cc[1] + C.org[1] + EY[q], cc[2] + C.org[2] + EZ[q]};
                    long t;
                    nb.c[q] = nb.f[q] = -1;
                    if (local(C, g, t) && regular(C, t)) { nb.c[q] = t; continue; }
                    int gf[3] = {2 * g[0], 2 * g[1], 2 * g[2]};
                    if (local(F, gf, t) && regular(F, t)) nb.f[q] = t;
                    else couplingOk = false;
                }
                nbsrc.push_back(nb);
            }
            preNb.assign(coinc.size() * 24, 0.);
        }
        f2c.clear();
        for (int kk = 0; kk < C.nz; ++kk)
            for (int j = 0; j < C.ny; ++j)
                for (int i = 0; i < C.nx; ++i) {
                    const long n = C.idx(i, j, kk);
                    if (C.type[n] != NT_IFACE) continue;
                    F2CNode fn;
                    fn.n = n;
                    const int c[3] = {i, j, kk};
                    int g[3], face[3];
                    geom[0].normal(c, face);
                    for (int a = 0; a < 3; ++a) g[a] = 2 * (c[a] + C.org[a]);
                    fineIdx(g, fn.partner);
                    int m = 0;
                    for (int dz = -1; dz <= 1; ++dz)
                        for (int dy = -1; dy <= 1; ++dy)
                            for (int dx = -1; dx <= 1; ++dx) {
                                int gg[3] = {g[0] + dx, g[1] + dy, g[2] + dz};
                                fineIdx(gg, fn.cube[m++]);
                            }
                    // populations arriving from the covered side are the missing ones
                    fn.mask = replaceMask(desc.f2c_replace, face);
                    f2c.push_back(fn);
                }
        if (isDC()) {
            f2c.clear();
            buildDirectCoupling();
        }
    }

    // the shared nodes of the direct coupling, in the order of the coincident C2F nodes
    void buildDirectCoupling() {
        Level& C = lev[0];
        Level& F = lev[1];
        const int dims[3] = {C.nx, C.ny, C.nz}, fd[3] = {F.nx, F.ny, F.nz};
        auto live = [&](Level& L, const int* dd, const int* c, long& out) {
            int cc[3];
            for (int a = 0; a < 3; ++a) {
                cc[a] = c[a];
                if (cc[a] < 0 || cc[a] >= dd[a]) {
                    if (!L.per[a]) return false;
                    cc[a] = (cc[a] % dd[a] + dd[a]) % dd[a];
                }
            }
            out = L.idx(cc[0], cc[1], cc[2]);
            return L.type[out] != NT_DEAD;
        };
        const unsigned all = (1u << Q) - 1u;
        const double w1[3] = {0.25, 0.5, 0.25};
        dc.clear();
        for (const C2FNode& cn : c2f) {
            if (cn.kind != 0) continue;
            DCNode dn;
            dn.nf = cn.n;
            dn.nc = cn.src;
            const int cf[3] = {(int)(cn.n % F.nx), (int)((cn.n / F.nx) % F.ny), (int)(cn.n / ((long)F.nx * F.ny))};
            const int cc[3] = {(int)(cn.src % C.nx), (int)((cn.src / C.nx) % C.ny), (int)(cn.src / ((long)C.nx * C.ny))};
            dn.vc = dn.vf = 0;
            for (int q = 0; q < Q; ++q) {
                const int e[3] = {EX[q], EY[q], EZ[q]};
                int sc[3], sf[3];
                long t;
                for (int a = 0; a < 3; ++a) { sc[a] = cc[a] - e[a]; sf[a] = cf[a] - e[a]; }
                if (live(C, dims, sc, t)) dn.vc |= 1u << q;
                if (live(F, fd, sf, t)) dn.vf |= 1u << q;
            }
            const unsigned both = dn.vc & dn.vf;
            dn.rc = (~dn.vc & all) | (desc.f2c_replace != ACP_F2C_MC ? both : 0u);
            dn.rf = (~dn.vf & all) | (desc.c2f_replace != ACP_C2F_MF ? both : 0u);
            // interface plane: spanned by the axes other than the first face axis
            int fa = 0, fnrm[3];
            geom[1].normal(cf, fnrm);
            for (int a = 0; a < 3; ++a)
                if (fnrm[a]) { fa = a; break; }
            const int b1 = fa == 0 ? 1 : 0, b2 = fa == 2 ? 1 : 2;
            for (int m = 0; m < 9; ++m) {
                const int d1 = m % 3 - 1, d2 = m / 3 - 1;
                int c2[3] = {cf[0], cf[1], cf[2]};
                c2[b1] += d1;
                c2[b2] += d2;
                long t;
                const bool ok = live(F, fd, c2, t) && F.type[t] == NT_IFACE;
                double w = 0;
                if (ok) {
                    if (desc.f2c_filter == ACP_F2C_NOFI) w = m == 4 ? 1. : 0.;
                    else if (desc.f2c_filter == ACP_F2C_LAG) w = 1.;
                    else w = w1[d1 + 1] * w1[d2 + 1];
                }
                dn.plane[m] = ok && w > 0 ? t : -1;
                dn.w[m] = dn.plane[m] >= 0 ? w : 0.;
                dn.pv[m] = 0;
                if (dn.plane[m] >= 0)
                    for (int q = 0; q < Q; ++q) {
                        const int sf[3] = {c2[0] - EX[q], c2[1] - EY[q], c2[2] - EZ[q]};
                        long tt;
                        if (live(F, fd, sf, tt)) dn.pv[m] |= 1u << q;
                    }
            }
            dc.push_back(dn);
        }
    }

    // second-order regularised non-equilibrium: 4.5 w_q H2_q : Pi with Pi =
    // sum_q H2_q neq_q, H2 in lattice units (e_a e_b - delta_ab / 3)
    void regularise(const double* neq, double* out) {
        double P[6] = {0, 0, 0, 0, 0, 0};
        for (int q = 0; q < Q; ++q) {
            P[0] += (EX[q] * EX[q] - 1. / 3.) * neq[q];
            P[1] += (EY[q] * EY[q] - 1. / 3.) * neq[q];
            P[2] += (EZ[q] * EZ[q] - 1. / 3.) * neq[q];
            P[3] += EX[q] * EY[q] * neq[q];
            P[4] += EX[q] * EZ[q] * neq[q];
            P[5] += EY[q] * EZ[q] * neq[q];
        }
        for (int q = 0; q < Q; ++q) {
            const double h = (EX[q] * EX[q] - 1. / 3.) * P[0] + (EY[q] * EY[q] - 1. / 3.) * P[1] +
                             (EZ[q] * EZ[q] - 1. / 3.) * P[2] +
                             2. * (EX[q] * EY[q] * P[3] + EX[q] * EZ[q] * P[4] + EY[q] * EZ[q] * P[5]);
            out[q] = 4.5 * k.w[q] * h;
        }
    }

    // direct coupling at the shared nodes (GridCoupling::interpolTimeDirectCoupling
    // and directCoupling, declared GridCoupling.h:28-29, called at
    // Lattice.cpp:14018-14058 and 14699-14739; bodies absent).  th < 1: the
    // fine side at t+1/2 from the coarse state blended in time; th == 1: both
    // sides at t+1.  The equilibrium is that of the merged population set
    // (each population from the level on which it is valid); the replaced
    // populations get that equilibrium plus the other level's rescaled
    // non-equilibrium -- population-wise (DC1) or regularised onto H2 (DC2).
    void directCouple(int cnew, int fnew, double th) {
        Level& C = lev[0];
        Level& F = lev[1];
        double* CB = C.f[cnew].data();
        double* FB = F.f[fnew].data();
        const bool dc2 = desc.coupling == ACP_COUPLING_DC2;
        const double aF2C = 2. * F.omega / C.omega;
#pragma omp parallel for num_threads(threads) schedule(static)
        for (long t = 0; t < (long)dc.size(); ++t) {
            const DCNode& dn = dc[t];
            const double* cp = &CB[dn.nc * Q];
            const double* fp = &FB[dn.nf * Q];
            double X[Q], eq[Q], rho, u[3];
            // populations whose source node is live on neither level keep the
            // coarse state of t (complete after the previous exchange); no
            // population that a level leaves unwritten is ever read
            for (int q = 0; q < Q; ++q) {
                if (dn.vc >> q & 1u) X[q] = (1. - th) * pre[t * Q + q] + th * cp[q];
                else if (th == 1. && (dn.vf >> q & 1u)) X[q] = fp[q];
                else X[q] = pre[t * Q + q];
            }
            splitEq(X, eq, rho, u, C.dt);
            double fnew_[Q], cnew_[Q];
            // fine side
            {
                double neq[Q], sc[Q];
                if (dc2) {
                    for (int q = 0; q < Q; ++q) {
                        const bool fineScaled = th == 1. && !(dn.vc >> q & 1u) && (dn.vf >> q & 1u);
                        neq[q] = (fineScaled ? aF2C : 1.) * (X[q] - eq[q]);
                    }
                    double r[Q];
                    regularise(neq, r);
                    const double aC2F = C.omega / (2. * F.omega);
                    for (int q = 0; q < Q; ++q) fnew_[q] = eq[q] + aC2F * r[q];
                } else {
                    for (int q = 0; q < Q; ++q) neq[q] = X[q] - eq[q];
                    rescale(neq, sc, true);
                    for (int q = 0; q < Q; ++q) fnew_[q] = (dn.vc >> q & 1u) ? eq[q] + sc[q] : eq[q];
                }
            }
            // coarse side (t+1): filtered fine populations in the interface plane
            if (th == 1.) {
                // each population filtered over the stencil nodes where it is valid
                double ff[Q], neq[Q], sc[Q];
                for (int q = 0; q < Q; ++q) {
                    double acc = 0, ws = 0;
                    for (int m = 0; m < 9; ++m)
                        if (dn.plane[m] >= 0 && (dn.pv[m] >> q & 1u)) {
                            acc += dn.w[m] * FB[dn.plane[m] * Q + q];
                            ws += dn.w[m];
                        }
                    ff[q] = ws > 0 ? acc / ws : 0.;
                }
                // fine non-equilibrium; the fine-missing populations take the
                // coarse one brought to the fine scale
                const double aC2F = C.omega / (2. * F.omega);
                for (int q = 0; q < Q; ++q) neq[q] = (dn.vf >> q & 1u) ? ff[q] - eq[q] : aC2F * (X[q] - eq[q]);
                if (dc2) {
                    for (int q = 0; q < Q; ++q) neq[q] *= aF2C;
                    regularise(neq, sc);
                    for (int q = 0; q < Q; ++q) cnew_[q] = eq[q] + sc[q];
                } else {
                    rescale(neq, sc, false);
                    for (int q = 0; q < Q; ++q) cnew_[q] = (dn.vf >> q & 1u) ? eq[q] + sc[q] : eq[q];
                }
            }
            for (int q = 0; q < Q; ++q)
                if (dn.rf >> q & 1u) FB[dn.nf * Q + q] = fnew_[q];
            if (th == 1.)
                for (int q = 0; q < Q; ++q)
                    if (dn.rc >> q & 1u) CB[dn.nc * Q + q] = cnew_[q];
        }
    }

    // the fine coupling nodes between coarse positions (mid, then centre)
    void interpolateHanging(int fnew) {
        double* FB = lev[1].f[fnew].data();
        for (const C2FNode& cn : c2f) {
            if (cn.kind == 0) continue;
            double v[Q];
            for (int q = 0; q < Q; ++q) {
                double acc = 0;
                for (int m = 0; m < 4; ++m)
                    if (cn.st[m] >= 0) acc += cn.w[m] * FB[cn.st[m] * Q + q];
                v[q] = acc;
            }
            for (int q = 0; q < Q; ++q)
                if (cn.mask >> q & 1u) FB[cn.n * Q + q] = v[q];
        }
    }

    // equilibrium of a population array's own moments and the non-equilibrium part
    void splitEq(const double* f, double* eq, double& rho, double* u, double) {
        plainMoments(k, f, rho, u);
        equilibrium(k, k.order, rho, u, eq);
    }

    // scale the non-equilibrium part between levels: population based
    // (SRTSTYLE) or moment based in the Gram-Schmidt basis (MRTSTYLE)
    void rescale(const double* neq, double* out, bool toFine) {
        const double wc = lev[0].omega, wf = lev[1].omega;
        if (desc.scaling_style == ACP_SCALING_SRT) {
            const double a = toFine ? wc / (2. * wf) : 2. * wf / wc;
            for (int q = 0; q < Q; ++q) out[q] = a * neq[q];
            return;
        }
        double m[Q];
        for (int r = 0; r < Q; ++r) {
            m[r] = 0;
            for (int q = 0; q < Q; ++q) m[r] += gsM.a[r][q] * neq[q];
            const bool visc = r == 1 || r == 9 || r == 11 || r == 13 || r == 14 || r == 15;
            const double a = visc ? (toFine ? wc / (2. * wf) : 2. * wf / wc) : (toFine ? 0.5 : 2.0);
            m[r] *= a;
        }
        for (int q = 0; q < Q; ++q) {
            out[q] = 0;
            for (int r = 0; r < Q; ++r) out[q] += gsMinv.a[q][r] * m[r];
        }
    }

    // C2F: coarse state (blend of `pre` and the coarse array `cnew` with
    // weight `th` on cnew) onto the fine array `fnew`
    void coarseToFine(int cnew, int fnew, double th) {
        Level& C = lev[0];
        Level& F = lev[1];
        double* FB = F.f[fnew].data();
        const double* CB = C.f[cnew].data();
        long ic = 0;
        const bool ps = !nbsrc.empty();
        for (const C2FNode& cn : c2f) {
            double v[Q];
            if (ps && cn.kind == 0) {
                // coarse stencil at the time of the fine state: regular coarse
                // neighbours blended between t and t+1, the others from the
                // regular fine node two cells away (Node.cpp:2244-2380)
                const NbSrc& nb = nbsrc[ic];
                double nbRho[6], nbU[6][3], dist[6];
                for (int d = 0; d < 6; ++d) {
                    dist[d] = k.spacing;
                    if (nb.c[d] >= 0) {
                        double r, u[3];
                        plainMoments(k, &CB[nb.c[d] * Q], r, u);
                        nbRho[d] = (1. - th) * preNb[ic * 24 + d * 4] + th * r;
                        for (int c = 0; c < 3; ++c) nbU[d][c] = (1. - th) * preNb[ic * 24 + d * 4 + 1 + c] + th * u[c];
                    } else {
                        plainMoments(k, &FB[nb.f[d] * Q], nbRho[d], nbU[d]);
                    }
                }
                strainAndPsi(k, nbRho, nbU, dist, &F.strain[cn.n * 6], &F.psi[cn.n * Q]);
            } else if (ps) {
                for (int c = 0; c < 6; ++c) {
                    double acc = 0;
                    for (int m = 0; m < 4; ++m)
                        if (cn.st[m] >= 0) acc += cn.w[m] * F.strain[cn.st[m] * 6 + c];
                    F.strain[cn.n * 6 + c] = acc;
                }
                for (int q = 0; q < Q; ++q) {
                    double acc = 0;
                    for (int m = 0; m < 4; ++m)
                        if (cn.st[m] >= 0) acc += cn.w[m] * F.psi[cn.st[m] * Q + q];
                    F.psi[cn.n * Q + q] = acc;
                }
            }
            if (cn.kind == 0) {
                double f[Q], eq[Q], rho, u[3], neq[Q], sc[Q];
                for (int q = 0; q < Q; ++q) f[q] = (1. - th) * pre[ic * Q + q] + th * CB[cn.src * Q + q];
                ++ic;
                splitEq(f, eq, rho, u, C.dt);
                for (int q = 0; q < Q; ++q) neq[q] = f[q] - eq[q];
                rescale(neq, sc, true);
                for (int q = 0; q < Q; ++q) v[q] = eq[q] + sc[q];
            } else {
                for (int q = 0; q < Q; ++q) {
                    double acc = 0;
                    for (int m = 0; m < 4; ++m)
                        if (cn.st[m] >= 0) acc += cn.w[m] * FB[cn.st[m] * Q + q];
                    v[q] = acc;
                }
            }
            for (int q = 0; q < Q; ++q)
                if (cn.mask >> q & 1u) FB[cn.n * Q + q] = v[q];
        }
    }

    // F2C: fine state at t+1 onto the coarse coupling nodes (NOFI: the
    // coincident node; LAG: arithmetic average of the non-equilibria of the
    // 3x3x3 fine neighbourhood; TOU: the separable (1/4, 1/2, 1/4) filter)
    void fineToCoarse(int fcur, int cnew) {
        Level& C = lev[0];
        Level& F = lev[1];
        const double* FA = F.f[fcur].data();
        double* CB = C.f[cnew].data();
        const double w1[3] = {0.25, 0.5, 0.25};
#pragma omp parallel for num_threads(threads) schedule(static)
        for (long t = 0; t < (long)f2c.size(); ++t) {
            const F2CNode& fn = f2c[t];
            double eq[Q], rho, u[3], neq[Q];
            splitEq(&FA[fn.partner * Q], eq, rho, u, F.dt);
            if (desc.f2c_filter == ACP_F2C_NOFI) {
                for (int q = 0; q < Q; ++q) neq[q] = FA[fn.partner * Q + q] - eq[q];
            } else {
                for (int q = 0; q < Q; ++q) neq[q] = 0.;
                int m = 0;
                for (int dz = 0; dz < 3; ++dz)
                    for (int dy = 0; dy < 3; ++dy)
                        for (int dx = 0; dx < 3; ++dx) {
                            const long nn = fn.cube[m++];
                            const double w = desc.f2c_filter == ACP_F2C_LAG ? 1. / 27. : w1[dx] * w1[dy] * w1[dz];
                            double e2[Q], r2, u2[3];
                            splitEq(&FA[nn * Q], e2, r2, u2, F.dt);
                            for (int q = 0; q < Q; ++q) neq[q] += w * (FA[nn * Q + q] - e2[q]);
                        }
            }
            double sc[Q];
            rescale(neq, sc, false);
            for (int q = 0; q < Q; ++q)
                if (fn.mask >> q & 1u) CB[fn.n * Q + q] = eq[q] + sc[q];
            if (!nbsrc.empty()) {
                // the fine partner's axis neighbours at t+1, fine spacing (Node.cpp:2383-2490)
                const int face[6] = {14, 16, 12, 10, 22, 4};  // +x +y -x -y +z -z in the 3x3x3 cube
                double nbRho[6], nbU[6][3], dist[6];
                for (int d = 0; d < 6; ++d) {
                    plainMoments(k, &FA[fn.cube[face[d]] * Q], nbRho[d], nbU[d]);
                    dist[d] = F.spacing;
                }
                strainAndPsi(k, nbRho, nbU, dist, &C.strain[fn.n * 6], &C.psi[fn.n * Q]);
            }
        }
    }

    void stepTwoLevel() {
        Level& C = lev[0];
        // coarse populations at t of the coincident coupling sources
        long ic = 0;
        for (const C2FNode& cn : c2f)
            if (cn.kind == 0) {
                for (int q = 0; q < Q; ++q) pre[ic * Q + q] = C.f[alt][cn.src * Q + q];
                if (!nbsrc.empty())
                    for (int d = 0; d < 6; ++d)
                        if (nbsrc[ic].c[d] >= 0) {
                            double r, u[3];
                            plainMoments(k, &C.f[alt][nbsrc[ic].c[d] * Q], r, u);
                            preNb[ic * 24 + d * 4] = r;
                            for (int c = 0; c < 3; ++c) preNb[ic * 24 + d * 4 + 1 + c] = u[c];
                        }
                ++ic;
            }
        const int cnew = 1 - alt;
        if (isDC()) {
            stepLevel(0, alt);                  // coarse step t -> t+1
            stepLevel(1, altf);                 // fine sub-step t -> t+1/2
            directCouple(cnew, 1 - altf, 0.5);  // shared nodes, fine side, t+1/2
            interpolateHanging(1 - altf);
            stepLevel(1, 1 - altf);             // fine sub-step t+1/2 -> t+1
            directCouple(cnew, altf, 1.0);      // shared nodes, both sides, t+1
            interpolateHanging(altf);
            alt = cnew;
            ++steps;
            return;
        }
        stepLevel(0, alt);                 // coarse step t -> t+1
        stepLevel(1, altf);                // fine sub-step t -> t+1/2
        coarseToFine(cnew, 1 - altf, 0.5);  // C2F at t+1/2 (linear in time)
        stepLevel(1, 1 - altf);            // fine sub-step t+1/2 -> t+1
        fineToCoarse(altf, cnew);          // F2C at t+1
        coarseToFine(cnew, altf, 1.0);     // C2F at t+1
        alt = cnew;
        ++steps;
    }
};

}  // namespace orc

using orc::Oracle;

extern "C" {

void* orc_create(const acp_case_desc* d, int threads, char* err, int errlen) {
    Oracle* o = new Oracle();
    o->desc = *d;
    o->threads = threads > 0 ? threads : omp_get_max_threads();
    if (!o->build()) {
        if (err && errlen > 0) std::snprintf(err, errlen, "%s", o->err.c_str());
        delete o;
        return nullptr;
    }
    return o;
}

int orc_init(void* h) {
    static_cast<Oracle*>(h)->init();
    return 0;
}

int orc_step(void* h, int n) {
    Oracle* o = static_cast<Oracle*>(h);
    for (int s = 0; s < n; ++s) {
        if (o->lev.size() == 2) o->stepTwoLevel();
        else o->stepSingle();
    }
    return 0;
}

int orc_dims(void* h, int level, int* dims) {
    Oracle* o = static_cast<Oracle*>(h);
    if (level < 0 || level >= (int)o->lev.size()) return -1;
    dims[0] = o->lev[level].nx; dims[1] = o->lev[level].ny; dims[2] = o->lev[level].nz;
    return 0;
}

// structure-of-arrays output: out[(q*nz + k)*ny + j)*nx + i]
int orc_read_populations(void* h, int level, double* out) {
    Oracle* o = static_cast<Oracle*>(h);
    if (level < 0 || level >= (int)o->lev.size()) return -1;
    const orc::Level& L = o->lev[level];
    const double* f = L.f[level == 0 ? o->alt : o->altf].data();
    for (long n = 0; n < L.N; ++n)
        for (int q = 0; q < orc::Q; ++q) out[(long)q * L.N + n] = f[n * orc::Q + q];
    return 0;
}

int orc_write_populations(void* h, int level, const double* in) {
    Oracle* o = static_cast<Oracle*>(h);
    if (level < 0 || level >= (int)o->lev.size()) return -1;
    orc::Level& L = o->lev[level];
    for (int a = 0; a < 2; ++a)
        for (long n = 0; n < L.N; ++n)
            for (int q = 0; q < orc::Q; ++q) L.f[a][n * orc::Q + q] = in[(long)q * L.N + n];
    return 0;
}

// the current array only (the other array keeps what the steps left in it,
// as the engine's acp_put_columns does)
int orc_write_current(void* h, int level, const double* in) {
    Oracle* o = static_cast<Oracle*>(h);
    if (level < 0 || level >= (int)o->lev.size()) return -1;
    orc::Level& L = o->lev[level];
    double* f = L.f[level == 0 ? o->alt : o->altf].data();
    for (long n = 0; n < L.N; ++n)
        for (int q = 0; q < orc::Q; ++q) f[n * orc::Q + q] = in[(long)q * L.N + n];
    return 0;
}

long long orc_steps_done(void* h) { return static_cast<Oracle*>(h)->steps; }

// pressure p = rho cs^2 (Node::calcPressure, Node.cpp:64-83) of the current
// state at probes (level, i, j, k) in the level's global node indices
int orc_probe_pressures(void* h, int n, const int* lijk, double* out) {
    Oracle* o = static_cast<Oracle*>(h);
    for (int m = 0; m < n; ++m) {
        const int l = lijk[4 * m];
        if (l < 0 || l >= (int)o->lev.size()) return -1;
        const orc::Level& L = o->lev[l];
        const int i = lijk[4 * m + 1] - L.org[0], j = lijk[4 * m + 2] - L.org[1], k = lijk[4 * m + 3] - L.org[2];
        if (i < 0 || i >= L.nx || j < 0 || j >= L.ny || k < 0 || k >= L.nz) return -1;
        const double* f = &L.f[l == 0 ? o->alt : o->altf][L.idx(i, j, k) * orc::Q];
        double rho = 0;
        for (int q = 0; q < orc::Q; ++q) rho += f[q];
        out[m] = rho * o->k.cs2;
    }
    return 0;
}

void orc_destroy(void* h) { delete static_cast<Oracle*>(h); }

}  // extern "C"

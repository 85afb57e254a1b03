// Host side of the engine: case validation, node classes and boundary wiring,
// device memory, kernel dispatch, CUDA-graph stepping and the C ABI of
// include/acp.h.
#include "../../include/acp.h"
#include "kernels.cuh"
#include "topology.h"
#include "handle.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <utility>
#include <algorithm>
#include <condition_variable>
#include <functional>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>

#include <pthread.h>
#include <string>
#include <vector>

using namespace acp;

namespace {

std::mutex g_constMutex;
bool g_constUploaded[64] = {false};

// this translation unit's copies of the constant tables, once per device
int uploadConstants(int device) {
    if (device < 0 || device >= 64) return ACP_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_constMutex);
    if (g_constUploaded[device]) return ACP_OK;
    ConstTables t;
    int s = makeConstTables(t);
    if (s) return s;
    if ((s = uploadTables(t))) return s;
    g_constUploaded[device] = true;
    return ACP_OK;
}

}  // namespace

namespace acp {

// Page-locked host blocks of the node-class arrays, kept for reuse once a
// lattice is destroyed: blocks of the same rounded size are handed out again
// (at most 1 GiB kept).  Without a usable device the blocks are ordinary heap
// memory.
struct HostBlocks {
    std::mutex m;
    std::map<size_t, std::vector<void*>> free;  // rounded size -> page-locked blocks
    std::unordered_map<void*, bool> pinned;     // live block -> page-locked
    size_t kept = 0;
};
static HostBlocks& hostBlocks() {
    static HostBlocks* b = new HostBlocks();  // kept until the process exits
    return *b;
}
static size_t roundHostBlock(size_t bytes) { return (bytes + (1u << 16) - 1) & ~(size_t)((1u << 16) - 1); }

void* hostBlockAlloc(size_t bytes) {
    HostBlocks& hb = hostBlocks();
    const size_t r = roundHostBlock(std::max<size_t>(bytes, 1));
    {
        std::lock_guard<std::mutex> g(hb.m);
        auto it = hb.free.find(r);
        if (it != hb.free.end() && !it->second.empty()) {
            void* p = it->second.back();
            it->second.pop_back();
            hb.kept -= r;
            hb.pinned[p] = true;
            return p;
        }
    }
    void* p = nullptr;
    bool pin = cudaMallocHost(&p, r) == cudaSuccess;
    if (!pin) {
        cudaGetLastError();
        p = std::malloc(r);
        if (!p) throw std::bad_alloc();
    }
    std::lock_guard<std::mutex> g(hb.m);
    hb.pinned[p] = pin;
    return p;
}

void hostBlockFree(void* p, size_t bytes) {
    if (!p) return;
    HostBlocks& hb = hostBlocks();
    const size_t r = roundHostBlock(std::max<size_t>(bytes, 1));
    bool pin = false;
    {
        std::lock_guard<std::mutex> g(hb.m);
        auto it = hb.pinned.find(p);
        if (it != hb.pinned.end()) {
            pin = it->second;
            hb.pinned.erase(it);
        }
        if (pin && hb.kept + r <= ((size_t)1 << 30)) {
            hb.free[r].push_back(p);
            hb.kept += r;
            return;
        }
    }
    if (pin) cudaFreeHost(p);
    else std::free(p);
}

// the lattice constant table (push masks)
int makeConstTables(ConstTables& t) {
    uint32_t* masks = t.masks;
    for (int c = 0; c < 54; ++c) masks[c] = 0;
    // coupling nodes: every direction except those leaving the level across its box faces
    for (int c = 0; c < 27; ++c) {
        const int f[3] = {c / 9 - 1, (c / 3) % 3 - 1, c % 3 - 1};
        uint32_t m = 0;
        for (int q = 0; q < 18; ++q) {
            const int e[3] = {ex(q), ey(q), ez(q)};
            bool out = false;
            for (int a = 0; a < 3; ++a)
                if (f[a] != 0 && e[a] == f[a]) out = true;
            if (!out) m |= 1u << q;
        }
        masks[27 + c] = m;
    }
    for (const BoundaryClass& b : kBoundaryClasses) {
        uint32_t m = 0;
        for (int k = 0; k < 5 && b.push[k] >= 0; ++k) m |= 1u << b.push[k];
        masks[faceCode(b.fx, b.fy, b.fz)] = m;
    }
    masks[CODE_FLUID] = 0x3FFFFu;
    return ACP_OK;
}

}  // namespace acp

namespace {

int validate(const acp_case_desc* d, std::string& why) {
    if (!d) { why = "null case"; return ACP_ERR_INVALID; }
    if (d->nx < 1 || d->ny < 1 || d->nz < 1) { why = "node counts must be positive"; return ACP_ERR_INVALID; }
    // element indices of a level are 32-bit: 19 populations x nodes < 2^31
    if ((long long)d->nx * d->ny * d->nz > 100000000LL) { why = "more than 1e8 nodes in one level"; return ACP_ERR_UNSUPPORTED; }
    if (d->op < 0 || d->op > 4) { why = "unknown collision model"; return ACP_ERR_INVALID; }
    if (d->eq_order < 2 || d->eq_order > 4) { why = "Wrong order of equilibrium! (2, 3 or 4)"; return ACP_ERR_INVALID; }
    if (!(d->spacing > 0) || !(d->speed_of_sound > 0) || !(d->density > 0) || !(d->kinematic_viscosity > 0)) {
        why = "spacing, speed of sound, density and viscosity must be positive";
        return ACP_ERR_INVALID;
    }
    if (d->storage < 0 || d->storage > 2) { why = "unknown storage form"; return ACP_ERR_INVALID; }
    const int dims[3] = {d->nx, d->ny, d->nz};
    for (int a = 0; a < 3; ++a) {
        if (d->bc[a] != ACP_BC_LODI && d->bc[a] != ACP_BC_PERIODIC) { why = "unknown boundary type"; return ACP_ERR_INVALID; }
        if (d->bc[a] == ACP_BC_LODI && dims[a] < 4) {
            // the second normal neighbour would be a boundary node of the
            // opposite face, whose new array the reference reads half-updated
            why = "a LODI axis needs at least 4 nodes";
            return ACP_ERR_UNSUPPORTED;
        }
    }
    for (int a = 0; a < 3; ++a)
        if (d->lodi_length_nodes[a] < 0) { why = "negative LODI length"; return ACP_ERR_INVALID; }
    if (d->max_level != 0 && d->max_level != 1) { why = "MaxLevel must be 0 or 1"; return ACP_ERR_INVALID; }
    if (d->max_level == 1) {
        if (d->layout != ACP_LAYOUT_BOX && d->layout != ACP_LAYOUT_SHELL) { why = "unknown refinement layout"; return ACP_ERR_INVALID; }
        if (d->coupling < ACP_COUPLING_STD || d->coupling > ACP_COUPLING_DC2) { why = "unknown coupling approach"; return ACP_ERR_INVALID; }
        if ((d->coupling == ACP_COUPLING_STD) != (d->overlap == 1)) {
            why = "Coupling-Approach STD needs Overlap 1, DC1 and DC2 need Overlap 0";
            return ACP_ERR_INVALID;
        }
        if (d->layout == ACP_LAYOUT_SHELL) {
            // the reference's layout: a coarse core inside a fine shell reaching every face
            const int ov = d->coupling == ACP_COUPLING_STD ? 1 : 0;
            const int refLo[3] = {d->ref_layer_x, d->ref_layer_yz, d->ref_layer_yz};
            for (int a = 0; a < 3; ++a) {
                if (d->bc[a] != ACP_BC_LODI) { why = "the shell layout has LODI boundaries on every face"; return ACP_ERR_UNSUPPORTED; }
                if (refLo[a] < 2 || d->ref_layer_yz < 2) { why = "refinement layers of at least 2 coarse cells"; return ACP_ERR_INVALID; }
                const int lo = refLo[a] - ov, hi = dims[a] - 1 - d->ref_layer_yz + ov;
                if (hi - lo < 4) { why = "the coarse core needs at least 4 coarse cells per axis"; return ACP_ERR_INVALID; }
            }
            const long long fine = (2LL * d->nx - 1) * (2LL * d->ny - 1) * (2LL * d->nz - 1);
            if (fine > 100000000LL) { why = "more than 1e8 nodes in the fine level"; return ACP_ERR_UNSUPPORTED; }
            return ACP_OK;
        }
        bool spans[3];
        for (int a = 0; a < 3; ++a) {
            if (d->box_lo[a] < 0 || d->box_hi[a] >= dims[a] || d->box_lo[a] > d->box_hi[a]) {
                why = "refined box outside the lattice";
                return ACP_ERR_INVALID;
            }
            spans[a] = d->box_lo[a] == 0 && d->box_hi[a] == dims[a] - 1;
            if (!(spans[a] && d->bc[a] == ACP_BC_PERIODIC) && d->box_hi[a] - d->box_lo[a] < 4) {
                why = "the refined box needs at least 4 coarse cells per axis";
                return ACP_ERR_INVALID;
            }
        }
        for (int a = 0; a < 3; ++a)
            if (d->bc[a] == ACP_BC_LODI && (d->box_lo[a] == 0 || d->box_hi[a] == dims[a] - 1))
                for (int b = 0; b < 3; ++b)
                    if (b != a && !spans[b]) {
                        // otherwise coupling nodes would sit on LODI faces
                        why = "a refined box touching a LODI face must span the other two axes";
                        return ACP_ERR_UNSUPPORTED;
                    }
        const long long fine = (2LL * (d->box_hi[0] - d->box_lo[0]) + 2) * (2LL * (d->box_hi[1] - d->box_lo[1]) + 2) *
                               (2LL * (d->box_hi[2] - d->box_lo[2]) + 2);
        if (fine > 100000000LL) { why = "more than 1e8 nodes in the fine level"; return ACP_ERR_UNSUPPORTED; }
    }
    return ACP_OK;
}

// Host threads of the set-up scans: created on first use and kept for the
// life of the process (starting threads for every scan cost as much as the
// scans of a 6 M-node level).  One scan runs at a time; callers on other
// threads wait for the pool.  A forked child starts a pool of its own.
class ScanPool {
  public:
    static constexpr int kMax = 16;
    static ScanPool& get() {
        static std::once_flag once;
        std::call_once(once, [] { pthread_atfork(nullptr, nullptr, [] { instance() = nullptr; }); });
        std::lock_guard<std::mutex> g(creation());
        if (!instance()) instance() = new ScanPool();  // kept until the process exits
        return *instance();
    }
    int threads() const { return T_; }
    // job(t) for t in [0, threads()), the caller running t = 0
    void run(const std::function<void(int)>& job) {
        std::lock_guard<std::mutex> one(busy_);
        {
            std::lock_guard<std::mutex> g(m_);
            job_ = &job;
            pending_ = T_ - 1;
            ++gen_;
        }
        cv_.notify_all();
        job(0);
        std::unique_lock<std::mutex> g(m_);
        done_.wait(g, [this] { return pending_ == 0; });
        job_ = nullptr;
    }

  private:
    ScanPool() : T_(std::max(1, std::min(kMax, (int)std::thread::hardware_concurrency()))) {
        for (int t = 1; t < T_; ++t) std::thread([this, t] { work(t); }).detach();
    }
    static ScanPool*& instance() {
        static ScanPool* p = nullptr;
        return p;
    }
    static std::mutex& creation() {
        static std::mutex m;
        return m;
    }
    void work(int t) {
        unsigned long long seen = 0;
        for (;;) {
            const std::function<void(int)>* job;
            {
                std::unique_lock<std::mutex> g(m_);
                cv_.wait(g, [&] { return gen_ != seen; });
                seen = gen_;
                job = job_;
            }
            (*job)(t);
            std::lock_guard<std::mutex> g(m_);
            if (--pending_ == 0) done_.notify_one();
        }
    }
    const int T_;
    std::mutex m_, busy_;
    std::condition_variable cv_, done_;
    const std::function<void(int)>* job_ = nullptr;
    int pending_ = 0;
    unsigned long long gen_ = 0;
};

// The node scans of the set-up run over the host's cores: rows (j, k) of a
// level split into contiguous ranges, one per pool thread (index t < 16), so
// that per-thread results concatenated in thread order are in node order.
template <typename F>
void forRows(long long rows, F&& fn) {
    if (rows < 256) {
        fn(0LL, rows, 0);
        return;
    }
    ScanPool& pool = ScanPool::get();
    const int T = pool.threads();
    if (T == 1) {
        fn(0LL, rows, 0);
        return;
    }
    const std::function<void(int)> job = [&fn, rows, T](int t) { fn(rows * t / T, rows * (t + 1) / T, t); };
    pool.run(job);
}

// LODI wiring and node classes of a level whose dead / coupling nodes are
// marked in L.code (CODE_DEAD, CODE_IFACE0 + class); the LODI faces are the
// domain faces the level's box reaches
int wireLevel(acp_handle* h, LevelHost& L, int level) {
    const acp_case_desc& d = h->d;
    const int dims[3] = {L.nx, L.ny, L.nz};
    const int dom[3] = {d.nx, d.ny, d.nz};
    int lodiLo[3], lodiHi[3];
    for (int a = 0; a < 3; ++a) {
        const bool lodi = d.bc[a] == ACP_BC_LODI;
        lodiLo[a] = lodi && L.off[a] == 0;
        lodiHi[a] = lodi && (L.off[a] + dims[a] - 1 == (dom[a] - 1) << level);
    }
    auto idx = [&](int i, int j, int k) { return ((long long)k * L.ny + j) * L.nx + i; };
    auto inRange = [&](int i, int j, int k, long long& out) {
        int c[3] = {i, j, k};
        for (int a = 0; a < 3; ++a)
            if (c[a] < 0 || c[a] >= dims[a]) {
                if (!L.per[a]) return false;
                c[a] = (c[a] % dims[a] + dims[a]) % dims[a];
            }
        out = idx(c[0], c[1], c[2]);
        return true;
    };
    auto faceOf = [&](int i, int j, int k, int* fc) {
        const int c[3] = {i, j, k};
        for (int a = 0; a < 3; ++a) fc[a] = (lodiLo[a] && c[a] == 0) ? -1 : ((lodiHi[a] && c[a] == dims[a] - 1) ? 1 : 0);
        return fc[0] || fc[1] || fc[2];
    };
    // live nodes on the LODI faces, in node order: a row on a y or z face is
    // scanned whole, any other row holds at most its two x-face nodes
    std::vector<long long> faceNodes;
    {
        std::vector<std::vector<long long>> part(ScanPool::kMax);
        forRows((long long)L.ny * L.nz, [&](long long r0, long long r1, int t) {
            for (long long r = r0; r < r1; ++r) {
                const int j = (int)(r % L.ny), k = (int)(r / L.ny);
                const bool whole = (lodiLo[1] && j == 0) || (lodiHi[1] && j == L.ny - 1) || (lodiLo[2] && k == 0) ||
                                   (lodiHi[2] && k == L.nz - 1);
                const long long row = r * L.nx;
                if (whole) {
                    for (int i = 0; i < L.nx; ++i)
                        if (L.code[row + i] != CODE_DEAD) part[t].push_back(row + i);
                    continue;
                }
                if (lodiLo[0] && L.code[row] != CODE_DEAD) part[t].push_back(row);
                if (lodiHi[0] && L.nx > 1 && L.code[row + L.nx - 1] != CODE_DEAD) part[t].push_back(row + L.nx - 1);
            }
        });
        for (auto& v : part) faceNodes.insert(faceNodes.end(), v.begin(), v.end());
    }
    for (const long long n : faceNodes) {
                const int i = (int)(n % L.nx), j = (int)((n / L.nx) % L.ny), k = (int)(n / ((long long)L.nx * L.ny));
                int fc[3];
                faceOf(i, j, k, fc);
                if (L.code[n] != CODE_FLUID) return fail(h, ACP_ERR_INVALID, "a coupling node on a LODI face");
                L.code[n] = (uint8_t)faceCode(fc[0], fc[1], fc[2]);
                const BoundaryClass* bc = boundaryClass(fc[0], fc[1], fc[2]);
                BNodeDev b;
                b.n = n;
                b.normalDir = bc->normalDir;
                if (!inRange(i + bc->n1[0], j + bc->n1[1], k + bc->n1[2], b.n1) ||
                    !inRange(i + bc->n2[0], j + bc->n2[1], k + bc->n2[2], b.n2))
                    return fail(h, ACP_ERR_INVALID, "normal neighbour outside the lattice");
                for (int m = 0; m < 4; ++m) b.t[m] = -1;
                b.transverse = 0;
                if ((fc[0] != 0) + (fc[1] != 0) + (fc[2] != 0) == 1) {
                    int t[4][3];
                    faceTangents(fc[0], fc[1], fc[2], t);
                    for (int m = 0; m < 4; ++m)
                        if (!inRange(i + t[m][0], j + t[m][1], k + t[m][2], b.t[m]))
                            return fail(h, ACP_ERR_INVALID, "tangent neighbour outside the lattice");
                    b.transverse = d.transverse ? 1 : 0;
                }
                (fc[0] != 0 ? L.lodiX : L.lodiZY).push_back(b);
            }
    L.active = L.N - L.dead;
    L.spacing = d.spacing / std::pow(2.0, (double)level);
    L.dt = d.spacing / (d.speed_of_sound * std::sqrt(3.0)) / std::pow(2.0, (double)level);
    const double cs2 = d.speed_of_sound * d.speed_of_sound;
    L.omega = (cs2 * L.dt) / (d.kinematic_viscosity + 0.5 * cs2 * L.dt);
    return ACP_OK;
}

// replaced populations of a coupling node on faces f (outward normals):
// all, the missing ones (arriving across a face), or missing and in-plane
uint32_t replaceMask(int mode, const int* f) {
    uint32_t m = 0;
    for (int q = 0; q < Q; ++q) {
        const int e[3] = {ex(q), ey(q), ez(q)};
        bool missing = false, inplane = false;
        for (int a = 0; a < 3; ++a)
            if (f[a] != 0) {
                if (e[a] == -f[a]) missing = true;
                if (e[a] == 0) inplane = true;
            }
        if (mode == 2 || missing || (mode == 1 && inplane)) m |= 1u << q;
    }
    return m;
}

// Coupling geometry of a level: its coupling nodes lie on the faces of the
// box [cl, ch] (local node indices) that are interfaces.  The level is live
// inside the box (`inside`: the fine level of the box layout, the coarse core
// of the shell layout) or outside it and on its faces (the coarse level of the
// box layout, the fine level of the shell layout), the nodes strictly inside
// being covered by the other level.
struct CouplingGeom {
    int cl[3], ch[3];
    int loIf[3], hiIf[3];
    bool inside;
    // outward normal of the level's live region at a coupling node
    void normal(const int* c, int* f) const {
        const int sg = inside ? 1 : -1;
        for (int a = 0; a < 3; ++a) f[a] = (loIf[a] && c[a] == cl[a]) ? -sg : ((hiIf[a] && c[a] == ch[a]) ? sg : 0);
    }
};

// node classes of a level from its coupling geometry: dead nodes, coupling
// nodes (pushing everywhere when the level lies outside its box, where the
// covered nodes exist in the array, else only within the level).  Row by row
// (j, k): a row crossing the box's interior holds at most one dead segment and
// a coupling node at each interface x face; a row on a y or z interface face
// is coupling over the whole x extent of the box; classes are then set per
// segment instead of testing every node.
void markLevel(LevelHost& L, const CouplingGeom& g) {
    L.code.resize(L.N);  // every row is filled with CODE_FLUID below before it is marked
    // coupling nodes and dead-node counts per pool thread, in node order
    std::vector<std::vector<long long>> part(ScanPool::kMax);
    std::vector<long long> dead(ScanPool::kMax, 0);
    auto setCoupling = [&](long long n, const int* c, int t) {
        int f[3];
        g.normal(c, f);
        L.code[n] = (uint8_t)(CODE_IFACE0 + (g.inside ? faceCode(f[0], f[1], f[2]) : CODE_FLUID));
        part[t].push_back(n);
    };
    // strictly-inside range of an axis (the covered nodes of a level outside its box)
    int dlo[3], dhi[3];
    for (int a = 0; a < 3; ++a) {
        dlo[a] = g.loIf[a] ? g.cl[a] + 1 : g.cl[a];
        dhi[a] = g.hiIf[a] ? g.ch[a] - 1 : g.ch[a];
    }
    forRows((long long)L.ny * L.nz, [&](long long r0, long long r1, int t) {
        std::fill(L.code.begin() + r0 * L.nx, L.code.begin() + r1 * L.nx, CODE_FLUID);
        for (long long r = r0; r < r1; ++r) {
            const int j = (int)(r % L.ny), k = (int)(r / L.ny);
            if (j < g.cl[1] || j > g.ch[1] || k < g.cl[2] || k > g.ch[2]) continue;  // row misses the box
            const long long row = r * L.nx;
            const bool faceRow = (g.loIf[1] && j == g.cl[1]) || (g.hiIf[1] && j == g.ch[1]) ||
                                 (g.loIf[2] && k == g.cl[2]) || (g.hiIf[2] && k == g.ch[2]);
            const bool innerRow = j >= dlo[1] && j <= dhi[1] && k >= dlo[2] && k <= dhi[2];
            if (faceRow) {
                // a face coordinate lies outside the strictly-inside range: nothing dead
                for (int i = std::max(0, g.cl[0]); i <= std::min(L.nx - 1, g.ch[0]); ++i) {
                    const int c[3] = {i, j, k};
                    setCoupling(row + i, c, t);
                }
                continue;
            }
            if (!g.inside && innerRow && dlo[0] <= dhi[0]) {
                const int i0 = std::max(0, dlo[0]), i1 = std::min(L.nx - 1, dhi[0]);
                if (i0 <= i1) {
                    std::fill(L.code.begin() + row + i0, L.code.begin() + row + i1 + 1, CODE_DEAD);
                    dead[t] += i1 - i0 + 1;
                }
            }
            // the x-face coupling nodes lie outside the dead segment, lower face first
            const int xs[2] = {g.loIf[0] ? g.cl[0] : -1, g.hiIf[0] ? g.ch[0] : -1};
            for (int e = 0; e < 2; ++e) {
                const int i = xs[e];
                if (i < 0 || i >= L.nx || (e == 1 && i == xs[0])) continue;
                const int c[3] = {i, j, k};
                setCoupling(row + i, c, t);
            }
        }
    });
    L.coupling.clear();
    L.dead = 0;
    for (int t = 0; t < ScanPool::kMax; ++t) {
        L.coupling.insert(L.coupling.end(), part[t].begin(), part[t].end());
        L.dead += dead[t];
    }
}

// Two levels.  Box layout: the fine level covers the box [box_lo, box_hi]
// (coarse node indices), the coarse level the domain with the box interior
// covered.  Shell layout (the reference's, Lattice.cpp:17-234): the coarse
// level is the core [RefinementLayerX - Overlap, nx-1 - RefinementLayerYZ +
// Overlap] x [RefinementLayerYZ - Overlap, n-1 - RefinementLayerYZ + Overlap]^2,
// the fine level the domain with the core covered.  STD couples with an
// overlap of one coarse cell, DC1/DC2 on shared nodes (Overlap 0).
int buildTwoLevel(acp_handle* h) {
    const acp_case_desc& d = h->d;
    const int dom[3] = {d.nx, d.ny, d.nz};
    const bool direct = d.coupling != ACP_COUPLING_STD;
    const int ov = direct ? 0 : 1;
    const bool shell = d.layout == ACP_LAYOUT_SHELL;
    LevelHost C, F;
    CouplingGeom gc, gf;
    int fd[3];
    if (!shell) {
        for (int a = 0; a < 3; ++a) {
            const int lo = d.box_lo[a], hi = d.box_hi[a];
            const bool spans = lo == 0 && hi == dom[a] - 1;
            const bool lodi = d.bc[a] == ACP_BC_LODI;
            gc.loIf[a] = gf.loIf[a] = !spans && !(lo == 0 && lodi);
            gc.hiIf[a] = gf.hiIf[a] = !spans && !(hi == dom[a] - 1 && lodi);
            C.per[a] = d.bc[a] == ACP_BC_PERIODIC;
            gc.cl[a] = gc.loIf[a] ? lo + ov : lo;
            gc.ch[a] = gc.hiIf[a] ? hi - ov : hi;
            F.per[a] = spans && d.bc[a] == ACP_BC_PERIODIC;
            fd[a] = F.per[a] ? 2 * dom[a] : 2 * (hi - lo) + 1;
            F.off[a] = 2 * lo;
            gf.cl[a] = 0;
            gf.ch[a] = fd[a] - 1;
        }
        C.nx = d.nx; C.ny = d.ny; C.nz = d.nz;
        gc.inside = false;
        gf.inside = true;
    } else {
        const int refLo[3] = {d.ref_layer_x, d.ref_layer_yz, d.ref_layer_yz};
        int cd[3];
        for (int a = 0; a < 3; ++a) {
            const int lo = refLo[a] - ov, hi = dom[a] - 1 - d.ref_layer_yz + ov;
            gc.loIf[a] = gf.loIf[a] = gc.hiIf[a] = gf.hiIf[a] = 1;
            cd[a] = hi - lo + 1;
            C.off[a] = lo;
            gc.cl[a] = 0;
            gc.ch[a] = cd[a] - 1;
            fd[a] = 2 * (dom[a] - 1) + 1;
            gf.cl[a] = 2 * (lo + ov);
            gf.ch[a] = 2 * (hi - ov);
        }
        C.nx = cd[0]; C.ny = cd[1]; C.nz = cd[2];
        gc.inside = true;
        gf.inside = false;
    }
    C.N = (long long)C.nx * C.ny * C.nz;
    markLevel(C, gc);
    int s = wireLevel(h, C, 0);
    if (s) return s;
    F.nx = fd[0]; F.ny = fd[1]; F.nz = fd[2];
    F.N = (long long)F.nx * F.ny * F.nz;
    markLevel(F, gf);
    if ((s = wireLevel(h, F, 1))) return s;
    // coupling lists; nodes addressed by their level-global indices
    auto local = [](const LevelHost& L, const int* g, long long& out) {
        int c[3];
        const int dd[3] = {L.nx, L.ny, L.nz};
        for (int a = 0; a < 3; ++a) {
            c[a] = g[a] - L.off[a];
            if (c[a] < 0 || c[a] >= dd[a]) {
                if (!L.per[a]) return false;
                c[a] = (c[a] % dd[a] + dd[a]) % dd[a];
            }
        }
        out = ((long long)c[2] * L.ny + c[1]) * L.nx + c[0];
        return true;
    };
    auto fineLocal = [&](const int* g, int& out) {
        long long n;
        if (!local(F, g, n)) return false;
        out = (int)n;
        return true;
    };
    // C2F records of the fine coupling nodes on the pool threads (contiguous
    // ranges of the node list; per-thread lists joined in thread order keep the
    // node order, and the first failing node's message is the one reported)
    const int T = ScanPool::kMax;
    std::vector<std::vector<C2FDev>> coincT(T), midT(T), cenT(T);
    std::vector<const char*> errT(T, nullptr);
    forRows((long long)F.coupling.size(), [&](long long i0, long long i1, int t) {
        for (long long i = i0; i < i1 && !errT[t]; ++i) {
                const long long n = F.coupling[i];
                const int c[3] = {(int)(n % F.nx), (int)((n / F.nx) % F.ny), (int)(n / ((long long)F.nx * F.ny))};
                int g[3], f[3], odd[3], nodd = 0;
                gf.normal(c, f);
                for (int a = 0; a < 3; ++a) {
                    g[a] = c[a] + F.off[a];
                    odd[a] = g[a] & 1;
                    nodd += odd[a];
                }
                C2FDev cn;
                cn.n = (int)n;
                cn.src = -1;
                // the direct coupling never overwrites the fine populations that only the fine level has
                cn.mask = replaceMask(direct && d.c2f_replace == ACP_C2F_FALL ? ACP_C2F_MFP : d.c2f_replace, f);
                for (int m = 0; m < 4; ++m) { cn.st[m] = -1; cn.w[m] = 0.f; }
                if (nodd == 0) {
                    int gc2[3];
                    for (int a = 0; a < 3; ++a) gc2[a] = g[a] / 2;
                    long long src;
                    if (!local(C, gc2, src) || C.code[src] == CODE_DEAD) {
                        errT[t] = "coarse source of a fine coupling node missing";
                        break;
                    }
                    cn.src = (int)src;
                    coincT[t].push_back(cn);
                    continue;
                }
                int ax = 0;
                for (int a = 2; a >= 0; --a)
                    if (odd[a]) { ax = a; break; }
                const int off[4] = {-3, -1, 1, 3};
                int pts[4];
                bool ok[4];
                for (int m = 0; m < 4; ++m) {
                    int gg[3] = {g[0], g[1], g[2]};
                    gg[ax] += off[m];
                    ok[m] = fineLocal(gg, pts[m]) && F.code[pts[m]] >= CODE_IFACE0 && F.code[pts[m]] != CODE_DEAD;
                }
                if (!ok[1] || !ok[2]) {
                    errT[t] = "interpolation stencil missing on the interface";
                    break;
                }
                if (ok[0] && ok[3]) {
                    const float w[4] = {-1.f / 16.f, 9.f / 16.f, 9.f / 16.f, -1.f / 16.f};
                    for (int m = 0; m < 4; ++m) { cn.st[m] = pts[m]; cn.w[m] = w[m]; }
                } else {
                    cn.st[0] = pts[1]; cn.w[0] = 0.5f;
                    cn.st[1] = pts[2]; cn.w[1] = 0.5f;
                }
                (nodd == 1 ? midT : cenT)[t].push_back(cn);
        }
    });
    for (int t = 0; t < T; ++t)
        if (errT[t]) return fail(h, ACP_ERR_INVALID, "%s", errT[t]);
    std::vector<C2FDev> coinc, mid, cen;
    for (int t = 0; t < T; ++t) {
        coinc.insert(coinc.end(), coincT[t].begin(), coincT[t].end());
        mid.insert(mid.end(), midT[t].begin(), midT[t].end());
        cen.insert(cen.end(), cenT[t].begin(), cenT[t].end());
    }
    h->nCoinc = (int)coinc.size();
    h->nMid = (int)mid.size();
    h->nCen = (int)cen.size();
    h->c2fHost.clear();
    h->c2fHost.insert(h->c2fHost.end(), coinc.begin(), coinc.end());
    h->c2fHost.insert(h->c2fHost.end(), mid.begin(), mid.end());
    h->c2fHost.insert(h->c2fHost.end(), cen.begin(), cen.end());
    h->f2cHost.clear();
    h->dcHost.clear();
    if (direct) {
        // the shared nodes, in the order of the coincident C2F nodes
        auto liveIn = [](const LevelHost& L, const int* c) {
            int cc[3];
            const int dd[3] = {L.nx, L.ny, L.nz};
            for (int a = 0; a < 3; ++a) {
                cc[a] = c[a];
                if (cc[a] < 0 || cc[a] >= dd[a]) {
                    if (!L.per[a]) return -1LL;
                    cc[a] = (cc[a] % dd[a] + dd[a]) % dd[a];
                }
            }
            const long long n = ((long long)cc[2] * L.ny + cc[1]) * L.nx + cc[0];
            return L.code[n] == CODE_DEAD ? -1LL : n;
        };
        const uint32_t all = (1u << Q) - 1u;
        const double w1[3] = {0.25, 0.5, 0.25};
        for (const C2FDev& cn : coinc) {
            DCDev dn;
            dn.nf = cn.n;
            dn.nc = cn.src;
            const int cf[3] = {(int)(cn.n % F.nx), (int)((cn.n / F.nx) % F.ny), (int)(cn.n / ((long long)F.nx * F.ny))};
            const int cc[3] = {(int)(cn.src % C.nx), (int)((cn.src / C.nx) % C.ny),
                               (int)(cn.src / ((long long)C.nx * C.ny))};
            dn.vc = dn.vf = 0;
            for (int q = 0; q < Q; ++q) {
                const int sc[3] = {cc[0] - ex(q), cc[1] - ey(q), cc[2] - ez(q)};
                const int sf[3] = {cf[0] - ex(q), cf[1] - ey(q), cf[2] - ez(q)};
                if (liveIn(C, sc) >= 0) dn.vc |= 1u << q;
                if (liveIn(F, sf) >= 0) dn.vf |= 1u << q;
            }
            const uint32_t both = dn.vc & dn.vf;
            dn.rc = (~dn.vc & all) | (d.f2c_replace != ACP_F2C_MC ? both : 0u);
            dn.rf = (~dn.vf & all) | (d.c2f_replace != ACP_C2F_MF ? both : 0u);
            int fa = 0, fn[3];
            gf.normal(cf, fn);
            for (int a = 0; a < 3; ++a)
                if (fn[a]) { fa = a; break; }
            const int b1 = fa == 0 ? 1 : 0, b2 = fa == 2 ? 1 : 2;
            for (int m = 0; m < 9; ++m) {
                const int d1 = m % 3 - 1, d2 = m / 3 - 1;
                int c2[3] = {cf[0], cf[1], cf[2]};
                c2[b1] += d1;
                c2[b2] += d2;
                const long long t = liveIn(F, c2);
                const bool ok = t >= 0 && F.code[t] >= CODE_IFACE0;
                double w = 0;
                if (ok) {
                    if (d.f2c_filter == ACP_F2C_NOFI) w = m == 4 ? 1. : 0.;
                    else if (d.f2c_filter == ACP_F2C_LAG) w = 1.;
                    else w = w1[d1 + 1] * w1[d2 + 1];
                }
                dn.plane[m] = ok && w > 0 ? (int)t : -1;
                dn.w[m] = dn.plane[m] >= 0 ? w : 0.;
                dn.pv[m] = 0;
                if (dn.plane[m] >= 0)
                    for (int q = 0; q < Q; ++q) {
                        const int sf[3] = {c2[0] - ex(q), c2[1] - ey(q), c2[2] - ez(q)};
                        if (liveIn(F, sf) >= 0) dn.pv[m] |= 1u << q;
                    }
            }
            h->dcHost.push_back(dn);
        }
    }
    // F2C records of the coarse coupling nodes (STD), on the pool threads as above
    std::vector<std::vector<F2CDev>> f2cT(T);
    std::fill(errT.begin(), errT.end(), nullptr);
    forRows(direct ? 0LL : (long long)C.coupling.size(), [&](long long i0, long long i1, int t) {
        for (long long i = i0; i < i1 && !errT[t]; ++i) {
                const long long n = C.coupling[i];
                const int c[3] = {(int)(n % C.nx), (int)((n / C.nx) % C.ny), (int)(n / ((long long)C.nx * C.ny))};
                int g[3], f[3];
                gc.normal(c, f);
                for (int a = 0; a < 3; ++a) g[a] = 2 * (c[a] + C.off[a]);
                F2CDev fn;
                fn.n = (int)n;
                fn.mask = replaceMask(d.f2c_replace, f);
                if (!fineLocal(g, fn.partner)) {
                    errT[t] = "fine partner outside the box";
                    break;
                }
                int m = 0;
                bool inside = true;
                for (int dz = -1; dz <= 1 && inside; ++dz)
                    for (int dy = -1; dy <= 1 && inside; ++dy)
                        for (int dx = -1; dx <= 1 && inside; ++dx) {
                            int gg[3] = {g[0] + dx, g[1] + dy, g[2] + dz};
                            inside = fineLocal(gg, fn.cube[m++]);
                        }
                if (!inside) {
                    errT[t] = "F2C neighbourhood outside the box";
                    break;
                }
                f2cT[t].push_back(fn);
        }
    });
    for (int t = 0; t < T; ++t)
        if (errT[t]) return fail(h, ACP_ERR_INVALID, "%s", errT[t]);
    for (int t = 0; t < T; ++t) h->f2cHost.insert(h->f2cHost.end(), f2cT[t].begin(), f2cT[t].end());
    // partner strain of the coupling nodes (STD scheme, HRR or RR with cubic-Mach)
    h->partner = !direct && (d.op == OP_HRR || (d.op == OP_RR && d.cubic_mach));
    h->nbHost.clear();
    if (h->partner) {
        // record t of a level's coupling list is the partner strain of its node
        // (the node -> record map is scattered on the device, k_scatter_slots)
        F.nSlots = (int)h->c2fHost.size();
        C.nSlots = (int)h->f2cHost.size();
        auto regular = [](const LevelHost& L, long long n) { return L.code[n] < CODE_IFACE0; };
        for (int t = 0; t < h->nCoinc; ++t) {
            const C2FDev& cn = h->c2fHost[t];
            const int cc[3] = {(int)(cn.src % C.nx), (int)((cn.src / C.nx) % C.ny), (int)(cn.src / ((long long)C.nx * C.ny))};
            C2FNbDev nb;
            for (int q = 0; q < 6; ++q) {
                const int g[3] = {cc[0] + C.off[0] + ex(q), cc[1] + C.off[1] + ey(q), cc[2] + C.off[2] + ez(q)};
                long long m;
                nb.c[q] = nb.f[q] = -1;
                if (local(C, g, m) && regular(C, m)) {
                    nb.c[q] = (int)m;
                    continue;
                }
                const int gf[3] = {2 * g[0], 2 * g[1], 2 * g[2]};
                if (!local(F, gf, m) || !regular(F, m))
                    return fail(h, ACP_ERR_INVALID, "partner strain stencil missing at a coupling node");
                nb.f[q] = (int)m;
            }
            h->nbHost.push_back(nb);
        }
    }
    h->host.push_back(std::move(C));
    h->host.push_back(std::move(F));
    return ACP_OK;
}

// node classes and LODI wiring of a single level
int buildSingleLevel(acp_handle* h) {
    const acp_case_desc& d = h->d;
    LevelHost L;
    L.nx = d.nx; L.ny = d.ny; L.nz = d.nz;
    L.N = (long long)L.nx * L.ny * L.nz;
    L.code.assign(L.N, CODE_FLUID);
    const int dims[3] = {L.nx, L.ny, L.nz};
    auto idx = [&](int i, int j, int k) { return ((long long)k * L.ny + j) * L.nx + i; };
    auto wrapped = [&](int i, int j, int k, long long& out) {
        int c[3] = {i, j, k};
        for (int a = 0; a < 3; ++a)
            if (c[a] < 0 || c[a] >= dims[a]) {
                if (d.bc[a] != ACP_BC_PERIODIC) return false;
                c[a] = (c[a] % dims[a] + dims[a]) % dims[a];
            }
        out = idx(c[0], c[1], c[2]);
        return true;
    };
    for (int k = 0; k < L.nz; ++k)
        for (int j = 0; j < L.ny; ++j)
            for (int i = 0; i < L.nx; ++i) {
                const int c[3] = {i, j, k};
                int fc[3];
                for (int a = 0; a < 3; ++a)
                    fc[a] = d.bc[a] == ACP_BC_LODI ? (c[a] == 0 ? -1 : (c[a] == dims[a] - 1 ? 1 : 0)) : 0;
                if (!fc[0] && !fc[1] && !fc[2]) continue;
                const long long n = idx(i, j, k);
                L.code[n] = (uint8_t)faceCode(fc[0], fc[1], fc[2]);
                const BoundaryClass* bc = boundaryClass(fc[0], fc[1], fc[2]);
                BNodeDev b;
                b.n = n;
                b.normalDir = bc->normalDir;
                if (!wrapped(i + bc->n1[0], j + bc->n1[1], k + bc->n1[2], b.n1) ||
                    !wrapped(i + bc->n2[0], j + bc->n2[1], k + bc->n2[2], b.n2))
                    return fail(h, ACP_ERR_INVALID, "normal neighbour outside the lattice");
                for (int m = 0; m < 4; ++m) b.t[m] = -1;
                const int nface = (fc[0] != 0) + (fc[1] != 0) + (fc[2] != 0);
                b.transverse = 0;
                if (nface == 1) {
                    int t[4][3];
                    faceTangents(fc[0], fc[1], fc[2], t);
                    for (int m = 0; m < 4; ++m)
                        if (!wrapped(i + t[m][0], j + t[m][1], k + t[m][2], b.t[m]))
                            return fail(h, ACP_ERR_INVALID, "tangent neighbour outside the lattice");
                    b.transverse = d.transverse ? 1 : 0;
                }
                (fc[0] != 0 ? L.lodiX : L.lodiZY).push_back(b);
            }
    for (int a = 0; a < 3; ++a) L.per[a] = d.bc[a] == ACP_BC_PERIODIC;
    L.active = L.N;
    L.spacing = d.spacing;
    L.dt = d.spacing / (d.speed_of_sound * std::sqrt(3.0));
    const double cs2 = d.speed_of_sound * d.speed_of_sound;
    L.omega = (cs2 * L.dt) / (d.kinematic_viscosity + 0.5 * cs2 * L.dt);
    h->host.push_back(std::move(L));
    return ACP_OK;
}

template <typename S>
using CollideFn = void (*)(LevelArgs<S>);

template <typename S, typename R, int OP>
CollideFn<S> pickOrder(int order, bool) {
    switch (order) {
        case 2: return k_collide_push<S, R, OP, 2, false, false>;
        case 3: return k_collide_push<S, R, OP, 3, false, false>;
        default: return k_collide_push<S, R, OP, 4, false, false>;
    }
}

template <typename S, typename R>
CollideFn<S> pickCollide(const acp_case_desc& d) {

    switch (d.op) {
        case OP_SRT:
            switch (d.eq_order) {
                case 2: return k_collide_push<S, R, OP_SRT, 2, false, false>;
                case 3: return k_collide_push<S, R, OP_SRT, 3, false, false>;
                default: return k_collide_push<S, R, OP_SRT, 4, false, false>;
            }
        case OP_MRT_GS:
            return d.mrt_writeback ? k_collide_push<S, R, OP_MRT_GS, 2, false, true>
                                   : k_collide_push<S, R, OP_MRT_GS, 2, false, false>;
        case OP_MRT_RM:
            return d.mrt_writeback ? k_collide_push<S, R, OP_MRT_RM, 2, false, true>
                                   : k_collide_push<S, R, OP_MRT_GS, 2, false, false>;
        default: return pickOrder<S, R, OP_RR>(d.eq_order, false);
    }
}

template <typename S>
using TiledFn = void (*)(LevelArgs<S>, int);

template <typename S, typename R>
TiledFn<S> pickTiled(const acp_case_desc& d) {
    const bool cubic = d.cubic_mach != 0;
    if (d.op == OP_RR) {
        switch (d.eq_order) {
            case 2: return k_collide_push_tiled<S, R, OP_RR, 2, true>;
            case 3: return k_collide_push_tiled<S, R, OP_RR, 3, true>;
            default: return k_collide_push_tiled<S, R, OP_RR, 4, true>;
        }
    }
    switch (d.eq_order) {
        case 2: return cubic ? k_collide_push_tiled<S, R, OP_HRR, 2, true> : k_collide_push_tiled<S, R, OP_HRR, 2, false>;
        case 3: return cubic ? k_collide_push_tiled<S, R, OP_HRR, 3, true> : k_collide_push_tiled<S, R, OP_HRR, 3, false>;
        default: return cubic ? k_collide_push_tiled<S, R, OP_HRR, 4, true> : k_collide_push_tiled<S, R, OP_HRR, 4, false>;
    }
}

template <typename S>
using MarchFn = void (*)(LevelArgs<S>, int, const int*);

// the march kernel of a case: FP64 compute with its launch bound, FP32
// compute (FP32 and FP16 storage) with its direct register cap
template <typename S, typename R, int OP, int ORDER, bool CUBIC>
MarchFn<S> marchKernel() {
    if constexpr (sizeof(R) == 8) return k_collide_push_march<S, R, OP, ORDER, CUBIC>;
    else return k_collide_push_march_f32<S, R, OP, ORDER, CUBIC>;
}
template <typename S, typename R>
MarchFn<S> pickMarch(const acp_case_desc& d) {
    const bool cubic = d.cubic_mach != 0;
    if (d.op == OP_RR) {
        switch (d.eq_order) {
            case 2: return marchKernel<S, R, OP_RR, 2, true>();
            case 3: return marchKernel<S, R, OP_RR, 3, true>();
            default: return marchKernel<S, R, OP_RR, 4, true>();
        }
    }
    switch (d.eq_order) {
        case 2: return cubic ? marchKernel<S, R, OP_HRR, 2, true>() : marchKernel<S, R, OP_HRR, 2, false>();
        case 3: return cubic ? marchKernel<S, R, OP_HRR, 3, true>() : marchKernel<S, R, OP_HRR, 3, false>();
        default: return cubic ? marchKernel<S, R, OP_HRR, 4, true>() : marchKernel<S, R, OP_HRR, 4, false>();
    }
}

template <typename S>
using LodiFn = void (*)(const S*, S*, const BNodeDev*, int, LodiArgs, LevelArgs<S>, int);

template <typename S>
LodiFn<S> pickLodi(int order) {
    return order == 2 ? k_lodi<S, 2> : (order == 3 ? k_lodi<S, 3> : k_lodi<S, 4>);
}


// events recorded between the kernels of a step, for acp_step_timed
struct PhaseTimer {
    cudaEvent_t ev[32];
    int kind[32];
    int n = 0;
    cudaStream_t stream;
    void mark(int k) {
        if (n < 32) {
            kind[n] = k;
            cudaEventRecord(ev[n], stream);
            ++n;
        }
    }
};

dim3 gridOf(const LevelHost& L, int bx) { return dim3((L.nx + bx - 1) / bx, L.ny, L.nz); }

// enqueue one step of a single level, reading array src
template <typename S, typename R>
int enqueueLevelLodi(acp_handle* h, int l, int src, PhaseTimer* tm, cudaStream_t st);

// part of a level's collide: every x tile, or (y-marching levels with an
// interior / boundary split of their tiles, LevelDev::cols) the tiles that
// touch no coupling or LODI node, or the others
enum { PART_ALL = 0, PART_INTERIOR = 1, PART_BOUNDARY = 2 };

template <typename S, typename R>
int enqueueLevelStep(acp_handle* h, int l, int src, PhaseTimer* tm = nullptr, cudaStream_t st = nullptr,
                     bool lodi = true, int part = PART_ALL) {
    if (!st) st = h->stream;
    const LevelHost& L = h->host[l];
    const LevelDev& D = h->dev[l];
    LevelArgs<S> a = levelArgs<S>(h, l, src);
    const int bx = 128;
    if (tm) tm->mark(-1);
    if (needsMoments(h->d) && marchesY(L)) {
        const int chunk = marchChunkFor(L, sizeof(R));
        dim3 grid((L.nx + MARCH_STEP - 1) / MARCH_STEP, (L.ny + chunk - 1) / chunk);
        const int* cols = nullptr;
        if (part != PART_ALL && D.nInner) {
            grid.x = part == PART_INTERIOR ? D.nInner : D.nOuter;
            cols = part == PART_INTERIOR ? D.cols : D.cols + D.nInner;
        }
        const MarchFn<S> k = pickMarch<S, R>(h->d);
        if (grid.x) k<<<grid, dim3(MARCH_TX, L.nz), marchSmemBytes<R>(L.nz), st>>>(a, chunk, cols);
        noteBulk(h->bulk, (const void*)k);
    } else if (needsMoments(h->d)) {
        const int chunk = tiledChunkFor(L, TiledMinBlocks<R>::value);
        dim3 grid((L.nx + TX - 1) / TX, (L.ny + TY - 1) / TY, (L.nz + chunk - 1) / chunk);
        const TiledFn<S> k = pickTiled<S, R>(h->d);
        k<<<grid, dim3(TX, TY), 0, st>>>(a, chunk);
        noteBulk(h->bulk, (const void*)k);
    } else {
        const auto k = pickCollide<S, R>(h->d);
        k<<<gridOf(L, bx), bx, 0, st>>>(a);
        noteBulk(h->bulk, (const void*)k);
    }
    if (tm) tm->mark(ACP_K_COLLIDE);
    return lodi ? enqueueLevelLodi<S, R>(h, l, src, tm, st) : ACP_OK;
}

// the LODI passes of a level after its collide + push (reading array src)
template <typename S, typename R>
int enqueueLevelLodi(acp_handle* h, int l, int src, PhaseTimer* tm, cudaStream_t st) {
    if (!st) st = h->stream;
    const LevelDev& D = h->dev[l];
    LevelArgs<S> a = levelArgs<S>(h, l, src);
    const LodiArgs p = lodiArgsOf(h, l);
    LodiFn<S> lf = pickLodi<S>(h->d.eq_order);
    // eight lanes per boundary node (one per stencil member) and small blocks
    // spread the few thousand nodes of a face over every SM
    const int tpn = lodiLanes(h->d.transverse);
    if (D.nLodiX) lf<<<(D.nLodiX * tpn + 63) / 64, 64, 0, st>>>(a.A, a.B, D.lodiX, D.nLodiX, p, a, tpn);
    if (D.nLodiZY) lf<<<(D.nLodiZY * tpn + 63) / 64, 64, 0, st>>>(a.A, a.B, D.lodiZY, D.nLodiZY, p, a, tpn);
    if (tm && (D.nLodiX || D.nLodiZY)) tm->mark(ACP_K_LODI);
    return ACP_OK;
}

// C2F onto the fine array `fdst` from the coarse array `cnew` (blended with
// the saved coarse state by weight 1 - th); with the direct coupling the
// shared nodes are coupled both ways (th == 1) or towards the fine level
template <typename S, typename R>
void enqueueC2F(acp_handle* h, int cnew, int fdst, R th) {
    LevelArgs<S> la = levelArgs<S>(h, 1, 0);
    const CouplingArgs c = couplingArgs(h);
    const S* Bc = (const S*)h->dev[0].f[cnew];
    S* Ff = (S*)h->dev[1].f[fdst];
    const R* pre = (const R*)h->dPre;
    const int o = h->d.eq_order;
    if (h->nCoinc && !h->dcHost.empty()) {
        const unsigned g = (h->nCoinc * DC_TPN + 127) / 128;  // a warp per shared node
        S* Bw = (S*)h->dev[0].f[cnew];
        const int dc2 = h->d.coupling == ACP_COUPLING_DC2;
        if (o == 2) k_dc_couple<S, R, 2><<<g, 128, 0, h->stream>>>(Bw, Ff, h->dDC, h->nCoinc, pre, th, dc2, c, la);
        else if (o == 3) k_dc_couple<S, R, 3><<<g, 128, 0, h->stream>>>(Bw, Ff, h->dDC, h->nCoinc, pre, th, dc2, c, la);
        else k_dc_couple<S, R, 4><<<g, 128, 0, h->stream>>>(Bw, Ff, h->dDC, h->nCoinc, pre, th, dc2, c, la);
    } else if (h->nCoinc) {
        const unsigned g = (h->nCoinc * coincidentThreadsPerNode(c) + 127) / 128;
        if (o == 2) k_c2f_coincident<S, R, 2><<<g, 128, 0, h->stream>>>(Bc, Ff, h->dC2F, h->nCoinc, pre, th, c, la);
        else if (o == 3) k_c2f_coincident<S, R, 3><<<g, 128, 0, h->stream>>>(Bc, Ff, h->dC2F, h->nCoinc, pre, th, c, la);
        else k_c2f_coincident<S, R, 4><<<g, 128, 0, h->stream>>>(Bc, Ff, h->dC2F, h->nCoinc, pre, th, c, la);
    }
    const int comps = interpComponents(h);
    if (h->nMid)
        k_c2f_interp<S, R><<<(h->nMid * comps + 255) / 256, 256, 0, h->stream>>>(Ff, h->dC2F + h->nCoinc, h->nMid, c,
                                                                                    la);
    if (h->nCen)
        k_c2f_interp<S, R><<<(h->nCen * comps + 255) / 256, 256, 0, h->stream>>>(Ff, h->dC2F + h->nCoinc + h->nMid,
                                                                                    h->nCen, c, la);
}

// one coarse step: single level, or the two-level sequence of
// Lattice::nestedTimeStepping* (Lattice.cpp:4354-5771)
template <typename S, typename R>
int enqueueStepT(acp_handle* h, int src, PhaseTimer* tm) {
    if (h->host.size() == 1) {
        enqueueLevelStep<S, R>(h, 0, src, tm);
    } else {
        LevelArgs<S> lc = levelArgs<S>(h, 0, src);
        const CouplingArgs c = couplingArgs(h);
        // in a captured graph three branches run side by side where the kernels
        // touch disjoint data: the coarse step (with the saving of the coupling
        // sources) beside the first fine sub-step; the fine level's LODI passes
        // (domain-face nodes and their normal neighbours) beside the coupling
        // kernels (coupling nodes: a coupling node on a LODI face is refused at
        // set-up); F2C (coarse coupling nodes from a fine cube two cells inside
        // the box) beside the last C2F (fine coupling nodes from regular coarse
        // nodes).  Timed runs (tm) keep one stream.
        const bool fork = tm == nullptr;
        cudaStream_t cs = h->stream, ls = h->stream, fs = h->stream;
        auto branch = [h](cudaStream_t to, cudaEvent_t ev) {
            cudaEventRecord(ev, h->stream);
            cudaStreamWaitEvent(to, ev, 0);
        };
        auto join = [h](cudaStream_t from, cudaEvent_t ev) {
            cudaEventRecord(ev, from);
            cudaStreamWaitEvent(h->stream, ev, 0);
        };
        if (fork) {
            branch(h->side, h->forkEv);
            cs = h->side;
            ls = h->side2;
            fs = h->side;
        }
        if (tm) tm->mark(-1);
        if (h->nCoinc)
            k_c2f_save<S, R><<<(h->nCoinc * coincidentThreadsPerNode(c) + 127) / 128, 128, 0, cs>>>(
                lc.A, h->dC2F, h->nCoinc, (R*)h->dPre, lc, c);
        if (tm) tm->mark(ACP_K_COUPLING);
        enqueueLevelStep<S, R>(h, 0, src, tm, cs);  // coarse t -> t+1
        enqueueLevelStep<S, R>(h, 1, 0, tm, h->stream, false);  // fine t -> t+1/2
        // the interior tiles of the next fine sub-step need only this one
        const bool split = fork && h->dev[1].nInner > 0;
        if (split) {
            branch(h->side3, h->splitEv[0]);
            enqueueLevelStep<S, R>(h, 1, 1, tm, h->side3, false, PART_INTERIOR);  // fine t+1/2 -> t+1, inside
        }
        if (fork) branch(ls, h->branchEv[0]);
        enqueueLevelLodi<S, R>(h, 1, 0, tm, ls);
        if (fork) join(h->side, h->joinEv);
        if (tm) tm->mark(-1);
        enqueueC2F<S, R>(h, 1 - src, 1, R(0.5));  // C2F at t+1/2
        if (tm) tm->mark(ACP_K_COUPLING);
        if (fork) join(ls, h->branchEv[1]);
        // the LODI passes at t+1, F2C and the last C2F read and write only
        // nodes within four of a LODI or coupling face: with the tiles split
        // they follow the face tiles and run beside the interior tiles' last
        // waves
        if (split) enqueueLevelStep<S, R>(h, 1, 1, tm, h->stream, false, PART_BOUNDARY);  // the face tiles
        else enqueueLevelStep<S, R>(h, 1, 1, tm, h->stream, false);                       // fine t+1/2 -> t+1
        if (fork) branch(ls, h->branchEv[2]);
        enqueueLevelLodi<S, R>(h, 1, 1, tm, ls);
        if (tm) tm->mark(-1);
        if (!h->f2cHost.empty()) {  // STD only: the direct coupling does F2C in its t+1 pass
            if (fork) branch(fs, h->branchEv[3]);
            LevelArgs<S> lf = levelArgs<S>(h, 1, 0);
            const unsigned g = ((unsigned)h->f2cHost.size() * 32 + 127) / 128;  // a warp per coarse node
            const S* Ff = (const S*)h->dev[1].f[0];
            S* Bc = (S*)h->dev[0].f[1 - src];
            const int n = (int)h->f2cHost.size();
            const int o = h->d.eq_order;
            if (o == 2) k_f2c<S, R, 2><<<g, 128, 0, fs>>>(Ff, Bc, h->dF2C, n, c, lf);
            else if (o == 3) k_f2c<S, R, 3><<<g, 128, 0, fs>>>(Ff, Bc, h->dF2C, n, c, lf);
            else k_f2c<S, R, 4><<<g, 128, 0, fs>>>(Ff, Bc, h->dF2C, n, c, lf);
        }
        enqueueC2F<S, R>(h, 1 - src, 0, R(1.0));  // C2F at t+1
        if (tm) tm->mark(ACP_K_COUPLING);
        if (fork) {
            if (!h->f2cHost.empty()) join(fs, h->branchEv[4]);
            join(ls, h->branchEv[5]);
            if (split) join(h->side3, h->splitEv[1]);
        }
    }
    if (h->nProbes) {
        launchProbes<S>(h, h->stream, 1 - src);
        if (tm) tm->mark(ACP_K_PROBES);
    }
    return ACP_OK;
}

int enqueueStep(acp_handle* h, int src, PhaseTimer* tm = nullptr) {
    switch (h->d.storage) {
        case ACP_STORE_F64: return enqueueStepT<double, double>(h, src, tm);
        case ACP_STORE_F32_DEV: return enqueueStepT<float, float>(h, src, tm);
        default: return enqueueStepT<__half, float>(h, src, tm);
    }
}

int launchesPerStep(const acp_handle* h) {
    int n = 0;
    for (size_t l = 0; l < h->host.size(); ++l) {
        const int per = 1 + (h->dev[l].nLodiX ? 1 : 0) + (h->dev[l].nLodiZY ? 1 : 0);
        n += l == 0 ? per : 2 * per;  // the fine level takes two sub-steps
    }
    if (h->host.size() == 2) {
        const int c2f = (h->nCoinc ? 1 : 0) + (h->nMid ? 1 : 0) + (h->nCen ? 1 : 0);
        n += (h->nCoinc ? 1 : 0) + 2 * c2f + (h->f2cHost.empty() ? 0 : 1);
        if (h->dev[1].nInner) ++n;  // the second fine collide as interior and boundary tiles
    }
    if (h->nProbes) ++n;
    return n;
}

void destroyGraphs(acp_handle* h) {
    for (int p = 0; p < 2; ++p)
        if (h->graph[p]) {
            cudaGraphExecDestroy(h->graph[p]);
            h->graph[p] = nullptr;
        }
}

int captureGraphs(acp_handle* h) {
    destroyGraphs(h);
    for (int p = 0; p < 2; ++p) {
        cudaGraph_t g;
        h->bulk.clear();
        CU(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        enqueueStep(h, p);
        cudaError_t e = cudaStreamEndCapture(h->stream, &g);
        if (e != cudaSuccess) return fail(h, ACP_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
        e = instantiateWithPriorities(&h->graph[p], g, h->bulk);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(h, ACP_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    }
    return ACP_OK;
}

template <typename S>
void launchToF64(acp_handle* h, int l, int arr, double* dst) {
    LevelArgs<S> a = levelArgs<S>(h, l, 0);
    long long total = h->host[l].N * Q;
    k_to_f64<S><<<(unsigned)((total + 255) / 256), 256, 0, h->stream>>>((const S*)h->dev[l].f[arr], dst, h->host[l].N,
                                                                         h->shift, a);
}
template <typename S>
void launchFromF64(acp_handle* h, int l, const double* src) {
    LevelArgs<S> a = levelArgs<S>(h, l, 0);
    long long total = h->host[l].N * Q;
    k_from_f64<S><<<(unsigned)((total + 255) / 256), 256, 0, h->stream>>>(src, (S*)h->dev[l].f[0], (S*)h->dev[l].f[1],
                                                                           h->host[l].N, h->shift, a);
}
template <typename S>
void launchInit(acp_handle* h, int l) {
    LevelArgs<S> a = levelArgs<S>(h, l, 0);
    const LevelHost& L = h->host[l];
    InitArgs ia;
    ia.ic = h->d.ic;
    ia.spacingLevel = h->d.spacing / std::pow(2.0, (double)l);
    ia.halfDomain[0] = h->d.domain_size[0] / 2.;
    ia.halfDomain[1] = h->d.domain_size[1] / 2.;
    ia.rho0 = h->d.density;
    ia.eps = h->d.ic_eps;
    ia.b = h->d.ic_b;
    ia.cell = 1.0 / std::pow(2.0, (double)l);
    for (int c = 0; c < 3; ++c) {
        ia.center[c] = h->d.ic_center[c];
        ia.off[c] = L.off[c];
    }
    ia.dims3 = h->d.ic_dims == 3;
    k_init<S><<<gridOf(L, 128), 128, 0, h->stream>>>(a, ia);
}

// node -> coupling record map of a level: slot[recs[t].n] = t (the map is
// -1 elsewhere, set by a memset before)
template <typename Rec>
__global__ void k_scatter_slots(int* slot, const Rec* recs, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) slot[recs[t].n] = t;
}

// Device memory of the lattices.  Blocks that a destroyed lattice (or a
// replaced probe set) frees are kept per device and rounded size and handed
// to the next allocation of that size, so a process that creates lattices
// one after another (a serving loop, repeated solves) skips cudaMalloc and
// cudaFree.  Sizes round up to 64 KiB below 1 MiB and to 2 MiB above; a
// device keeps at most a quarter of its memory this way; an allocation that
// cudaMalloc refuses first returns the kept blocks of its device and retries.
// Freeing synchronises the device first, as cudaFree does.
struct DeviceBlocks {
    std::mutex m;
    std::map<std::pair<int, size_t>, std::vector<void*>> free;  // (device, rounded size) -> blocks
    std::unordered_map<void*, std::pair<int, size_t>> live;     // block -> (device, rounded size)
    std::map<int, size_t> kept, limit;                            // per device: bytes kept, most kept
};
DeviceBlocks& deviceBlocks() {
    static DeviceBlocks* b = new DeviceBlocks();  // kept until the process exits
    return *b;
}
size_t roundDeviceBlock(size_t bytes) {
    const size_t g = bytes <= ((size_t)1 << 20) ? ((size_t)1 << 16) : ((size_t)2 << 20);
    return (std::max<size_t>(bytes, 1) + g - 1) / g * g;
}
void releaseDeviceBlocks(int device) {
    DeviceBlocks& db = deviceBlocks();
    std::vector<void*> out;
    {
        std::lock_guard<std::mutex> g(db.m);
        for (auto& kv : db.free)
            if (kv.first.first == device) {
                out.insert(out.end(), kv.second.begin(), kv.second.end());
                kv.second.clear();
            }
        db.kept[device] = 0;
    }
    for (void* p : out) cudaFree(p);
}

int devAlloc(acp_handle* h, void** p, size_t bytes) {
    DeviceBlocks& db = deviceBlocks();
    const size_t r = roundDeviceBlock(bytes);
    {
        std::lock_guard<std::mutex> g(db.m);
        auto it = db.free.find({h->device, r});
        if (it != db.free.end() && !it->second.empty()) {
            *p = it->second.back();
            it->second.pop_back();
            db.kept[h->device] -= r;
            db.live[*p] = {h->device, r};
            h->devBytes += bytes;
            return ACP_OK;
        }
    }
    cudaError_t e = cudaMalloc(p, r);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        releaseDeviceBlocks(h->device);
        e = cudaMalloc(p, r);
    }
    if (e != cudaSuccess) return fail(h, ACP_ERR_NOMEM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    std::lock_guard<std::mutex> g(db.m);
    db.live[*p] = {h->device, r};
    if (!db.limit.count(h->device)) {
        size_t fr = 0, total = 0;
        db.limit[h->device] = cudaMemGetInfo(&fr, &total) == cudaSuccess ? total / 4 : 0;
    }
    h->devBytes += bytes;
    return ACP_OK;
}

// returns a block of devAlloc (kept for reuse) or frees any other device pointer
void devFree(void* p) {
    if (!p) return;
    cudaDeviceSynchronize();  // no kernel may still use the block when it is handed out again
    DeviceBlocks& db = deviceBlocks();
    {
        std::lock_guard<std::mutex> g(db.m);
        auto it = db.live.find(p);
        if (it != db.live.end()) {
            const int dev = it->second.first;
            const size_t r = it->second.second;
            db.live.erase(it);
            if (db.kept[dev] + r <= db.limit[dev]) {
                db.free[{dev, r}].push_back(p);
                db.kept[dev] += r;
                return;
            }
        }
    }
    cudaFree(p);
}

size_t estimateBytes(const acp_case_desc& d) {
    const size_t per = 2 * Q * storageBytes(d.storage) + 1;  // two population arrays and the node class
    long long nodes = (long long)d.nx * d.ny * d.nz;
    long long surf = 2LL * ((long long)d.nx * d.ny + (long long)d.ny * d.nz + (long long)d.nx * d.nz);
    if (d.max_level == 1 && d.layout == ACP_LAYOUT_SHELL) {
        // coarse core (at most the domain) and the fine level over the whole domain
        const long long fine = (2LL * d.nx - 1) * (2LL * d.ny - 1) * (2LL * d.nz - 1);
        const long long fsurf = 2 * ((2LL * d.nx) * (2LL * d.ny) + (2LL * d.ny) * (2LL * d.nz) + (2LL * d.nx) * (2LL * d.nz));
        const size_t rb = d.storage == ACP_STORE_F64 ? 8 : 4;
        return (size_t)(nodes + fine) * per + (size_t)fsurf * sizeof(BNodeDev) +
               (size_t)surf * (sizeof(C2FDev) + sizeof(F2CDev) / 4 + sizeof(DCDev) / 4 + Q * rb);
    }
    if (d.max_level == 1) {
        const int dom[3] = {d.nx, d.ny, d.nz};
        long long f[3];
        for (int a = 0; a < 3; ++a) {
            const bool spans = d.box_lo[a] == 0 && d.box_hi[a] == dom[a] - 1;
            f[a] = spans && d.bc[a] == ACP_BC_PERIODIC ? 2LL * dom[a] : 2LL * (d.box_hi[a] - d.box_lo[a]) + 1;
        }
        nodes += f[0] * f[1] * f[2];
        const long long fsurf = 2 * (f[0] * f[1] + f[1] * f[2] + f[0] * f[2]);
        surf += fsurf;
        // coupling lists and the saved coarse populations
        const size_t rb = d.storage == ACP_STORE_F64 ? 8 : 4;
        return (size_t)nodes * per + (size_t)surf * sizeof(BNodeDev) +
               (size_t)fsurf * (sizeof(C2FDev) + sizeof(F2CDev) / 4 + sizeof(DCDev) / 4 + Q * rb);
    }
    return (size_t)nodes * per + (size_t)surf * sizeof(BNodeDev);
}

}  // namespace

// Device scratch of acp_read_populations_window: the FP64 copy of one window
// of nodes lives in this fixed array instead of a per-call allocation.
static __device__ __align__(256) double g_windowScratch[(size_t)ACP_WINDOW_MAX_NODES * Q];

namespace {
// device address of g_windowScratch in the current context (the handle's
// device is current).  It is looked up on every call rather than cached: the
// address belongs to the context the module was loaded into, so after the
// application destroys and recreates a device's context (cudaDeviceReset)
// the next call gets the new address instead of a stale one.  The lookup
// allocates nothing.
int windowScratch(acp_handle* h, double** out) {
    double* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_windowScratch);
    if (e != cudaSuccess) return fail(h, ACP_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    *out = p;
    return ACP_OK;
}

template <typename S>
void launchWindow(acp_handle* h, int l, int arr, long long begin, int count, double* dst) {
    LevelArgs<S> a = levelArgs<S>(h, l, 0);
    const long long total = (long long)count * Q;
    k_to_f64_window<S><<<(unsigned)((total + 255) / 256), 256, 0, h->stream>>>((const S*)h->dev[l].f[arr], dst,
                                                                                h->host[l].N, begin, count, h->shift, a);
}
}  // namespace

extern "C" {

void acp_default_case(acp_case_desc* d) {
    std::memset(d, 0, sizeof *d);
    d->spacing = 2.0e-2;
    d->domain_size[0] = 3.0; d->domain_size[1] = 3.0; d->domain_size[2] = 0.4;
    d->nx = 151; d->ny = 151; d->nz = 21;
    d->density = 1.17621;
    d->kinematic_viscosity = 1.49e-5;
    d->speed_of_sound = 347.3;
    d->mach = 0.0;
    d->op = ACP_OP_HRR;
    d->eq_order = 3;
    d->hybrid_sigma = 0.98;
    d->bc[0] = d->bc[1] = d->bc[2] = ACP_BC_LODI;
    d->k1 = 1.0;
    d->ref_layer_yz = 4; d->ref_layer_x = 75; d->overlap = 1;
    d->c2f_replace = ACP_C2F_FALL;
    d->f2c_replace = ACP_F2C_CALL;
    d->ic = ACP_IC_REFERENCE;
    d->ic_eps = 1e-3; d->ic_b = 6.0; d->ic_dims = 2;
    d->storage = ACP_STORE_F64;
}

int acp_estimate_bytes(const acp_case_desc* d, size_t* bytes) {
    std::string why;
    int s = validate(d, why);
    if (s) return s;
    *bytes = estimateBytes(*d);
    return ACP_OK;
}

// The x tiles of the fine level's y-marching collide (STD coupling, x not
// periodic) split into those with no coupling or LODI node within reach and
// the others (LevelDev::cols).  A tile reads and pushes within x0 - 1 ..
// x0 + 30; four more nodes each side are kept clear, the depth of the fine
// nodes F2C and the partner strain read behind a coupling face.  The second
// fine sub-step runs the first kind beside the first C2F and the fine LODI
// passes (those write only coupling and LODI nodes of the array the tiles
// read, and read only LODI nodes of the array the tiles write), and F2C and
// the last C2F beside its last waves.
int splitFineTiles(acp_handle* h) {
    const LevelHost& F = h->host[1];
    if (!h->dcHost.empty() || !needsMoments(h->d) || !marchesY(F) || F.per[0]) return ACP_OK;
    const int ntx = (F.nx + MARCH_STEP - 1) / MARCH_STEP;
    std::vector<char> hit(ntx, 0);
    auto mark = [&](long long n) {
        const int x = (int)(n % F.nx);
        for (int bx = std::max(0, (x - 34) / MARCH_STEP - 1); bx <= std::min(ntx - 1, (x + 5) / MARCH_STEP + 1); ++bx)
            if (x >= bx * MARCH_STEP - 5 && x <= bx * MARCH_STEP + 34) hit[bx] = 1;
    };
    for (const long long n : F.coupling) mark(n);
    for (const BNodeDev& b : F.lodiX) mark(b.n);
    for (const BNodeDev& b : F.lodiZY) mark(b.n);
    std::vector<int> cols;
    for (int bx = 0; bx < ntx; ++bx)
        if (!hit[bx]) cols.push_back(bx);
    const int inner = (int)cols.size();
    if (inner == 0 || inner == ntx) return ACP_OK;
    for (int bx = 0; bx < ntx; ++bx)
        if (hit[bx]) cols.push_back(bx);
    LevelDev& D = h->dev[1];
    int s = devAlloc(h, (void**)&D.cols, cols.size() * sizeof(int));
    if (s) return s;
    CU(h, cudaMemcpyAsync(D.cols, cols.data(), cols.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    D.nInner = inner;
    D.nOuter = ntx - inner;
    return ACP_OK;
}

int acp_create(const acp_case_desc* d, int device, acp_handle** out) {
    if (!out) return ACP_ERR_INVALID;
    *out = nullptr;
    std::string why;
    int s = validate(d, why);
    acp_handle* h = new acp_handle();
    if (s) {
        h->err = why;
        *out = h;  // handle carries the error text; caller destroys it
        return s;
    }
    h->d = *d;
    if (device < 0) {
        if (cudaGetDevice(&h->device) != cudaSuccess) h->device = 0;
    } else {
        h->device = device;
    }
    *out = h;
    CU(h, cudaSetDevice(h->device));
    if ((s = uploadConstants(h->device))) return fail(h, s, "uploading lattice constants failed");
    h->c = d->speed_of_sound * std::sqrt(3.0);
    h->kappa = 1.0 / (6.0 * h->c * h->c);
    h->shift = d->storage == ACP_STORE_F64 ? 0.0 : d->density;
    if (d->eq_order == 4) {
        // projection of the orthogonalised fourth-order Hermite terms on H2,
        // nonzero when kappa differs from the lattice-unit value 1/6
        for (int q = 0; q < Q; ++q) {
            const double hxx = ex(q) * ex(q) - 1.0 / 3.0, hyy = ey(q) * ey(q) - 1.0 / 3.0, hzz = ez(q) * ez(q) - 1.0 / 3.0;
            const double h2[6] = {hxx, hyy, hzz, (double)(ex(q) * ey(q)), (double)(ex(q) * ez(q)), (double)(ey(q) * ez(q))};
            double f0 = hxx * hyy + h->kappa * hzz;
            double f1 = hxx * hzz + h->kappa * hyy + 2.0 / 7.0 * f0;
            double f2 = hyy * hzz + h->kappa * hxx + 2.0 / 7.0 * f0 + 2.0 / 5.0 * f1;
            const double h4[3] = {8.0 / 7.0 * f0, 56.0 / 45.0 * f1, 40.0 / 27.0 * f2};
            for (int ab = 0; ab < 6; ++ab)
                for (int k = 0; k < 3; ++k) h->m4[ab * 3 + k] += wq(q) * h2[ab] * h4[k];
        }
    }
    for (int q = 0; q < Q; ++q) h->hscale[q] = 1.0f;
    if (d->storage == ACP_STORE_F16_DEV) {
        // power-of-two scale per population: the deviation w_q * drho of a
        // pulse of relative amplitude eps stays inside the FP16 normal range
        const double amp = std::max(d->ic == ACP_IC_GAUSSIAN ? d->ic_eps : 0.01, 1e-6) * d->density;
        for (int q = 0; q < Q; ++q) {
            const double mag = 4.0 * amp * wq(q);
            h->hscale[q] = (float)std::ldexp(1.0, (int)std::ceil(std::log2(mag)) - 14);
        }
    }
    s = d->max_level == 1 ? buildTwoLevel(h) : buildSingleLevel(h);
    if (s) return s;
    CU(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->ownStream = true;
    CU(h, cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
    CU(h, cudaEventCreateWithFlags(&h->forkEv, cudaEventDisableTiming));
    CU(h, cudaEventCreateWithFlags(&h->joinEv, cudaEventDisableTiming));
    CU(h, cudaStreamCreateWithFlags(&h->side2, cudaStreamNonBlocking));
    for (cudaEvent_t& e : h->branchEv) CU(h, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CU(h, cudaStreamCreateWithFlags(&h->side3, cudaStreamNonBlocking));
    for (cudaEvent_t& e : h->splitEv) CU(h, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    if ((s = devAlloc(h, (void**)&h->dErr, sizeof(int)))) return s;
    CU(h, cudaMemsetAsync(h->dErr, 0, sizeof(int), h->stream));
    h->dev.resize(h->host.size());
    const size_t sb = storageBytes(d->storage);
    for (size_t l = 0; l < h->host.size(); ++l) {
        LevelHost& L = h->host[l];
        LevelDev& D = h->dev[l];
        for (int a = 0; a < 2; ++a)
            if ((s = devAlloc(h, &D.f[a], (size_t)L.N * Q * sb))) return s;
        if ((s = devAlloc(h, (void**)&D.code, (size_t)L.N))) return s;
        CU(h, cudaMemcpyAsync(D.code, L.code.data(), (size_t)L.N, cudaMemcpyHostToDevice, h->stream));
        D.nLodiX = (int)L.lodiX.size();
        D.nLodiZY = (int)L.lodiZY.size();
        if (D.nLodiX) {
            if ((s = devAlloc(h, (void**)&D.lodiX, L.lodiX.size() * sizeof(BNodeDev)))) return s;
            CU(h, cudaMemcpyAsync(D.lodiX, L.lodiX.data(), L.lodiX.size() * sizeof(BNodeDev), cudaMemcpyHostToDevice,
                                  h->stream));
        }
        if (D.nLodiZY) {
            if ((s = devAlloc(h, (void**)&D.lodiZY, L.lodiZY.size() * sizeof(BNodeDev)))) return s;
            CU(h, cudaMemcpyAsync(D.lodiZY, L.lodiZY.data(), L.lodiZY.size() * sizeof(BNodeDev),
                                  cudaMemcpyHostToDevice, h->stream));
        }
    }
    if (h->host.size() == 2) {
        const size_t rb = d->storage == ACP_STORE_F64 ? sizeof(double) : sizeof(float);
        if (!h->c2fHost.empty()) {
            if ((s = devAlloc(h, (void**)&h->dC2F, h->c2fHost.size() * sizeof(C2FDev)))) return s;
            CU(h, cudaMemcpyAsync(h->dC2F, h->c2fHost.data(), h->c2fHost.size() * sizeof(C2FDev),
                                  cudaMemcpyHostToDevice, h->stream));
        }
        if (h->nCoinc && (s = devAlloc(h, &h->dPre, (size_t)h->nCoinc * Q * rb))) return s;
        if (h->partner) {
            for (int l = 0; l < 2; ++l) {
                LevelHost& L = h->host[l];
                LevelDev& D = h->dev[l];
                if ((s = devAlloc(h, (void**)&D.slot, (size_t)L.N * sizeof(int)))) return s;
                CU(h, cudaMemsetAsync(D.slot, 0xFF, (size_t)L.N * sizeof(int), h->stream));  // -1: no record
                if ((s = devAlloc(h, (void**)&D.sg, std::max<size_t>(1, (size_t)L.nSlots) * 12 * sizeof(double)))) return s;
                CU(h, cudaMemsetAsync(D.sg, 0, std::max<size_t>(1, (size_t)L.nSlots) * 12 * sizeof(double), h->stream));
            }
            if (h->nCoinc) {
                if ((s = devAlloc(h, (void**)&h->dNb, h->nbHost.size() * sizeof(C2FNbDev)))) return s;
                CU(h, cudaMemcpyAsync(h->dNb, h->nbHost.data(), h->nbHost.size() * sizeof(C2FNbDev),
                                      cudaMemcpyHostToDevice, h->stream));
                if ((s = devAlloc(h, &h->dPreNb, (size_t)h->nCoinc * 24 * rb))) return s;
            }
        }
        if (!h->dcHost.empty()) {
            if ((s = devAlloc(h, (void**)&h->dDC, h->dcHost.size() * sizeof(DCDev)))) return s;
            CU(h, cudaMemcpyAsync(h->dDC, h->dcHost.data(), h->dcHost.size() * sizeof(DCDev), cudaMemcpyHostToDevice,
                                  h->stream));
        }
        if (!h->f2cHost.empty()) {
            if ((s = devAlloc(h, (void**)&h->dF2C, h->f2cHost.size() * sizeof(F2CDev)))) return s;
            CU(h, cudaMemcpyAsync(h->dF2C, h->f2cHost.data(), h->f2cHost.size() * sizeof(F2CDev),
                                  cudaMemcpyHostToDevice, h->stream));
        }
        if (h->partner) {
            const int nf = (int)h->c2fHost.size(), nc = (int)h->f2cHost.size();
            if (nf) k_scatter_slots<C2FDev><<<(nf + 255) / 256, 256, 0, h->stream>>>(h->dev[1].slot, h->dC2F, nf);
            if (nc) k_scatter_slots<F2CDev><<<(nc + 255) / 256, 256, 0, h->stream>>>(h->dev[0].slot, h->dF2C, nc);
            CU(h, cudaGetLastError());
        }
        if ((s = splitFineTiles(h))) return s;
    }
    CU(h, cudaStreamSynchronize(h->stream));
    return ACP_OK;
}

int acp_init(acp_handle* h) {
    if (!h || h->dev.empty()) return ACP_ERR_STATE;
    CU(h, cudaSetDevice(h->device));
    for (size_t l = 0; l < h->host.size(); ++l) {
        switch (h->d.storage) {
            case ACP_STORE_F64: launchInit<double>(h, (int)l); break;
            case ACP_STORE_F32_DEV: launchInit<float>(h, (int)l); break;
            default: launchInit<__half>(h, (int)l); break;
        }
    }
    CU(h, cudaGetLastError());
    for (size_t l = 0; l < h->dev.size(); ++l)
        if (h->dev[l].sg)
            CU(h, cudaMemsetAsync(h->dev[l].sg, 0, std::max<size_t>(1, (size_t)h->host[l].nSlots) * 12 * sizeof(double),
                                  h->stream));
    h->cur = 0;
    h->steps = 0;
    if (h->dCounter) CU(h, cudaMemsetAsync(h->dCounter, 0, sizeof(int), h->stream));
    CU(h, cudaMemsetAsync(h->dErr, 0, sizeof(int), h->stream));
    int s = captureGraphs(h);
    if (s) return s;
    h->inited = true;
    return ACP_OK;
}

int acp_step(acp_handle* h, int n) {
    if (!h || !h->inited) return ACP_ERR_STATE;
    if (h->batch) return fail(h, ACP_ERR_STATE, "the case is stepped by its batch (acp_batch_step)");
    if (n < 0) return fail(h, ACP_ERR_INVALID, "negative step count");
    CU(h, cudaSetDevice(h->device));
    for (int s = 0; s < n; ++s) {
        CU(h, cudaGraphLaunch(h->graph[h->cur], h->stream));
        h->cur ^= 1;
        ++h->steps;
    }
    return ACP_OK;
}

int acp_sync(acp_handle* h) {
    if (!h) return ACP_ERR_INVALID;
    if (h->dev.empty()) return ACP_ERR_STATE;
    CU(h, cudaSetDevice(h->device));
    joinBatch(h);
    int flag = 0;
    CU(h, cudaMemcpyAsync(&flag, h->dErr, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CU(h, cudaStreamSynchronize(h->stream));
    if (flag) return fail(h, ACP_ERR_NUMERIC, "boundary density left [0.5, 1.5] x rho0 or became NaN");
    return ACP_OK;
}

int acp_level_dims(acp_handle* h, int level, int dims[3]) {
    if (!h || level < 0 || level >= (int)h->host.size()) return ACP_ERR_INVALID;
    dims[0] = h->host[level].nx; dims[1] = h->host[level].ny; dims[2] = h->host[level].nz;
    return ACP_OK;
}

int acp_level_origin(acp_handle* h, int level, int origin[3]) {
    if (!h || !origin || level < 0 || level >= (int)h->host.size()) return ACP_ERR_INVALID;
    for (int a = 0; a < 3; ++a) origin[a] = h->host[level].off[a];
    return ACP_OK;
}

int acp_active_updates(acp_handle* h, long long* coarse, long long* fine) {
    if (!h || h->host.empty()) return ACP_ERR_STATE;
    *coarse = h->host[0].active;
    *fine = h->host.size() > 1 ? h->host[1].active : 0;
    return ACP_OK;
}

// FP64 populations of ping-pong array `arr` of a level into host memory
static int readArray(acp_handle* h, int level, int arr, double* out) {
    CU(h, cudaSetDevice(h->device));
    joinBatch(h);
    const LevelHost& L = h->host[level];
    double* tmp = nullptr;
    CU(h, cudaMallocAsync((void**)&tmp, (size_t)L.N * Q * sizeof(double), h->stream));
    switch (h->d.storage) {
        case ACP_STORE_F64: launchToF64<double>(h, level, arr, tmp); break;
        case ACP_STORE_F32_DEV: launchToF64<float>(h, level, arr, tmp); break;
        default: launchToF64<__half>(h, level, arr, tmp); break;
    }
    cudaError_t e = cudaMemcpyAsync(out, tmp, (size_t)L.N * Q * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    cudaFreeAsync(tmp, h->stream);
    if (e != cudaSuccess) return fail(h, ACP_ERR_CUDA, "copy: %s", cudaGetErrorString(e));
    CU(h, cudaStreamSynchronize(h->stream));
    return ACP_OK;
}

int acp_read_populations(acp_handle* h, int level, double* out) {
    if (!h || !out || level < 0 || level >= (int)h->host.size()) return ACP_ERR_INVALID;
    return readArray(h, level, level == 0 ? h->cur : 0, out);
}

int acp_node_kind(acp_handle* h, int level, int i, int j, int k, int* id, int* face_class) {
    if (!h || !id || !face_class || level < 0 || level >= (int)h->host.size()) return ACP_ERR_INVALID;
    const LevelHost& L = h->host[level];
    const int c[3] = {i - L.off[0], j - L.off[1], k - L.off[2]};
    *id = -1;
    *face_class = CODE_FLUID;
    if (c[0] < 0 || c[1] < 0 || c[2] < 0 || c[0] >= L.nx || c[1] >= L.ny || c[2] >= L.nz) return ACP_OK;
    const uint8_t code = L.code[((long long)c[2] * L.ny + c[1]) * L.nx + c[0]];
    if (code == CODE_DEAD) return ACP_OK;
    if (code == CODE_FLUID) {
        *id = 0;
    } else if (code < CODE_IFACE0) {
        *id = 1;
        *face_class = code;
    } else {
        *id = 2;
        *face_class = code - CODE_IFACE0;
    }
    return ACP_OK;
}

int acp_read_populations_other(acp_handle* h, int level, double* out) {
    if (!h || !out || level < 0 || level >= (int)h->host.size()) return ACP_ERR_INVALID;
    return readArray(h, level, level == 0 ? (h->cur ^ 1) : 1, out);
}

// the x-columns [x0, x0 + ncols) of a single-level case's current array in
// storage form, as one strided copy: the array is 19 * nz * ny rows of nx
// values, the columns a block of ncols values in every row
static int columnsCopy(acp_handle* h, int ncols, void* dst, size_t dpitch, const void* src, size_t spitch,
                       size_t rows) {
    const size_t sb = storageBytes(h->d.storage);
    CU(h, cudaMemcpy2DAsync(dst, dpitch, src, spitch, (size_t)ncols * sb, rows, cudaMemcpyDefault, h->stream));
    CU(h, cudaStreamSynchronize(h->stream));
    return ACP_OK;
}

static int columnsCheck(acp_handle* h, int x0, int ncols) {
    if (!h || h->host.size() != 1) return h ? fail(h, ACP_ERR_UNSUPPORTED, "columns: single-level cases only")
                                            : ACP_ERR_INVALID;
    if (!h->inited) return fail(h, ACP_ERR_STATE, "columns: case not initialised");
    if (h->batch) return fail(h, ACP_ERR_STATE, "columns: the case is stepped by a batch");
    const LevelHost& L = h->host[0];
    if (ncols < 0 || x0 < 0 || x0 > L.nx - ncols) return fail(h, ACP_ERR_INVALID, "columns [%d, %d) outside 0..%d", x0,
                                                               x0 + ncols, L.nx);
    return ACP_OK;
}

int acp_get_columns(acp_handle* h, int x0, int ncols, void* buf) {
    int s = columnsCheck(h, x0, ncols);
    if (s) return s;
    if (!buf) return fail(h, ACP_ERR_INVALID, "columns: null buffer");
    CU(h, cudaSetDevice(h->device));
    const LevelHost& L = h->host[0];
    const size_t sb = storageBytes(h->d.storage);
    const char* arr = (const char*)h->dev[0].f[h->cur] + (size_t)x0 * sb;
    return columnsCopy(h, ncols, buf, (size_t)ncols * sb, arr, (size_t)L.nx * sb, (size_t)Q * L.ny * L.nz);
}

int acp_put_columns(acp_handle* h, int x0, int ncols, const void* buf) {
    int s = columnsCheck(h, x0, ncols);
    if (s) return s;
    if (!buf) return fail(h, ACP_ERR_INVALID, "columns: null buffer");
    CU(h, cudaSetDevice(h->device));
    const LevelHost& L = h->host[0];
    const size_t sb = storageBytes(h->d.storage);
    char* arr = (char*)h->dev[0].f[h->cur] + (size_t)x0 * sb;
    return columnsCopy(h, ncols, arr, (size_t)L.nx * sb, buf, (size_t)ncols * sb, (size_t)Q * L.ny * L.nz);
}

int acp_copy_columns(acp_handle* dst, int dst_x0, acp_handle* src, int src_x0, int ncols) {
    int s = columnsCheck(dst, dst_x0, ncols);
    if (s) return s;
    if ((s = columnsCheck(src, src_x0, ncols))) return fail(dst, s, "source: %s", src->err.c_str());
    const LevelHost& D = dst->host[0];
    const LevelHost& S = src->host[0];
    if (D.ny != S.ny || D.nz != S.nz || dst->d.storage != src->d.storage || dst->shift != src->shift)
        return fail(dst, ACP_ERR_INVALID, "columns: the cases differ in ny, nz or storage form");
    CU(dst, cudaSetDevice(src->device));
    CU(dst, cudaStreamSynchronize(src->stream));  // the source's queued steps
    CU(dst, cudaSetDevice(dst->device));
    const size_t sb = storageBytes(dst->d.storage);
    char* d = (char*)dst->dev[0].f[dst->cur] + (size_t)dst_x0 * sb;
    const char* sp = (const char*)src->dev[0].f[src->cur] + (size_t)src_x0 * sb;
    return columnsCopy(dst, ncols, d, (size_t)D.nx * sb, sp, (size_t)S.nx * sb, (size_t)Q * D.ny * D.nz);
}

int acp_read_populations_window(acp_handle* h, int level, long long begin, int count, double* out) {
    if (!h || !out || level < 0 || level >= (int)h->host.size()) return ACP_ERR_INVALID;
    const LevelHost& L = h->host[level];
    if (count < 0 || count > ACP_WINDOW_MAX_NODES)
        return fail(h, ACP_ERR_INVALID, "window of %d nodes: at most %d (ACP_WINDOW_MAX_NODES) per call", count,
                    ACP_WINDOW_MAX_NODES);
    // count is in [0, ACP_WINDOW_MAX_NODES], so L.N - count cannot overflow
    if (begin < 0 || begin > L.N - count)
        return fail(h, ACP_ERR_INVALID, "window of %d nodes at %lld outside the level's %lld nodes", count, begin, L.N);
    if (count == 0) return ACP_OK;
    CU(h, cudaSetDevice(h->device));
    joinBatch(h);
    double* scratch = nullptr;
    int s = windowScratch(h, &scratch);
    if (s) return s;
    const int arr = level == 0 ? h->cur : 0;
    switch (h->d.storage) {
        case ACP_STORE_F64: launchWindow<double>(h, level, arr, begin, count, scratch); break;
        case ACP_STORE_F32_DEV: launchWindow<float>(h, level, arr, begin, count, scratch); break;
        default: launchWindow<__half>(h, level, arr, begin, count, scratch); break;
    }
    CU(h, cudaGetLastError());
    CU(h, cudaMemcpyAsync(out, scratch, (size_t)count * Q * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CU(h, cudaStreamSynchronize(h->stream));
    return ACP_OK;
}

int acp_write_populations(acp_handle* h, int level, const double* in) {
    if (!h || !in || level < 0 || level >= (int)h->host.size()) return ACP_ERR_INVALID;
    CU(h, cudaSetDevice(h->device));
    joinBatch(h);
    const LevelHost& L = h->host[level];
    double* tmp = nullptr;
    CU(h, cudaMallocAsync((void**)&tmp, (size_t)L.N * Q * sizeof(double), h->stream));
    cudaError_t e = cudaMemcpyAsync(tmp, in, (size_t)L.N * Q * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        switch (h->d.storage) {
            case ACP_STORE_F64: launchFromF64<double>(h, level, tmp); break;
            case ACP_STORE_F32_DEV: launchFromF64<float>(h, level, tmp); break;
            default: launchFromF64<__half>(h, level, tmp); break;
        }
    }
    cudaFreeAsync(tmp, h->stream);
    if (e != cudaSuccess) return fail(h, ACP_ERR_CUDA, "copy: %s", cudaGetErrorString(e));
    CU(h, cudaStreamSynchronize(h->stream));
    return ACP_OK;
}

namespace {
// checkpoint file: header, then per level both population arrays (storage
// bytes) and the partner-strain records.  The header names everything that
// gives the stored values their meaning: the storage form with its shift and
// FP16 scales, the operator and its options, the coupling and layout.
struct CheckpointHeader {
    char magic[8];
    int abi, storage, levels, cur;
    long long steps;
    long long dims[2][3];
    long long slots[2];
    int op, eqOrder, cubic, mrtWriteback, coupling, layout, scalingStyle, f2cFilter;
    double shift;
    float hscale[Q];
    int pad;
};
constexpr char kCheckpointMagic[8] = {'A', 'C', 'P', 'C', 'K', 'P', 'T', '2'};

CheckpointHeader checkpointHeader(const acp_handle* h) {
    CheckpointHeader c;
    std::memset(&c, 0, sizeof c);
    std::memcpy(c.magic, kCheckpointMagic, sizeof c.magic);
    c.abi = ACP_ABI_VERSION;
    c.storage = h->d.storage;
    c.levels = (int)h->host.size();
    c.cur = h->cur;
    c.steps = h->steps;
    for (size_t l = 0; l < h->host.size() && l < 2; ++l) {
        c.dims[l][0] = h->host[l].nx;
        c.dims[l][1] = h->host[l].ny;
        c.dims[l][2] = h->host[l].nz;
        c.slots[l] = h->dev[l].sg ? h->host[l].nSlots : 0;
    }
    c.op = h->d.op;
    c.eqOrder = h->d.eq_order;
    c.cubic = h->d.cubic_mach;
    c.mrtWriteback = h->d.mrt_writeback;
    c.coupling = h->d.coupling;
    c.layout = h->d.max_level == 1 ? h->d.layout : -1;
    c.scalingStyle = h->d.scaling_style;
    c.f2cFilter = h->d.f2c_filter;
    c.shift = h->shift;
    for (int q = 0; q < Q; ++q) c.hscale[q] = h->hscale[q];
    return c;
}

// the case fields of two headers agree (everything but parity and step count)
bool sameCase(const CheckpointHeader& a, const CheckpointHeader& b) {
    return a.abi == b.abi && a.storage == b.storage && a.levels == b.levels &&
           std::memcmp(a.dims, b.dims, sizeof a.dims) == 0 && std::memcmp(a.slots, b.slots, sizeof a.slots) == 0 &&
           a.op == b.op && a.eqOrder == b.eqOrder && a.cubic == b.cubic && a.mrtWriteback == b.mrtWriteback &&
           a.coupling == b.coupling && a.layout == b.layout && a.scalingStyle == b.scalingStyle &&
           a.f2cFilter == b.f2cFilter && a.shift == b.shift && std::memcmp(a.hscale, b.hscale, sizeof a.hscale) == 0;
}

// device regions of the state, in file order
std::vector<std::pair<void*, size_t>> checkpointRegions(acp_handle* h) {
    std::vector<std::pair<void*, size_t>> r;
    const size_t sb = storageBytes(h->d.storage);
    for (size_t l = 0; l < h->host.size(); ++l) {
        for (int a = 0; a < 2; ++a) r.push_back({h->dev[l].f[a], (size_t)h->host[l].N * Q * sb});
        if (h->dev[l].sg) r.push_back({h->dev[l].sg, std::max<size_t>(1, (size_t)h->host[l].nSlots) * 12 * sizeof(double)});
    }
    return r;
}
constexpr size_t kCheckpointChunk = 64u << 20;  // host staging per copy
}  // namespace

int acp_checkpoint_save(acp_handle* h, const char* path) {
    if (!h || !path) return ACP_ERR_INVALID;
    if (!h->inited) return fail(h, ACP_ERR_STATE, "checkpoint before acp_init");
    if (h->batch) return fail(h, ACP_ERR_STATE, "the case belongs to a batch");
    CU(h, cudaSetDevice(h->device));
    CU(h, cudaStreamSynchronize(h->stream));
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(h, ACP_ERR_INVALID, "cannot write %s", path);
    const CheckpointHeader hd = checkpointHeader(h);
    bool ok = std::fwrite(&hd, sizeof hd, 1, f) == 1;
    std::vector<char> buf;
    for (const auto& reg : checkpointRegions(h)) {
        for (size_t o = 0; ok && o < reg.second; o += kCheckpointChunk) {
            const size_t n = std::min(kCheckpointChunk, reg.second - o);
            buf.resize(n);
            const cudaError_t e = cudaMemcpy(buf.data(), (const char*)reg.first + o, n, cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) {
                std::fclose(f);
                return fail(h, ACP_ERR_CUDA, "checkpoint copy: %s", cudaGetErrorString(e));
            }
            ok = std::fwrite(buf.data(), 1, n, f) == n;
        }
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return fail(h, ACP_ERR_INVALID, "writing %s failed", path);
    return ACP_OK;
}

int acp_checkpoint_load(acp_handle* h, const char* path) {
    if (!h || !path) return ACP_ERR_INVALID;
    if (!h->inited) return fail(h, ACP_ERR_STATE, "restore before acp_init");
    if (h->batch) return fail(h, ACP_ERR_STATE, "the case belongs to a batch");
    CU(h, cudaSetDevice(h->device));
    CU(h, cudaStreamSynchronize(h->stream));
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(h, ACP_ERR_INVALID, "cannot read %s", path);
    CheckpointHeader hd;
    if (std::fread(&hd, sizeof hd, 1, f) != 1 || std::memcmp(hd.magic, kCheckpointMagic, sizeof hd.magic) != 0) {
        std::fclose(f);
        return fail(h, ACP_ERR_INVALID, "%s is not a checkpoint of this engine", path);
    }
    const CheckpointHeader mine = checkpointHeader(h);
    if (!sameCase(hd, mine) || (hd.cur != 0 && hd.cur != 1) || hd.steps < 0) {
        std::fclose(f);
        return fail(h, ACP_ERR_INVALID,
                    "%s holds another case (storage form, shift, level shape, operator, coupling or layout)", path);
    }
    // the file must hold exactly the state regions: checked before any device write
    const auto regions = checkpointRegions(h);
    long long want = (long long)sizeof hd;
    for (const auto& reg : regions) want += (long long)reg.second;
    if (std::fseek(f, 0, SEEK_END) != 0 || std::ftell(f) != want || std::fseek(f, (long)sizeof hd, SEEK_SET) != 0) {
        std::fclose(f);
        return fail(h, ACP_ERR_INVALID, "%s is truncated or too long (%lld bytes expected)", path, want);
    }
    std::vector<char> buf;
    for (const auto& reg : regions) {
        for (size_t o = 0; o < reg.second; o += kCheckpointChunk) {
            const size_t n = std::min(kCheckpointChunk, reg.second - o);
            buf.resize(n);
            if (std::fread(buf.data(), 1, n, f) != n) {
                std::fclose(f);
                return fail(h, ACP_ERR_INVALID, "reading %s failed; the case's state is undefined", path);
            }
            const cudaError_t e = cudaMemcpy((char*)reg.first + o, buf.data(), n, cudaMemcpyHostToDevice);
            if (e != cudaSuccess) {
                std::fclose(f);
                return fail(h, ACP_ERR_CUDA, "restore copy: %s; the case's state is undefined", cudaGetErrorString(e));
            }
        }
    }
    std::fclose(f);
    h->cur = hd.cur;
    h->steps = hd.steps;
    // probe series restart empty: the counter is reset, the step count continues
    if (h->dCounter) CU(h, cudaMemset(h->dCounter, 0, sizeof(int)));
    CU(h, cudaMemset(h->dErr, 0, sizeof(int)));
    return ACP_OK;
}

int acp_write_vtk(acp_handle* h, const char* prefix, int binary) {
    if (!h || !prefix || (binary != 0 && binary != 1)) return ACP_ERR_INVALID;
    if (h->dev.empty()) return ACP_ERR_STATE;
    CU(h, cudaSetDevice(h->device));
    joinBatch(h);
    const acp_case_desc& d = h->d;
    const double cs2 = d.speed_of_sound * d.speed_of_sound;
    for (size_t l = 0; l < h->host.size(); ++l) {
        const LevelHost& L = h->host[l];
        const size_t N = (size_t)L.N;
        const int arr = l == 0 ? h->cur : 0;
        double* tmp = nullptr;
        CU(h, cudaMallocAsync((void**)&tmp, N * 4 * sizeof(double), h->stream));
        const unsigned grid = (unsigned)((N + 255) / 256);
        switch (d.storage) {
            case ACP_STORE_F64:
                k_fields4<double><<<grid, 256, 0, h->stream>>>((const double*)h->dev[l].f[arr], tmp, L.N, h->shift, h->c,
                                                                levelArgs<double>(h, (int)l, 0));
                break;
            case ACP_STORE_F32_DEV:
                k_fields4<float><<<grid, 256, 0, h->stream>>>((const float*)h->dev[l].f[arr], tmp, L.N, h->shift, h->c,
                                                               levelArgs<float>(h, (int)l, 0));
                break;
            default:
                k_fields4<__half><<<grid, 256, 0, h->stream>>>((const __half*)h->dev[l].f[arr], tmp, L.N, h->shift, h->c,
                                                                levelArgs<__half>(h, (int)l, 0));
                break;
        }
        std::vector<double> v(N * 4);
        cudaError_t e = cudaMemcpyAsync(v.data(), tmp, N * 4 * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
        cudaFreeAsync(tmp, h->stream);
        if (e != cudaSuccess) return fail(h, ACP_ERR_CUDA, "copy: %s", cudaGetErrorString(e));
        CU(h, cudaStreamSynchronize(h->stream));
        const double* rho = v.data();
        const double* u[3] = {v.data() + N, v.data() + 2 * N, v.data() + 3 * N};
        const std::string path = std::string(prefix) + (h->host.size() > 1 ? "_level" + std::to_string(l) : "") + ".vtk";
        FILE* f = std::fopen(path.c_str(), "wb");
        if (!f) return fail(h, ACP_ERR_INVALID, "cannot write %s", path.c_str());
        const double sp = d.spacing / std::pow(2.0, (double)l);
        std::fprintf(f, "# vtk DataFile Version 3.0\nacPulse_vcLBM level %d\n%s\nDATASET STRUCTURED_POINTS\n", (int)l,
                     binary ? "BINARY" : "ASCII");
        std::fprintf(f, "DIMENSIONS %d %d %d\n", L.nx, L.ny, L.nz);
        std::fprintf(f, "ORIGIN %.8g %.8g %.8g\n", L.off[0] * sp, L.off[1] * sp, L.off[2] * sp);
        std::fprintf(f, "SPACING %.8g %.8g %.8g\nPOINT_DATA %zu\n", sp, sp, sp, N);
        // values in file order: big-endian FP64 (binary) or %.8g text
        std::vector<unsigned char> be;
        auto put = [&](const double* x, size_t n, size_t stride, int per) {
            if (binary) {
                be.resize(n * per * 8);
                for (size_t m = 0; m < n; ++m)
                    for (int k = 0; k < per; ++k) {
                        uint64_t w;
                        std::memcpy(&w, x + m + k * stride, 8);
                        for (int b = 0; b < 8; ++b) be[(m * per + k) * 8 + b] = (unsigned char)(w >> (56 - 8 * b));
                    }
                std::fwrite(be.data(), 1, be.size(), f);
                std::fputc('\n', f);
            } else {
                for (size_t m = 0; m < n; ++m)
                    for (int k = 0; k < per; ++k) std::fprintf(f, k + 1 < per ? "%.8g " : "%.8g\n", x[m + k * stride]);
            }
        };
        std::vector<double> p(N);
        for (size_t m = 0; m < N; ++m) p[m] = rho[m] * cs2;
        std::fprintf(f, "SCALARS Pressure double 1\nLOOKUP_TABLE default\n");
        put(p.data(), N, 0, 1);
        std::fprintf(f, "SCALARS Density double 1\nLOOKUP_TABLE default\n");
        put(rho, N, 0, 1);
        std::fprintf(f, "VECTORS Velocity double\n");
        put(u[0], N, N, 3);
        if (std::fclose(f) != 0) return fail(h, ACP_ERR_INVALID, "writing %s failed", path.c_str());
    }
    return ACP_OK;
}

int acp_read_field(acp_handle* h, int level, int field, double* out) {
    if (!h || !out || level < 0 || level >= (int)h->host.size() || field < 0 || field > 4) return ACP_ERR_INVALID;
    CU(h, cudaSetDevice(h->device));
    joinBatch(h);
    const LevelHost& L = h->host[level];
    const int arr = level == 0 ? h->cur : 0;
    double* tmp = nullptr;
    CU(h, cudaMallocAsync((void**)&tmp, (size_t)L.N * sizeof(double), h->stream));
    const unsigned grid = (unsigned)((L.N + 255) / 256);
    const double cs = h->d.speed_of_sound;
    switch (h->d.storage) {
        case ACP_STORE_F64:
            k_field<double><<<grid, 256, 0, h->stream>>>((const double*)h->dev[level].f[arr], tmp, L.N, h->shift, h->c,
                                                          cs, field, levelArgs<double>(h, level, 0));
            break;
        case ACP_STORE_F32_DEV:
            k_field<float><<<grid, 256, 0, h->stream>>>((const float*)h->dev[level].f[arr], tmp, L.N, h->shift, h->c,
                                                         cs, field, levelArgs<float>(h, level, 0));
            break;
        default:
            k_field<__half><<<grid, 256, 0, h->stream>>>((const __half*)h->dev[level].f[arr], tmp, L.N, h->shift, h->c,
                                                          cs, field, levelArgs<__half>(h, level, 0));
            break;
    }
    cudaError_t e = cudaMemcpyAsync(out, tmp, (size_t)L.N * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    cudaFreeAsync(tmp, h->stream);
    if (e != cudaSuccess) return fail(h, ACP_ERR_CUDA, "copy: %s", cudaGetErrorString(e));
    CU(h, cudaStreamSynchronize(h->stream));
    return ACP_OK;
}

int acp_set_probes(acp_handle* h, int n, const int* lijk) {
    if (!h || n < 0 || (n > 0 && !lijk)) return ACP_ERR_INVALID;
    if (h->batch) return fail(h, ACP_ERR_STATE, "the case belongs to a batch");
    CU(h, cudaSetDevice(h->device));
    std::vector<long long> nodes(n);
    std::vector<int> levels(n);
    for (int m = 0; m < n; ++m) {
        const int l = lijk[4 * m];
        if (l < 0 || l >= (int)h->host.size()) return fail(h, ACP_ERR_INVALID, "probe %d: no level %d", m, l);
        const LevelHost& L = h->host[l];
        const int i = lijk[4 * m + 1] - L.off[0], j = lijk[4 * m + 2] - L.off[1], k = lijk[4 * m + 3] - L.off[2];
        if (i < 0 || i >= L.nx || j < 0 || j >= L.ny || k < 0 || k >= L.nz)
            return fail(h, ACP_ERR_INVALID, "probe %d outside its level", m);
        nodes[m] = ((long long)k * L.ny + j) * L.nx + i;
        if (L.code[nodes[m]] == CODE_DEAD) return fail(h, ACP_ERR_INVALID, "probe %d on a node covered by the fine level", m);
        levels[m] = l;
    }
    if (h->dProbeNodes) { devFree(h->dProbeNodes); h->dProbeNodes = nullptr; }
    if (h->dProbeLevels) { devFree(h->dProbeLevels); h->dProbeLevels = nullptr; }
    if (h->dSeries) { devFree(h->dSeries); h->dSeries = nullptr; }
    if (!h->dCounter) {
        int s = devAlloc(h, (void**)&h->dCounter, sizeof(int));
        if (s) return s;
    }
    h->nProbes = n;
    h->probeCapacity = 1 << 16;
    if (n) {
        int s = devAlloc(h, (void**)&h->dProbeNodes, n * sizeof(long long));
        if (s) return s;
        if ((s = devAlloc(h, (void**)&h->dProbeLevels, n * sizeof(int)))) return s;
        if ((s = devAlloc(h, (void**)&h->dSeries, (size_t)n * h->probeCapacity * sizeof(double)))) return s;
        CU(h, cudaMemcpyAsync(h->dProbeNodes, nodes.data(), n * sizeof(long long), cudaMemcpyHostToDevice, h->stream));
        CU(h, cudaMemcpyAsync(h->dProbeLevels, levels.data(), n * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    }
    CU(h, cudaMemsetAsync(h->dCounter, 0, sizeof(int), h->stream));
    CU(h, cudaStreamSynchronize(h->stream));
    if (h->inited) return captureGraphs(h);
    return ACP_OK;
}

int acp_read_probes(acp_handle* h, double* out, int max_samples, int* n_samples) {
    if (!h || !n_samples) return ACP_ERR_INVALID;
    CU(h, cudaSetDevice(h->device));
    joinBatch(h);
    int cnt = 0;
    if (h->dCounter) CU(h, cudaMemcpyAsync(&cnt, h->dCounter, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CU(h, cudaStreamSynchronize(h->stream));
    cnt = std::min(cnt, h->probeCapacity);
    const int take = std::min(cnt, max_samples);
    if (take > 0 && out && h->nProbes)
        CU(h, cudaMemcpy(out, h->dSeries, (size_t)take * h->nProbes * sizeof(double), cudaMemcpyDeviceToHost));
    *n_samples = take;
    return ACP_OK;
}

int acp_steps_done(acp_handle* h, long long* steps) {
    if (!h || !steps) return ACP_ERR_INVALID;
    *steps = h->steps;
    return ACP_OK;
}

int acp_set_stream(acp_handle* h, void* stream) {
    if (!h) return ACP_ERR_INVALID;
    if (h->batch) return fail(h, ACP_ERR_STATE, "the case belongs to a batch");
    CU(h, cudaSetDevice(h->device));
    CU(h, cudaStreamSynchronize(h->stream));
    if (h->ownStream && stream) {
        cudaStreamDestroy(h->stream);
        h->ownStream = false;
    }
    if (stream) {
        h->stream = (cudaStream_t)stream;
    } else if (!h->ownStream) {
        CU(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        h->ownStream = true;
    }
    if (h->inited) return captureGraphs(h);
    return ACP_OK;
}

int acp_device_bytes(acp_handle* h, size_t* bytes) {
    if (!h || !bytes) return ACP_ERR_INVALID;
    *bytes = h->devBytes;
    return ACP_OK;
}

int acp_step_timed(acp_handle* h, int n, double* kernel_ms) {
    if (!h || !h->inited || !kernel_ms || n < 0) return ACP_ERR_INVALID;
    if (h->batch) return fail(h, ACP_ERR_STATE, "the case is stepped by its batch (acp_batch_step)");
    CU(h, cudaSetDevice(h->device));
    double acc[ACP_K_COUNT] = {0, 0, 0, 0, 0};
    PhaseTimer tm;
    tm.stream = h->stream;
    for (int e = 0; e < 32; ++e) CU(h, cudaEventCreate(&tm.ev[e]));
    int status = ACP_OK;
    for (int s = 0; s < n && status == ACP_OK; ++s) {
        tm.n = 0;
        enqueueStep(h, h->cur, &tm);
        h->cur ^= 1;
        ++h->steps;
        cudaError_t e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) { status = fail(h, ACP_ERR_CUDA, "timed step: %s", cudaGetErrorString(e)); break; }
        for (int m = 1; m < tm.n; ++m) {
            float ms = 0;
            cudaEventElapsedTime(&ms, tm.ev[m - 1], tm.ev[m]);
            if (tm.kind[m] >= 0) acc[tm.kind[m]] += ms;
        }
    }
    for (int e = 0; e < 32; ++e) cudaEventDestroy(tm.ev[e]);
    for (int k = 0; k < ACP_K_COUNT; ++k) kernel_ms[k] = n ? acc[k] / n : 0.0;
    return status;
}

int acp_launches_per_step(acp_handle* h, int* launches) {
    if (!h || !launches || h->dev.empty()) return ACP_ERR_INVALID;
    *launches = launchesPerStep(h);
    return ACP_OK;
}

int acp_boundary_wiring(const acp_case_desc* d, long long* rows, long long max_rows, long long* count) {
    if (!count) return ACP_ERR_INVALID;
    std::string why;
    int s = validate(d, why);
    if (s) return s;
    acp_handle tmp;
    tmp.d = *d;
    if ((s = buildSingleLevel(&tmp))) return s;
    const LevelHost& L = tmp.host[0];
    std::vector<const BNodeDev*> all;
    for (const BNodeDev& b : L.lodiX) all.push_back(&b);
    for (const BNodeDev& b : L.lodiZY) all.push_back(&b);
    std::sort(all.begin(), all.end(), [](const BNodeDev* a, const BNodeDev* b) { return a->n < b->n; });
    *count = (long long)all.size();
    if (!rows) return ACP_OK;
    for (long long r = 0; r < (long long)all.size() && r < max_rows; ++r) {
        const BNodeDev& b = *all[r];
        const long long i = b.n % L.nx, j = (b.n / L.nx) % L.ny, k = b.n / ((long long)L.nx * L.ny);
        const int code = L.code[b.n];
        const int fx = code / 9 - 1, fy = (code / 3) % 3 - 1, fz = code % 3 - 1;
        const BoundaryClass* bc = boundaryClass(fx, fy, fz);
        long long mask = 0;
        for (int m = 0; m < 5 && bc->push[m] >= 0; ++m) mask |= 1LL << bc->push[m];
        long long* o = rows + 12 * r;
        o[0] = i; o[1] = j; o[2] = k; o[3] = b.normalDir; o[4] = b.n1; o[5] = b.n2;
        for (int m = 0; m < 4; ++m) o[6 + m] = b.t[m];
        o[10] = bc->corner;
        o[11] = mask;
    }
    return ACP_OK;
}

int acp_destroy(acp_handle* h) {
    if (!h) return ACP_OK;
    if (h->batch) return fail(h, ACP_ERR_STATE, "destroy the batch before its cases");
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    destroyGraphs(h);
    for (LevelDev& D : h->dev) {
        devFree(D.f[0]);
        devFree(D.f[1]);
        devFree(D.code);
        devFree(D.lodiX);
        devFree(D.lodiZY);
        devFree(D.slot);
        devFree(D.sg);
        devFree(D.cols);
    }
    devFree(h->dNb);
    devFree(h->dPreNb);
    devFree(h->dErr);
    devFree(h->dC2F);
    devFree(h->dF2C);
    devFree(h->dDC);
    devFree(h->dPre);
    devFree(h->dProbeNodes);
    devFree(h->dProbeLevels);
    devFree(h->dSeries);
    devFree(h->dCounter);
    if (h->ownStream && h->stream) cudaStreamDestroy(h->stream);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->forkEv) cudaEventDestroy(h->forkEv);
    if (h->joinEv) cudaEventDestroy(h->joinEv);
    if (h->side2) cudaStreamDestroy(h->side2);
    for (cudaEvent_t e : h->branchEv)
        if (e) cudaEventDestroy(e);
    if (h->side3) cudaStreamDestroy(h->side3);
    for (cudaEvent_t e : h->splitEv)
        if (e) cudaEventDestroy(e);
    delete h;
    return ACP_OK;
}

const char* acp_last_error(const acp_handle* h) { return h ? h->err.c_str() : "null handle"; }

const char* acp_status_string(int s) {
    switch (s) {
        case ACP_OK: return "ok";
        case ACP_ERR_INVALID: return "invalid argument";
        case ACP_ERR_CUDA: return "CUDA error";
        case ACP_ERR_NOMEM: return "out of memory";
        case ACP_ERR_UNSUPPORTED: return "unsupported";
        case ACP_ERR_NUMERIC: return "numerical blow-up";
        case ACP_ERR_TIMEOUT: return "device wait timed out";
        case ACP_ERR_BUDGET: return "HBM budget exhausted";
        case ACP_ERR_STATE: return "call out of order";
        default: return "unknown status";
    }
}

int acp_abi_version(void) { return ACP_ABI_VERSION; }

}  // extern "C"

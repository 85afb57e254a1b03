// The engine's handle (the state behind acp_handle of include/acp.h) and the
// helpers that build kernel arguments from it; shared by the single-case
// engine (engine.cu) and the batched engine (batch.cu).
#pragma once
#include "../../include/acp.h"
#include "kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

struct acp_batch;

namespace acp {

// page-locked host blocks kept for reuse (engine.cu): the node-class arrays
// live in them, so their upload is a direct DMA instead of a staged copy of
// pageable memory; without a device they are ordinary heap blocks
void* hostBlockAlloc(size_t bytes);
void hostBlockFree(void* p, size_t bytes);

// allocator of the node-class arrays: page-locked host blocks (above), and a
// resize that leaves new elements uninitialised (the set-up scans write the
// arrays in full, row ranges on several threads, so a zero fill first would
// be a second serial pass over them)
template <typename T>
struct NoInitAlloc {
    using value_type = T;
    template <typename U>
    struct rebind {
        using other = NoInitAlloc<U>;
    };
    NoInitAlloc() = default;
    template <typename U>
    NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
    T* allocate(size_t n) { return static_cast<T*>(hostBlockAlloc(n * sizeof(T))); }
    void deallocate(T* p, size_t n) noexcept { hostBlockFree(p, n * sizeof(T)); }
    template <typename U>
    void construct(U*) noexcept {}
    template <typename U, typename... A>
    void construct(U* p, A&&... a) {
        ::new ((void*)p) U(std::forward<A>(a)...);
    }
    template <typename U>
    bool operator==(const NoInitAlloc<U>&) const noexcept { return true; }
    template <typename U>
    bool operator!=(const NoInitAlloc<U>&) const noexcept { return false; }
};

struct LevelHost {
    int nx = 0, ny = 0, nz = 0;
    long long N = 0;
    int off[3] = {0, 0, 0};  // box origin in this level's global node index
    int per[3] = {0, 0, 0};  // periodic axes of this level
    std::vector<uint8_t, NoInitAlloc<uint8_t>> code;
    std::vector<long long> coupling;  // coupling nodes in node order (two levels)
    long long dead = 0;               // nodes covered by the other level
    std::vector<BNodeDev> lodiX, lodiZY;
    int nSlots = 0;  // partner-strain records kept (the device map LevelDev::slot; 0: none)
    long long active = 0;
    double omega = 0, dt = 0, spacing = 0;
};

struct LevelDev {
    void* f[2] = {nullptr, nullptr};
    uint8_t* code = nullptr;
    BNodeDev* lodiX = nullptr;
    BNodeDev* lodiZY = nullptr;
    int nLodiX = 0, nLodiZY = 0;
    // x tiles of the y-marching collide split for the second fine sub-step:
    // cols[0, nInner) touch no coupling or LODI node (they may run while the
    // coupling kernels do), cols[nInner, nInner + nOuter) the others; nInner
    // = 0: no split
    int* cols = nullptr;
    int nInner = 0, nOuter = 0;
    int* slot = nullptr;    // see LevelHost::slot
    double* sg = nullptr;   // [12][nSlots] partner strain S and cubic-Mach gradient G
};

inline size_t storageBytes(int storage) {
    return storage == ACP_STORE_F64 ? 8 : (storage == ACP_STORE_F32_DEV ? 4 : 2);
}

}  // namespace acp

struct acp_handle {
    acp_case_desc d;
    int device = 0;
    std::vector<acp::LevelHost> host;
    std::vector<acp::LevelDev> dev;
    int cur = 0;  // array holding the current state (0 or 1) of the coarse level
    bool inited = false;
    long long steps = 0;
    cudaStream_t stream = nullptr;
    bool ownStream = false;
    cudaStream_t side = nullptr;  // second branch of a captured step (coarse level beside the fine sub-step)
    cudaEvent_t forkEv = nullptr, joinEv = nullptr;
    // third branch of a captured step: the fine level's LODI passes beside the
    // coupling kernels, F2C beside the last C2F (disjoint node sets)
    cudaStream_t side2 = nullptr;
    cudaEvent_t branchEv[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    // fourth branch: the interior tiles of the second fine sub-step beside the
    // first C2F and the fine LODI passes (LevelDev::cols)
    cudaStream_t side3 = nullptr;
    cudaEvent_t splitEv[2] = {nullptr, nullptr};
    cudaGraphExec_t graph[2] = {nullptr, nullptr};  // one step starting from cur == 0 / cur == 1
    // two-level coupling (fine state always in array 0 between coarse steps)
    std::vector<acp::C2FDev> c2fHost;
    std::vector<acp::F2CDev> f2cHost;
    std::vector<acp::DCDev> dcHost;  // direct coupling: the shared nodes
    acp::DCDev* dDC = nullptr;
    int nCoinc = 0, nMid = 0, nCen = 0;
    acp::C2FDev* dC2F = nullptr;
    acp::F2CDev* dF2C = nullptr;
    void* dPre = nullptr;  // coarse populations before the coarse step, [Q][nCoinc]
    // partner strain of the coupling nodes (STD; HRR, or RR with cubic-Mach)
    bool partner = false;
    std::vector<acp::C2FNbDev> nbHost;
    acp::C2FNbDev* dNb = nullptr;
    void* dPreNb = nullptr;  // [24][nCoinc] drho, u of the coincident nodes' coarse neighbours at t
    int* dErr = nullptr;
    // probes
    long long* dProbeNodes = nullptr;
    int* dProbeLevels = nullptr;
    int nProbes = 0;
    double* dSeries = nullptr;
    int* dCounter = nullptr;
    int probeCapacity = 0;
    size_t devBytes = 0;
    std::string err;
    double c = 0, kappa = 0, shift = 0;
    float hscale[acp::Q];
    double m4[18] = {0};  // sum_q w_q H2_q (x) H4_q(kappa) (fourth-order equilibria)
    acp_batch* batch = nullptr;  // the batch this case belongs to (stepped only through it)
    std::vector<const void*> bulk;  // collide kernels launched while capturing the step graphs
};

namespace acp {

inline int fail(acp_handle* h, int code, const char* fmt, ...) {
    if (h) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        std::vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        h->err = buf;
    }
    return code;
}

// adds a collide kernel to the set kept for instantiateWithPriorities
inline void noteBulk(std::vector<const void*>& bulk, const void* f) {
    if (std::find(bulk.begin(), bulk.end(), f) == bulk.end()) bulk.push_back(f);
}

// Instantiates a captured step graph with every kernel but the collide
// launches (`bulk`: the kernels that fill the SMs) at the device's greatest
// stream priority.  The small latency-bound phases (LODI, coupling, probes)
// of one branch then take the block slots that free up while another
// branch's collide runs, instead of waiting behind its remaining waves.
// Priorities change no dependency of the graph.
inline cudaError_t instantiateWithPriorities(cudaGraphExec_t* exec, cudaGraph_t g, const std::vector<const void*>& bulk) {
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess && greatest != least) {
        size_t n = 0;
        if (cudaGraphGetNodes(g, nullptr, &n) == cudaSuccess && n) {
            std::vector<cudaGraphNode_t> nodes(n);
            if (cudaGraphGetNodes(g, nodes.data(), &n) == cudaSuccess)
                for (cudaGraphNode_t nd : nodes) {
                    cudaGraphNodeType t;
                    cudaKernelNodeParams kp;
                    if (cudaGraphNodeGetType(nd, &t) != cudaSuccess || t != cudaGraphNodeTypeKernel ||
                        cudaGraphKernelNodeGetParams(nd, &kp) != cudaSuccess)
                        continue;
                    bool isBulk = false;
                    for (const void* f : bulk) isBulk = isBulk || f == (const void*)kp.func;
                    cudaKernelNodeAttrValue v = {};
                    v.priority = isBulk ? least : greatest;
                    cudaGraphKernelNodeSetAttribute(nd, cudaKernelNodeAttributePriority, &v);
                }
        }
        cudaGetLastError();  // a node left at the default priority is not an error
    }
    return cudaGraphInstantiateWithFlags(exec, g, cudaGraphInstantiateFlagUseNodePriority);
}

#define CU(h, call)                                                                                       \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess) return fail((h), ACP_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// kernel arguments of level l of a case, reading array src
template <typename S>
LevelArgs<S> levelArgs(const acp_handle* h, int l, int src) {
    const LevelHost& L = h->host[l];
    const LevelDev& D = h->dev[l];
    LevelArgs<S> a;
    a.nx = L.nx; a.ny = L.ny; a.nz = L.nz;
    a.N = L.N;
    a.Ni = (int)L.N;
    for (int ax = 0; ax < 3; ++ax) a.per[ax] = L.per[ax];
    a.A = (const S*)D.f[src];
    a.B = (S*)D.f[1 - src];
    for (int q = 0; q < Q; ++q) {
        a.Aq[q] = a.A + (size_t)q * (size_t)L.N;
        a.Bq[q] = a.B + (size_t)q * (size_t)L.N;
    }
    a.code = D.code;
    a.shift = h->shift;
    a.omega = L.omega;
    a.kappa = h->kappa;
    a.sigma = h->d.hybrid_sigma;
    for (int q = 0; q < Q; ++q) a.hscale[q] = h->hscale[q];
    for (int c = 0; c < 18; ++c) a.m4[c] = h->m4[c];
    a.slot = D.slot;
    a.sg = D.sg;
    a.nSlots = L.nSlots;
    return a;
}

inline CouplingArgs couplingArgs(const acp_handle* h) {
    CouplingArgs c;
    c.Nc = h->host[0].N;
    c.Nf = h->host[1].N;
    c.shiftC = h->shift;
    c.kappa = h->kappa;
    c.omegaC = h->host[0].omega;
    c.omegaF = h->host[1].omega;
    c.alphaC2F = c.omegaC / (2.0 * c.omegaF);
    c.alphaF2C = 2.0 * c.omegaF / c.omegaC;
    c.mrtStyle = h->d.scaling_style == ACP_SCALING_MRT;
    c.filter = h->d.f2c_filter;
    c.partner = h->partner ? 1 : 0;
    c.nSlotsF = h->host[1].nSlots;
    c.nSlotsC = h->host[0].nSlots;
    c.nb = h->dNb;
    c.preNb = h->dPreNb;
    c.sgF = h->dev[1].sg;
    c.sgC = h->dev[0].sg;
    c.slotF = h->dev[1].slot;
    return c;
}

// components one C2F interpolation thread handles per hanging node: the
// populations, and the partner strain when it is kept
inline int interpComponents(const acp_handle* h) { return Q + (h->partner ? 12 : 0); }

// LODI arguments of level l (Node::LODIpressureOutlet's constants: L is the
// node count times the coarse spacing on every level, Node.cpp:311)
inline LodiArgs lodiArgsOf(const acp_handle* h, int l) {
    const LevelHost& L = h->host[l];
    LodiArgs p;
    p.N = L.N;
    p.shift = h->shift;
    p.cs = h->d.speed_of_sound;
    p.c = h->c;
    p.mach = h->d.mach;
    p.k1 = h->d.k1;
    p.rho0 = h->d.density;
    p.dt = L.dt;
    p.localSpacing = h->d.spacing * std::pow(2.0, -(double)l);
    p.kappa = h->kappa;
    const int dims[3] = {h->d.nx, h->d.ny, h->d.nz};
    for (int a = 0; a < 3; ++a)
        p.domainLength[a] = (h->d.lodi_length_nodes[a] > 0 ? h->d.lodi_length_nodes[a] : dims[a]) * h->d.spacing;
    p.order = h->d.eq_order;
    p.errorFlag = h->dErr;
    return p;
}

// event recorded after a batch's last enqueued step (defined with the batch)
cudaEvent_t batchDoneEvent(acp_batch* b);

// a case stepped by a batch: order the case's own stream after the batch's work
inline void joinBatch(acp_handle* h) {
    if (h && h->batch) cudaStreamWaitEvent(h->stream, batchDoneEvent(h->batch), 0);
}

// probe sampling after a step whose coarse level wrote array coarseNew
template <typename S>
void launchProbes(const acp_handle* h, cudaStream_t st, int coarseNew) {
    LevelArgs<S> a = levelArgs<S>(h, 0, 0);
    const S* fine = h->host.size() > 1 ? (const S*)h->dev[1].f[0] : nullptr;
    const long long Nf = h->host.size() > 1 ? h->host[1].N : 0;
    k_probes<S><<<1, 128, 0, st>>>((const S*)h->dev[0].f[coarseNew], h->host[0].N, fine, Nf, a, h->dProbeNodes,
                                   h->dProbeLevels, h->nProbes, h->shift,
                                   h->d.speed_of_sound * h->d.speed_of_sound, h->dSeries, h->dCounter,
                                   h->probeCapacity);
}

inline bool needsMoments(const acp_case_desc& d) { return d.op == OP_HRR || (d.op == OP_RR && d.cubic_mach); }

// z chunk of a tiled kernel launch (one block per TX x TY column and chunk):
// short chunks of about eight planes, each block passing its chunk plus the
// plane on either side (those mostly come from L2, where the neighbouring
// chunk's block has just read them), shortened down to six planes until the
// launch fills the `perSM` resident blocks of each of B200's 148 SMs.  Many
// short blocks balance better than one wave of long ones: on 192^3 nodes
// (HRR, FP32) chunks of 8 take 349 us per step against 449 us for chunks of
// 39.  A periodic z axis of at most three planes stays resident, and a
// periodic axis shorter than the chunk goes to one block per column.
inline int tiledChunkFor(const LevelHost& L, int perSM) {
    if (L.per[2] && L.nz <= 3) return L.nz;
    const long long bxy = (long long)((L.nx + TX - 1) / TX) * ((L.ny + TY - 1) / TY);
    int chunk = 8;
    while (chunk > 6 && bxy * ((L.nz + chunk - 1) / chunk) < (long long)perSM * 148) --chunk;
    return std::min(chunk, L.nz);
}

// The y-marching form of the neighbour-moment collide (k_collide_push_march)
// takes levels whose z axis is periodic and at most MARCH_MAX_NZ planes deep.
inline bool marchesY(const LevelHost& L) { return L.per[2] && L.nz <= MARCH_MAX_NZ; }

// y rows per march block.  Every block reloads two rows at its chunk's ends,
// yet short chunks win: a block's rows are serial (load, barrier, collide),
// so the SM hides latency only across blocks, and many short-lived blocks
// also balance the tail.  Measured on the fine level of the 1024 x 512 x 3
// two-level HRR workload (collide time per coarse step): FP32 (alternating
// march directions, 56 registers) 2 rows 562 us, 3 rows 536, 4 rows 528,
// 8 rows 545, 16 rows 599; FP64 (prefetch) 4 rows 1104 us, 8 rows 1087.
// ACP_MARCH_YCHUNK overrides the choice.
inline int marchChunkFor(const LevelHost& L, size_t realBytes) {
    if (const char* e = std::getenv("ACP_MARCH_YCHUNK")) {
        const int v = std::atoi(e);
        if (v > 0) return std::min(v, L.ny);
    }
    return std::min(realBytes == 8 ? 8 : 4, L.ny);
}

// z chunk of the batched engine's persistent tiled work items: a periodic z
// axis of at most three planes is resident at once; otherwise chunks give
// >= 4 blocks per SM
inline int tiledChunk(const LevelHost& L) {
    if (L.per[2] && L.nz <= 3) return L.nz;
    const int bxy = ((L.nx + TX - 1) / TX) * ((L.ny + TY - 1) / TY);
    const int want = (4 * 148 + bxy - 1) / bxy;
    return std::max(8, (L.nz + want - 1) / want);
}

}  // namespace acp

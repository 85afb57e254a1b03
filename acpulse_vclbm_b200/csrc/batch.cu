// Batched engine: many pulse cases of uneven sizes, operators, storage forms
// and refinement layouts advance together.  Cases are split into homogeneous
// groups (same kernel templates and phase sequence); each group runs the
// phase sequence of one coarse step (Lattice::timeStepping* /
// nestedTimeStepping*, Lattice.cpp:1496-15051) on its own stream branch, and
// every phase of a group is ONE persistent launch over a work list of
// (case, block) items for all of the group's cases.  The step is captured as
// one CUDA graph per ping-pong parity.  An autotuner picks the persistent grid
// size, the item order and the z-chunk of the tiled kernel by timing them on
// the live batch.
#include "../../include/acp.h"
#include "handle.h"
#include "kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <tuple>
#include <vector>

namespace acp {

struct WorkItem {
    int c;           // case record
    int bx, by, bz;  // block coordinates within the case's launch
};

template <typename S>
struct BatchLevel {
    LevelArgs<S> a[2];  // reading array 0 / 1
    LodiArgs lodi;
    const BNodeDev* lodiX;
    const BNodeDev* lodiZY;
    int nLodiX, nLodiZY;
    int zChunk;
    int pad;
};

template <typename S>
struct BatchCase {
    BatchLevel<S> lv[2];
    CouplingArgs cpl;
    const C2FDev* c2f;
    const F2CDev* f2c;
    const DCDev* dc;
    void* pre;
    int nCoinc, nMid, nCen, nF2C;
    int base;  // coarse array read at the batch's even steps
    int dc2;
};

// copy a kernel-argument record into shared memory (all threads of the block)
template <typename T>
__device__ __forceinline__ void stage(T* dst, const T* src) {
    static_assert(sizeof(T) % 4 == 0, "records are copied as 32-bit words");
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int nt = blockDim.x * blockDim.y;
    for (int k = tid; k < (int)(sizeof(T) / 4); k += nt)
        reinterpret_cast<int*>(dst)[k] = reinterpret_cast<const int*>(src)[k];
}

// the coarse level reads array base ^ flip, the fine level the sub-step's array
template <typename S>
__device__ __forceinline__ int srcOf(const BatchCase<S>& bc, int level, int fineSrc, int flip) {
    return level == 0 ? (bc.base ^ flip) : fineSrc;
}

template <typename S, typename R, int OP, int ORDER, bool CUBIC, bool MRTWB>
__global__ void __launch_bounds__(128) kb_collide(const BatchCase<S>* __restrict__ cases,
                                                  const WorkItem* __restrict__ items, int n, int level, int fineSrc,
                                                  int flip) {
    __shared__ LevelArgs<S> sa;
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const WorkItem it = items[w];
        const BatchCase<S>& bc = cases[it.c];
        stage(&sa, &bc.lv[level].a[srcOf(bc, level, fineSrc, flip)]);
        __syncthreads();
        collidePushBody<S, R, OP, ORDER, CUBIC, MRTWB>(sa, it.bx, it.by, it.bz);
        __syncthreads();
    }
}

template <typename S, typename R, int OP, int ORDER, bool CUBIC>
__global__ void __launch_bounds__(TX * TY, TiledMinBlocks<R>::value)
    kb_tiled(const BatchCase<S>* __restrict__ cases, const WorkItem* __restrict__ items, int n, int level, int fineSrc,
             int flip) {
    __shared__ LevelArgs<S> sa;
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const WorkItem it = items[w];
        const BatchCase<S>& bc = cases[it.c];
        stage(&sa, &bc.lv[level].a[srcOf(bc, level, fineSrc, flip)]);
        __syncthreads();
        tiledBody<S, R, OP, ORDER, CUBIC>(sa, bc.lv[level].zChunk, it.bx, it.by, it.bz);
        __syncthreads();
    }
}

// the y-marching collide (periodic z of at most MARCH_MAX_NZ planes) over
// (case, x tile, y chunk) items; every case of the group has the same number
// of z planes on the level (blockDim.y)
template <typename S, typename R, int OP, int ORDER, bool CUBIC>
__device__ __forceinline__ void kbMarchBody(const BatchCase<S>* __restrict__ cases, const WorkItem* __restrict__ items,
                                            int n, int level, int fineSrc, int flip) {
    __shared__ LevelArgs<S> sa;
    extern __shared__ __align__(16) unsigned char marchSmem[];
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const WorkItem it = items[w];
        const BatchCase<S>& bc = cases[it.c];
        stage(&sa, &bc.lv[level].a[srcOf(bc, level, fineSrc, flip)]);
        __syncthreads();
        if (MarchPrefetch<R>::value)
            marchBodyPrefetch<S, R, OP, ORDER, CUBIC>(sa, bc.lv[level].zChunk, it.bx, it.by,
                                                      reinterpret_cast<MomR<R>*>(marchSmem));
        else
            marchBody<S, R, OP, ORDER, CUBIC>(sa, bc.lv[level].zChunk, it.bx, it.by,
                                              reinterpret_cast<MomR<R>*>(marchSmem));
        __syncthreads();
    }
}
template <typename S, typename R, int OP, int ORDER, bool CUBIC>
__global__ void __launch_bounds__(MARCH_TX * MARCH_MAX_NZ, TiledMinBlocks<R>::value)
    kb_march(const BatchCase<S>* __restrict__ cases, const WorkItem* __restrict__ items, int n, int level, int fineSrc,
             int flip) {
    kbMarchBody<S, R, OP, ORDER, CUBIC>(cases, items, n, level, fineSrc, flip);
}
template <typename S, typename R, int OP, int ORDER, bool CUBIC>
__global__ void __maxnreg__(ACP_MARCH_REGS_F32)
    kb_march_f32(const BatchCase<S>* __restrict__ cases, const WorkItem* __restrict__ items, int n, int level,
                 int fineSrc, int flip) {
    kbMarchBody<S, R, OP, ORDER, CUBIC>(cases, items, n, level, fineSrc, flip);
}

template <typename S, int ORDER>
__global__ void __launch_bounds__(128) kb_lodi(const BatchCase<S>* __restrict__ cases,
                                               const WorkItem* __restrict__ items, int n, int level, int fineSrc,
                                               int flip, int zy, int tpn) {
    __shared__ LevelArgs<S> sa;
    __shared__ LodiArgs sp;
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const WorkItem it = items[w];
        const BatchCase<S>& bc = cases[it.c];
        const BatchLevel<S>& L = bc.lv[level];
        stage(&sa, &L.a[srcOf(bc, level, fineSrc, flip)]);
        stage(&sp, &L.lodi);
        __syncthreads();
        lodiBody<S, ORDER>(sa.A, sa.B, zy ? L.lodiZY : L.lodiX, zy ? L.nLodiZY : L.nLodiX, sp, sa, it.bx, tpn);
        __syncthreads();
    }
}

template <typename S, typename R>
__global__ void __launch_bounds__(128) kb_c2f_save(const BatchCase<S>* __restrict__ cases,
                                                   const WorkItem* __restrict__ items, int n, int flip) {
    __shared__ LevelArgs<S> sa;
    __shared__ CouplingArgs sc;
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const WorkItem it = items[w];
        const BatchCase<S>& bc = cases[it.c];
        stage(&sa, &bc.lv[0].a[bc.base ^ flip]);
        stage(&sc, &bc.cpl);
        __syncthreads();
        c2fSaveBody<S, R>(sa.A, bc.c2f, bc.nCoinc, (R*)bc.pre, sa, sc, it.bx);
        __syncthreads();
    }
}

// C2F (STD: coincident nodes; DC: the shared nodes) onto fine array fdst
template <typename S, typename R, int ORDER>
__global__ void __launch_bounds__(128) kb_c2f_coincident(const BatchCase<S>* __restrict__ cases,
                                                         const WorkItem* __restrict__ items, int n, int flip,
                                                         int fdst, R th, int direct) {
    __shared__ LevelArgs<S> sa;
    __shared__ CouplingArgs sc;
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const WorkItem it = items[w];
        const BatchCase<S>& bc = cases[it.c];
        stage(&sa, &bc.lv[1].a[fdst]);
        stage(&sc, &bc.cpl);
        __syncthreads();
        S* Bc = bc.lv[0].a[bc.base ^ flip].B;  // the coarse array written by this step
        S* Ff = const_cast<S*>(sa.A);
        if (direct) dcCoupleBody<S, R, ORDER>(Bc, Ff, bc.dc, bc.nCoinc, (const R*)bc.pre, th, bc.dc2, sc, sa, it.bx);
        else c2fCoincidentBody<S, R, ORDER>(Bc, Ff, bc.c2f, bc.nCoinc, (const R*)bc.pre, th, sc, sa, it.bx);
        __syncthreads();
    }
}

template <typename S, typename R>
__global__ void __launch_bounds__(256) kb_c2f_interp(const BatchCase<S>* __restrict__ cases,
                                                     const WorkItem* __restrict__ items, int n, int fdst,
                                                     int centre) {
    __shared__ LevelArgs<S> sa;
    __shared__ CouplingArgs sc;
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const WorkItem it = items[w];
        const BatchCase<S>& bc = cases[it.c];
        stage(&sa, &bc.lv[1].a[fdst]);
        stage(&sc, &bc.cpl);
        __syncthreads();
        const C2FDev* nodes = bc.c2f + bc.nCoinc + (centre ? bc.nMid : 0);
        c2fInterpBody<S, R>(const_cast<S*>(sa.A), nodes, centre ? bc.nCen : bc.nMid, sc, sa, it.bx);
        __syncthreads();
    }
}

template <typename S, typename R, int ORDER>
__global__ void __launch_bounds__(128) kb_f2c(const BatchCase<S>* __restrict__ cases,
                                              const WorkItem* __restrict__ items, int n, int flip) {
    __shared__ LevelArgs<S> sa;
    __shared__ CouplingArgs sc;
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const WorkItem it = items[w];
        const BatchCase<S>& bc = cases[it.c];
        stage(&sa, &bc.lv[1].a[0]);
        stage(&sc, &bc.cpl);
        __syncthreads();
        f2cBody<S, R, ORDER>(sa.A, bc.lv[0].a[bc.base ^ flip].B, bc.f2c, bc.nF2C, sc, sa, it.bx);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// host side

template <typename S>
using KbCollide = void (*)(const BatchCase<S>*, const WorkItem*, int, int, int, int);
template <typename S>
using KbLodi = void (*)(const BatchCase<S>*, const WorkItem*, int, int, int, int, int, int);
template <typename S>
using KbSave = void (*)(const BatchCase<S>*, const WorkItem*, int, int);
template <typename S, typename R>
using KbCoinc = void (*)(const BatchCase<S>*, const WorkItem*, int, int, int, R, int);
template <typename S>
using KbInterp = void (*)(const BatchCase<S>*, const WorkItem*, int, int, int);
template <typename S>
using KbF2C = void (*)(const BatchCase<S>*, const WorkItem*, int, int);

template <typename S, typename R>
KbCollide<S> pickBatchCollide(const acp_case_desc& d) {
    if (needsMoments(d)) {
        const bool cubic = d.cubic_mach != 0;
        if (d.op == OP_RR) {
            switch (d.eq_order) {
                case 2: return kb_tiled<S, R, OP_RR, 2, true>;
                case 3: return kb_tiled<S, R, OP_RR, 3, true>;
                default: return kb_tiled<S, R, OP_RR, 4, true>;
            }
        }
        switch (d.eq_order) {
            case 2: return cubic ? kb_tiled<S, R, OP_HRR, 2, true> : kb_tiled<S, R, OP_HRR, 2, false>;
            case 3: return cubic ? kb_tiled<S, R, OP_HRR, 3, true> : kb_tiled<S, R, OP_HRR, 3, false>;
            default: return cubic ? kb_tiled<S, R, OP_HRR, 4, true> : kb_tiled<S, R, OP_HRR, 4, false>;
        }
    }
    switch (d.op) {
        case OP_SRT:
            switch (d.eq_order) {
                case 2: return kb_collide<S, R, OP_SRT, 2, false, false>;
                case 3: return kb_collide<S, R, OP_SRT, 3, false, false>;
                default: return kb_collide<S, R, OP_SRT, 4, false, false>;
            }
        case OP_MRT_GS:
            return d.mrt_writeback ? kb_collide<S, R, OP_MRT_GS, 2, false, true> : kb_collide<S, R, OP_MRT_GS, 2, false, false>;
        case OP_MRT_RM:
            return d.mrt_writeback ? kb_collide<S, R, OP_MRT_RM, 2, false, true> : kb_collide<S, R, OP_MRT_GS, 2, false, false>;
        default:
            switch (d.eq_order) {
                case 2: return kb_collide<S, R, OP_RR, 2, false, false>;
                case 3: return kb_collide<S, R, OP_RR, 3, false, false>;
                default: return kb_collide<S, R, OP_RR, 4, false, false>;
            }
    }
}

template <typename S, typename R, int OP, int ORDER, bool CUBIC>
KbCollide<S> batchMarchKernel() {
    if constexpr (sizeof(R) == 8) return kb_march<S, R, OP, ORDER, CUBIC>;
    else return kb_march_f32<S, R, OP, ORDER, CUBIC>;
}
template <typename S, typename R>
KbCollide<S> pickBatchMarch(const acp_case_desc& d) {
    const bool cubic = d.cubic_mach != 0;
    if (d.op == OP_RR) {
        switch (d.eq_order) {
            case 2: return batchMarchKernel<S, R, OP_RR, 2, true>();
            case 3: return batchMarchKernel<S, R, OP_RR, 3, true>();
            default: return batchMarchKernel<S, R, OP_RR, 4, true>();
        }
    }
    switch (d.eq_order) {
        case 2: return cubic ? batchMarchKernel<S, R, OP_HRR, 2, true>() : batchMarchKernel<S, R, OP_HRR, 2, false>();
        case 3: return cubic ? batchMarchKernel<S, R, OP_HRR, 3, true>() : batchMarchKernel<S, R, OP_HRR, 3, false>();
        default: return cubic ? batchMarchKernel<S, R, OP_HRR, 4, true>() : batchMarchKernel<S, R, OP_HRR, 4, false>();
    }
}

template <typename S>
KbLodi<S> pickBatchLodi(int o) { return o == 2 ? kb_lodi<S, 2> : (o == 3 ? kb_lodi<S, 3> : kb_lodi<S, 4>); }
template <typename S, typename R>
KbCoinc<S, R> pickBatchCoinc(int o) {
    return o == 2 ? kb_c2f_coincident<S, R, 2> : (o == 3 ? kb_c2f_coincident<S, R, 3> : kb_c2f_coincident<S, R, 4>);
}
template <typename S, typename R>
KbF2C<S> pickBatchF2C(int o) { return o == 2 ? kb_f2c<S, R, 2> : (o == 3 ? kb_f2c<S, R, 3> : kb_f2c<S, R, 4>); }

// z planes of a level when its neighbour-moment collide is the y-marching
// one (those planes are the block's second dimension), else 0
int marchPlanes(const acp_handle* h, int l) {
    const LevelHost& L = h->host[l];
    return needsMoments(h->d) && marchesY(L) ? L.nz : 0;
}

using GroupKey = std::tuple<int, int, int, int, int, int, int, int, int>;

// the kernel-template key of a case: cases with equal keys form one group
GroupKey groupKey(const acp_handle* h) {
    const acp_case_desc& d = h->d;
    const int levels = (int)h->host.size();
    const bool mrt = d.op == OP_MRT_GS || d.op == OP_MRT_RM;
    const int op = (mrt && !d.mrt_writeback) ? -1 : d.op;  // the reference's MRT no-op forms share a kernel
    return std::make_tuple(d.storage, op, mrt ? 0 : d.eq_order, d.cubic_mach && (d.op == OP_RR || d.op == OP_HRR),
                           mrt ? d.mrt_writeback : 0, levels, levels == 2 ? (d.coupling != ACP_COUPLING_STD) : 0,
                           marchPlanes(h, 0), levels == 2 ? marchPlanes(h, 1) : 0);
}

struct Range {
    int off = 0, count = 0;
};

struct TuneConfig {
    int persist = 0;      // 0: one block per item; k > 0: k x the resident blocks of the device
    int largestFirst = 0; // item order: cases by descending node count
    int chunkScale = 1;   // multiplier of the tiled kernel's z chunk
};

struct Group {
    std::vector<int> members;  // indices into acp_batch::cases
    int storage = 0;
    int levels = 1;
    bool direct = false;
    bool tiled = false;
    int marchNz[2] = {0, 0};  // per level: z planes of the y-marching collide (0: not marching)
    int lodiTpn = LODI_TPN_CLASSICAL;  // lanes per LODI node: lodiLanes of the members (any with transverse terms: 8)
    void* dCases = nullptr;
    WorkItem* dItems = nullptr;
    // item ranges per phase
    Range collide[2], lodiX[2], lodiZY[2], save, coinc, mid, cen, f2c;
    cudaStream_t stream = nullptr;
    cudaEvent_t joined = nullptr;
    cudaStream_t side = nullptr;  // the coarse step beside the first fine sub-step
    cudaEvent_t sideFork = nullptr, sideJoin = nullptr;
    int resident[9] = {0};  // resident blocks per SM of each batch kernel (occupancy; 6, 7: march per level)
};

}  // namespace acp

using namespace acp;

struct acp_batch {
    std::vector<acp_handle*> cases;
    std::vector<Group> groups;
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t forked = nullptr, done = nullptr;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int flip = 0;
    long long steps = 0;
    TuneConfig cfg;
    std::string err;
    std::string report;
    std::vector<const void*> bulk;  // collide kernels of the captured step (instantiateWithPriorities)
};

namespace acp {

cudaEvent_t batchDoneEvent(acp_batch* b) { return b ? b->done : nullptr; }

namespace {

int bfail(acp_batch* b, int code, const char* fmt, ...) {
    if (b) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        std::vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        b->err = buf;
    }
    return code;
}

#define BCU(b, call)                                                                                       \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) return bfail((b), ACP_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// base: the coarse array the case reads when the batch's step counter is even
template <typename S>
BatchCase<S> caseRecord(const acp_handle* h, int chunkScale, int base) {
    BatchCase<S> r;
    std::memset(&r, 0, sizeof r);
    for (size_t l = 0; l < h->host.size(); ++l) {
        BatchLevel<S>& L = r.lv[l];
        L.a[0] = levelArgs<S>(h, (int)l, 0);
        L.a[1] = levelArgs<S>(h, (int)l, 1);
        L.lodi = lodiArgsOf(h, (int)l);
        L.lodiX = h->dev[l].lodiX;
        L.lodiZY = h->dev[l].lodiZY;
        L.nLodiX = h->dev[l].nLodiX;
        L.nLodiZY = h->dev[l].nLodiZY;
        const LevelHost& H = h->host[l];
        // the y-marching collide takes its y chunk in the same field
        if (marchPlanes(h, (int)l))
            L.zChunk = std::min(H.ny, marchChunkFor(H, h->d.storage == ACP_STORE_F64 ? 8 : 4) * chunkScale);
        else
            L.zChunk = (H.per[2] && H.nz <= 3) ? H.nz : std::min(H.nz, tiledChunk(H) * chunkScale);
    }
    if (h->host.size() == 2) {
        r.cpl = couplingArgs(h);
        r.c2f = h->dC2F;
        r.f2c = h->dF2C;
        r.dc = h->dDC;
        r.pre = h->dPre;
        r.nCoinc = h->nCoinc;
        r.nMid = h->nMid;
        r.nCen = h->nCen;
        r.nF2C = (int)h->f2cHost.size();
        r.dc2 = h->d.coupling == ACP_COUPLING_DC2;
    }
    r.base = base;
    return r;
}

// blocks of a level's collide launch that hold at least one live node
void collideItems(const LevelHost& L, int c, bool tiled, bool march, int zChunk, std::vector<WorkItem>& out) {
    auto live = [&](int i0, int i1, int j0, int j1, int k0, int k1) {
        for (int k = k0; k < k1; ++k)
            for (int j = j0; j < j1; ++j) {
                const uint8_t* row = L.code.data() + ((long long)k * L.ny + j) * L.nx;
                for (int i = i0; i < i1; ++i)
                    if (row[i] != CODE_DEAD) return true;
            }
        return false;
    };
    if (march) {
        // x tiles of MARCH_STEP collided nodes, y chunks of zChunk rows, whole z columns
        const int gx = (L.nx + MARCH_STEP - 1) / MARCH_STEP, gy = (L.ny + zChunk - 1) / zChunk;
        for (int by = 0; by < gy; ++by)
            for (int bx = 0; bx < gx; ++bx)
                if (live(bx * MARCH_STEP, std::min(L.nx, bx * MARCH_STEP + MARCH_STEP), by * zChunk,
                         std::min(L.ny, by * zChunk + zChunk), 0, L.nz))
                    out.push_back({c, bx, by, 0});
    } else if (tiled) {
        const int gx = (L.nx + TX - 1) / TX, gy = (L.ny + TY - 1) / TY, gz = (L.nz + zChunk - 1) / zChunk;
        for (int bz = 0; bz < gz; ++bz)
            for (int by = 0; by < gy; ++by)
                for (int bx = 0; bx < gx; ++bx)
                    if (live(bx * TX, std::min(L.nx, bx * TX + TX), by * TY, std::min(L.ny, by * TY + TY), bz * zChunk,
                             std::min(L.nz, bz * zChunk + zChunk)))
                        out.push_back({c, bx, by, bz});
    } else {
        const int gx = (L.nx + 127) / 128;
        for (int k = 0; k < L.nz; ++k)
            for (int j = 0; j < L.ny; ++j)
                for (int bx = 0; bx < gx; ++bx)
                    if (live(bx * 128, std::min(L.nx, bx * 128 + 128), j, j + 1, k, k + 1)) out.push_back({c, bx, j, k});
    }
}

void blockItems(int c, long long threads, int block, std::vector<WorkItem>& out) {
    const long long nb = (threads + block - 1) / block;
    for (long long b = 0; b < nb; ++b) out.push_back({c, (int)b, 0, 0});
}

template <typename S>
void releaseGroup(Group& g) {
    cudaFree(g.dCases);
    cudaFree(g.dItems);
    g.dCases = nullptr;
    g.dItems = nullptr;
}

// case records and work lists of one group under the tuning configuration
template <typename S>
int buildGroup(acp_batch* b, Group& g) {
    releaseGroup<S>(g);
    std::vector<int> order(g.members.size());
    std::iota(order.begin(), order.end(), 0);
    if (b->cfg.largestFirst) {
        auto size = [&](int m) {
            const acp_handle* h = b->cases[g.members[m]];
            long long n = 0;
            for (const LevelHost& L : h->host) n += L.active;
            return n;
        };
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return size(x) > size(y); });
    }
    std::vector<BatchCase<S>> recs;
    for (int m : order) {
        const acp_handle* h = b->cases[g.members[m]];
        recs.push_back(caseRecord<S>(h, b->cfg.chunkScale, h->cur ^ b->flip));
    }
    std::vector<WorkItem> items;
    auto phase = [&](Range& r, auto&& fill) {
        r.off = (int)items.size();
        for (int c = 0; c < (int)recs.size(); ++c) fill(c, b->cases[g.members[order[c]]]);
        r.count = (int)items.size() - r.off;
    };
    for (int l = 0; l < g.levels; ++l) {
        phase(g.collide[l], [&](int c, const acp_handle* h) {
            collideItems(h->host[l], c, g.tiled, g.marchNz[l] > 0, recs[c].lv[l].zChunk, items);
        });
        phase(g.lodiX[l], [&](int c, const acp_handle* h) { blockItems(c, h->dev[l].nLodiX * g.lodiTpn, 128, items); });
        phase(g.lodiZY[l], [&](int c, const acp_handle* h) { blockItems(c, h->dev[l].nLodiZY * g.lodiTpn, 128, items); });
    }
    if (g.levels == 2) {
        phase(g.save, [&](int c, const acp_handle* h) {
            blockItems(c, (long long)h->nCoinc * coincidentThreadsPerNode(couplingArgs(h)), 128, items);
        });
        phase(g.coinc, [&](int c, const acp_handle* h) {
            blockItems(c, (long long)h->nCoinc * (h->dcHost.empty() ? coincidentThreadsPerNode(couplingArgs(h)) : DC_TPN),
                       128, items);
        });
        phase(g.mid, [&](int c, const acp_handle* h) {
            blockItems(c, (long long)h->nMid * interpComponents(h), 256, items);
        });
        phase(g.cen, [&](int c, const acp_handle* h) {
            blockItems(c, (long long)h->nCen * interpComponents(h), 256, items);
        });
        phase(g.f2c, [&](int c, const acp_handle* h) { blockItems(c, (long long)h->f2cHost.size() * 32, 128, items); });
    }
    BCU(b, cudaMalloc(&g.dCases, std::max<size_t>(1, recs.size()) * sizeof(BatchCase<S>)));
    BCU(b, cudaMalloc((void**)&g.dItems, std::max<size_t>(1, items.size()) * sizeof(WorkItem)));
    BCU(b, cudaMemcpyAsync(g.dCases, recs.data(), recs.size() * sizeof(BatchCase<S>), cudaMemcpyHostToDevice, b->stream));
    if (!items.empty())
        BCU(b, cudaMemcpyAsync(g.dItems, items.data(), items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice, b->stream));
    BCU(b, cudaStreamSynchronize(b->stream));
    return ACP_OK;
}

int gridFor(const acp_batch* b, int items, int residentPerSm) {
    if (items <= 0) return 0;
    if (b->cfg.persist <= 0) return items;
    const long long cap = (long long)b->cfg.persist * std::max(1, residentPerSm) * b->sms;
    return (int)std::min<long long>(items, cap);
}

template <typename S, typename R>
int occupancy(Group& g, const acp_case_desc& d) {
    auto occ = [](const void* fn, int block) {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, block, 0) != cudaSuccess) n = 1;
        return std::max(1, n);
    };
    const int o = d.eq_order;
    g.resident[0] = occ((const void*)pickBatchCollide<S, R>(d), g.tiled ? TX * TY : 128);
    g.resident[1] = occ((const void*)pickBatchLodi<S>(o), 128);
    g.resident[2] = occ((const void*)kb_c2f_save<S, R>, 128);
    g.resident[3] = occ((const void*)pickBatchCoinc<S, R>(o), 128);
    g.resident[4] = occ((const void*)kb_c2f_interp<S, R>, 256);
    g.resident[5] = occ((const void*)pickBatchF2C<S, R>(o), 128);
    for (int l = 0; l < 2; ++l)
        if (g.marchNz[l]) {
            int m = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&m, (const void*)pickBatchMarch<S, R>(d),
                                                              MARCH_TX * g.marchNz[l],
                                                              marchSmemBytes<R>(g.marchNz[l])) != cudaSuccess)
                m = 1;
            g.resident[6 + l] = std::max(1, m);
        }
    return ACP_OK;
}

// one coarse step of a group (the sequence of the single-case engine, every
// phase one launch over all of the group's cases)
template <typename S, typename R>
void enqueueGroup(acp_batch* b, Group& g, int flip) {
    const acp_case_desc& d = b->cases[g.members[0]]->d;
    const BatchCase<S>* cs = (const BatchCase<S>*)g.dCases;
    const WorkItem* it = g.dItems;
    cudaStream_t st = g.stream;
    const int o = d.eq_order;
    KbCollide<S> collide = pickBatchCollide<S, R>(d);
    noteBulk(b->bulk, (const void*)collide);
    for (int l = 0; l < g.levels; ++l)
        if (g.marchNz[l]) noteBulk(b->bulk, (const void*)pickBatchMarch<S, R>(d));
    KbLodi<S> lodi = pickBatchLodi<S>(o);
    const dim3 cblock = g.tiled ? dim3(TX, TY) : dim3(128);
    auto levelStep = [&](int l, int fineSrc, cudaStream_t ls) {
        if (g.collide[l].count && g.marchNz[l])
            pickBatchMarch<S, R>(d)<<<gridFor(b, g.collide[l].count, g.resident[6 + l]), dim3(MARCH_TX, g.marchNz[l]),
                                      marchSmemBytes<R>(g.marchNz[l]), ls>>>(cs, it + g.collide[l].off,
                                                                             g.collide[l].count, l, fineSrc, flip);
        else if (g.collide[l].count)
            collide<<<gridFor(b, g.collide[l].count, g.resident[0]), cblock, 0, ls>>>(cs, it + g.collide[l].off,
                                                                                     g.collide[l].count, l, fineSrc,
                                                                                     flip);
        if (g.lodiX[l].count)
            lodi<<<gridFor(b, g.lodiX[l].count, g.resident[1]), 128, 0, ls>>>(cs, it + g.lodiX[l].off,
                                                                             g.lodiX[l].count, l, fineSrc, flip, 0,
                                                                             g.lodiTpn);
        if (g.lodiZY[l].count)
            lodi<<<gridFor(b, g.lodiZY[l].count, g.resident[1]), 128, 0, ls>>>(cs, it + g.lodiZY[l].off,
                                                                              g.lodiZY[l].count, l, fineSrc, flip, 1,
                                                                              g.lodiTpn);
    };
    if (g.levels == 1) {
        levelStep(0, 0, st);
        return;
    }
    KbCoinc<S, R> coinc = pickBatchCoinc<S, R>(o);
    auto c2f = [&](int fdst, R th) {
        if (g.coinc.count)
            coinc<<<gridFor(b, g.coinc.count, g.resident[3]), 128, 0, st>>>(cs, it + g.coinc.off, g.coinc.count, flip,
                                                                            fdst, th, g.direct ? 1 : 0);
        if (g.mid.count)
            kb_c2f_interp<S, R><<<gridFor(b, g.mid.count, g.resident[4]), 256, 0, st>>>(cs, it + g.mid.off,
                                                                                       g.mid.count, fdst, 0);
        if (g.cen.count)
            kb_c2f_interp<S, R><<<gridFor(b, g.cen.count, g.resident[4]), 256, 0, st>>>(cs, it + g.cen.off,
                                                                                       g.cen.count, fdst, 1);
    };
    // the coarse step (and the saving of the coupling sources) beside the first fine sub-step
    cudaEventRecord(g.sideFork, st);
    cudaStreamWaitEvent(g.side, g.sideFork, 0);
    if (g.save.count)
        kb_c2f_save<S, R><<<gridFor(b, g.save.count, g.resident[2]), 128, 0, g.side>>>(cs, it + g.save.off,
                                                                                      g.save.count, flip);
    levelStep(0, 0, g.side);  // coarse t -> t+1
    levelStep(1, 0, st);      // fine t -> t+1/2
    cudaEventRecord(g.sideJoin, g.side);
    cudaStreamWaitEvent(st, g.sideJoin, 0);
    c2f(1, R(0.5));   // C2F (or direct coupling, fine side) at t+1/2
    levelStep(1, 1, st);  // fine t+1/2 -> t+1
    if (g.f2c.count)
        pickBatchF2C<S, R>(o)<<<gridFor(b, g.f2c.count, g.resident[5]), 128, 0, st>>>(cs, it + g.f2c.off,
                                                                                      g.f2c.count, flip);
    c2f(0, R(1));     // C2F at t+1 (direct coupling: both sides)
}

// pressure probes of a case after the step (as the single-case engine samples them)
void enqueueProbes(const acp_batch* b, acp_handle* h, cudaStream_t st, int flip) {
    if (!h->nProbes) return;
    const int coarseNew = 1 - (h->cur ^ b->flip ^ flip);
    switch (h->d.storage) {
        case ACP_STORE_F64: launchProbes<double>(h, st, coarseNew); break;
        case ACP_STORE_F32_DEV: launchProbes<float>(h, st, coarseNew); break;
        default: launchProbes<__half>(h, st, coarseNew); break;
    }
}

int enqueueBatchStep(acp_batch* b, int flip) {
    BCU(b, cudaEventRecord(b->forked, b->stream));
    for (Group& g : b->groups) {
        BCU(b, cudaStreamWaitEvent(g.stream, b->forked, 0));
        switch (g.storage) {
            case ACP_STORE_F64: enqueueGroup<double, double>(b, g, flip); break;
            case ACP_STORE_F32_DEV: enqueueGroup<float, float>(b, g, flip); break;
            default: enqueueGroup<__half, float>(b, g, flip); break;
        }
        for (int m : g.members) enqueueProbes(b, b->cases[m], g.stream, flip);
        BCU(b, cudaEventRecord(g.joined, g.stream));
        BCU(b, cudaStreamWaitEvent(b->stream, g.joined, 0));
    }
    BCU(b, cudaGetLastError());
    return ACP_OK;
}

void destroyBatchGraphs(acp_batch* b) {
    for (int p = 0; p < 2; ++p)
        if (b->graph[p]) {
            cudaGraphExecDestroy(b->graph[p]);
            b->graph[p] = nullptr;
        }
}

int buildAll(acp_batch* b) {
    destroyBatchGraphs(b);
    for (Group& g : b->groups) {
        int s;
        switch (g.storage) {
            case ACP_STORE_F64: s = buildGroup<double>(b, g); break;
            case ACP_STORE_F32_DEV: s = buildGroup<float>(b, g); break;
            default: s = buildGroup<__half>(b, g); break;
        }
        if (s) return s;
    }
    // one graph per parity of the batch's step counter
    for (int p = 0; p < 2; ++p) {
        cudaGraph_t graph;
        b->bulk.clear();
        BCU(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        int s = enqueueBatchStep(b, p);
        cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
        if (s) return s;
        if (e != cudaSuccess) return bfail(b, ACP_ERR_CUDA, "batch graph capture: %s", cudaGetErrorString(e));
        e = instantiateWithPriorities(&b->graph[p], graph, b->bulk);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return bfail(b, ACP_ERR_CUDA, "batch graph instantiate: %s", cudaGetErrorString(e));
    }
    return ACP_OK;
}

int runSteps(acp_batch* b, int n) {
    for (int s = 0; s < n; ++s) {
        BCU(b, cudaGraphLaunch(b->graph[b->flip], b->stream));
        b->flip ^= 1;
        ++b->steps;
        for (acp_handle* h : b->cases) {
            h->cur ^= 1;
            ++h->steps;
        }
    }
    BCU(b, cudaEventRecord(b->done, b->stream));
    return ACP_OK;
}

}  // namespace
}  // namespace acp

namespace {
std::mutex g_batchConstMutex;
bool g_batchConstUploaded[64] = {false};

// batch.cu's own copies of the constant tables, once per device
int uploadBatchConstants(int device) {
    if (device < 0 || device >= 64) return ACP_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_batchConstMutex);
    if (g_batchConstUploaded[device]) return ACP_OK;
    ConstTables t;
    int s = makeConstTables(t);
    if (s) return s;
    if ((s = uploadTables(t))) return s;
    g_batchConstUploaded[device] = true;
    return ACP_OK;
}
}  // namespace

extern "C" {

int acp_batch_create(acp_handle* const* cases, int n, acp_batch** out) {
    if (!out) return ACP_ERR_INVALID;
    *out = nullptr;
    acp_batch* b = new acp_batch();
    *out = b;
    if (n <= 0 || !cases) return bfail(b, ACP_ERR_INVALID, "a batch needs at least one case");
    for (int i = 0; i < n; ++i) {
        acp_handle* h = cases[i];
        if (!h || !h->inited) return bfail(b, ACP_ERR_STATE, "case %d is not initialised", i);
        if (h->batch) return bfail(b, ACP_ERR_STATE, "case %d already belongs to a batch", i);
        if (h->device != cases[0]->device) return bfail(b, ACP_ERR_INVALID, "cases on different devices");
        for (int j = 0; j < i; ++j)
            if (cases[j] == h) return bfail(b, ACP_ERR_INVALID, "case %d appears twice", i);
    }
    b->device = cases[0]->device;
    BCU(b, cudaSetDevice(b->device));
    if (int s0 = uploadBatchConstants(b->device)) return bfail(b, s0, "uploading lattice constants failed");
    BCU(b, cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device));
    BCU(b, cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    BCU(b, cudaEventCreateWithFlags(&b->forked, cudaEventDisableTiming));
    BCU(b, cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming));
    std::map<GroupKey, int> index;
    for (int i = 0; i < n; ++i) {
        acp_handle* h = cases[i];
        BCU(b, cudaStreamSynchronize(h->stream));  // the case's own pending work
        b->cases.push_back(h);
        const int levels = (int)h->host.size();
        auto key = groupKey(h);
        auto f = index.find(key);
        if (f == index.end()) {
            Group g;
            g.storage = h->d.storage;
            g.levels = levels;
            g.direct = levels == 2 && h->d.coupling != ACP_COUPLING_STD;
            g.tiled = needsMoments(h->d);
            for (int l = 0; l < levels; ++l) g.marchNz[l] = marchPlanes(h, l);
            index[key] = (int)b->groups.size();
            b->groups.push_back(g);
            f = index.find(key);
        }
        b->groups[f->second].members.push_back(i);
        b->groups[f->second].lodiTpn = std::max(b->groups[f->second].lodiTpn, lodiLanes(h->d.transverse));
    }
    for (Group& g : b->groups) {
        BCU(b, cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
        BCU(b, cudaEventCreateWithFlags(&g.joined, cudaEventDisableTiming));
        BCU(b, cudaStreamCreateWithFlags(&g.side, cudaStreamNonBlocking));
        BCU(b, cudaEventCreateWithFlags(&g.sideFork, cudaEventDisableTiming));
        BCU(b, cudaEventCreateWithFlags(&g.sideJoin, cudaEventDisableTiming));
        const acp_case_desc& d = b->cases[g.members[0]]->d;
        switch (g.storage) {
            case ACP_STORE_F64: occupancy<double, double>(g, d); break;
            case ACP_STORE_F32_DEV: occupancy<float, float>(g, d); break;
            default: occupancy<__half, float>(g, d); break;
        }
    }
    int s = buildAll(b);
    if (s) return s;
    for (acp_handle* h : b->cases) h->batch = b;
    return ACP_OK;
}

int acp_batch_step(acp_batch* b, int n) {
    if (!b || b->cases.empty() || !b->graph[0]) return ACP_ERR_STATE;
    if (n < 0) return bfail(b, ACP_ERR_INVALID, "negative step count");
    BCU(b, cudaSetDevice(b->device));
    return runSteps(b, n);
}

int acp_batch_sync(acp_batch* b) {
    if (!b || b->cases.empty()) return ACP_ERR_STATE;
    BCU(b, cudaSetDevice(b->device));
    BCU(b, cudaStreamSynchronize(b->stream));
    for (acp_handle* h : b->cases) {
        int s = acp_sync(h);
        if (s) return bfail(b, s, "case %s", acp_last_error(h));
    }
    return ACP_OK;
}

int acp_batch_tune(acp_batch* b, int trial_steps, char* report, size_t report_len) {
    if (!b || b->cases.empty()) return ACP_ERR_STATE;
    if (trial_steps <= 0) return bfail(b, ACP_ERR_INVALID, "trial_steps must be positive");
    BCU(b, cudaSetDevice(b->device));
    bool any3d = false;
    for (acp_handle* h : b->cases)
        for (const LevelHost& L : h->host)
            if (needsMoments(h->d) && !(L.per[2] && L.nz <= 3) && L.nz > 8) any3d = true;
    std::vector<TuneConfig> cands;
    for (int persist : {0, 1, 2, 4})
        for (int lf : {0, 1})
            for (int cs : any3d ? std::vector<int>{1, 2} : std::vector<int>{1}) cands.push_back({persist, lf, cs});
    cudaEvent_t e0, e1;
    BCU(b, cudaEventCreate(&e0));
    BCU(b, cudaEventCreate(&e1));
    std::string rep;
    float best = 1e30f;
    TuneConfig bestCfg = b->cfg;
    for (const TuneConfig& c : cands) {
        b->cfg = c;
        int s = buildAll(b);
        if (s) return s;
        if ((s = runSteps(b, 1))) return s;  // warm
        BCU(b, cudaEventRecord(e0, b->stream));
        if ((s = runSteps(b, trial_steps))) return s;
        BCU(b, cudaEventRecord(e1, b->stream));
        BCU(b, cudaEventSynchronize(e1));
        float ms = 0;
        BCU(b, cudaEventElapsedTime(&ms, e0, e1));
        ms /= trial_steps;
        char line[160];
        std::snprintf(line, sizeof line, "persist=%d largest_first=%d chunk_scale=%d: %.4f ms/step\n", c.persist,
                      c.largestFirst, c.chunkScale, ms);
        rep += line;
        if (ms < best) {
            best = ms;
            bestCfg = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->cfg = bestCfg;
    int s = buildAll(b);
    if (s) return s;
    char line[160];
    std::snprintf(line, sizeof line, "chosen: persist=%d largest_first=%d chunk_scale=%d (%.4f ms/step)\n",
                  bestCfg.persist, bestCfg.largestFirst, bestCfg.chunkScale, best);
    rep += line;
    b->report = rep;
    if (report && report_len) {
        std::snprintf(report, report_len, "%s", rep.c_str());
    }
    return ACP_OK;
}

int acp_batch_configure(acp_batch* b, int persist, int largest_first, int chunk_scale) {
    if (!b || b->cases.empty()) return ACP_ERR_STATE;
    if (persist < 0 || chunk_scale < 1) return bfail(b, ACP_ERR_INVALID, "persist >= 0 and chunk_scale >= 1");
    BCU(b, cudaSetDevice(b->device));
    BCU(b, cudaStreamSynchronize(b->stream));
    b->cfg = {persist, largest_first ? 1 : 0, chunk_scale};
    return buildAll(b);
}

int acp_batch_info(acp_batch* b, int* groups, int* launches_per_step, long long* updates_per_step) {
    if (!b) return ACP_ERR_INVALID;
    int launches = 0;
    long long upd = 0;
    for (const Group& g : b->groups) {
        const Range* rs[] = {&g.collide[0], &g.collide[1], &g.lodiX[0], &g.lodiX[1], &g.lodiZY[0], &g.lodiZY[1],
                             &g.save, &g.f2c};
        for (const Range* r : rs)
            if (r->count) ++launches;
        for (int l = 1; l < g.levels; ++l) {
            // fine collide and LODI run in both sub-steps
            launches += (g.collide[l].count ? 1 : 0) + (g.lodiX[l].count ? 1 : 0) + (g.lodiZY[l].count ? 1 : 0);
        }
        launches += 2 * ((g.coinc.count ? 1 : 0) + (g.mid.count ? 1 : 0) + (g.cen.count ? 1 : 0));
        for (int m : g.members) {
            const acp_handle* h = b->cases[m];
            upd += h->host[0].active + (h->host.size() > 1 ? 2 * h->host[1].active : 0);
            if (h->nProbes) ++launches;
        }
    }
    if (groups) *groups = (int)b->groups.size();
    if (launches_per_step) *launches_per_step = launches;
    if (updates_per_step) *updates_per_step = upd;
    return ACP_OK;
}

int acp_batch_destroy(acp_batch* b) {
    if (!b) return ACP_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    destroyBatchGraphs(b);
    for (Group& g : b->groups) {
        cudaFree(g.dCases);
        cudaFree(g.dItems);
        if (g.stream) cudaStreamDestroy(g.stream);
        if (g.joined) cudaEventDestroy(g.joined);
        if (g.side) cudaStreamDestroy(g.side);
        if (g.sideFork) cudaEventDestroy(g.sideFork);
        if (g.sideJoin) cudaEventDestroy(g.sideJoin);
    }
    for (acp_handle* h : b->cases)
        if (h->batch == b) h->batch = nullptr;
    if (b->forked) cudaEventDestroy(b->forked);
    if (b->done) cudaEventDestroy(b->done);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return ACP_OK;
}

const char* acp_batch_last_error(const acp_batch* b) { return b ? b->err.c_str() : "null batch"; }

}  // extern "C"

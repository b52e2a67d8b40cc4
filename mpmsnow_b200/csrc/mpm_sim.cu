// Host orchestration of the CUDA implicit MPM snow step and the C-ABI of include/mpm_gpu.h.
//
// One step (Sim::advance, Sim.cpp:57-134) runs as:
//   ballistic update + per-body centre-of-mass / bounding box (one device->host read of B small records)
//   -> per-body grid geometry on the host (Grid.cpp:171-213) -> tile keys, counting sort, state permutation
//   -> P2G mass / velocity, forces, explicit momenta + collisions + initial guess, rhs + Jacobi diagonal
//   -> conjugate residuals, all bodies batched, FP64 segmented reductions, device-side termination
//   -> G2P + F update, plasticity (all particles), collide + advect, body segmentation for the next step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "../../include/mpm_gpu.h"
#include "mpm_kernels.h"
#include "mpm_types.h"

using namespace mpm;

namespace mpm {
long long kernel_launch_count();
void kernel_launch_add(int n);
}

namespace {

struct CudaError {
    cudaError_t e;
    const char* where;
};

#define CK(x)                                                   \
    do {                                                        \
        cudaError_t _e = (x);                                   \
        if (_e != cudaSuccess) throw CudaError{_e, #x};         \
    } while (0)

// device buffers that follow the scene's size: the first allocation reserves twice the need, later growth 50 %,
// so that a run of steps rarely allocates (fresh device memory took up to hundreds of milliseconds to map here)
template <class T> void grow(T*& p, size_t& cap, size_t need) {
    if (need <= cap && p) return;
    size_t n = std::max(p ? need + need / 2 : 2 * need, (size_t)(cap * 1.5)) + 16;
    if (p) CK(cudaFree(p));
    p = nullptr;
    CK(cudaMalloc(&p, n * sizeof(T)));
    cap = n;
}

struct VarInfo {
    const char* name;
    int comps;
};
const VarInfo kVars[] = {{"p", 3}, {"v", 3}, {"F", 9}, {"Fp", 9}, {"FinvTrans", 9}, {"R", 9}, {"Ginv", 9}, {"m", 1},
                         {"volume", 1}, {"J", 1}, {"mu", 1}, {"lambda", 1}, {"mu0", 1}, {"lambda0", 1}};

}  // namespace

struct mpm_sim {
    int device = 0;
    float* collPhi[kMaxColliders] = {};  // grid colliders' samples (device), per collider slot
    float* collVel[kMaxColliders] = {};
    int dim = 3;   // the reference's Sim dimension (Sim.h:88-89): grids span axes 0 .. dim - 1
    cudaStream_t stream = nullptr;
    // the step's second stream, at the device's greatest priority: the advection and the segmentation run there
    // beside the plasticity pass, which touches other particle arrays; evFork / evJoin order them after G2P and
    // before the step's scalars are read
    cudaStream_t side = nullptr;
    cudaEvent_t evFork = nullptr, evJoin = nullptr;
    StepParams sp{};
    int N = 0;
    PartArrays P{}, Q{};        // current state and permutation target
    float* staging = nullptr;   // N * 9 floats
    OpRec opRec{nullptr, nullptr, nullptr};  // the operator's per-particle records of the current step (70 words each)
    int* slotOf = nullptr;
    int* key = nullptr;
    int* rank = nullptr;
    int* inv = nullptr;   // the counting sort's inverse permutation (destination slot -> source slot)
    bool hasMu0 = false;

    int B = 0, nBallistic = 0;  // bodies from the last segmentation
    std::vector<BodyGrid> grids;
    std::vector<int> bodyCount;
    BodyGrid* dGrids = nullptr; size_t capGrids = 0;
    BodyAccum* dAcc = nullptr; size_t capAcc = 0;
    BodySolve* dSolve = nullptr; size_t capSolve = 0;
    int* dChunkBody = nullptr; size_t capChunk = 0;
    int* dCounter = nullptr; size_t capCounter = 0;
    double* dPartial = nullptr; size_t capPartial = 0;
    std::vector<int> chunkBody;
    long long Gtot = 0;
    int nChunks = 0, totalTiles = 0;

    NodeArrays nd{};
    size_t capNodes = 0;
    cudaMemPool_t pool = nullptr;   // the handle's stream-ordered pool (node arrays)
    void* nodeBlock = nullptr;
    float* dbgA = nullptr; float* dbgB = nullptr; float* dbgC = nullptr;
    size_t capDbg = 0;
    TileArrays T{};
    TileArrays contactT{};   // the tiles of T near collided nodes (the rhs's DF(vc))
    size_t capTiles = 0;
    // [0] listCount [1] ndone [2] fp64 count [3] err [4..7] segmentation scalars [8] contact tile count
    // [10] warm-start err
    // [16..21] segmentation bounding box
    int* dScalars = nullptr;
    int* hScalars = nullptr;   // pinned mirror; [20 + 4 k] the CR loop's snapshots of [1..3]
    bool segValid = true;      // the last body segmentation completed without error
    SegArrays S{};
    int2* segEdges[2] = {nullptr, nullptr};  // the segmentations' spanning forests: the last one's, the next one's
    int hashBits = 0;
    size_t capSeg = 0;
    int* scanTmp = nullptr; size_t capScan = 0;
    bool gridsValid = false;
    std::string lastError;
    size_t capN = 0;
    // phase profiler: CUDA events on the launching stream around each launch
    struct ProfRec {
        int phase;
        int a, b;        // event pool indices
        int slot;        // operator launches: particle counter slot, else -1
        double particles, nodes;
    };
    bool profOn = false;
    std::vector<ProfRec> recs;
    std::vector<cudaEvent_t> evPool;
    size_t evUsed = 0;
    unsigned long long* dProc = nullptr;
    int procUsed = 0;
    // learned warm start
    struct WarmStart {
        bool on = false;
        bool net = false;                  // a network is installed (else the guess is p*/m and the history)
        bool useHist = false;
        bool extrapolate = false;          // without a network: add h1 - h2 to the guess
        // the last two records (see mpm_nn.h): [0] h1 of the previous step, [1] h2 of the one before
        float* hist[2] = {nullptr, nullptr};
        size_t capHist[2] = {0, 0};
        std::vector<BodyGrid> histGrids[2];  // the grids each record belongs to
        bool histValid[2] = {false, false};
        void* wf[mpmnn::kLayers] = {};     // bf16 forward packs
        float* bias[mpmnn::kLayers] = {};
        float featScale[mpmnn::kFeat] = {};
        float outScale = 1.f, density = 400.f, lightMass = 0.f;
        int minNodes = 0;
        void* feat = nullptr;              // bf16 [G][16]
        void* actA = nullptr;              // bf16 [G][32]
        void* actB = nullptr;
        float* out = nullptr;              // fp32 [G][3]
        size_t cap = 0;                    // nodes
        unsigned char* blockFlag = nullptr;  // 2 bytes per node: distance to the nearest heavy node
        int* blockList = nullptr;            // kLayers lists of 8 x 16 x 1 output blocks, capBlocks apart
        int* blockCount = nullptr;           // kLayers counts
        size_t capBlocks = 0;
    } ws;
};

namespace {
enum Phase {
    PH_GRID_SETUP, PH_P2G_MASS, PH_P2G_FORCE, PH_NODE, PH_OP_RHS_DIAG, PH_OP, PH_CR_NODE, PH_G2P,
    PH_PLASTICITY, PH_ADVECT, PH_SEGMENT, PH_PREPARE, PH_HOST_GEOMETRY, PH_WARM_START, PH_COUNT
};
const char* kPhaseNames[PH_COUNT] = {"bin_sort_permute", "p2g_mass_momentum", "p2g_force", "node_explicit_rhs",
                                     "op_rhs_diag", "op_apply", "cr_node", "g2p_F", "plasticity_svd", "advect",
                                     "segment_bodies", "prepare_com_bbox", "host_geometry_sync", "warm_start_net"};
constexpr int kProcSlots = 16384;
constexpr int kScalars = 32;

cudaEvent_t pool_event(mpm_sim* sim) {
    if (sim->evUsed == sim->evPool.size()) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        sim->evPool.push_back(e);
    }
    return sim->evPool[sim->evUsed++];
}
// begin a profiled phase; returns the record index or -1
int pbegin(mpm_sim* sim, int phase, double particles, double nodes, bool countParticles = false,
           cudaStream_t on = nullptr) {
    if (!sim->profOn) return -1;
    mpm_sim::ProfRec r;
    r.phase = phase;
    r.a = (int)sim->evUsed;
    CK(cudaEventRecord(pool_event(sim), on ? on : sim->stream));
    r.b = -1;
    r.slot = (countParticles && sim->procUsed < kProcSlots) ? sim->procUsed++ : -1;
    r.particles = particles;
    r.nodes = nodes;
    sim->recs.push_back(r);
    return (int)sim->recs.size() - 1;
}
void pend(mpm_sim* sim, int idx, cudaStream_t on = nullptr) {
    if (idx < 0) return;
    sim->recs[idx].b = (int)sim->evUsed;
    CK(cudaEventRecord(pool_event(sim), on ? on : sim->stream));
}
unsigned long long* pslot(mpm_sim* sim, int idx) {
    if (idx < 0 || sim->recs[idx].slot < 0) return nullptr;
    return sim->dProc + sim->recs[idx].slot;
}
}  // namespace

namespace {

float* alloc_f(size_t n) { float* p = nullptr; CK(cudaMalloc(&p, n * sizeof(float))); return p; }
int* alloc_i(size_t n) { int* p = nullptr; CK(cudaMalloc(&p, n * sizeof(int))); return p; }

void alloc_part(PartArrays& A, int N) {
    A.x = alloc_f(3ull * N); A.v = alloc_f(3ull * N);
    A.F = alloc_f(9ull * N); A.Fp = alloc_f(9ull * N); A.R = alloc_f(9ull * N); A.FiT = alloc_f(9ull * N); A.Gi = alloc_f(9ull * N);
    A.m = alloc_f(N); A.vol = alloc_f(N); A.J = alloc_f(N); A.mu = alloc_f(N); A.lam = alloc_f(N);
    A.mu0 = nullptr; A.lam0 = nullptr;
    A.orig = alloc_i(N); A.body = alloc_i(N);
}
void free_part(PartArrays& A) {
    float* fs[] = {A.x, A.v, A.F, A.Fp, A.R, A.FiT, A.Gi, A.m, A.vol, A.J, A.mu, A.lam, A.mu0, A.lam0};
    for (float* p : fs) if (p) cudaFree(p);
    if (A.orig) cudaFree(A.orig);
    if (A.body) cudaFree(A.body);
    A = PartArrays{};
}

float** var_ptr(PartArrays& A, const std::string& name, int& comps) {
    comps = 0;
    for (auto& v : kVars) if (name == v.name) comps = v.comps;
    if (name == "p") return &A.x;
    if (name == "v") return &A.v;
    if (name == "F") return &A.F;
    if (name == "Fp") return &A.Fp;
    if (name == "FinvTrans") return &A.FiT;
    if (name == "R") return &A.R;
    if (name == "Ginv") return &A.Gi;
    if (name == "m") return &A.m;
    if (name == "volume") return &A.vol;
    if (name == "J") return &A.J;
    if (name == "mu") return &A.mu;
    if (name == "lambda") return &A.lam;
    if (name == "mu0") return &A.mu0;
    if (name == "lambda0") return &A.lam0;
    return nullptr;
}

__global__ void k_fill_f(float* a, size_t n, float v) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}
__global__ void k_iota(int* a, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
}
__global__ void k_identity9(float* a, int N) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    for (int k = 0; k < 9; ++k) a[(size_t)k * N + i] = (k % 4 == 0) ? 1.f : 0.f;
}
__global__ void k_gather_i(const int* state, const int* slotOf, int* out, int N) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) out[i] = state[slotOf[i]];
}
__global__ void k_debug_cells(PartArrays P, int N, const int* slotOf, const BodyGrid* grids, float h, int* body, int* cell3,
                              int* voxel3) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int s = slotOf[i];
    int b = P.body[s];
    body[i] = b;
    float x[3] = {P.x[s], P.x[N + s], P.x[2 * (size_t)N + s]};
    const float vs = 4.0f * h;  // 2 * supportRadius() * gridSize (Grid.cpp:359)
    for (int a = 0; a < 3; ++a) voxel3[3 * i + a] = (int)floorf(__fdiv_rn(x[a], vs));
    if (b < 0) { cell3[3 * i] = cell3[3 * i + 1] = cell3[3 * i + 2] = -1; return; }
    for (int a = 0; a < 3; ++a)
        cell3[3 * i + a] = grids[b].n[a] == 1 ? 0 : (int)floorf(__fdiv_rn(__fsub_rn(x[a], grids[b].mn[a]), h));
}

void fill_f(float* a, size_t n, float v, cudaStream_t s) {
    if (n) k_fill_f<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, n, v);
}

mpm_status set_err(mpm_sim* sim, mpm_status st, const std::string& msg) {
    if (sim) sim->lastError = msg;
    return st;
}

// Collider slot i from a C-ABI descriptor; a grid collider's samples are copied into device memory the handle
// owns (replacing the slot's previous ones)
mpm_status set_collider(mpm_sim* sim, int i, const mpm_collider& c) {
    if (c.kind != MPM_COLLIDER_PLANE && c.kind != MPM_COLLIDER_CYLINDER && c.kind != MPM_COLLIDER_GRID)
        return MPM_ERR_UNSUPPORTED;
    DevCollider& dc = sim->sp.coll[i];
    float*& phi = sim->collPhi[i];
    float*& vel = sim->collVel[i];
    if (c.kind == MPM_COLLIDER_GRID) {
        const long long cnt = (long long)c.grid_dims[0] * c.grid_dims[1] * c.grid_dims[2];
        if (c.grid_dims[0] < 2 || c.grid_dims[1] < 2 || c.grid_dims[2] < 2 || cnt > (1ll << 31) || !c.grid_phi ||
            !(c.coeffs[3] > 0.f))
            return MPM_ERR_INVALID_ARGUMENT;
        if (phi) CK(cudaFree(phi));
        if (vel) CK(cudaFree(vel));
        phi = vel = nullptr;
        CK(cudaMalloc(&phi, sizeof(float) * cnt));
        CK(cudaMemcpy(phi, c.grid_phi, sizeof(float) * cnt, cudaMemcpyHostToDevice));
        if (c.grid_velocity) {
            CK(cudaMalloc(&vel, 3 * sizeof(float) * cnt));
            CK(cudaMemcpy(vel, c.grid_velocity, 3 * sizeof(float) * cnt, cudaMemcpyHostToDevice));
        }
        for (int k = 0; k < 3; ++k) dc.n[k] = c.grid_dims[k];
    } else {
        for (int k = 0; k < 3; ++k) dc.n[k] = 0;
    }
    dc.kind = c.kind;
    for (int k = 0; k < 4; ++k) dc.c[k] = c.coeffs[k];
    for (int k = 0; k < 3; ++k) dc.vel[k] = c.velocity[k];
    dc.friction = c.friction;
    dc.sticky = c.sticky;
    dc.phi = c.kind == MPM_COLLIDER_GRID ? phi : nullptr;
    dc.v = c.kind == MPM_COLLIDER_GRID ? vel : nullptr;
    return MPM_OK;
}

mpm_status from_device_error(mpm_sim* sim, int e) {
    if (e & ERR_NAN_MASSES) return set_err(sim, MPM_ERR_NAN_MASSES, "nans in splatted masses!");
    if (e & ERR_NAN_VELOCITIES) return set_err(sim, MPM_ERR_NAN_VELOCITIES, "nans in splatted velocities!");
    if (e & ERR_NAN_STRESS) return set_err(sim, MPM_ERR_NAN_STRESS, "nans in dEnergyDensitydF matrix!");
    if (e & ERR_NAN_MOMENTA) return set_err(sim, MPM_ERR_NAN_MOMENTA, "nan in explicit momenta!");
    if (e & ERR_HARDNESS) return set_err(sim, MPM_ERR_INFINITE_HARDNESS, "infinite hardness!!!");
    if (e & ERR_NAN_PARTICLE_V) return set_err(sim, MPM_ERR_NAN_PARTICLE_VELOCITY, "nans in particle velocity data!");
    if (e & ERR_STENCIL_OOB) return set_err(sim, MPM_ERR_INTERNAL, "particle stencil outside its grid");
    if (e & ERR_SEGMENT) return set_err(sim, MPM_ERR_INTERNAL, "body segmentation: a union did not complete");
    return MPM_OK;
}

// ---- body segmentation (Sim::calculateBodies) ------------------------------------------------------------
void segment(mpm_sim* sim, cudaStream_t on = nullptr) {
    const int N = sim->N;
    int bits = 10;
    while ((1ll << bits) < 2ll * N && bits < 30) ++bits;
    if (bits != sim->hashBits || !sim->S.count) {
        SegArrays& S = sim->S;
        if (S.count) { cudaFree(S.count); cudaFree(S.start); }
        S.count = alloc_i(1ull << bits);
        S.start = alloc_i(1ull << bits);
        sim->hashBits = bits;
    }
    if (!sim->S.sorted) {
        SegArrays& S = sim->S;
        S.sorted = alloc_i(N); S.rank = alloc_i(N); S.parent = alloc_i(N); S.size = alloc_i(N); S.minOrig = alloc_i(N);
        S.mark = alloc_i(N); S.mrank = alloc_i(N);
        CK(cudaMalloc(&S.xs, sizeof(float4) * std::max(N, 1)));
        S.nbodies = sim->dScalars + 4;
        S.bbox = reinterpret_cast<unsigned int*>(sim->dScalars + 16);
        for (int2*& e : sim->segEdges) CK(cudaMalloc(&e, sizeof(int2) * std::max(N, 1)));
        S.useEdges = 0;  // the first segmentation of the particles searches its sampled links
    }
    grow(sim->scanTmp, sim->capScan, scan_tmp_ints(std::max<long long>(1ll << bits, N)));
    // the last segmentation's forest in, this one's out; the segmentations run in stream order (the step's side
    // stream joins the main stream before the next step), so the two buffers alternate safely
    sim->S.edgeIn = sim->segEdges[0];
    sim->S.edgeOut = sim->segEdges[1];
    sim->S.slotOf = sim->slotOf;
    launch_segment(sim->P, N, sim->sp.h, sim->S, bits, sim->scanTmp, sim->dScalars + 3, on ? on : sim->stream);
    std::swap(sim->segEdges[0], sim->segEdges[1]);
    sim->S.useEdges = N > 0 ? 1 : 0;
}

void read_scalars(mpm_sim* sim) {
    CK(cudaMemcpyAsync(sim->hScalars, sim->dScalars, 8 * sizeof(int), cudaMemcpyDeviceToHost, sim->stream));
    CK(cudaStreamSynchronize(sim->stream));
}

// Node arrays: one block from the handle's own stream-ordered memory pool, carved into the arrays.  A body
// whose box grows past the capacity reallocates it; freeing and allocating through the pool on the stream takes
// no device-wide synchronisation and reuses the pool's memory (plain cudaFree / cudaMalloc of the arrays took
// from 5 ms up to a second here).
void ensure_nodes(mpm_sim* sim, size_t G) {
    if (G <= sim->capNodes && sim->nodeBlock) return;
    if (!sim->pool) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = sim->device;
        CK(cudaMemPoolCreate(&sim->pool, &props));
        uint64_t keep = UINT64_MAX;  // the pool keeps freed memory for the next growth
        CK(cudaMemPoolSetAttribute(sim->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    if (sim->nodeBlock) CK(cudaFreeAsync(sim->nodeBlock, sim->stream));
    sim->nodeBlock = nullptr;
    // the first reservation is twice the first grid: growing later maps fresh memory on the stream, which took
    // up to hundreds of milliseconds here
    const size_t cap = std::max(sim->nodeBlock ? G + G / 2 : 2 * G, (size_t)(sim->capNodes * 1.5)) + 1024;
    auto al = [](size_t bytes) { return (bytes + 255) / 256 * 256; };
    const size_t a1 = al(cap * sizeof(float)), a3 = al(3 * cap * sizeof(float)), af = al(cap);
    CK(cudaMallocFromPoolAsync(&sim->nodeBlock, a1 + 16 * a3 + af, sim->pool, sim->stream));
    char* q = static_cast<char*>(sim->nodeBlock);
    NodeArrays& n = sim->nd;
    n.mass = reinterpret_cast<float*>(q);
    q += a1;
    float** vec[] = {&n.vel, &n.prev, &n.frc, &n.pstar, &n.b, &n.vc, &n.diag, &n.x, &n.rpc, &n.p, &n.Ap, &n.Ar, &n.dxp,
                     &n.df, &n.vfin, &n.x0};
    for (float** v : vec) {
        *v = reinterpret_cast<float*>(q);
        q += a3;
    }
    n.flag = reinterpret_cast<signed char*>(q);
    sim->capNodes = cap;
}

ReduceArrays reduce_arrays(mpm_sim* sim) {
    ReduceArrays R;
    R.partial = sim->dPartial;
    R.counter = sim->dCounter;
    R.chunkBody = sim->dChunkBody;
    R.ndone = sim->dScalars + 1;
    R.fp64Count = sim->dScalars + 2;
    return R;
}

// Build every body's grid (Grid::Grid, Grid.cpp:156-263 up to the splats): geometry, binning, state sort.
mpm_status build_grids(mpm_sim* sim, bool ballisticUpdate) {
    const int N = sim->N, B = sim->B;
    cudaStream_t s = sim->stream;
    grow(sim->dAcc, sim->capAcc, (size_t)std::max(B, 1));
    std::vector<BodyAccum> acc(std::max(B, 1));
    for (auto& a : acc) {
        std::memset(&a, 0, sizeof(a));
        for (int k = 0; k < 3; ++k) { a.bmin[k] = 0xffffffffu; a.bmax[k] = 0u; }
    }
    CK(cudaMemcpyAsync(sim->dAcc, acc.data(), sizeof(BodyAccum) * acc.size(), cudaMemcpyHostToDevice, s));
    StepParams sp = sim->sp;
    if (!ballisticUpdate) sp.nfields = -1;  // the constructor's grids (Sim.cpp:44-49) move nothing
    int pr = pbegin(sim, PH_PREPARE, N, 0);
    launch_prepare(sim->P, N, sp, sim->dAcc, B, sim->dScalars + 3, s);
    pend(sim, pr);
    if (B == 0) return MPM_OK;
    pr = pbegin(sim, PH_HOST_GEOMETRY, 0, 0);
    CK(cudaMemcpyAsync(acc.data(), sim->dAcc, sizeof(BodyAccum) * B, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    // geometry — Grid.cpp:194-213 (float arithmetic on the host, separately rounded)
    const float h = sim->sp.h;
    sim->grids.resize(B);
    sim->bodyCount.resize(B);
    sim->chunkBody.clear();
    long long nodeOff = 0;
    int tileOff = 0, cta = 0;
    for (int b = 0; b < B; ++b) {
        BodyGrid& g = sim->grids[b];
        const BodyAccum& a = acc[b];
        sim->bodyCount[b] = a.count;
        float mass = (float)a.mass;
        for (int k = 0; k < 3; ++k) g.fv[k] = ballisticUpdate ? (float)(a.mom[k] / a.mass) : 0.f;
        (void)mass;
        long long ncell = 1;
        for (int k = 0; k < 3; ++k) {
            if (k >= sim->dim) {  // Grid.cpp:203-207: the axes a lower-dimensional grid does not span
                g.mn[k] = 0.f;
                g.n[k] = 1;
                g.T[k] = 1;
                continue;
            }
            volatile float lo = ordered_to_float(a.bmin[k]);
            volatile float hi = ordered_to_float(a.bmax[k]);
            volatile float qlo = lo / h, qhi = hi / h;
            int cellMin = int(std::floor((float)qlo)) - 2 - 1;
            int cellMax = int(std::ceil((float)qhi)) + 2 + 1;
            volatile float mn = (float)cellMin * h;
            g.mn[k] = mn;
            g.n[k] = cellMax - cellMin;
            g.T[k] = (g.n[k] + kTile - 1) / kTile;
            ncell *= g.n[k];
        }
        if (ncell > 4000000000LL || ncell <= 0) return set_err(sim, MPM_ERR_GRID_TOO_BIG, "grid is too big");
        long long padded = (ncell + kNodeChunk - 1) / kNodeChunk * kNodeChunk;
        g.nodeOff = nodeOff;
        g.tileOff = tileOff;
        g.ctaBegin = cta;
        g.ctaEnd = cta + (int)(padded / kNodeChunk);
        for (int c = g.ctaBegin; c < g.ctaEnd; ++c) sim->chunkBody.push_back(b);
        cta = g.ctaEnd;
        nodeOff += padded;
        tileOff += g.T[0] * g.T[1] * g.T[2];
    }
    sim->Gtot = nodeOff;
    sim->nChunks = cta;
    sim->totalTiles = tileOff;
    pend(sim, pr);  // host geometry done; the stream was idle since the prepare kernel
    pr = pbegin(sim, PH_GRID_SETUP, N, (double)nodeOff);
    grow(sim->dGrids, sim->capGrids, (size_t)B);
    grow(sim->dChunkBody, sim->capChunk, (size_t)cta);
    grow(sim->dCounter, sim->capCounter, (size_t)B);
    grow(sim->dPartial, sim->capPartial, (size_t)cta * 8);
    grow(sim->dSolve, sim->capSolve, (size_t)B);
    CK(cudaMemcpyAsync(sim->dGrids, sim->grids.data(), sizeof(BodyGrid) * B, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(sim->dChunkBody, sim->chunkBody.data(), sizeof(int) * cta, cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(sim->dCounter, 0, sizeof(int) * B, s));
    CK(cudaMemsetAsync(sim->dSolve, 0, sizeof(BodySolve) * B, s));
    ensure_nodes(sim, (size_t)sim->Gtot);
    NodeArrays& nd = sim->nd;
    CK(cudaMemsetAsync(nd.mass, 0, sizeof(float) * sim->Gtot, s));
    CK(cudaMemsetAsync(nd.vel, 0, 3 * sizeof(float) * sim->Gtot, s));
    CK(cudaMemsetAsync(nd.df, 0, 3 * sizeof(float) * sim->Gtot, s));
    CK(cudaMemsetAsync(nd.diag, 0, 3 * sizeof(float) * sim->Gtot, s));
    CK(cudaMemsetAsync(nd.frc, 0, 3 * sizeof(float) * sim->Gtot, s));  // the force pass adds, k_node_vel adds g m
    // binning and the counting sort by (tile, cell within tile); one extra bucket for ballistic particles
    size_t cells1 = (size_t)sim->totalTiles * kTileCells + 1;
    if (cells1 > sim->capTiles || !sim->T.count) {
        TileArrays& T = sim->T;
        if (T.count) { cudaFree(T.count); cudaFree(T.start); cudaFree(T.list); cudaFree(T.listBody); }
        size_t cap = std::max(sim->capTiles ? cells1 + cells1 / 2 : 2 * cells1, (size_t)(sim->capTiles * 1.5)) + 64;
        T.count = alloc_i(cap); T.start = alloc_i(cap);
        T.list = alloc_i(cap / kTileCells + 64); T.listBody = alloc_i(cap / kTileCells + 64);
        TileArrays& C = sim->contactT;
        if (C.list) { cudaFree(C.list); cudaFree(C.listBody); }
        C.list = alloc_i(cap / kTileCells + 64); C.listBody = alloc_i(cap / kTileCells + 64);
        sim->capTiles = cap;
    }
    sim->T.listCount = sim->dScalars + 0;
    sim->contactT.count = sim->T.count;
    sim->contactT.start = sim->T.start;
    sim->contactT.listCount = sim->dScalars + 8;
    // the tile kernels' scheduling counters (zeroed at allocation; every launch leaves them at 0); the two lists
    // are used by one launch at a time on the handle's stream
    sim->T.sched = sim->dScalars + 28;
    sim->contactT.sched = sim->dScalars + 28;
    CK(cudaMemsetAsync(sim->T.count, 0, sizeof(int) * cells1, s));
    CK(cudaMemsetAsync(sim->T.listCount, 0, sizeof(int), s));
    launch_keys(sim->P, N, sim->dGrids, sim->totalTiles, h, sim->key, sim->rank, sim->T.count, sim->dScalars + 3, s);
    grow(sim->scanTmp, sim->capScan, scan_tmp_ints((long long)cells1));
    scan_exclusive(sim->T.count, sim->T.start, (long long)cells1, sim->scanTmp, sim->dScalars + 7, s);
    // permute the particle state into tile order
    PartArrays& A = sim->P;
    PartArrays& Bq = sim->Q;
    if ((A.mu0 == nullptr) != (A.lam0 == nullptr)) return set_err(sim, MPM_ERR_INTERNAL, "mu0 / lambda0 half allocated");
    if (A.mu0) {
        if (!Bq.mu0) Bq.mu0 = alloc_f(std::max(N, 1));
        if (!Bq.lam0) Bq.lam0 = alloc_f(std::max(N, 1));
    }
    PermuteWords w;
    w.n = 0;
    auto add = [&](const void* src, void* dst, int comps) {
        for (int c = 0; c < comps; ++c) {
            w.src[w.n] = static_cast<const unsigned int*>(src) + (size_t)c * N;
            w.dst[w.n++] = static_cast<unsigned int*>(dst) + (size_t)c * N;
        }
    };
    add(A.x, Bq.x, 3);
    add(A.v, Bq.v, 3);
    add(A.F, Bq.F, 9);
    add(A.Fp, Bq.Fp, 9);
    add(A.R, Bq.R, 9);
    add(A.FiT, Bq.FiT, 9);
    add(A.Gi, Bq.Gi, 9);
    add(A.m, Bq.m, 1);
    add(A.vol, Bq.vol, 1);
    add(A.J, Bq.J, 1);
    add(A.mu, Bq.mu, 1);
    add(A.lam, Bq.lam, 1);
    if (A.mu0) {
        add(A.mu0, Bq.mu0, 1);
        add(A.lam0, Bq.lam0, 1);
    }
    add(A.orig, Bq.orig, 1);
    add(A.body, Bq.body, 1);
    launch_permute_state(sim->key, sim->rank, sim->T.start, N, w, A.orig, sim->slotOf, sim->inv, s);
    std::swap(sim->P, sim->Q);
    launch_tile_list(sim->T.start, sim->dGrids, B, sim->totalTiles, sim->T.list, sim->T.listBody, sim->T.listCount, s);
    // heavy tiles first (the contact list's arrays, rebuilt later in the step, serve as scratch)
    launch_tile_order(sim->T.start, sim->T.list, sim->T.listBody, sim->T.listCount, sim->contactT.list,
                      sim->contactT.listBody, s);
    pend(sim, pr);
    return MPM_OK;
}

void init_state(mpm_sim* sim) {
    const int N = sim->N;
    cudaStream_t s = sim->stream;
    PartArrays& P = sim->P;
    CK(cudaMemsetAsync(P.v, 0, 3 * sizeof(float) * N, s));
    k_identity9<<<(N + 255) / 256, 256, 0, s>>>(P.F, N);
    k_identity9<<<(N + 255) / 256, 256, 0, s>>>(P.Fp, N);
    k_identity9<<<(N + 255) / 256, 256, 0, s>>>(P.R, N);
    k_identity9<<<(N + 255) / 256, 256, 0, s>>>(P.FiT, N);
    k_identity9<<<(N + 255) / 256, 256, 0, s>>>(P.Gi, N);
    CK(cudaMemsetAsync(P.vol, 0, sizeof(float) * N, s));
    fill_f(P.J, N, 1.f, s);
    fill_f(P.mu, N, sim->sp.mu, s);
    fill_f(P.lam, N, sim->sp.lambda, s);
    k_iota<<<(N + 255) / 256, 256, 0, s>>>(P.orig, N);
    k_iota<<<(N + 255) / 256, 256, 0, s>>>(sim->slotOf, N);
}

mpm_status guarded(mpm_sim* sim, const std::function<mpm_status()>& fn) {
    try {
        return fn();
    } catch (CudaError& e) {
        char buf[512];
        std::snprintf(buf, sizeof(buf), "CUDA error %s (%s) at %s", cudaGetErrorName(e.e), cudaGetErrorString(e.e), e.where);
        if (sim) sim->lastError = buf;
        return e.e == cudaErrorMemoryAllocation ? MPM_ERR_OUT_OF_MEMORY : MPM_ERR_CUDA;
    } catch (std::exception& e) {
        if (sim) sim->lastError = e.what();
        return MPM_ERR_INTERNAL;
    }
}

// Stencil-sized tile kernels launch over at most this many CTAs (they loop over the tile list).
int max_tiles(mpm_sim* sim) { return std::max(1, sim->totalTiles); }

void fill_stats(mpm_sim* sim, int B, const std::vector<BodySolve>& hs, int fp64, mpm_step_stats* stats) {
    if (!stats) return;
    stats->num_bodies = B;
    stats->num_ballistic = sim->nBallistic;
    stats->fp64_svd_particles = fp64;
    for (int b = 0; b < B && b < (int)hs.size(); ++b) {
        stats->total_iterations += hs[b].iterations;
        stats->max_iterations_used = std::max(stats->max_iterations_used, hs[b].iterations);
        if (b < 64) {
            stats->iterations[b] = hs[b].iterations;
            stats->b_norm2[b] = hs[b].bNorm2;
            stats->r_norm2[b] = hs[b].rNorm2;
            stats->exit_reason[b] = hs[b].exitReason;
        }
    }
}

mpm_status stop_here(mpm_sim* sim, int B, mpm_step_stats* stats) {
    std::vector<BodySolve> hs(B);
    if (B > 0) CK(cudaMemcpyAsync(hs.data(), sim->dSolve, sizeof(BodySolve) * B, cudaMemcpyDeviceToHost, sim->stream));
    read_scalars(sim);
    fill_stats(sim, B, hs, sim->hScalars[2], stats);
    sim->gridsValid = B > 0;
    return from_device_error(sim, sim->hScalars[3]);
}

// the learned warm start for every body with at least ws.minNodes grid nodes: features -> 4 convolutions ->
// x0 (replaces the uniform guess that k_node_rhs wrote)
mpmnn::NnNorm ws_norm(const mpm_sim* sim, const StepParams& sp) {
    const mpm_sim::WarmStart& w = sim->ws;
    mpmnn::NnNorm nn{};
    nn.inv_mass_unit = 1.f / (w.density * sp.h * sp.h * sp.h);
    nn.inv_vel_unit = sp.dt / sp.h;
    nn.vel_unit = sp.h / sp.dt;
    nn.dt = sp.dt;
    for (int a = 0; a < 3; ++a) {
        float g = 0.f;
        for (int k = 0; k < sp.nfields; ++k) g += sp.gravity[k][a];
        nn.gdt[a] = sp.dt * g;
    }
    for (int k = 0; k < mpmnn::kFeat; ++k) nn.feat_scale[k] = w.featScale[k];
    nn.out_scale = w.outScale;
    nn.light_mass = w.lightMass;
    return nn;
}

// the previous solve's history of body b mapped onto its current grid (none when there is no history, the body
// is new, or the two boxes do not overlap)
mpmnn::WsHist ws_hist(const mpm_sim* sim, int b, float h, int which) {
    const mpm_sim::WarmStart& w = sim->ws;
    mpmnn::WsHist H{};
    if (!w.useHist || !w.histValid[which] || b >= (int)w.histGrids[which].size()) return H;
    const BodyGrid& g = sim->grids[b];
    const BodyGrid& p = w.histGrids[which][b];
    bool overlap = true;
    for (int a = 0; a < 3; ++a) {
        H.off[a] = (int)std::lrint((double)(g.mn[a] - p.mn[a]) / (double)h);
        H.n[a] = p.n[a];
        if (H.off[a] >= p.n[a] || H.off[a] + g.n[a] <= 0) overlap = false;
    }
    if (!overlap) return mpmnn::WsHist{};
    H.h = w.hist[which];
    H.nodeOff = p.nodeOff;
    return H;
}

// the learned warm start for every body with at least ws.minNodes grid nodes: features -> 4 convolutions ->
// guess (replaces the uniform guess that k_node_rhs wrote); without a network, the guess from p*/m and the
// history alone
mpm_status warm_start(mpm_sim* sim, const StepParams& sp) {
    mpm_sim::WarmStart& w = sim->ws;
    cudaStream_t s = sim->stream;
    int* err = sim->dScalars + 10;
    CK(cudaMemsetAsync(err, 0, sizeof(int), s));
    size_t need = 0, needBlocks = 0;
    for (int b = 0; b < sim->B; ++b) {
        const BodyGrid& g = sim->grids[b];
        const size_t G = (size_t)g.n[0] * g.n[1] * g.n[2];
        if ((long long)G >= w.minNodes) {
            need = std::max(need, G);
            needBlocks = std::max(needBlocks, (size_t)mpmnn::tile_blocks(g.n[0], g.n[1], g.n[2]));
        }
    }
    if (need == 0) return MPM_OK;
    // buffers from the handle's pool (stream-ordered, no device-wide synchronisation when they grow)
    auto palloc = [&](void** p, size_t bytes) { CK(cudaMallocFromPoolAsync(p, bytes, sim->pool, s)); };
    if (w.net && need > w.cap) {
        void* old[] = {w.feat, w.actA, w.actB, w.out, w.blockFlag};
        for (void* p : old) if (p) CK(cudaFreeAsync(p, s));
        const size_t cap = need + need / 2;
        palloc(&w.feat, cap * 16 * sizeof(__nv_bfloat16));
        palloc(&w.actA, cap * 32 * sizeof(__nv_bfloat16));
        palloc(&w.actB, cap * 32 * sizeof(__nv_bfloat16));
        palloc((void**)&w.out, cap * 3 * sizeof(float));
        palloc((void**)&w.blockFlag, 2 * cap);
        w.cap = cap;
    }
    if (w.net && (needBlocks > w.capBlocks || !w.blockCount)) {
        void* old[] = {w.blockList, w.blockCount};
        for (void* p : old) if (p) CK(cudaFreeAsync(p, s));
        const size_t cap = needBlocks + needBlocks / 2 + 1;
        palloc((void**)&w.blockList, cap * mpmnn::kLayers * sizeof(int));
        palloc((void**)&w.blockCount, mpmnn::kLayers * sizeof(int));
        w.capBlocks = cap;
    }
    const mpmnn::NnNorm nn = ws_norm(sim, sp);
    for (int b = 0; b < sim->B; ++b) {
        const BodyGrid& g = sim->grids[b];
        const long long G = (long long)g.n[0] * g.n[1] * g.n[2];
        if (G < w.minNodes || G == 0) continue;
        const mpmnn::WsHist H = ws_hist(sim, b, sp.h, 0), H2 = ws_hist(sim, b, sp.h, 1);
        if (w.net) {
            launch_ws_features(sim->nd, g, sp, nn, H, w.feat, s);
            // each layer's output blocks: within reach of the heavy nodes, the only ones that read the output
            // (the seed threshold sits just under the guess's heavy test, so rounding cannot drop a heavy node)
            const float heavyMass = 0.999f * nn.light_mass / nn.inv_mass_unit;
            CK(mpmnn::layer_blocks(sim->nd.mass + g.nodeOff, heavyMass, g.n[0], g.n[1], g.n[2], mpmnn::kLayers,
                                   w.blockFlag, w.blockList, (long long)w.capBlocks, w.blockCount, s));
            kernel_launch_add(4);
            const void* in = w.feat;
            void* outs[3] = {w.actA, w.actB, w.actA};
            for (int l = 0; l < mpmnn::kLayers; ++l) {
                const bool last = l == mpmnn::kLayers - 1;
                CK(mpmnn::conv3d_tiled(in, mpmnn::kCinPad[l], w.wf[l], w.bias[l], mpmnn::kCout[l], mpmnn::kCoutPad[l],
                                       last ? 0 : 1, 0, nullptr, last ? nullptr : outs[l], last ? w.out : nullptr, 3,
                                       g.n[0], g.n[1], g.n[2], 1, w.blockList + (size_t)l * w.capBlocks,
                                       w.blockCount + l, err, s));
                kernel_launch_add(1);
                if (!last) in = outs[l];
            }
        }
        launch_ws_apply(sim->nd, g, sp, nn, H, H2, w.net ? w.out : nullptr, !w.net && w.extrapolate, s);
    }
    return MPM_OK;
}

// after the solve: the history of every body for the next step's warm start
mpm_status ws_record(mpm_sim* sim, const StepParams& sp) {
    mpm_sim::WarmStart& w = sim->ws;
    const size_t need = 3 * (size_t)sim->Gtot;
    // the previous record becomes h2; the new one is written over the buffer of the one before
    std::swap(w.hist[0], w.hist[1]);
    std::swap(w.capHist[0], w.capHist[1]);
    std::swap(w.histGrids[0], w.histGrids[1]);
    std::swap(w.histValid[0], w.histValid[1]);
    if (need > w.capHist[0]) {
        if (w.hist[0]) CK(cudaFreeAsync(w.hist[0], sim->stream));
        w.hist[0] = nullptr;
        w.capHist[0] = 0;
        CK(cudaMallocFromPoolAsync((void**)&w.hist[0], (need + need / 2) * sizeof(float), sim->pool, sim->stream));
        w.capHist[0] = need + need / 2;
    }
    launch_ws_record(sim->nd, sim->dGrids, sim->dChunkBody, sim->nChunks, ws_norm(sim, sp), w.hist[0], sim->stream);
    w.histGrids[0] = sim->grids;
    w.histValid[0] = true;
    return MPM_OK;
}

mpm_status step_impl(mpm_sim* sim, float dt, const mpm_solve_params* solve, int stopPhase, mpm_cancel_fn cancel,
                     void* cancelCtx, mpm_iterate_fn iterate, void* iterCtx, mpm_step_stats* stats) {
    const long long launches0 = kernel_launch_count();
    const int N = sim->N;
    cudaStream_t s = sim->stream;
    StepParams sp = sim->sp;
    sp.dt = dt;
    sp.maxIters = solve ? solve->max_iterations : 60;
    sp.tol = solve ? solve->tolerance : 1e-5f;
    sim->sp.dt = dt;
    sim->gridsValid = false;
    CK(cudaMemsetAsync(sim->dScalars, 0, 4 * sizeof(int), s));
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (!sim->segValid) {  // the last segmentation failed: run it again before using its partition
        segment(sim);
        read_scalars(sim);
        sim->B = sim->hScalars[4];
        sim->nBallistic = sim->hScalars[5];
        sim->segValid = (sim->hScalars[3] & ERR_SEGMENT) == 0;
        if (!sim->segValid) return from_device_error(sim, sim->hScalars[3]);
        CK(cudaMemsetAsync(sim->dScalars, 0, 4 * sizeof(int), s));
    }
    const int B = sim->B;
    int pr = -1;
    mpm_status st = build_grids(sim, true);
    if (st != MPM_OK) return st;
    bool forked = false;  // the plasticity pass is running on the side stream
    if (B > 0) {
        const int mt = max_tiles(sim);
        NodeArrays nd = sim->nd;
        ReduceArrays R = reduce_arrays(sim);
        const BodyGrid* G = sim->dGrids;
        const int* cb = sim->dChunkBody;
        const int nc = sim->nChunks;
        int* err = sim->dScalars + 3;
        double NB = 0;
        for (int b = 0; b < B; ++b) NB += sim->bodyCount[b];
        const double GN = (double)sim->Gtot;
        // one particle pass: masses and momenta (Grid.cpp:62-150), internal forces (:405-428), the Jacobi
        // diagonal's dFidXi sums (:484-531) and the operator records; then the node passes
        pr = pbegin(sim, PH_P2G_FORCE, NB, GN);
        launch_p2g_force(sim->P, N, sim->T, mt, G, sp.h, nd, nd.diag, sim->opRec, true, err, s);
        pend(sim, pr);
        pr = pbegin(sim, PH_NODE, 0, GN);
        launch_node_mass(nd, G, cb, nc, err, s);
        pend(sim, pr);
        pr = pbegin(sim, PH_NODE, 0, GN);
        launch_node_vel(nd, G, cb, nc, sp, err, s);
        pend(sim, pr);
        pr = pbegin(sim, PH_NODE, 0, GN);
        launch_node_explicit(nd, G, cb, nc, sp, sim->dSolve, R, err, s);
        pend(sim, pr);
        // DF(vc) of the rhs (Grid.cpp:983-1002): vc is zero away from collided nodes, so only the tiles whose
        // window holds one take part
        pr = pbegin(sim, PH_OP_RHS_DIAG, NB, GN, true);
        launch_contact_tiles(sim->T, mt, G, nd.flag, sim->contactT, s);
        launch_op(sim->P, N, sim->contactT, mt, G, sp.h, nd.vc, nd.df, sim->opRec, sim->dSolve, false, s, pslot(sim, pr));
        pend(sim, pr);
        pr = pbegin(sim, PH_NODE, 0, GN);
        launch_node_rhs(nd, G, cb, nc, sp, sim->dSolve, R, err, s);
        pend(sim, pr);
        if (sim->ws.on) {
            pr = pbegin(sim, PH_WARM_START, 0, GN);
            st = warm_start(sim, sp);
            pend(sim, pr);
            if (st != MPM_OK) return st;
        }
        if (stopPhase == 1) return stop_here(sim, B, stats);
        // conjugate residuals: A x, A p, then the loop
        pr = pbegin(sim, PH_OP, NB, GN, true);
        launch_op(sim->P, N, sim->T, mt, G, sp.h, nd.dxp, nd.df, sim->opRec, sim->dSolve, true, s, pslot(sim, pr));
        pend(sim, pr);
        pr = pbegin(sim, PH_CR_NODE, 0, GN);
        launch_node_cr_init1(nd, G, cb, nc, sp, sim->dSolve, s);
        pend(sim, pr);
        pr = pbegin(sim, PH_OP, NB, GN, true);
        launch_op(sim->P, N, sim->T, mt, G, sp.h, nd.dxp, nd.df, sim->opRec, sim->dSolve, true, s, pslot(sim, pr));
        pend(sim, pr);
        pr = pbegin(sim, PH_CR_NODE, 0, GN);
        launch_node_cr_init2(nd, G, cb, nc, sp, sim->dSolve, R, s);
        pend(sim, pr);
        // every iteration ends with a snapshot of the finished-body count (hScalars[20 + 4 (it % 3)]); the host
        // waits for the one from two iterations back, so at most two iterations run past convergence while the
        // queue still holds the next iteration's launches
        cudaEvent_t evs[3];
        for (cudaEvent_t& e : evs) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        std::vector<BodySolve> hs;
        std::vector<float> xb;
        for (int it = 0; it <= sp.maxIters; ++it) {
            std::vector<int> doneBefore;
            if (iterate) {
                hs.resize(B);
                CK(cudaMemcpyAsync(hs.data(), sim->dSolve, sizeof(BodySolve) * B, cudaMemcpyDeviceToHost, s));
                CK(cudaStreamSynchronize(s));
                for (int b = 0; b < B; ++b) doneBefore.push_back(hs[b].done);
            }
            pr = pbegin(sim, PH_CR_NODE, 0, GN);
            launch_node_cr_update(nd, G, cb, nc, sp, sim->dSolve, R, it, s);
            pend(sim, pr);
            if (iterate) {
                for (int b = 0; b < B; ++b) {
                    if (doneBefore[b]) continue;
                    const BodyGrid& g = sim->grids[b];
                    size_t cnt = 3ull * g.n[0] * g.n[1] * g.n[2];
                    xb.resize(cnt);
                    CK(cudaMemcpyAsync(xb.data(), nd.x + 3 * g.nodeOff, cnt * sizeof(float), cudaMemcpyDeviceToHost, s));
                    CK(cudaStreamSynchronize(s));
                    iterate(iterCtx, b, it, xb.data(), cnt);
                }
            }
            pr = pbegin(sim, PH_OP, NB, GN, true);
            launch_op(sim->P, N, sim->T, mt, G, sp.h, nd.dxp, nd.df, sim->opRec, sim->dSolve, true, s, pslot(sim, pr));
            pend(sim, pr);
            pr = pbegin(sim, PH_CR_NODE, 0, 2 * GN);
            launch_node_cr_ar(nd, G, cb, nc, sp, sim->dSolve, R, it, s);
            launch_node_cr_p(nd, G, cb, nc, sp, sim->dSolve, R, it, s);
            pend(sim, pr);
            {
                const int slot = it % 3;
                CK(cudaMemcpyAsync(sim->hScalars + 20 + 4 * slot, sim->dScalars + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
                CK(cudaEventRecord(evs[slot], s));
                if (it >= 2) {
                    const int back = (it - 2) % 3;
                    CK(cudaEventSynchronize(evs[back]));
                    if (sim->hScalars[20 + 4 * back] >= B) break;
                }
            }
        }
        for (cudaEvent_t& e : evs) cudaEventDestroy(e);
        launch_node_final(nd, G, cb, nc, sim->dSolve, s);
        if (sim->ws.on && sim->ws.useHist) ws_record(sim, sp);
        if (stopPhase == 2) return stop_here(sim, B, stats);
        // the grid phases' NaN checks before any particle moves: the reference throws from the splats and the
        // explicit update (Grid.cpp:233-260, 675-677), so a failed step leaves the particles where they were
        CK(cudaMemcpyAsync(sim->hScalars + 3, sim->dScalars + 3, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (sim->hScalars[3] & kGridErrors) {
            const int e = sim->hScalars[3];
            segment(sim);
            read_scalars(sim);
            sim->B = sim->hScalars[4];
            sim->nBallistic = sim->hScalars[5];
            sim->segValid = (sim->hScalars[3] & ERR_SEGMENT) == 0;
            return from_device_error(sim, e);
        }
        if (cancel) {
            if (cancel(cancelCtx)) {  // Sim.cpp:107-111
                segment(sim);
                read_scalars(sim);
                sim->B = sim->hScalars[4];
                sim->nBallistic = sim->hScalars[5];
                sim->segValid = (sim->hScalars[3] & ERR_SEGMENT) == 0;
                if (!sim->segValid) return from_device_error(sim, ERR_SEGMENT);
                return set_err(sim, MPM_ERR_CANCELLED, "cancelled");
            }
        }
        pr = pbegin(sim, PH_G2P, NB, GN);
        launch_g2p(sim->P, N, sim->T, mt, G, sp.h, dt, nd, s);
        pend(sim, pr);
        if (stopPhase != 0) {
            pr = pbegin(sim, PH_PLASTICITY, N, 0);
            launch_plasticity(sim->P, N, sp, sim->dScalars + 2, err, s);
            pend(sim, pr);
            return stop_here(sim, B, stats);
        }
        // the advection and the segmentation (x, v, body ids) on the high-priority side stream, beside the
        // plasticity pass (F, Fp, R, F^-T, G^-1, J, mu, lambda) here; the two share only atomically updated
        // scalars ([2] and [3]); the segmentation's CTAs go first, the plasticity pass fills the SMs around them
        CK(cudaEventRecord(sim->evFork, s));
        CK(cudaStreamWaitEvent(sim->side, sim->evFork, 0));
        pr = pbegin(sim, PH_PLASTICITY, N, 0);
        launch_plasticity(sim->P, N, sp, sim->dScalars + 2, err, s);
        pend(sim, pr);
        forked = true;
    }
    if (stopPhase != 0) return stop_here(sim, B, stats);  // no bodies: particles stay untouched
    cudaStream_t sa = forked ? sim->side : s;
    pr = pbegin(sim, PH_ADVECT, N, 0, false, sa);
    launch_advect(sim->P, N, sp, sa);
    pend(sim, pr, sa);
    pr = pbegin(sim, PH_SEGMENT, N, 0, false, sa);
    segment(sim, sa);
    pend(sim, pr, sa);
    if (forked) {
        CK(cudaEventRecord(sim->evJoin, sim->side));
        CK(cudaStreamWaitEvent(s, sim->evJoin, 0));
    }
    // the solves' stats and the scalars: [2] FP64 SVD count, [3] error bits, [4], [5] the next step's bodies
    std::vector<BodySolve> hs(B);
    if (B > 0) CK(cudaMemcpyAsync(hs.data(), sim->dSolve, sizeof(BodySolve) * B, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(sim->hScalars, sim->dScalars, 6 * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (sim->ws.on) CK(cudaMemcpyAsync(sim->hScalars + 10, sim->dScalars + 10, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const int errBits = sim->hScalars[3];
    const int fp64 = sim->hScalars[2];
    sim->gridsValid = B > 0;
    const int nextB = sim->hScalars[4], nextBallistic = sim->hScalars[5];
    sim->segValid = (errBits & ERR_SEGMENT) == 0;
    if (sim->ws.on && sim->hScalars[10]) {
        sim->B = nextB;
        sim->nBallistic = nextBallistic;
        return set_err(sim, MPM_ERR_INTERNAL, "warm start network: a tensor-core wait timed out");
    }
    fill_stats(sim, B, hs, fp64, stats);  // this step's bodies and ballistic count
    sim->B = nextB;
    sim->nBallistic = nextBallistic;
    if (stats) stats->kernel_launches = (int)(kernel_launch_count() - launches0);
    return from_device_error(sim, errBits);
}

}  // namespace

// =========================================================================================================
// C-ABI
// =========================================================================================================
extern "C" {

int mpm_abi_version(void) { return MPM_ABI_VERSION; }

const char* mpm_status_string(mpm_status s) {
    switch (s) {
        case MPM_OK: return "ok";
        case MPM_ERR_INVALID_ARGUMENT: return "invalid argument";
        case MPM_ERR_CUDA: return "CUDA error";
        case MPM_ERR_NO_DEVICE: return "no CUDA device";
        case MPM_ERR_NAN_MASSES: return "nans in splatted masses!";
        case MPM_ERR_NAN_VELOCITIES: return "nans in splatted velocities!";
        case MPM_ERR_NAN_MOMENTA: return "nan in explicit momenta!";
        case MPM_ERR_NAN_STRESS: return "nans in dEnergyDensitydF matrix!";
        case MPM_ERR_INFINITE_HARDNESS: return "infinite hardness!!!";
        case MPM_ERR_NAN_PARTICLE_VELOCITY: return "nans in particle velocity data!";
        case MPM_ERR_GRID_TOO_BIG: return "grid is too big";
        case MPM_ERR_UNKNOWN_VARIABLE: return "Material point data has no variable of that name";
        case MPM_ERR_WRONG_SIZE: return "wrong element count";
        case MPM_ERR_UNSUPPORTED: return "unsupported";
        case MPM_ERR_CANCELLED: return "cancelled";
        case MPM_ERR_INTERNAL: return "internal error";
        case MPM_ERR_OUT_OF_MEMORY: return "out of device memory";
        case MPM_ERR_TOO_MANY_PARTICLES: return "more particles than the no-allocation entry point's maximum (262144)";
    }
    return "unknown status";
}

const char* mpm_last_error(const mpm_sim* sim) { return sim ? sim->lastError.c_str() : ""; }

mpm_status mpm_create(const mpm_scene_desc* d, size_t n, const float* x, const float* masses, mpm_sim** out) {
    if (!d || !out || (n > 0 && (!x || !masses))) return MPM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (d->dimension < 1 || d->dimension > 3 || d->shape_function != 0) return MPM_ERR_UNSUPPORTED;
    if (d->num_colliders < 0 || d->num_colliders > kMaxColliders) return MPM_ERR_UNSUPPORTED;
    if (d->num_gravity_fields < 0 || d->num_gravity_fields > kMaxFields) return MPM_ERR_UNSUPPORTED;
    if (!(d->grid_size > 0.f) || n > 0x7fffffffull / 9) return MPM_ERR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return MPM_ERR_NO_DEVICE;
    if (d->device < 0 || d->device >= ndev) return MPM_ERR_INVALID_ARGUMENT;
    mpm_sim* sim = new mpm_sim();
    mpm_status st = guarded(sim, [&]() -> mpm_status {
        sim->device = d->device;
        sim->dim = d->dimension;
        CK(cudaSetDevice(sim->device));
        CK(cudaStreamCreateWithFlags(&sim->stream, cudaStreamNonBlocking));
        int leastPrio = 0, greatestPrio = 0;
        CK(cudaDeviceGetStreamPriorityRange(&leastPrio, &greatestPrio));
        CK(cudaStreamCreateWithPriority(&sim->side, cudaStreamNonBlocking, greatestPrio));
        CK(cudaEventCreateWithFlags(&sim->evFork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&sim->evJoin, cudaEventDisableTiming));
        StepParams& sp = sim->sp;
        sp.h = d->grid_size;
        // SnowConstitutiveModel.cpp:23-24
        const float E = d->youngs_modulus, nu = d->poisson_ratio;
        sp.mu = E / (2 * (1 + nu));
        sp.lambda = E * nu / ((1 + nu) * (1 - 2 * nu));
        sp.xi = d->hardening;
        sp.thetaC = d->compressive_strength;
        sp.thetaS = d->tensile_strength;
        sp.ncoll = d->num_colliders;
        for (int i = 0; i < sp.ncoll; ++i) {
            const mpm_status cs = set_collider(sim, i, d->colliders[i]);
            if (cs != MPM_OK) return cs;
        }
        sp.nfields = d->num_gravity_fields;
        for (int i = 0; i < sp.nfields; ++i)
            for (int k = 0; k < 3; ++k) sp.gravity[i][k] = d->gravity[3 * i + k];
        const int N = (int)n;
        sim->N = N;
        const int Na = std::max(N, 1);
        alloc_part(sim->P, Na);
        alloc_part(sim->Q, Na);
        sim->staging = alloc_f(9ull * Na);
        sim->opRec.base = alloc_i(Na);
        CK(cudaMemset(sim->opRec.base, 0xff, sizeof(int) * Na));  // no records yet: window base -1
        CK(cudaMalloc(&sim->opRec.w4, sizeof(float4) * kOpRecW4 * Na));
        CK(cudaMalloc(&sim->opRec.m4, sizeof(float4) * kOpRecM4 * Na));
        sim->slotOf = alloc_i(Na);
        sim->key = alloc_i(Na);
        sim->rank = alloc_i(Na);
        sim->inv = alloc_i(Na);
        CK(cudaMalloc(&sim->dScalars, kScalars * sizeof(int)));
        CK(cudaMemset(sim->dScalars, 0, kScalars * sizeof(int)));
        CK(cudaMallocHost(&sim->hScalars, kScalars * sizeof(int)));
        init_state(sim);
        if (N > 0) {
            CK(cudaMemcpyAsync(sim->staging, x, 3ull * N * sizeof(float), cudaMemcpyHostToDevice, sim->stream));
            launch_scatter_user(sim->staging, sim->slotOf, sim->P.x, N, 3, sim->stream);
            CK(cudaMemcpyAsync(sim->P.m, masses, (size_t)N * sizeof(float), cudaMemcpyHostToDevice, sim->stream));
            // Sim.cpp:40-49: bodies, then each body's grid and its particle volumes
            segment(sim);
            read_scalars(sim);
            sim->B = sim->hScalars[4];
            sim->nBallistic = sim->hScalars[5];
            if (sim->hScalars[3]) return from_device_error(sim, sim->hScalars[3]);
            mpm_status s2 = build_grids(sim, false);
            if (s2 != MPM_OK) return s2;
            if (sim->B > 0) {
                const int mt = max_tiles(sim);
                int* err = sim->dScalars + 3;
                launch_p2g_mass_momentum(sim->P, N, sim->T, mt, sim->dGrids, sp.h, sim->nd, err, sim->stream);
                launch_node_mass(sim->nd, sim->dGrids, sim->dChunkBody, sim->nChunks, err, sim->stream);
                launch_volumes(sim->P, N, sim->T, mt, sim->dGrids, sp.h, sim->nd, sim->stream);
            }
            read_scalars(sim);
            if (sim->hScalars[3]) return from_device_error(sim, sim->hScalars[3]);
        }
        CK(cudaStreamSynchronize(sim->stream));
        return MPM_OK;
    });
    if (st != MPM_OK) {
        mpm_destroy(sim);
        return st;
    }
    *out = sim;
    return MPM_OK;
}

void mpm_destroy(mpm_sim* sim) {
    if (!sim) return;
    cudaSetDevice(sim->device);
    if (sim->side) cudaStreamSynchronize(sim->side);
    if (sim->stream) cudaStreamSynchronize(sim->stream);
    free_part(sim->P);
    free_part(sim->Q);
    void* ps[] = {sim->staging, sim->opRec.base, sim->opRec.w4, sim->opRec.m4, sim->slotOf, sim->key, sim->rank, sim->inv, sim->dGrids, sim->dAcc, sim->dSolve,
                  sim->dChunkBody, sim->dCounter, sim->dPartial, sim->dScalars, sim->scanTmp, sim->dbgA, sim->dbgB, sim->dbgC,
                  sim->T.count, sim->T.start, sim->T.list, sim->T.listBody, sim->contactT.list, sim->contactT.listBody,
                  sim->S.count, sim->S.start, sim->S.sorted,
                  sim->S.rank, sim->S.parent, sim->S.size, sim->S.minOrig, sim->S.mark, sim->S.mrank, sim->S.xs,
                  sim->segEdges[0], sim->segEdges[1]};
    for (void* p : ps) if (p) cudaFree(p);
    for (int i = 0; i < kMaxColliders; ++i) {
        if (sim->collPhi[i]) cudaFree(sim->collPhi[i]);
        if (sim->collVel[i]) cudaFree(sim->collVel[i]);
    }
    // the handle's pool: node arrays and the warm start's growing buffers
    void* pooled[] = {sim->nodeBlock, sim->ws.feat, sim->ws.actA, sim->ws.actB, sim->ws.out, sim->ws.blockFlag,
                      sim->ws.blockList, sim->ws.blockCount, sim->ws.hist[0], sim->ws.hist[1]};
    for (void* p : pooled) if (p) cudaFreeAsync(p, sim->stream);
    if (sim->stream) cudaStreamSynchronize(sim->stream);
    if (sim->pool) cudaMemPoolDestroy(sim->pool);
    if (sim->hScalars) cudaFreeHost(sim->hScalars);
    if (sim->dProc) cudaFree(sim->dProc);
    for (int l = 0; l < mpmnn::kLayers; ++l) {
        if (sim->ws.wf[l]) cudaFree(sim->ws.wf[l]);
        if (sim->ws.bias[l]) cudaFree(sim->ws.bias[l]);
    }
    for (cudaEvent_t e : sim->evPool) cudaEventDestroy(e);
    if (sim->evFork) cudaEventDestroy(sim->evFork);
    if (sim->evJoin) cudaEventDestroy(sim->evJoin);
    if (sim->side) cudaStreamDestroy(sim->side);
    if (sim->stream) cudaStreamDestroy(sim->stream);
    delete sim;
}

void* mpm_get_stream(mpm_sim* sim) { return sim ? (void*)sim->stream : nullptr; }

mpm_status mpm_set_colliders(mpm_sim* sim, int num_colliders, const mpm_collider* colliders) {
    if (!sim || num_colliders < 0 || (num_colliders > 0 && !colliders)) return MPM_ERR_INVALID_ARGUMENT;
    if (num_colliders > kMaxColliders) return MPM_ERR_UNSUPPORTED;
    return guarded(sim, [&]() -> mpm_status {
        CK(cudaSetDevice(sim->device));
        CK(cudaStreamSynchronize(sim->stream));
        for (int i = 0; i < num_colliders; ++i) {
            const mpm_status st = set_collider(sim, i, colliders[i]);
            if (st != MPM_OK) return st;
        }
        sim->sp.ncoll = num_colliders;
        return MPM_OK;
    });
}

mpm_status mpm_seed_particles(const mpm_collider* sdf, const float* bbox_min, const float* bbox_max, float h,
                              float density, int device, float* x_out, float* v_out, float* m_out, size_t capacity,
                              size_t* count) {
    if (!sdf || sdf->kind != MPM_COLLIDER_GRID || !bbox_min || !bbox_max || !(h > 0.f) || !count ||
        (capacity > 0 && (!x_out || !v_out || !m_out)))
        return MPM_ERR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return MPM_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return MPM_ERR_INVALID_ARGUMENT;
    // the lattice of SOP_MPMSim.cpp:174-180: ceil(size / h) sites per axis (float division, as there)
    SeedLattice L{};
    L.sites = 1;
    for (int a = 0; a < 3; ++a) {
        const float size = bbox_max[a] - bbox_min[a];
        L.dims[a] = std::max(0, (int)std::ceil(size / h));
        L.bmin[a] = (double)bbox_min[a];
        L.sites *= L.dims[a];
    }
    L.h = (double)h;
    if (L.sites > (1ll << 31) - 1) return MPM_ERR_INVALID_ARGUMENT;
    *count = 0;
    if (L.sites == 0) return MPM_OK;
    mpm_sim tmp;  // a scratch handle: owns the field's device copy and the seeding buffers for this call
    mpm_status st = guarded(&tmp, [&]() -> mpm_status {
        tmp.device = device;
        CK(cudaSetDevice(device));
        CK(cudaStreamCreateWithFlags(&tmp.stream, cudaStreamNonBlocking));
        const mpm_status cs = set_collider(&tmp, 0, *sdf);
        if (cs != MPM_OK) return cs;
        int* flag = alloc_i((size_t)L.sites);
        int* pos = alloc_i((size_t)L.sites);
        int* scratch = alloc_i(scan_tmp_ints(L.sites) + 8);
        int* total = scratch + scan_tmp_ints(L.sites);
        float *dx = nullptr, *dv = nullptr, *dm = nullptr;
        auto release = [&]() {
            void* ps[] = {flag, pos, scratch, dx, dv, dm};
            for (void* p : ps) if (p) cudaFree(p);
        };
        launch_seed(tmp.sp.coll[0], L, 0.f, flag, pos, scratch, total, nullptr, nullptr, nullptr, false, tmp.stream);
        int n = 0;
        cudaError_t e = cudaMemcpyAsync(&n, total, sizeof(int), cudaMemcpyDeviceToHost, tmp.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(tmp.stream);
        if (e != cudaSuccess) { release(); throw CudaError{e, "seed count"}; }
        *count = (size_t)n;
        if ((size_t)n > capacity) { release(); return MPM_ERR_WRONG_SIZE; }
        if (n > 0) {
            // SOP_MPMSim.cpp:187: initialDensity * h * h * h in float
            const float mass = density * h * h * h;
            e = cudaMalloc(&dx, 3 * sizeof(float) * n);
            if (e == cudaSuccess) e = cudaMalloc(&dv, 3 * sizeof(float) * n);
            if (e == cudaSuccess) e = cudaMalloc(&dm, sizeof(float) * n);
            if (e == cudaSuccess) {
                launch_seed(tmp.sp.coll[0], L, mass, flag, pos, scratch, total, dx, dv, dm, true, tmp.stream);
                e = cudaMemcpyAsync(x_out, dx, 3 * sizeof(float) * n, cudaMemcpyDeviceToHost, tmp.stream);
            }
            if (e == cudaSuccess) e = cudaMemcpyAsync(v_out, dv, 3 * sizeof(float) * n, cudaMemcpyDeviceToHost, tmp.stream);
            if (e == cudaSuccess) e = cudaMemcpyAsync(m_out, dm, sizeof(float) * n, cudaMemcpyDeviceToHost, tmp.stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(tmp.stream);
        }
        release();
        if (e != cudaSuccess) throw CudaError{e, "seed particles"};
        return MPM_OK;
    });
    for (int i = 0; i < kMaxColliders; ++i) {
        if (tmp.collPhi[i]) cudaFree(tmp.collPhi[i]);
        if (tmp.collVel[i]) cudaFree(tmp.collVel[i]);
        tmp.collPhi[i] = tmp.collVel[i] = nullptr;
    }
    if (tmp.stream) cudaStreamDestroy(tmp.stream);
    tmp.stream = nullptr;
    return st;
}

mpm_status mpm_set_collider(mpm_sim* sim, int index, const mpm_collider* collider) {
    if (!sim || !collider || index < 0 || index >= sim->sp.ncoll) return MPM_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&]() -> mpm_status {
        CK(cudaSetDevice(sim->device));
        CK(cudaStreamSynchronize(sim->stream));  // no step in flight reads the slot's samples
        return set_collider(sim, index, *collider);
    });
}

mpm_status mpm_set_warm_start(mpm_sim* sim, const mpm_warm_start* model) {
    if (!sim) return MPM_ERR_INVALID_ARGUMENT;
    if (model && ((!model->weights) != (!model->biases) || !(model->density > 0.f) || model->min_nodes < 0 ||
                  model->use_history < 0 || model->use_history > 2 ||
                  !(model->light_mass >= 0.f) || !std::isfinite(model->output_scale)))
        return MPM_ERR_INVALID_ARGUMENT;
    if (model && sim->dim != 3)  // the network is a 3-D convolution over the grid
        return set_err(sim, MPM_ERR_UNSUPPORTED, "the learned warm start needs a 3-D simulation");
    return guarded(sim, [&]() -> mpm_status {
        CK(cudaSetDevice(sim->device));
        CK(cudaStreamSynchronize(sim->stream));
        mpm_sim::WarmStart& w = sim->ws;
        w.on = false;
        w.histValid[0] = w.histValid[1] = false;
        if (!model) return MPM_OK;
        for (int k = 0; k < mpmnn::kFeat; ++k)
            if (!std::isfinite(model->feature_scale[k])) return MPM_ERR_INVALID_ARGUMENT;
        if (model->weights) {
            size_t wo = 0, bo = 0;
            for (int l = 0; l < mpmnn::kLayers; ++l) {
                for (int i = 0; i < mpmnn::layer_weight_count(l); ++i)
                    if (!std::isfinite(model->weights[wo + i])) return MPM_ERR_INVALID_ARGUMENT;
                for (int i = 0; i < mpmnn::kCout[l]; ++i)
                    if (!std::isfinite(model->biases[bo + i])) return MPM_ERR_INVALID_ARGUMENT;
                wo += mpmnn::layer_weight_count(l);
                bo += mpmnn::kCout[l];
            }
            float* tmp = nullptr;
            CK(cudaMalloc((void**)&tmp, (size_t)mpmnn::layer_weight_count(1) * sizeof(float)));
            wo = bo = 0;
            for (int l = 0; l < mpmnn::kLayers; ++l) {
                const int nw = mpmnn::layer_weight_count(l);
                if (!w.wf[l]) CK(cudaMalloc(&w.wf[l], (size_t)nw * sizeof(__nv_bfloat16)));
                if (!w.bias[l]) CK(cudaMalloc((void**)&w.bias[l], 32 * sizeof(float)));
                CK(cudaMemcpyAsync(tmp, model->weights + wo, (size_t)nw * sizeof(float), cudaMemcpyHostToDevice, sim->stream));
                CK(mpmnn::pack_weights(tmp, mpmnn::kCinPad[l], mpmnn::kCoutPad[l], mpmnn::kCinPad[l], mpmnn::kCoutPad[l],
                                       w.wf[l], nullptr, sim->stream));
                std::vector<float> bz(32, 0.f);
                for (int i = 0; i < mpmnn::kCout[l]; ++i) bz[i] = model->biases[bo + i];
                CK(cudaMemcpyAsync(w.bias[l], bz.data(), 32 * sizeof(float), cudaMemcpyHostToDevice, sim->stream));
                CK(cudaStreamSynchronize(sim->stream));
                wo += nw;
                bo += mpmnn::kCout[l];
            }
            cudaFree(tmp);
        }
        for (int k = 0; k < mpmnn::kFeat; ++k) w.featScale[k] = model->feature_scale[k];
        w.outScale = model->output_scale;
        w.lightMass = model->light_mass;
        w.density = model->density;
        w.minNodes = model->min_nodes;
        w.net = model->weights != nullptr;
        w.useHist = model->use_history != 0;
        w.extrapolate = model->use_history == 2;
        w.on = true;
        return MPM_OK;
    });
}

mpm_status mpm_profile_enable(mpm_sim* sim, int enable) {
    if (!sim) return MPM_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&]() -> mpm_status {
        CK(cudaSetDevice(sim->device));
        CK(cudaStreamSynchronize(sim->stream));
        sim->recs.clear();
        sim->evUsed = 0;
        sim->procUsed = 0;
        if (!sim->dProc) CK(cudaMalloc(&sim->dProc, sizeof(unsigned long long) * kProcSlots));
        CK(cudaMemsetAsync(sim->dProc, 0, sizeof(unsigned long long) * kProcSlots, sim->stream));
        CK(cudaStreamSynchronize(sim->stream));
        sim->profOn = enable != 0;
        return MPM_OK;
    });
}

int mpm_profile_read(mpm_sim* sim, mpm_phase_profile* out, int max) {
    if (!sim) return 0;
    mpm_status st = guarded(sim, [&]() -> mpm_status {
        CK(cudaSetDevice(sim->device));
        CK(cudaStreamSynchronize(sim->stream));
        std::vector<unsigned long long> proc(std::max(sim->procUsed, 1));
        if (sim->procUsed > 0)
            CK(cudaMemcpy(proc.data(), sim->dProc, sizeof(unsigned long long) * sim->procUsed, cudaMemcpyDeviceToHost));
        std::vector<mpm_phase_profile> agg(PH_COUNT);
        for (int p = 0; p < PH_COUNT; ++p) {
            std::memset(&agg[p], 0, sizeof(agg[p]));
            std::snprintf(agg[p].name, sizeof(agg[p].name), "%s", kPhaseNames[p]);
        }
        for (const auto& r : sim->recs) {
            if (r.b < 0) continue;
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, sim->evPool[r.a], sim->evPool[r.b]));
            mpm_phase_profile& a = agg[r.phase];
            a.launches += 1;
            a.total_ms += ms;
            a.particles += r.slot >= 0 ? (double)proc[r.slot] : r.particles;
            a.nodes += r.nodes;
        }
        for (int p = 0; p < PH_COUNT && p < max; ++p) out[p] = agg[p];
        return MPM_OK;
    });
    return st == MPM_OK ? (int)PH_COUNT : -1;
}

mpm_status mpm_step_ex(mpm_sim* sim, float dt, const mpm_solve_params* solve, int stop_phase, mpm_cancel_fn cancel,
                       void* cancel_ctx, mpm_iterate_fn iterate, void* iterate_ctx, mpm_step_stats* stats) {
    if (!sim || stop_phase < 0 || stop_phase > 2) return MPM_ERR_INVALID_ARGUMENT;
    if (solve && solve->max_iterations < 0) return MPM_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&]() {
        CK(cudaSetDevice(sim->device));
        return step_impl(sim, dt, solve, stop_phase, cancel, cancel_ctx, iterate, iterate_ctx, stats);
    });
}

mpm_status mpm_step(mpm_sim* sim, float dt, const mpm_solve_params* solve, mpm_step_stats* stats) {
    return mpm_step_ex(sim, dt, solve, 0, nullptr, nullptr, nullptr, nullptr, stats);
}

size_t mpm_num_particles(const mpm_sim* sim) { return sim ? (size_t)sim->N : 0; }

mpm_status mpm_variable_info(const mpm_sim* sim, const char* name, int* components) {
    if (!sim || !name) return MPM_ERR_INVALID_ARGUMENT;
    int comps = 0;
    float** p = var_ptr(const_cast<mpm_sim*>(sim)->P, name, comps);
    if (!p || (!*p && sim->N > 0)) return MPM_ERR_UNKNOWN_VARIABLE;
    if (components) *components = comps;
    return MPM_OK;
}

static mpm_status get_var(mpm_sim* sim, const char* name, float* dst, size_t count, bool device) {
    if (!sim || !name || (!dst && count)) return MPM_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&]() -> mpm_status {
        CK(cudaSetDevice(sim->device));
        int comps = 0;
        float** p = var_ptr(sim->P, name, comps);
        if (!p || !*p) return set_err(sim, MPM_ERR_UNKNOWN_VARIABLE, std::string("Material point data has no variable named '") + name + "'");
        if (count != (size_t)comps * sim->N) return set_err(sim, MPM_ERR_WRONG_SIZE, "element count does not match the variable");
        if (sim->N == 0) return MPM_OK;
        float* target = device ? dst : sim->staging;
        launch_gather_user(*p, sim->slotOf, target, sim->N, comps, sim->stream);
        if (!device) CK(cudaMemcpyAsync(dst, sim->staging, count * sizeof(float), cudaMemcpyDeviceToHost, sim->stream));
        CK(cudaStreamSynchronize(sim->stream));
        return MPM_OK;
    });
}
static mpm_status set_var(mpm_sim* sim, const char* name, const float* src, size_t count, bool device) {
    if (!sim || !name || (!src && count)) return MPM_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&]() -> mpm_status {
        CK(cudaSetDevice(sim->device));
        int comps = 0;
        float** p = var_ptr(sim->P, name, comps);
        if (!p) return set_err(sim, MPM_ERR_UNKNOWN_VARIABLE, std::string("Material point data has no variable named '") + name + "'");
        if (count != (size_t)comps * sim->N) return set_err(sim, MPM_ERR_WRONG_SIZE, "element count does not match the variable");
        if (!*p) {
            // the per-particle Lame extension is created on first write, both parameters in both state
            // buffers, initialised from the current mu / lambda
            const size_t n1 = std::max(sim->N, 1);
            sim->P.mu0 = alloc_f(n1);
            sim->P.lam0 = alloc_f(n1);
            if (!sim->Q.mu0) sim->Q.mu0 = alloc_f(n1);
            if (!sim->Q.lam0) sim->Q.lam0 = alloc_f(n1);
            CK(cudaMemcpyAsync(sim->P.mu0, sim->P.mu, sizeof(float) * sim->N, cudaMemcpyDeviceToDevice, sim->stream));
            CK(cudaMemcpyAsync(sim->P.lam0, sim->P.lam, sizeof(float) * sim->N, cudaMemcpyDeviceToDevice, sim->stream));
        }
        if (sim->N == 0) return MPM_OK;
        const float* srcd = src;
        if (!device) {
            CK(cudaMemcpyAsync(sim->staging, src, count * sizeof(float), cudaMemcpyHostToDevice, sim->stream));
            srcd = sim->staging;
        }
        launch_scatter_user(srcd, sim->slotOf, *p, sim->N, comps, sim->stream);
        // base Lame parameters also seed the current ones, as SnowConstitutiveModel::setParticles seeds mu and
        // lambda from the model's base values (SnowConstitutiveModel.cpp:156-157)
        const std::string nm(name);
        if (nm == "mu0") launch_scatter_user(srcd, sim->slotOf, sim->P.mu, sim->N, 1, sim->stream);
        if (nm == "lambda0") launch_scatter_user(srcd, sim->slotOf, sim->P.lam, sim->N, 1, sim->stream);
        CK(cudaStreamSynchronize(sim->stream));
        return MPM_OK;
    });
}

mpm_status mpm_get_variable(mpm_sim* sim, const char* name, float* dst, size_t count) { return get_var(sim, name, dst, count, false); }
mpm_status mpm_set_variable(mpm_sim* sim, const char* name, const float* src, size_t count) { return set_var(sim, name, src, count, false); }
mpm_status mpm_get_variable_device(mpm_sim* sim, const char* name, float* dst, size_t count) { return get_var(sim, name, dst, count, true); }
mpm_status mpm_set_variable_device(mpm_sim* sim, const char* name, const float* src, size_t count) { return set_var(sim, name, src, count, true); }

mpm_status mpm_get_bodies(mpm_sim* sim, int* body_of_particle, int* num_bodies, int* num_ballistic) {
    if (!sim) return MPM_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&]() -> mpm_status {
        CK(cudaSetDevice(sim->device));
        if (num_bodies) *num_bodies = sim->B;
        if (num_ballistic) *num_ballistic = sim->nBallistic;
        if (body_of_particle && sim->N > 0) {
            int* tmp = reinterpret_cast<int*>(sim->staging);
            k_gather_i<<<(sim->N + 255) / 256, 256, 0, sim->stream>>>(sim->P.body, sim->slotOf, tmp, sim->N);
            CK(cudaMemcpyAsync(body_of_particle, tmp, sizeof(int) * sim->N, cudaMemcpyDeviceToHost, sim->stream));
            CK(cudaStreamSynchronize(sim->stream));
        }
        return MPM_OK;
    });
}

mpm_status mpm_debug_grid_info(mpm_sim* sim, int body, float* min3, int* n3, float* fv3, int* num_particles) {
    if (!sim || !sim->gridsValid || body < 0 || body >= (int)sim->grids.size()) return MPM_ERR_INVALID_ARGUMENT;
    const BodyGrid& g = sim->grids[body];
    for (int k = 0; k < 3; ++k) {
        if (min3) min3[k] = g.mn[k];
        if (n3) n3[k] = g.n[k];
        if (fv3) fv3[k] = g.fv[k];
    }
    if (num_particles) *num_particles = sim->bodyCount[body];
    return MPM_OK;
}

mpm_status mpm_debug_grid_get(mpm_sim* sim, int body, const char* name, float* dst, size_t count) {
    if (!sim || !name || !dst || !sim->gridsValid || body < 0 || body >= (int)sim->grids.size()) return MPM_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&]() -> mpm_status {
        CK(cudaSetDevice(sim->device));
        const BodyGrid& g = sim->grids[body];
        const size_t G = (size_t)g.n[0] * g.n[1] * g.n[2];
        std::string nm(name);
        NodeArrays& n = sim->nd;
        if (nm == "masses") {
            if (count != G) return MPM_ERR_WRONG_SIZE;
            CK(cudaMemcpyAsync(dst, n.mass + g.nodeOff, G * sizeof(float), cudaMemcpyDeviceToHost, sim->stream));
        } else if (nm == "nodeCollided") {
            if (count != G) return MPM_ERR_WRONG_SIZE;
            std::vector<signed char> f(G);
            CK(cudaMemcpyAsync(f.data(), n.flag + g.nodeOff, G, cudaMemcpyDeviceToHost, sim->stream));
            CK(cudaStreamSynchronize(sim->stream));
            for (size_t i = 0; i < G; ++i) dst[i] = (float)f[i];
            return MPM_OK;
        } else {
            const float* src = nullptr;
            if (nm == "prevVelocities") src = n.prev;
            else if (nm == "forces") src = n.frc;
            else if (nm == "explicitMomenta") src = n.pstar;
            else if (nm == "rhs") src = n.b;
            else if (nm == "vc") src = n.vc;
            else if (nm == "diag") src = n.diag;
            else if (nm == "x0") src = n.x0;
            else if (nm == "solution") src = n.x;
            else if (nm == "velocities") src = n.vfin;
            if (!src) return set_err(sim, MPM_ERR_UNKNOWN_VARIABLE, "unknown grid array");
            if (count != 3 * G) return MPM_ERR_WRONG_SIZE;
            CK(cudaMemcpyAsync(dst, src + 3 * g.nodeOff, 3 * G * sizeof(float), cudaMemcpyDeviceToHost, sim->stream));
        }
        CK(cudaStreamSynchronize(sim->stream));
        return MPM_OK;
    });
}

mpm_status mpm_debug_apply(mpm_sim* sim, int body, const char* op, const float* in, float* out, size_t count, float dt) {
    if (!sim || !op || !in || !out || !sim->gridsValid || body < 0 || body >= (int)sim->grids.size()) return MPM_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&]() -> mpm_status {
        CK(cudaSetDevice(sim->device));
        const BodyGrid& g = sim->grids[body];
        const size_t G = (size_t)g.n[0] * g.n[1] * g.n[2];
        if (count != 3 * G) return MPM_ERR_WRONG_SIZE;
        std::string o(op);
        if (o != "A" && o != "DF") return MPM_ERR_INVALID_ARGUMENT;
        cudaStream_t s = sim->stream;
        if (sim->capDbg < 3 * (size_t)sim->Gtot) {
            if (sim->dbgA) { cudaFree(sim->dbgA); cudaFree(sim->dbgB); cudaFree(sim->dbgC); }
            sim->dbgA = alloc_f(3 * sim->Gtot); sim->dbgB = alloc_f(3 * sim->Gtot); sim->dbgC = alloc_f(3 * sim->Gtot);
            sim->capDbg = 3 * sim->Gtot;
        }
        CK(cudaMemsetAsync(sim->dbgA, 0, 3 * sizeof(float) * sim->Gtot, s));
        CK(cudaMemsetAsync(sim->dbgB, 0, 3 * sizeof(float) * sim->Gtot, s));
        CK(cudaMemcpyAsync(sim->dbgA + 3 * g.nodeOff, in, 3 * G * sizeof(float), cudaMemcpyHostToDevice, s));
        StepParams sp = sim->sp;
        sp.dt = dt;
        const int mt = max_tiles(sim);
        // the operator records of the current particle state: one force pass into a scratch force array
        {
            NodeArrays scratch = sim->nd;
            scratch.frc = sim->dbgB;
            launch_p2g_force(sim->P, sim->N, sim->T, mt, sim->dGrids, sp.h, scratch, nullptr, sim->opRec, false,
                             sim->dScalars + 3, s);
        }
        CK(cudaMemsetAsync(sim->dbgB, 0, 3 * sizeof(float) * sim->Gtot, s));
        if (o == "DF") {
            launch_op(sim->P, sim->N, sim->T, mt, sim->dGrids, sp.h, sim->dbgA, sim->dbgB, sim->opRec, sim->dSolve, false, s);
            CK(cudaMemcpyAsync(out, sim->dbgB + 3 * g.nodeOff, 3 * G * sizeof(float), cudaMemcpyDeviceToHost, s));
        } else {
            launch_node_project(sim->nd, sim->dGrids, sim->dChunkBody, sim->nChunks, sp, sim->dbgA, sim->dbgC, s);
            launch_op(sim->P, sim->N, sim->T, mt, sim->dGrids, sp.h, sim->dbgC, sim->dbgB, sim->opRec, sim->dSolve, false, s);
            launch_node_combine(sim->nd, sim->dGrids, sim->dChunkBody, sim->nChunks, sp, sim->dbgC, sim->dbgB, sim->dbgA, s);
            CK(cudaMemcpyAsync(out, sim->dbgA + 3 * g.nodeOff, 3 * G * sizeof(float), cudaMemcpyDeviceToHost, s));
        }
        CK(cudaStreamSynchronize(s));
        return MPM_OK;
    });
}

mpm_status mpm_debug_particle_cells(mpm_sim* sim, int* body, int* cell3, int* voxel3) {
    if (!sim || !body || !cell3 || !voxel3 || !sim->gridsValid) return MPM_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&]() -> mpm_status {
        CK(cudaSetDevice(sim->device));
        const int N = sim->N;
        if (N == 0) return MPM_OK;
        int *db = nullptr, *dc = nullptr, *dv = nullptr;
        CK(cudaMalloc(&db, sizeof(int) * N));
        CK(cudaMalloc(&dc, sizeof(int) * 3 * N));
        CK(cudaMalloc(&dv, sizeof(int) * 3 * N));
        k_debug_cells<<<(N + 255) / 256, 256, 0, sim->stream>>>(sim->P, N, sim->slotOf, sim->dGrids, sim->sp.h, db, dc, dv);
        CK(cudaMemcpyAsync(body, db, sizeof(int) * N, cudaMemcpyDeviceToHost, sim->stream));
        CK(cudaMemcpyAsync(cell3, dc, sizeof(int) * 3 * N, cudaMemcpyDeviceToHost, sim->stream));
        CK(cudaMemcpyAsync(voxel3, dv, sizeof(int) * 3 * N, cudaMemcpyDeviceToHost, sim->stream));
        CK(cudaStreamSynchronize(sim->stream));
        cudaFree(db); cudaFree(dc); cudaFree(dv);
        return MPM_OK;
    });
}

}  // extern "C"

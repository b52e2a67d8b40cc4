// CUDA kernels of the implicit MPM snow time step for B200 (sm_100a).
//
// Particle work runs per 4x4x4-cell tile: a CTA stages the tile's 7x7x7-node window of the grid in shared
// memory, its particles gather from / scatter into the window with shared-memory atomics, and the window is
// flushed to HBM with one global atomic per node.  Node work runs per 1024-node chunk; chunks never straddle
// bodies, so per-body reductions are segmented: each CTA stores an FP64 partial and the last CTA of a body
// (counter in HBM) sums that body's partials in a fixed order, which keeps the solver scalars deterministic.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>

#include "mpm_device.cuh"
#include "mpm_kernels.h"

namespace mpm {

// launches issued by this library (host threads may step different handles at once: relaxed atomic counts)
static std::atomic<long long> g_kernel_launches{0};
long long kernel_launch_count() { return g_kernel_launches.load(std::memory_order_relaxed); }
void kernel_launch_add(int n) { g_kernel_launches.fetch_add(n, std::memory_order_relaxed); }

namespace {

__device__ __forceinline__ void ld3(const float* a, size_t N, size_t i, float o[3]) {
    o[0] = a[i]; o[1] = a[N + i]; o[2] = a[2 * N + i];
}
__device__ __forceinline__ void st3(float* a, size_t N, size_t i, const float o[3]) {
    a[i] = o[0]; a[N + i] = o[1]; a[2 * N + i] = o[2];
}
__device__ __forceinline__ void ld9(const float* a, size_t N, size_t i, float o[9]) {
#pragma unroll
    for (int k = 0; k < 9; ++k) o[k] = a[k * N + i];
}
__device__ __forceinline__ void st9(float* a, size_t N, size_t i, const float o[9]) {
#pragma unroll
    for (int k = 0; k < 9; ++k) a[k * N + i] = o[k];
}

// ---------------------------------------------------------------------------------------------------------
// scan (exclusive prefix sum of ints), 1024 elements per CTA, recursive over block totals
// ---------------------------------------------------------------------------------------------------------
constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr int kScanBlock = kScanThreads * kScanItems;

__global__ void k_block_scan(const int* in, int* out, long long n, int* blockSums, int* total) {
    __shared__ int warpSums[kScanThreads / 32];
    const long long base = (long long)blockIdx.x * kScanBlock + (long long)threadIdx.x * kScanItems;
    int v[kScanItems];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? in[base + k] : 0;
        sum += v[k];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warpSums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int ws = lane < kScanThreads / 32 ? warpSums[lane] : 0;
        int wi = ws;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < kScanThreads / 32) warpSums[lane] = wi - ws;
        if (lane == kScanThreads / 32 - 1) {
            if (blockSums) blockSums[blockIdx.x] = wi;
            if (total && gridDim.x == 1) *total = wi;
        }
    }
    __syncthreads();
    int run = warpSums[warp] + incl - sum;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
}

__global__ void k_add_offsets(int* out, long long n, const int* offs) {
    const long long base = (long long)blockIdx.x * kScanBlock;
    const int add = offs[blockIdx.x];
    for (int k = threadIdx.x; k < kScanBlock; k += blockDim.x)
        if (base + k < n) out[base + k] += add;
}

// ---------------------------------------------------------------------------------------------------------
// deterministic block reduction of K doubles; result valid in thread 0
// ---------------------------------------------------------------------------------------------------------
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double (*sh)[kNodeThreads / 32]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[k][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double s = 0;
            for (int w = 0; w < kNodeThreads / 32; ++w) s += sh[k][w];
            v[k] = s;
        }
    }
    __syncthreads();
}

// Store this CTA's partials; returns true in the last CTA of the body, with `tot` = the body's sums
// (valid in every thread of that CTA).
template <int K>
__device__ bool segmented_reduce(double (&v)[K], const ReduceArrays& R, int b, int ctaBegin, int ctaEnd, double (&tot)[K]) {
    __shared__ double sh[K][kNodeThreads / 32];
    __shared__ double res[K];
    __shared__ int isLast;
    block_sum<K>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) R.partial[(size_t)blockIdx.x * 8 + k] = v[k];
        __threadfence();
        int prev = atomicAdd(&R.counter[b], 1);
        isLast = prev == ctaEnd - ctaBegin - 1;
    }
    __syncthreads();
    if (!isLast) return false;
    __threadfence();
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0;
    for (int c = ctaBegin + threadIdx.x; c < ctaEnd; c += blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] += __ldcg(&R.partial[(size_t)c * 8 + k]);
    block_sum<K>(acc, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) res[k] = acc[k];
        R.counter[b] = 0;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) tot[k] = res[k];
    return true;
}

// node chunk context
struct NodeCtx {
    int b;
    BodyGrid g;
    long long G;   // nodes of this body
    long long l0;  // first local node of this CTA
};
__device__ __forceinline__ NodeCtx node_ctx(const BodyGrid* grids, const int* chunkBody) {
    NodeCtx c;
    c.b = chunkBody[blockIdx.x];
    c.g = grids[c.b];
    c.G = (long long)c.g.n[0] * c.g.n[1] * c.g.n[2];
    c.l0 = (long long)(blockIdx.x - c.g.ctaBegin) * kNodeChunk;
    return c;
}
__device__ __forceinline__ void node_pos(const NodeCtx& c, long long l, float h, float x[3]) {
    int i = (int)(l % c.g.n[0]);
    long long r = l / c.g.n[0];
    int j = (int)(r % c.g.n[1]);
    int k = (int)(r / c.g.n[1]);
    // Grid.cpp:668 m_gridSize * i + m_min[0], separately rounded
    x[0] = __fadd_rn(__fmul_rn(h, (float)i), c.g.mn[0]);
    x[1] = __fadd_rn(__fmul_rn(h, (float)j), c.g.mn[1]);
    x[2] = __fadd_rn(__fmul_rn(h, (float)k), c.g.mn[2]);
}
__device__ __forceinline__ void ldn(const float* a, long long node, float o[3]) {
    o[0] = a[3 * node]; o[1] = a[3 * node + 1]; o[2] = a[3 * node + 2];
}
__device__ __forceinline__ void stn(float* a, long long node, const float o[3]) {
    a[3 * node] = o[0]; a[3 * node + 1] = o[1]; a[3 * node + 2] = o[2];
}

// tile context
struct TileCtx {
    int b;
    BodyGrid g;
    int wo[3];   // window origin node (tile * 4 - 1)
    int ps, pe;  // particle slots
    int tile;    // global tile id; its cells' particle ranges are T.start[tile * 64 + c]
};
__device__ __forceinline__ TileCtx tile_ctx(const TileArrays& T, const BodyGrid* grids, int li) {
    TileCtx c;
    int tile = T.list[li];
    c.b = T.listBody[li];
    c.g = grids[c.b];
    int lt = tile - c.g.tileOff;
    int tx = lt % c.g.T[0];
    int r = lt / c.g.T[0];
    int ty = r % c.g.T[1];
    int tz = r / c.g.T[1];
    c.wo[0] = tx * kTile - 1;
    c.wo[1] = ty * kTile - 1;
    c.wo[2] = tz * kTile - 1;
    c.ps = T.start[tile * kTileCells];
    c.pe = T.start[(tile + 1) * kTileCells];
    c.tile = tile;
    return c;
}
// global node of window entry w, or -1 if outside the grid
__device__ __forceinline__ long long win_node(const TileCtx& c, int w) {
    int lx = w % kWin, r = w / kWin, ly = r % kWin, lz = r / kWin;
    int gx = c.wo[0] + lx, gy = c.wo[1] + ly, gz = c.wo[2] + lz;
    if (gx < 0 || gy < 0 || gz < 0 || gx >= c.g.n[0] || gy >= c.g.n[1] || gz >= c.g.n[2]) return -1;
    return c.g.nodeOff + gx + (long long)c.g.n[0] * (gy + (long long)c.g.n[1] * gz);
}
// window offset of a particle's stencil (cell - 1 - wo); false if it falls outside the window
__device__ __forceinline__ bool win_base(const TileCtx& c, const Stencil& s, int& w0) {
    int lx = s.cell[0] - 1 - c.wo[0], ly = s.cell[1] - 1 - c.wo[1], lz = s.cell[2] - 1 - c.wo[2];
    if (lx < 0 || ly < 0 || lz < 0 || lx > kWin - 4 || ly > kWin - 4 || lz > kWin - 4) return false;
    w0 = lx + kWin * (ly + kWin * lz);
    return true;
}

__device__ __forceinline__ int read_list_count(const TileArrays& T) { return *T.listCount; }
// Adds a CTA's window accumulator to a node array with NC components per node ([NC node + c], x fastest): the
// accumulator holds STRIDE values per window node, the NC to add at offset OFF.  A window row (7 nodes along x)
// is NC * 7 consecutive floats of the node array: one thread per row adds them with 16-byte vector atomics over
// the row's 16-byte-aligned middle (addresses checked, not assumed) and scalar atomics at its ends, skipping
// all-zero groups and the window's nodes outside the grid.
template <int NC, int STRIDE, int OFF>
__device__ void flush_window(const TileCtx& c, const float* acc, float* out) {
    for (int row = threadIdx.x; row < kWin * kWin; row += blockDim.x) {
        const int ly = row % kWin, lz = row / kWin;
        const int gy = c.wo[1] + ly, gz = c.wo[2] + lz;
        if (gy < 0 || gz < 0 || gy >= c.g.n[1] || gz >= c.g.n[2]) continue;
        const int xa = max(0, -c.wo[0]), xb = min(kWin, c.g.n[0] - c.wo[0]);
        if (xa >= xb) continue;
        const long long node0 = c.g.nodeOff + (c.wo[0] + xa) + (long long)c.g.n[0] * (gy + (long long)c.g.n[1] * gz);
        float* o = out + NC * node0;
        const float* a = acc + STRIDE * (kWin * row + xa);
        const int cnt = NC * (xb - xa);
        auto val = [&](int k) { return a[STRIDE * (k / NC) + OFF + k % NC]; };
        int k = 0;
        for (; k < cnt && (reinterpret_cast<uintptr_t>(o + k) & 15u) != 0; ++k) {
            const float v = val(k);
            if (v != 0.f) atomicAdd(o + k, v);
        }
        for (; k + 4 <= cnt; k += 4) {
            const float4 v = make_float4(val(k), val(k + 1), val(k + 2), val(k + 3));
            if (v.x != 0.f || v.y != 0.f || v.z != 0.f || v.w != 0.f) atomicAdd(reinterpret_cast<float4*>(o + k), v);
        }
        for (; k < cnt; ++k) {
            const float v = val(k);
            if (v != 0.f) atomicAdd(o + k, v);
        }
    }
}

// Persistent tile kernels take their tiles from a shared counter, one at a time, so that a CTA that drew light
// tiles (a body's surface, a tilted slab's faces) takes more of them: the launch ends one tile after the mean
// instead of at the CTA with the heaviest fixed share.  `slot` is a shared int of the calling CTA.
__device__ __forceinline__ int next_tile(const TileArrays& T, int* slot) {
    if (threadIdx.x == 0) *slot = atomicAdd(&T.sched[0], 1);
    __syncthreads();
    const int li = *slot;
    __syncthreads();
    return li;
}
// every CTA calls this once after its last tile; the last one resets the counters for the next launch
__device__ __forceinline__ void tiles_done(const TileArrays& T) {
    if (threadIdx.x == 0 && atomicAdd(&T.sched[1], 1) == (int)gridDim.x - 1) {
        T.sched[0] = 0;
        T.sched[1] = 0;
    }
}

}  // namespace

// =========================================================================================================
// scan
// =========================================================================================================
size_t scan_tmp_ints(long long n) {
    size_t t = 0;
    long long m = n;
    while (m > 1) {
        m = (m + kScanBlock - 1) / kScanBlock;
        t += (size_t)m + 32;
    }
    return t + 64;
}

void scan_exclusive(const int* in, int* out, long long n, int* tmp, int* total, cudaStream_t s) {
    long long nb = (n + kScanBlock - 1) / kScanBlock;
    if (nb < 1) nb = 1;
    if (nb == 1) {
        ++g_kernel_launches; k_block_scan<<<1, kScanThreads, 0, s>>>(in, out, n, nullptr, total);
        return;
    }
    int* sums = tmp;
    ++g_kernel_launches; k_block_scan<<<(unsigned)nb, kScanThreads, 0, s>>>(in, out, n, sums, nullptr);
    scan_exclusive(sums, sums, nb, tmp + nb + 32, total, s);
    ++g_kernel_launches; k_add_offsets<<<(unsigned)nb, kScanThreads, 0, s>>>(out, n, sums);
}

// =========================================================================================================
// step start: ballistic update (Sim.cpp:66-73) and per-body centre-of-mass velocity + bounding box
// (Sim.cpp:84-93, Grid.cpp:175-191)
// =========================================================================================================
// One wave of CTAs, each over a contiguous range of particles.  Particles of one body are contiguous in storage
// (tile-sorted), so a range almost always holds one body: each thread sums its particles per body (flushing
// with atomics where the body changes), the CTA reduces in shared memory and issues one set of atomics; a range
// over several bodies flushes per thread.
constexpr int kPrepThreads = 256;
__global__ void __launch_bounds__(kPrepThreads) k_prepare(PartArrays P, int N, StepParams sp, BodyAccum* acc, int B,
                                                          int chunk) {
    __shared__ double sd[4][kPrepThreads / 32];
    __shared__ unsigned int su[6][kPrepThreads / 32];
    __shared__ int sc[kPrepThreads / 32];
    __shared__ int sCur;
    // a thread's sums over its particles of body `cur`, flushed with atomics when the body changes (rare: the
    // particles are in the previous step's body order)
    int cur = -1, cnt = 0;
    double d[4] = {0.0, 0.0, 0.0, 0.0};
    unsigned int lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, hi[3] = {0u, 0u, 0u};
    auto flush = [&]() {
        if (cnt == 0) return;
        BodyAccum& A = acc[cur];
        for (int k = 0; k < 3; ++k) {
            atomicAdd(&A.mom[k], d[k]);
            atomicMin(&A.bmin[k], lo[k]);
            atomicMax(&A.bmax[k], hi[k]);
        }
        atomicAdd(&A.mass, d[3]);
        atomicAdd(&A.count, cnt);
        cnt = 0;
        for (int k = 0; k < 4; ++k) d[k] = 0.0;
        for (int k = 0; k < 3; ++k) { lo[k] = 0xffffffffu; hi[k] = 0u; }
    };
    const int beg = blockIdx.x * chunk, end = min(N, beg + chunk);
    for (int i = beg + threadIdx.x; i < end; i += kPrepThreads) {
        int b = P.body[i];
        const float m = P.m[i];
        float v[3];
        ld3(P.v, N, i, v);
        if (b < 0 && sp.nfields >= 0) {  // ballistic update (Sim.cpp:66-73)
            float a[3] = {0.f, 0.f, 0.f};
            for (int f = 0; f < sp.nfields; ++f)
                for (int k = 0; k < 3; ++k) a[k] = __fadd_rn(a[k], __fmul_rn(sp.gravity[f][k], m));
            for (int k = 0; k < 3; ++k) v[k] = __fadd_rn(v[k], __fmul_rn(sp.dt, __fdiv_rn(a[k], m)));
            st3(P.v, N, i, v);
        }
        if (b >= B || b < 0) continue;
        if (b != cur) {
            flush();
            cur = b;
        }
        float x[3];
        ld3(P.x, N, i, x);
        d[0] += (double)v[0] * m;
        d[1] += (double)v[1] * m;
        d[2] += (double)v[2] * m;
        d[3] += (double)m;
        for (int k = 0; k < 3; ++k) {
            lo[k] = min(lo[k], float_to_ordered(x[k]));
            hi[k] = max(hi[k], float_to_ordered(x[k]));
        }
        ++cnt;
    }
    // one atomic set per CTA when every thread's sums belong to the same body (the common case)
    if (threadIdx.x == 0) sCur = -1;
    __syncthreads();
    if (cnt > 0) sCur = cur;  // any one of them
    __syncthreads();
    const int b0 = sCur;
    const bool uniform = __syncthreads_and(cnt == 0 || cur == b0);
    if (b0 < 0) return;
    if (!uniform) {
        flush();
        return;
    }
    for (int o = 16; o > 0; o >>= 1) {
        for (int k = 0; k < 4; ++k) d[k] += __shfl_down_sync(0xffffffffu, d[k], o);
        for (int k = 0; k < 3; ++k) {
            lo[k] = min(lo[k], __shfl_down_sync(0xffffffffu, lo[k], o));
            hi[k] = max(hi[k], __shfl_down_sync(0xffffffffu, hi[k], o));
        }
        cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        for (int k = 0; k < 4; ++k) sd[k][warp] = d[k];
        for (int k = 0; k < 3; ++k) { su[k][warp] = lo[k]; su[3 + k][warp] = hi[k]; }
        sc[warp] = cnt;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kPrepThreads / 32; ++w) {
            for (int k = 0; k < 4; ++k) sd[k][0] += sd[k][w];
            for (int k = 0; k < 3; ++k) { su[k][0] = min(su[k][0], su[k][w]); su[3 + k][0] = max(su[3 + k][0], su[3 + k][w]); }
            sc[0] += sc[w];
        }
        BodyAccum& A = acc[b0];
        for (int k = 0; k < 3; ++k) {
            atomicAdd(&A.mom[k], sd[k][0]);
            atomicMin(&A.bmin[k], su[k][0]);
            atomicMax(&A.bmax[k], su[3 + k][0]);
        }
        atomicAdd(&A.mass, sd[3][0]);
        atomicAdd(&A.count, sc[0]);
    }
}

// one wave of CTAs, each over a contiguous range of particles (a multiple of the block size)
void launch_prepare(const PartArrays& P, int N, const StepParams& sp, BodyAccum* acc, int B, int* err, cudaStream_t s) {
    if (N <= 0) return;
    const int blocks = std::min((N + kPrepThreads - 1) / kPrepThreads, 148 * 8);
    const int per = (N + blocks - 1) / blocks;
    const int chunk = (per + kPrepThreads - 1) / kPrepThreads * kPrepThreads;
    const int grid = (N + chunk - 1) / chunk;
    ++g_kernel_launches; k_prepare<<<grid, kPrepThreads, 0, s>>>(P, N, sp, acc, B, chunk);
}

// =========================================================================================================
// binning: tile key per particle (cell index bit-exact with the reference's stencil base), counting sort
// =========================================================================================================
// key = global tile * 64 + cell within the tile (x fastest): particles end up grouped by tile and, inside a tile,
// by cell; ballistic particles go to the last bucket.
__global__ void k_keys(PartArrays P, int N, const BodyGrid* grids, int totalTiles, float h, int* key, int* rank,
                       int* cellCount, int* err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < N;
    const int b = valid ? P.body[i] : -1;
    int k = valid ? totalTiles * kTileCells : -1;
    if (b >= 0) {
        const BodyGrid& g = grids[b];
        float x[3], frac[3];
        int cell[3];
        ld3(P.x, N, i, x);
        stencil_cells(x, g.mn, g.n, h, cell, frac);
        int t[3], l[3];
        bool ok = true;
        for (int d = 0; d < 3; ++d) {
            if (g.n[d] == 1) {  // an axis of a lower-dimensional grid: one node, one tile
                t[d] = l[d] = 0;
                continue;
            }
            if (cell[d] < 1 || cell[d] + 2 >= g.n[d]) ok = false;
            int c = min(max(cell[d], 1), g.n[d] - 3);
            t[d] = c / kTile;
            l[d] = c - t[d] * kTile;
        }
        if (!ok) atomicOr(err, ERR_STENCIL_OOB);
        k = (g.tileOff + t[0] + g.T[0] * (t[1] + g.T[1] * t[2])) * kTileCells + l[0] + kTile * (l[1] + kTile * l[2]);
    }
    // particles arrive in the previous step's cell order: lanes sharing a key take one atomic per group
    // (all 32 lanes reach this point; lanes past N carry key -1 and write nothing)
    const unsigned int grp = __match_any_sync(0xffffffffu, k);
    const int lane = threadIdx.x & 31, leader = __ffs(grp) - 1;
    int base = 0;
    if (lane == leader && valid) base = atomicAdd(&cellCount[k], __popc(grp));
    base = __shfl_sync(grp, base, leader);
    if (valid) {
        key[i] = k;
        rank[i] = base + __popc(grp & ((1u << lane) - 1u));
    }
}

void launch_keys(const PartArrays& P, int N, const BodyGrid* grids, int totalTiles, float h, int* key, int* rank,
                 int* tileCount, int* err, cudaStream_t s) {
    if (N <= 0) return;
    ++g_kernel_launches; k_keys<<<(N + 255) / 256, 256, 0, s>>>(P, N, grids, totalTiles, h, key, rank, tileCount, err);
}

// the non-empty tiles, with one atomic per warp for their list positions
__global__ void k_tile_list(const int* cellStart, const BodyGrid* grids, int B, int totalTiles, int* list, int* listBody,
                            int* listCount) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool keep = t < totalTiles && cellStart[(t + 1) * kTileCells] != cellStart[t * kTileCells];
    const unsigned ballot = __ballot_sync(0xffffffffu, keep);
    if (!ballot) return;
    const int lane = threadIdx.x & 31, leader = __ffs(ballot) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(listCount, __popc(ballot));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (!keep) return;
    int lo = 0, hi = B - 1;
    while (lo < hi) {  // last body with tileOff <= t
        int mid = (lo + hi + 1) >> 1;
        if (grids[mid].tileOff <= t) lo = mid; else hi = mid - 1;
    }
    const int idx = base + __popc(ballot & ((1u << lane) - 1u));
    list[idx] = t;
    listBody[idx] = lo;
}
void launch_tile_list(const int* tileCount, const BodyGrid* grids, int B, int totalTiles, int* list, int* listBody,
                      int* listCount, cudaStream_t s) {
    if (totalTiles <= 0) return;
    ++g_kernel_launches; k_tile_list<<<(totalTiles + 255) / 256, 256, 0, s>>>(tileCount, grids, B, totalTiles, list, listBody, listCount);
}

// The tile list ordered by decreasing particle count (16 classes of 64 particles), so that the tile kernels'
// dynamic scheduling hands out the heavy tiles first and ends on light ones (longest-processing-time first): one
// CTA counting-sorts the list through the scratch arrays tmp / tmpBody.
constexpr int kOrderThreads = 1024;
__global__ void __launch_bounds__(kOrderThreads) k_tile_order(const int* cellStart, int* list, int* listBody,
                                                              const int* listCount, int* tmp, int* tmpBody) {
    __shared__ int hist[16];
    const int n = *listCount;
    if (threadIdx.x < 16) hist[threadIdx.x] = 0;
    __syncthreads();
    auto cls = [&](int t) {
        const int cnt = cellStart[(t + 1) * kTileCells] - cellStart[t * kTileCells];
        return 15 - min(cnt >> 6, 15);
    };
    for (int li = threadIdx.x; li < n; li += kOrderThreads) atomicAdd(&hist[cls(list[li])], 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int c = 0; c < 16; ++c) {
            const int h = hist[c];
            hist[c] = acc;
            acc += h;
        }
    }
    __syncthreads();
    for (int li = threadIdx.x; li < n; li += kOrderThreads) {
        const int t = list[li];
        const int pos = atomicAdd(&hist[cls(t)], 1);
        tmp[pos] = t;
        tmpBody[pos] = listBody[li];
    }
    __syncthreads();
    for (int li = threadIdx.x; li < n; li += kOrderThreads) {
        list[li] = tmp[li];
        listBody[li] = tmpBody[li];
    }
}
void launch_tile_order(const int* cellStart, int* list, int* listBody, const int* listCount, int* tmp, int* tmpBody,
                       cudaStream_t s) {
    ++g_kernel_launches;
    k_tile_order<<<1, kOrderThreads, 0, s>>>(cellStart, list, listBody, listCount, tmp, tmpBody);
}

// The counting sort's permutation in two passes: the first computes each particle's slot d = tileStart[key] + rank,
// maps the caller's index to it (slotOf) and records the inverse (inv[d] = source slot); the second gathers every
// 32-bit word of the particle state (up to 64 component arrays, their loads in flight together) into slot order,
// so that the writes are aligned and coalesced.
__global__ void __launch_bounds__(256) k_permute_state(const int* __restrict__ key, const int* __restrict__ rank,
                                                       const int* __restrict__ tileStart, int N, PermuteWords w,
                                                       const int* __restrict__ orig, int* slotOf, int* inv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int d = tileStart[key[i]] + rank[i];
    slotOf[orig[i]] = d;
    inv[d] = i;
}
__global__ void __launch_bounds__(256) k_permute_gather(int N, PermuteWords w, const int* __restrict__ inv) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N) return;
    const int i = inv[j];
    int f = 0;
    for (; f + 8 <= w.n; f += 8) {
        unsigned int v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = __ldg(w.src[f + k] + i);
#pragma unroll
        for (int k = 0; k < 8; ++k) w.dst[f + k][j] = v[k];
    }
    for (; f < w.n; ++f) w.dst[f][j] = __ldg(w.src[f] + i);
}
void launch_permute_state(const int* key, const int* rank, const int* tileStart, int N, const PermuteWords& w,
                          const int* orig, int* slotOf, int* inv, cudaStream_t s) {
    if (N <= 0) return;
    ++g_kernel_launches; k_permute_state<<<(N + 255) / 256, 256, 0, s>>>(key, rank, tileStart, N, w, orig, slotOf, inv);
    ++g_kernel_launches; k_permute_gather<<<(N + 255) / 256, 256, 0, s>>>(N, w, inv);
}
// state (SoA, slot order) -> caller order, interleaved comps per particle
__global__ void k_gather_user(const float* state, const int* slotOf, float* out, int N, int comps) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int s = slotOf[i];
    for (int c = 0; c < comps; ++c) out[(size_t)i * comps + c] = state[(size_t)c * N + s];
}
void launch_gather_user(const float* state, const int* slotOf, float* out, int N, int comps, cudaStream_t s) {
    if (N <= 0) return;
    ++g_kernel_launches; k_gather_user<<<(N + 255) / 256, 256, 0, s>>>(state, slotOf, out, N, comps);
}
__global__ void k_scatter_user(const float* in, const int* slotOf, float* state, int N, int comps) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int s = slotOf[i];
    for (int c = 0; c < comps; ++c) state[(size_t)c * N + s] = in[(size_t)i * comps + c];
}
void launch_scatter_user(const float* in, const int* slotOf, float* state, int N, int comps, cudaStream_t s) {
    if (N <= 0) return;
    ++g_kernel_launches; k_scatter_user<<<(N + 255) / 256, 256, 0, s>>>(in, slotOf, state, N, comps);
}

// Particle volumes — Grid::computeParticleVolumes, Grid.cpp:265-292
__global__ void __launch_bounds__(kTileThreads) k_volumes(PartArrays P, int N, TileArrays T, const BodyGrid* grids, float h,
                                                           NodeArrays nd) {
    __shared__ float gm[kWin3];
    __shared__ int sTile;
    const int nl = read_list_count(T);
    const float cellVolume = h * h * h;
    for (int li = next_tile(T, &sTile); li < nl; li = next_tile(T, &sTile)) {
        TileCtx c = tile_ctx(T, grids, li);
        for (int w = threadIdx.x; w < kWin3; w += blockDim.x) {
            long long node = win_node(c, w);
            gm[w] = node >= 0 ? nd.mass[node] : 0.f;
        }
        __syncthreads();
        for (int i = c.ps + threadIdx.x; i < c.pe; i += blockDim.x) {
            float x[3];
            ld3(P.x, N, i, x);
            Stencil s;
            stencil_eval<false>(x, c.g.mn, c.g.n, h, s);
            int w0;
            if (!win_base(c, s, w0)) continue;
            float density = 0.f;
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int j = 0; j < 4; ++j)
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        density += s.w[0][q] * s.w[1][j] * s.w[2][k] * gm[w0 + q + kWin * (j + kWin * k)] / cellVolume;
            P.vol[i] = P.m[i] / density;
        }
        __syncthreads();
    }
    tiles_done(T);
}

// =========================================================================================================
// The implicit operator's particle pass (ForceDifferentialSplatter, Grid.cpp:569-611) through the step's
// operator records.  The force pass (k_force_warp) also sums the dFidXi diagonal (dFidXiSplatter,
// Grid.cpp:484-531) through linearity: dEdFDifferential is linear in dF, so the reference's 192 evaluations per
// particle reduce to the particle's 9x9 map M (built there) and a quadratic form per node.
// =========================================================================================================
// fm is linear in G: fm = M vec(G) with the 9x9 matrix M = vol L^T H L, H the Hessian of the energy density
// (dEdFDifferential) and L: G -> G F; M is symmetric because H is.  The force pass, once per step and with the
// particle state already loaded for the stress, evaluates M in closed form and stores its 45 upper entries with
// the particle's window base and 24 B-spline weights (OpRec), and sums the Jacobi diagonal from M's diagonal 3x3
// blocks.  DF(vc) for the rhs (on the tiles that touch a collided node) and the CR operator passes of the step
// read those 280 B per particle in place of x, F, R, F^-T, G^-1, J, mu, lambda and the volume, and do 81 FMA in
// place of the stencil evaluation and the linearisation.  The weights are stored rather than re-evaluated so
// that the operator uses bit for bit the values of the step's other passes: at a stencil's tail nodes, whose
// masses are tiny, an operator built from differently rounded weights disagrees with the masses and the
// diagonal, which slows CR and degrades the converged velocities.
// position of M[r][c], r <= c, in the upper triangle stored column by column
__host__ __device__ constexpr int msym_index(int r, int c) { return c * (c + 1) / 2 + r; }
static_assert(msym_index(8, 8) == kOpRecM - 1 && kOpRecM <= 4 * kOpRecM4, "upper triangle of a 9x9 matrix");

// The force pass's per-particle work (the particle's state already loaded by its CTA's tile pass): its force
// matrix fmOut = vol P F^T from the stress (ForceSplatter, Grid.cpp:405-428), the operator's map M in closed form
// written to the step's records (the upper triangle, four entries per float4), and M's diagonal blocks as the
// Jacobi diagonal's quadratic forms S[6 a + slot].
__device__ __forceinline__ void force_particle(const PartArrays& P, int N, int i, const OpRec& opr, float fmOut[9],
                                               float S[18], int* err) {
    // (vol P) F^T of the particle's stress
    float F[9], R[9], FiT[9], Gi[9], Ps[9], fm[9];
    ld9(P.F, N, i, F);
    ld9(P.R, N, i, R);
    ld9(P.FiT, N, i, FiT);
    const float vol = P.vol[i], J = P.J[i], mu = P.mu[i], lam = P.lam[i];
    snow_stress(F, R, FiT, J, mu, lam, Ps);
    float nrm = 0.f;
#pragma unroll
    for (int k = 0; k < 9; ++k) nrm += Ps[k] * Ps[k];
    if (!isfinite(nrm)) atomicOr(err, ERR_NAN_STRESS);
#pragma unroll
    for (int k = 0; k < 9; ++k) Ps[k] *= vol;
    mat_mul_bt(Ps, F, fm);
#pragma unroll
    for (int k = 0; k < 9; ++k) fmOut[k] = fm[k];
    // the operator's map M in closed form.  dEdFDifferential at dF = G F, times vol and F^T, is
    //   vol [2 mu G F F^T + lam J (2J - 1) <G, C> C - lam J (J - 1) C G^T C - 2 mu R Omega(g) F^T]
    // with C = F^-T F^T from the stored F^-T (the identity unless F was set since the last
    // plasticity pass, which the reference's formula then evaluates as it stands), g = G^-1 w and
    // w_k = <G, Q_k>, Q_k = R E_k F^T for the antisymmetric basis E_k = e_i e_j^T - e_j e_i^T,
    // (i, j) = (0, 1), (0, 2), (1, 2), of the rotation's axial vector (SnowConstitutiveModel.cpp:
    // 218-287).  Entry (row (a, c), column (b, d)) is therefore 2 mu [a = b] (F F^T)_dc
    // + lam J (2J - 1) C_ac C_bd - lam J (J - 1) C_ad C_bc - 2 mu sum_kl (G^-1)_kl (Q_k)_ac (Q_l)_bd,
    // times vol, the same as column (b, d) of the column-by-column evaluation.  Entries on and above
    // the diagonal go to the records, four at a time.
    ld9(P.Gi, N, i, Gi);
    float q[3][9], B[9];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int ei = k == 2 ? 1 : 0, ej = k == 0 ? 1 : 2;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int cc = 0; cc < 3; ++cc)
                q[k][3 * a + cc] = R[3 * a + ei] * F[3 * cc + ej] - R[3 * a + ej] * F[3 * cc + ei];
    }
    float Cm[9];
    mat_mul_bt(F, F, B);
    mat_mul_bt(FiT, F, Cm);
    const float m2 = 2.0f * mu, s1 = lam * J * (2.0f * J - 1.0f), s2 = lam * J * (J - 1.0f);
    float4* Mo = opr.m4 + i;
    float grp[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int col = 0; col < 9; ++col) {
        const int b = col / 3, d = col % 3;
        float hk[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) hk[k] = Gi[3 * k] * q[0][col] + Gi[3 * k + 1] * q[1][col] + Gi[3 * k + 2] * q[2][col];
#pragma unroll
        for (int row = 0; row <= col; ++row) {
            const int a = row / 3, cc = row % 3;
            float v = -m2 * (q[0][row] * hk[0] + q[1][row] * hk[1] + q[2][row] * hk[2]);
            if (a == b) v += m2 * B[3 * d + cc];
            v += s1 * Cm[3 * a + cc] * Cm[3 * b + d];
            v -= s2 * Cm[3 * a + d] * Cm[3 * b + cc];
            const int e = msym_index(row, col);
            grp[e & 3] = vol * v;
            if (a == b) {
                // M's diagonal block of axis a: the coefficient of g_c g_d in that axis's
                // diagonal -g^T M_aa g (dForceidXi, Grid.cpp:841-867), stored as
                // {c = d = 0, 1, 2; 2 x (0, 1), (0, 2), (1, 2)}
                const int slot = cc == d ? cc : (cc == 0 ? (d == 1 ? 3 : 4) : 5);
                S[6 * a + slot] = cc == d ? vol * v : 2.0f * (vol * v);
            }
            if ((e & 3) == 3 || e == kOpRecM - 1) {
                Mo[(size_t)(e >> 2) * N] = make_float4(grp[0], grp[1], grp[2], grp[3]);
                grp[0] = grp[1] = grp[2] = grp[3] = 0.f;
            }
        }
    }
}

// G2P — updateParticleVelocities (Grid.cpp:1049-1081) fused with updateDeformationGradients (:1018-1047).  The
// window holds per node the solved velocity v and its change d = v - prev as float4s; the 64-node sums are
// separable: per stencil row (y, z) they contract over x first (sv = sum_q v wx_q, sdv = sum_q v dwx_q,
// sd = sum_q d wx_q), then the row's y / z factors give FLIP, PIC and the velocity gradient.  PIC adds the frame
// velocity times the sum of the weights.
__global__ void __launch_bounds__(kTileThreads) k_g2p(PartArrays P, int N, TileArrays T, const BodyGrid* grids, float h,
                                                       float dt, NodeArrays nd) {
    __shared__ float4 wv[kWin3];
    __shared__ float4 wd[kWin3];
    __shared__ int sTile;
    const int nl = read_list_count(T);
    const float alpha = 0.95f, beta = 1.0f - alpha;
    for (int li = next_tile(T, &sTile); li < nl; li = next_tile(T, &sTile)) {
        TileCtx c = tile_ctx(T, grids, li);
        for (int w = threadIdx.x; w < kWin3; w += blockDim.x) {
            long long node = win_node(c, w);
            float v[3] = {0.f, 0.f, 0.f}, pv[3] = {0.f, 0.f, 0.f};
            if (node >= 0) {
                ldn(nd.vfin, node, v);
                ldn(nd.prev, node, pv);
            }
            wv[w] = make_float4(v[0], v[1], v[2], 0.f);
            wd[w] = make_float4(v[0] - pv[0], v[1] - pv[1], v[2] - pv[2], 0.f);
        }
        __syncthreads();
        for (int i = c.ps + threadIdx.x; i < c.pe; i += blockDim.x) {
            float x[3];
            ld3(P.x, N, i, x);
            Stencil s;
            stencil_eval<true>(x, c.g.mn, c.g.n, h, s);
            int w0;
            if (!win_base(c, s, w0)) continue;
            float vflip[3], vpic[3] = {0.f, 0.f, 0.f}, dv[9], wsum = 0.f;
            ld3(P.v, N, i, vflip);
#pragma unroll
            for (int k = 0; k < 9; ++k) dv[k] = 0.f;
            float wx = 0.f;
#pragma unroll
            for (int q = 0; q < 4; ++q) wx += s.w[0][q];
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float wjk = s.w[1][j] * s.w[2][k], dwjk = s.dw[1][j] * s.w[2][k], wjdk = s.w[1][j] * s.dw[2][k];
                    const int wr = w0 + kWin * (j + kWin * k);
                    float sv[3] = {0.f, 0.f, 0.f}, sdv[3] = {0.f, 0.f, 0.f}, sd[3] = {0.f, 0.f, 0.f};
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const float4 a = wv[wr + q], b = wd[wr + q];
                        const float wq = s.w[0][q], dq = s.dw[0][q];
                        sv[0] += a.x * wq; sv[1] += a.y * wq; sv[2] += a.z * wq;
                        sdv[0] += a.x * dq; sdv[1] += a.y * dq; sdv[2] += a.z * dq;
                        sd[0] += b.x * wq; sd[1] += b.y * wq; sd[2] += b.z * wq;
                    }
                    wsum += wx * wjk;
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        vflip[a] += wjk * sd[a];
                        vpic[a] += wjk * sv[a];
                        dv[3 * a] -= sdv[a] * wjk;
                        dv[3 * a + 1] -= sv[a] * dwjk;
                        dv[3 * a + 2] -= sv[a] * wjdk;
                    }
                }
#pragma unroll
            for (int a = 0; a < 3; ++a) vpic[a] += wsum * c.g.fv[a];
            float vn[3] = {alpha * vflip[0] + beta * vpic[0], alpha * vflip[1] + beta * vpic[1], alpha * vflip[2] + beta * vpic[2]};
            st3(P.v, N, i, vn);
            float F[9], Mx[9], Fn[9];
            ld9(P.F, N, i, F);
#pragma unroll
            for (int k = 0; k < 9; ++k) Mx[k] = dt * dv[k] + ((k % 4 == 0) ? 1.f : 0.f);
            mat_mul(Mx, F, Fn);
            st9(P.F, N, i, Fn);
        }
        __syncthreads();
    }
    tiles_done(T);
}

static inline int tile_grid(int maxTiles) {
    int g = maxTiles < 148 * 8 ? maxTiles : 148 * 8;
    return g < 1 ? 1 : g;
}

void launch_volumes(const PartArrays& P, int N, const TileArrays& T, int maxTiles, const BodyGrid* grids, float h,
                    NodeArrays nd, cudaStream_t s) {
    ++g_kernel_launches; k_volumes<<<tile_grid(maxTiles), kTileThreads, 0, s>>>(P, N, T, grids, h, nd);
}
// ---------------------------------------------------------------------------------------------------------
// The CR operator pass, warp-autonomous: the pass a CR iteration runs (ForceDifferentialSplatter, Grid.cpp:
// 569-611, through the step's operator records).  A CTA stages the tile's 7 x 7 x 7 window of the input vector
// and an accumulator in shared memory; each of its warps then takes a quarter of the tile's particles in rounds
// of 32 with no CTA-wide barrier until the flush:
//   lane = particle: its record (18 float4 loads), the gather G = sum_i in_i grad(w_i)^T from the window
//     (separable: contracted over x, then y and z), fm = M vec(G), staged with its 24 weights in the warp's own
//     shared-memory slots;
//   lane = (run of the round's particles in one cell, stencil z-layer, stencil y-row): the scatter
//     -fm grad(w_i) summed over the run's particles into 4 nodes x 3 components of registers (packed FP32x2
//     FMA over node pairs), added to the accumulator once per run.
// Particles are sorted by cell within the tile, so a round's particles form a few runs of one cell each.
// ---------------------------------------------------------------------------------------------------------
constexpr int kApplyWarps = 4;
constexpr int kApplyThreads = 32 * kApplyWarps;
constexpr int kApplyMinBlocks = 6;
constexpr int kApplyRec = 36;   // staged per particle: fm[9] (+3 unused) | wx | dwx | wy | dwy | wz | dwz
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__global__ void __launch_bounds__(kApplyThreads, kApplyMinBlocks)
    k_op_apply(TileArrays T, const BodyGrid* grids, const float* __restrict__ in, float* out, OpRec opr, int N,
               const BodySolve* solve, int skipDone, unsigned long long* procCount) {
    __shared__ float4 win[kWin3];
    __shared__ float acc[3 * kWin3];
    __shared__ __align__(16) float rec[kApplyWarps][32 * kApplyRec];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float* R = &rec[warp][lane * kApplyRec];
    const float* Rw = rec[warp];
    __shared__ int sTile;
    const int nl = read_list_count(T);
    for (int li = next_tile(T, &sTile); li < nl; li = next_tile(T, &sTile)) {
        TileCtx c = tile_ctx(T, grids, li);
        if (skipDone && solve[c.b].done) continue;  // uniform over the CTA
        if (procCount && threadIdx.x == 0) atomicAdd(procCount, (unsigned long long)(c.pe - c.ps));
        for (int w = threadIdx.x; w < kWin3; w += kApplyThreads) {
            const long long node = win_node(c, w);
            win[w] = node >= 0 ? make_float4(__ldg(&in[3 * node]), __ldg(&in[3 * node + 1]), __ldg(&in[3 * node + 2]), 0.f)
                               : make_float4(0.f, 0.f, 0.f, 0.f);
            acc[3 * w] = acc[3 * w + 1] = acc[3 * w + 2] = 0.f;
        }
        __syncthreads();
        const int np = c.pe - c.ps;
        const int wb = c.ps + (int)(((long long)np * warp) / kApplyWarps);
        const int we = c.ps + (int)(((long long)np * (warp + 1)) / kApplyWarps);
        for (int r0 = wb; r0 < we; r0 += 32) {
            const int i = r0 + lane;
            int w0 = -1;
            if (i < we) {
                w0 = __ldg(&opr.base[i]);
                // a window base has lx, ly, lz in [0, kWin - 4]; anything else (no record) contributes nothing
                if ((unsigned)w0 > (unsigned)((kWin - 4) * (1 + kWin + kWin * kWin))) w0 = -1;
            }
            int cl = -1;  // the particle's cell within the tile, x fastest
            if (w0 >= 0) {
                const int lx = w0 % kWin, ly = (w0 / kWin) % kWin, lz = w0 / (kWin * kWin);
                cl = lx + kTile * (ly + kTile * lz);
                const float4* Wi = opr.w4 + i;
                const float4 gwx = __ldg(Wi), gdwx = __ldg(Wi + N), gwy = __ldg(Wi + 2 * (size_t)N),
                             gdwy = __ldg(Wi + 3 * (size_t)N), gwz = __ldg(Wi + 4 * (size_t)N),
                             gdwz = __ldg(Wi + 5 * (size_t)N);
                const float wx[4] = {gwx.x, gwx.y, gwx.z, gwx.w}, dwx[4] = {gdwx.x, gdwx.y, gdwx.z, gdwx.w};
                const float wy[4] = {gwy.x, gwy.y, gwy.z, gwy.w}, dwy[4] = {gdwy.x, gdwy.y, gdwy.z, gdwy.w};
                const float wz[4] = {gwz.x, gwz.y, gwz.z, gwz.w}, dwz[4] = {gdwz.x, gdwz.y, gdwz.z, gdwz.w};
                // G = sum_i dx_i grad(w_i)^T, grad(w_i) = -(dwx wy wz, wx dwy wz, wx wy dwz): over x first
                float Gm[9];
#pragma unroll
                for (int k = 0; k < 9; ++k) Gm[k] = 0.f;
#pragma unroll 1
                for (int k = 0; k < 4; ++k) {
                    const float wzk = k == 0 ? wz[0] : k == 1 ? wz[1] : k == 2 ? wz[2] : wz[3];
                    const float dwzk = k == 0 ? dwz[0] : k == 1 ? dwz[1] : k == 2 ? dwz[2] : dwz[3];
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const float wjk = wy[j] * wzk, dwjk = dwy[j] * wzk, wjdk = wy[j] * dwzk;
                        const int wr = w0 + kWin * (j + kWin * k);
                        float sx[3] = {0.f, 0.f, 0.f}, sdx[3] = {0.f, 0.f, 0.f};
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const float4 d = win[wr + q];
                            sx[0] += d.x * wx[q]; sdx[0] += d.x * dwx[q];
                            sx[1] += d.y * wx[q]; sdx[1] += d.y * dwx[q];
                            sx[2] += d.z * wx[q]; sdx[2] += d.z * dwx[q];
                        }
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            Gm[3 * a] -= sdx[a] * wjk;
                            Gm[3 * a + 1] -= sx[a] * dwjk;
                            Gm[3 * a + 2] -= sx[a] * wjdk;
                        }
                    }
                }
                // fm = M vec(G), M symmetric from its upper triangle (45 entries in 12 float4 groups)
                float fm[9];
#pragma unroll
                for (int k = 0; k < 9; ++k) fm[k] = 0.f;
                const float4* Mi = opr.m4 + i;
                float4 grp = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int b = 0; b < 9; ++b)
#pragma unroll
                    for (int a = 0; a <= b; ++a) {
                        const int e = msym_index(a, b);
                        if ((e & 3) == 0) grp = __ldg(Mi + (size_t)(e >> 2) * N);
                        const float mv = (e & 3) == 0 ? grp.x : (e & 3) == 1 ? grp.y : (e & 3) == 2 ? grp.z : grp.w;
                        fm[a] += mv * Gm[b];
                        if (b != a) fm[b] += mv * Gm[a];
                    }
                float4* R4 = reinterpret_cast<float4*>(R);
                R4[0] = make_float4(fm[0], fm[1], fm[2], fm[3]);
                R4[1] = make_float4(fm[4], fm[5], fm[6], fm[7]);
                R4[2] = make_float4(fm[8], __int_as_float(cl), 0.f, 0.f);
                R4[3] = gwx; R4[4] = gdwx; R4[5] = gwy; R4[6] = gdwy; R4[7] = gwz; R4[8] = gdwz;
            }
            __syncwarp();
            // runs of equal cells among the round's lanes; a lane without a particle ends a run
            const int prev = __shfl_up_sync(0xffffffffu, cl, 1);
            const unsigned heads = __ballot_sync(0xffffffffu, cl >= 0 && (lane == 0 || prev != cl));
            const unsigned breaks = heads | __ballot_sync(0xffffffffu, cl < 0);
            const int nrun = __popc(heads);
            for (int item = lane; item < 16 * nrun; item += 32) {
                const int run = item >> 4, kz = (item >> 2) & 3, jy = item & 3;
                const int sl = __fns(heads, 0, run + 1);
                const unsigned after = sl >= 31 ? 0u : breaks & (0xffffffffu << (sl + 1));
                const int el = after ? __ffs(after) - 1 : 32;
                // -fm grad(w) over the row (jy, kz): dwx (fm[:,0] wy wz) + wx (fm[:,1] dwy wz + fm[:,2] wy dwz)
                float2 a01[3] = {f2(0.f, 0.f), f2(0.f, 0.f), f2(0.f, 0.f)}, a23[3] = {f2(0.f, 0.f), f2(0.f, 0.f), f2(0.f, 0.f)};
                for (int p = sl; p < el; ++p) {
                    const float* Rp = Rw + p * kApplyRec;
                    const float4 f0 = *reinterpret_cast<const float4*>(Rp), f1 = *reinterpret_cast<const float4*>(Rp + 4);
                    const float f8 = Rp[8];
                    const float4 gx = *reinterpret_cast<const float4*>(Rp + 12), gdx = *reinterpret_cast<const float4*>(Rp + 16);
                    const float wyj = Rp[20 + jy], dwyj = Rp[24 + jy], wzk = Rp[28 + kz], dwzk = Rp[32 + kz];
                    // the row's three weight products, formed once for the three components
                    const float wzy = wzk * wyj, wzdy = wzk * dwyj, dzwy = dwzk * wyj;
                    const float fmv[9] = {f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, f1.z, f1.w, f8};
                    const float2 wx01 = f2(gx.x, gx.y), wx23 = f2(gx.z, gx.w);
                    const float2 dwx01 = f2(gdx.x, gdx.y), dwx23 = f2(gdx.z, gdx.w);
#pragma unroll
                    for (int cc = 0; cc < 3; ++cc) {
                        const float U = fmv[3 * cc] * wzy;
                        const float V = fmv[3 * cc + 1] * wzdy + fmv[3 * cc + 2] * dzwy;
                        const float2 U2 = f2(U, U), V2 = f2(V, V);
                        a01[cc] = __ffma2_rn(U2, dwx01, __ffma2_rn(V2, wx01, a01[cc]));
                        a23[cc] = __ffma2_rn(U2, dwx23, __ffma2_rn(V2, wx23, a23[cc]));
                    }
                }
                // the run's cell (staged beside fm) places the row: its stencil starts at the cell's window offset
                const int cell = __float_as_int(Rw[sl * kApplyRec + 9]);
                const int cx = cell & 3, cy = (cell >> 2) & 3, cz = cell >> 4;
                float* dst = &acc[3 * (cx + kWin * ((cy + jy) + kWin * (cz + kz)))];
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) {
                    atomicAdd(&dst[cc], a01[cc].x);
                    atomicAdd(&dst[3 + cc], a01[cc].y);
                    atomicAdd(&dst[6 + cc], a23[cc].x);
                    atomicAdd(&dst[9 + cc], a23[cc].y);
                }
            }
            __syncwarp();
        }
        __syncthreads();
        flush_window<3, 3, 0>(c, acc, out);
        __syncthreads();
    }
    tiles_done(T);
}

// ---------------------------------------------------------------------------------------------------------
// The force pass, warp-autonomous like k_op_apply: per tile, each warp takes a quarter of its particles in rounds
// of 32.  Lane = particle: its stencil, weights and window base written to the step's operator records, its
// force matrix, M in closed form (records) and M's diagonal blocks (force_particle), staged in the warp's slots.
// Lane = (run of one cell, stencil z-layer, y-row): the internal forces -vol P F^T grad(w) (ForceSplatter,
// Grid.cpp:405-428) and the dFidXi sums of the Jacobi diagonal (dFidXiSplatter, Grid.cpp:484-531) of 4 nodes,
// summed over the run and added to the CTA's accumulators once per run.
// ---------------------------------------------------------------------------------------------------------
constexpr int kForceRec = 60;  // fm[9], cell, -, - | wx dwx wy dwy wz dwz | S[18], -, - | m, m (v - v_frame)
template <bool MASS>
__global__ void __launch_bounds__(kApplyThreads, 4)
    k_force_warp(PartArrays P, int N, TileArrays T, const BodyGrid* grids, float h, float* frc, float* diagOut,
                 float* massOut, float* momOut, OpRec opr, int* err) {
    __shared__ float acc[3 * kWin3];
    __shared__ float dacc[3 * kWin3];
    __shared__ float macc[MASS ? 4 * kWin3 : 1];
    __shared__ __align__(16) float rec[kApplyWarps][32 * kForceRec];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float* R = &rec[warp][lane * kForceRec];
    const float* Rw = rec[warp];
    __shared__ int sTile;
    const int nl = read_list_count(T);
    for (int li = next_tile(T, &sTile); li < nl; li = next_tile(T, &sTile)) {
        TileCtx c = tile_ctx(T, grids, li);
        for (int e = threadIdx.x; e < 3 * kWin3; e += kApplyThreads) acc[e] = dacc[e] = 0.f;
        if (MASS)
            for (int e = threadIdx.x; e < 4 * kWin3; e += kApplyThreads) macc[e] = 0.f;
        __syncthreads();
        const int np = c.pe - c.ps;
        const int wb = c.ps + (int)(((long long)np * warp) / kApplyWarps);
        const int we = c.ps + (int)(((long long)np * (warp + 1)) / kApplyWarps);
        for (int r0 = wb; r0 < we; r0 += 32) {
            const int i = r0 + lane;
            int cl = -1;
            if (i < we) {
                float x[3], frac[3];
                int cell[3];
                ld3(P.x, N, i, x);
                stencil_cells(x, c.g.mn, c.g.n, h, cell, frac);
                const int lx = cell[0] - 1 - c.wo[0], ly = cell[1] - 1 - c.wo[1], lz = cell[2] - 1 - c.wo[2];
                if (lx >= 0 && ly >= 0 && lz >= 0 && lx <= kWin - 4 && ly <= kWin - 4 && lz <= kWin - 4) {
                    if (MASS) {  // the particle's mass and momentum relative to the frame (MassSplatter, VelocitySplatter)
                        float v[3];
                        ld3(P.v, N, i, v);
                        const float m = P.m[i];
                        reinterpret_cast<float4*>(R)[14] =
                            make_float4(m, m * (v[0] - c.g.fv[0]), m * (v[1] - c.g.fv[1]), m * (v[2] - c.g.fv[2]));
                    }
                    opr.base[i] = lx + kWin * (ly + kWin * lz);
                    cl = lx + kTile * (ly + kTile * lz);
                    float wgt[6][4];
#pragma unroll
                    for (int q = 0; q < 4; ++q)
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            wgt[2 * a][q] = stencil_w(c.g.n[a] == 1, q, frac[a]);
                            wgt[2 * a + 1][q] = stencil_dw(c.g.n[a] == 1, q, frac[a], h);
                        }
                    float4* R4 = reinterpret_cast<float4*>(R);
                    float4* Wo = opr.w4 + i;
#pragma unroll
                    for (int g = 0; g < kOpRecW4; ++g) {
                        const float4 v4 = make_float4(wgt[g][0], wgt[g][1], wgt[g][2], wgt[g][3]);
                        Wo[(size_t)g * N] = v4;
                        R4[3 + g] = v4;
                    }
                    float fm[9], S[18];
                    force_particle(P, N, i, opr, fm, S, err);
                    R4[0] = make_float4(fm[0], fm[1], fm[2], fm[3]);
                    R4[1] = make_float4(fm[4], fm[5], fm[6], fm[7]);
                    R4[2] = make_float4(fm[8], __int_as_float(cl), 0.f, 0.f);
#pragma unroll
                    for (int g = 0; g < 4; ++g) R4[9 + g] = make_float4(S[4 * g], S[4 * g + 1], S[4 * g + 2], S[4 * g + 3]);
                    R4[13] = make_float4(S[16], S[17], 0.f, 0.f);
                } else {
                    opr.base[i] = -1;
                    atomicOr(err, ERR_STENCIL_OOB);
                }
            }
            __syncwarp();
            const int prev = __shfl_up_sync(0xffffffffu, cl, 1);
            const unsigned heads = __ballot_sync(0xffffffffu, cl >= 0 && (lane == 0 || prev != cl));
            const unsigned breaks = heads | __ballot_sync(0xffffffffu, cl < 0);
            const int nrun = __popc(heads);
            for (int item = lane; item < 16 * nrun; item += 32) {
                const int run = item >> 4, kz = (item >> 2) & 3, jy = item & 3;
                const int sl = __fns(heads, 0, run + 1);
                const unsigned after = sl >= 31 ? 0u : breaks & (0xffffffffu << (sl + 1));
                const int el = after ? __ffs(after) - 1 : 32;
                float2 a01[3] = {f2(0.f, 0.f), f2(0.f, 0.f), f2(0.f, 0.f)}, a23[3] = {f2(0.f, 0.f), f2(0.f, 0.f), f2(0.f, 0.f)};
                float dg[4][3];
#pragma unroll
                for (int q = 0; q < 4; ++q) dg[q][0] = dg[q][1] = dg[q][2] = 0.f;
                for (int p = sl; p < el; ++p) {
                    const float* Rp = Rw + p * kForceRec;
                    const float4 f0 = *reinterpret_cast<const float4*>(Rp), f1 = *reinterpret_cast<const float4*>(Rp + 4);
                    const float f8 = Rp[8];
                    const float4 gx = *reinterpret_cast<const float4*>(Rp + 12), gdx = *reinterpret_cast<const float4*>(Rp + 16);
                    const float wyj = Rp[20 + jy], dwyj = Rp[24 + jy], wzk = Rp[28 + kz], dwzk = Rp[32 + kz];
                    // the row's three weight products, formed once for the three components
                    const float wzy = wzk * wyj, wzdy = wzk * dwyj, dzwy = dwzk * wyj;
                    const float fmv[9] = {f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, f1.z, f1.w, f8};
                    const float2 wx01 = f2(gx.x, gx.y), wx23 = f2(gx.z, gx.w);
                    const float2 dwx01 = f2(gdx.x, gdx.y), dwx23 = f2(gdx.z, gdx.w);
#pragma unroll
                    for (int cc = 0; cc < 3; ++cc) {
                        const float U = fmv[3 * cc] * wzy;
                        const float V = fmv[3 * cc + 1] * wzdy + fmv[3 * cc + 2] * dzwy;
                        const float2 U2 = f2(U, U), V2 = f2(V, V);
                        a01[cc] = __ffma2_rn(U2, dwx01, __ffma2_rn(V2, wx01, a01[cc]));
                        a23[cc] = __ffma2_rn(U2, dwx23, __ffma2_rn(V2, wx23, a23[cc]));
                    }
                    // diag_ax -= S0 g0^2 + S1 g1^2 + S2 g2^2 + S3 g0 g1 + S4 g0 g2 + S5 g1 g2 with
                    // g = -(dwx wy wz, wx dwy wz, wx wy dwz), grouped by the x factors dwx^2, wx^2 and dwx wx
                    const float wy2 = wyj * wyj, dwy2 = dwyj * dwyj, wydwy = wyj * dwyj;
                    const float wz2 = wzk * wzk, dwz2 = dwzk * dwzk, wzdwz = wzk * dwzk;
                    const float yz0 = wy2 * wz2, yz1 = dwy2 * wz2, yz2 = wy2 * dwz2, yz3 = wydwy * wz2, yz4 = wy2 * wzdwz,
                                yz5 = wydwy * wzdwz;
                    const float wxs[4] = {gx.x, gx.y, gx.z, gx.w}, dwxs[4] = {gdx.x, gdx.y, gdx.z, gdx.w};
#pragma unroll
                    for (int ax = 0; ax < 3; ++ax) {
                        const float* S = Rp + 36 + 6 * ax;
                        const float A = S[0] * yz0;
                        const float B = S[1] * yz1 + S[2] * yz2 + S[5] * yz5;
                        const float Cc = S[3] * yz3 + S[4] * yz4;
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                            dg[q][ax] -= A * (dwxs[q] * dwxs[q]) + B * (wxs[q] * wxs[q]) + Cc * (dwxs[q] * wxs[q]);
                    }
                }
                const int cell = __float_as_int(Rw[sl * kForceRec + 9]);
                const int cx = cell & 3, cy = (cell >> 2) & 3, cz = cell >> 4;
                const int w = 3 * (cx + kWin * ((cy + jy) + kWin * (cz + kz)));
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) {
                    atomicAdd(&acc[w + cc], a01[cc].x);
                    atomicAdd(&acc[w + 3 + cc], a01[cc].y);
                    atomicAdd(&acc[w + 6 + cc], a23[cc].x);
                    atomicAdd(&acc[w + 9 + cc], a23[cc].y);
                }
#pragma unroll
                for (int q = 0; q < 4; ++q)
#pragma unroll
                    for (int ax = 0; ax < 3; ++ax) atomicAdd(&dacc[w + 3 * q + ax], dg[q][ax]);
            }
            if (MASS) {
                // node mass and momentum sum_p w (m_p, m_p (v_p - v_frame)) over the same runs, rows and layers
                for (int item = lane; item < 16 * nrun; item += 32) {
                    const int run = item >> 4, kz = (item >> 2) & 3, jy = item & 3;
                    const int sl = __fns(heads, 0, run + 1);
                    const unsigned after = sl >= 31 ? 0u : breaks & (0xffffffffu << (sl + 1));
                    const int el = after ? __ffs(after) - 1 : 32;
                    float a[4][4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) a[q][0] = a[q][1] = a[q][2] = a[q][3] = 0.f;
                    for (int p = sl; p < el; ++p) {
                        const float* Rp = Rw + p * kForceRec;
                        const float4 m4 = *reinterpret_cast<const float4*>(Rp + 56);
                        const float4 wx4 = *reinterpret_cast<const float4*>(Rp + 12);
                        const float wjk = Rp[20 + jy] * Rp[28 + kz];
                        const float wq[4] = {wx4.x * wjk, wx4.y * wjk, wx4.z * wjk, wx4.w * wjk};
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            a[q][0] += wq[q] * m4.x; a[q][1] += wq[q] * m4.y; a[q][2] += wq[q] * m4.z;
                            a[q][3] += wq[q] * m4.w;
                        }
                    }
                    const int cell = __float_as_int(Rw[sl * kForceRec + 9]);
                    const int cx = cell & 3, cy = (cell >> 2) & 3, cz = cell >> 4;
                    float* dst = &macc[4 * (cx + kWin * ((cy + jy) + kWin * (cz + kz)))];
#pragma unroll
                    for (int q = 0; q < 4; ++q)
#pragma unroll
                        for (int ch = 0; ch < 4; ++ch) atomicAdd(&dst[4 * q + ch], a[q][ch]);
                }
            }
            __syncwarp();
        }
        __syncthreads();
        flush_window<3, 3, 0>(c, acc, frc);
        if (diagOut) flush_window<3, 3, 0>(c, dacc, diagOut);
        if (MASS) {
            flush_window<1, 4, 0>(c, macc, massOut);
            flush_window<3, 4, 1>(c, macc, momOut);
        }
        __syncthreads();
    }
    tiles_done(T);
}

// The apply pass runs one wave of persistent CTAs (SMs x resident CTAs per SM), each striding over the tile list.
static int op_apply_grid(int maxTiles) {
    static int sms[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    int n = dev >= 0 && dev < 64 ? sms[dev] : 0;
    if (n == 0) {
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        if (dev >= 0 && dev < 64) sms[dev] = n;
    }
    const int g = n * kApplyMinBlocks;
    return std::max(1, std::min(maxTiles, g));
}
void launch_op(const PartArrays& P, int N, const TileArrays& T, int maxTiles, const BodyGrid* grids, float h, const float* in,
               float* out, OpRec rec, const BodySolve* solve, bool skipDone, cudaStream_t s, unsigned long long* procCount) {
    ++g_kernel_launches;
    k_op_apply<<<op_apply_grid(maxTiles), kApplyThreads, 0, s>>>(T, grids, in, out, rec, N, solve, skipDone ? 1 : 0,
                                                                 procCount);
}

// The tiles whose 7 x 7 x 7-node window holds a collided node (nodeCollided >= 0, where the collision velocity
// vc can be non-zero): the only tiles whose particles see a non-zero vc, so DF(vc) for the rhs runs over them
// alone.  One warp per listed tile.
__global__ void k_contact_tiles(TileArrays T, const BodyGrid* grids, const signed char* __restrict__ flag, int* list,
                                int* listBody, int* listCount) {
    const int li = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (li >= read_list_count(T)) return;
    const TileCtx c = tile_ctx(T, grids, li);
    bool hit = false;
    for (int w = lane; w < kWin3 && !hit; w += 32) {
        const long long node = win_node(c, w);
        hit = node >= 0 && flag[node] >= 0;
    }
    if (__any_sync(0xffffffffu, hit) && lane == 0) {
        const int k = atomicAdd(listCount, 1);
        list[k] = T.list[li];
        listBody[k] = T.listBody[li];
    }
}
void launch_contact_tiles(const TileArrays& T, int maxTiles, const BodyGrid* grids, const signed char* flag, TileArrays C,
                          cudaStream_t s) {
    cudaMemsetAsync(C.listCount, 0, sizeof(int), s);
    ++g_kernel_launches;
    k_contact_tiles<<<(unsigned)((maxTiles + 7) / 8), 256, 0, s>>>(T, grids, flag, C.list, C.listBody, C.listCount);
}
// P2G of mass and momentum in one pass — MassSplatter and VelocitySplatter (Grid.cpp:62-150): m_i = sum_p w_ip m_p
// and the momentum sum_p w_ip m_p (v_p - v_frame); k_node_vel divides the latter by m_i, which is the
// reference's sum_p w_ip (m_p / m_i)(v_p - v_frame) up to summation order.  Warp-autonomous like the operator
// pass: each warp takes a quarter of the tile's particles in rounds of 32; lane = particle stages m,
// m (v - v_frame) and its 12 weights; lane = (run of one cell, stencil z-layer, y-row) sums 4 nodes x 4 channels
// over the run and adds them to the CTA's window accumulator once per run.
constexpr int kP2GWarps = 4;
constexpr int kP2GWRec = 20;  // m4 | wx | wy | wz | cell
__global__ void __launch_bounds__(32 * kP2GWarps, 6) k_p2g_warp(PartArrays P, int N, TileArrays T, const BodyGrid* grids,
                                                                 float h, NodeArrays nd, int* err) {
    __shared__ float acc[4 * kWin3];
    __shared__ __align__(16) float rec[kP2GWarps][32 * kP2GWRec];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float* R = &rec[warp][lane * kP2GWRec];
    const float* Rw = rec[warp];
    __shared__ int sTile;
    const int nl = read_list_count(T);
    for (int li = next_tile(T, &sTile); li < nl; li = next_tile(T, &sTile)) {
        TileCtx c = tile_ctx(T, grids, li);
        for (int e = threadIdx.x; e < 4 * kWin3; e += blockDim.x) acc[e] = 0.f;
        __syncthreads();
        const int np = c.pe - c.ps;
        const int wb = c.ps + (int)(((long long)np * warp) / kP2GWarps);
        const int we = c.ps + (int)(((long long)np * (warp + 1)) / kP2GWarps);
        for (int r0 = wb; r0 < we; r0 += 32) {
            const int i = r0 + lane;
            int cl = -1;
            if (i < we) {
                float x[3], frac[3], v[3];
                int cell[3];
                ld3(P.x, N, i, x);
                stencil_cells(x, c.g.mn, c.g.n, h, cell, frac);
                const int lx = cell[0] - 1 - c.wo[0], ly = cell[1] - 1 - c.wo[1], lz = cell[2] - 1 - c.wo[2];
                if (lx < 0 || ly < 0 || lz < 0 || lx > kWin - 4 || ly > kWin - 4 || lz > kWin - 4) {
                    atomicOr(err, ERR_STENCIL_OOB);
                } else {
                    cl = lx + kTile * (ly + kTile * lz);
                    ld3(P.v, N, i, v);
                    const float m = P.m[i];
                    float4* R4 = reinterpret_cast<float4*>(R);
                    R4[0] = make_float4(m, m * (v[0] - c.g.fv[0]), m * (v[1] - c.g.fv[1]), m * (v[2] - c.g.fv[2]));
                    float wxs[4], wys[4], wzs[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        wxs[q] = stencil_w(c.g.n[0] == 1, q, frac[0]);
                        wys[q] = stencil_w(c.g.n[1] == 1, q, frac[1]);
                        wzs[q] = stencil_w(c.g.n[2] == 1, q, frac[2]);
                    }
                    R4[1] = make_float4(wxs[0], wxs[1], wxs[2], wxs[3]);
                    R4[2] = make_float4(wys[0], wys[1], wys[2], wys[3]);
                    R4[3] = make_float4(wzs[0], wzs[1], wzs[2], wzs[3]);
                    R[16] = __int_as_float(cl);
                }
            }
            __syncwarp();
            const int prev = __shfl_up_sync(0xffffffffu, cl, 1);
            const unsigned heads = __ballot_sync(0xffffffffu, cl >= 0 && (lane == 0 || prev != cl));
            const unsigned breaks = heads | __ballot_sync(0xffffffffu, cl < 0);
            const int nrun = __popc(heads);
            for (int item = lane; item < 16 * nrun; item += 32) {
                const int run = item >> 4, kz = (item >> 2) & 3, jy = item & 3;
                const int sl = __fns(heads, 0, run + 1);
                const unsigned after = sl >= 31 ? 0u : breaks & (0xffffffffu << (sl + 1));
                const int el = after ? __ffs(after) - 1 : 32;
                float a[4][4];
#pragma unroll
                for (int q = 0; q < 4; ++q) a[q][0] = a[q][1] = a[q][2] = a[q][3] = 0.f;
                for (int p = sl; p < el; ++p) {
                    const float* Rp = Rw + p * kP2GWRec;
                    const float4 m4 = *reinterpret_cast<const float4*>(Rp), wx4 = *reinterpret_cast<const float4*>(Rp + 4);
                    const float wjk = Rp[8 + jy] * Rp[12 + kz];
                    const float wq[4] = {wx4.x * wjk, wx4.y * wjk, wx4.z * wjk, wx4.w * wjk};
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        a[q][0] += wq[q] * m4.x; a[q][1] += wq[q] * m4.y; a[q][2] += wq[q] * m4.z; a[q][3] += wq[q] * m4.w;
                    }
                }
                const int cell = __float_as_int(Rw[sl * kP2GWRec + 16]);
                const int cx = cell & 3, cy = (cell >> 2) & 3, cz = cell >> 4;
                float* dst = &acc[4 * (cx + kWin * ((cy + jy) + kWin * (cz + kz)))];
#pragma unroll
                for (int q = 0; q < 4; ++q)
#pragma unroll
                    for (int ch = 0; ch < 4; ++ch) atomicAdd(&dst[4 * q + ch], a[q][ch]);
            }
            __syncwarp();
        }
        __syncthreads();
        flush_window<1, 4, 0>(c, acc, nd.mass);
        flush_window<3, 4, 1>(c, acc, nd.vel);
        __syncthreads();
    }
    tiles_done(T);
}

void launch_p2g_mass_momentum(const PartArrays& P, int N, const TileArrays& T, int maxTiles, const BodyGrid* grids, float h,
                              NodeArrays nd, int* err, cudaStream_t s) {
    ++g_kernel_launches;
    k_p2g_warp<<<std::max(1, std::min(maxTiles, 148 * 6)), 32 * kP2GWarps, 0, s>>>(P, N, T, grids, h, nd, err);
}
void launch_p2g_force(const PartArrays& P, int N, const TileArrays& T, int maxTiles, const BodyGrid* grids, float h,
                      NodeArrays nd, float* diagOut, OpRec rec, bool withMass, int* err, cudaStream_t s) {
    ++g_kernel_launches;
    const int grid = std::max(1, std::min(maxTiles, 148 * 4));
    if (withMass)
        k_force_warp<true><<<grid, kApplyThreads, 0, s>>>(P, N, T, grids, h, nd.frc, diagOut, nd.mass, nd.vel, rec, err);
    else
        k_force_warp<false><<<grid, kApplyThreads, 0, s>>>(P, N, T, grids, h, nd.frc, diagOut, nullptr, nullptr, rec, err);
}
void launch_g2p(const PartArrays& P, int N, const TileArrays& T, int maxTiles, const BodyGrid* grids, float h, float dt,
                NodeArrays nd, cudaStream_t s) {
    ++g_kernel_launches; k_g2p<<<tile_grid(maxTiles), kTileThreads, 0, s>>>(P, N, T, grids, h, dt, nd);
}

// =========================================================================================================
// node kernels
// =========================================================================================================
#define NODE_LOOP(c)                                                     \
    for (int qq = 0; qq < kNodeChunk / kNodeThreads; ++qq)                \
        for (long long l = (c).l0 + threadIdx.x + (long long)qq * kNodeThreads, node = (c).g.nodeOff + l, once = 1; \
             once; once = 0)

// masses: clamp negatives, NaN check (Grid.cpp:226-241)
__global__ void k_node_mass(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int* err) {
    NodeCtx c = node_ctx(grids, chunkBody);
    NODE_LOOP(c) {
        if (l >= c.G) continue;
        float m = nd.mass[node];
        if (m < 0.f) { m = 0.f; nd.mass[node] = 0.f; }
        if (!isfinite(m)) atomicOr(err, ERR_NAN_MASSES);
    }
}
void launch_node_mass(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, int* err, cudaStream_t s) {
    if (nChunks > 0) { ++g_kernel_launches; k_node_mass<<<nChunks, kNodeThreads, 0, s>>>(nd, grids, chunkBody, err); }
}

// velocities: momentum / mass (see k_p2g_warp), NaN check (Grid.cpp:250-260), prev = v (:262), field forces
// at the nodes (:446-458) added to the internal forces that the force pass summed before it
__global__ void k_node_vel(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, StepParams sp, int* err) {
    NodeCtx c = node_ctx(grids, chunkBody);
    NODE_LOOP(c) {
        if (l >= c.G) continue;
        float v[3];
        ldn(nd.vel, node, v);  // the splatted momentum
        float m = nd.mass[node];
        for (int a = 0; a < 3; ++a) v[a] = m > 0.f ? v[a] / m : 0.f;
        stn(nd.vel, node, v);
        if (!isfinite(v[0]) || !isfinite(v[1]) || !isfinite(v[2])) atomicOr(err, ERR_NAN_VELOCITIES);
        stn(nd.prev, node, v);
        float f[3] = {0.f, 0.f, 0.f}, fi[3];
        for (int k = 0; k < sp.nfields; ++k)
            for (int a = 0; a < 3; ++a) f[a] = __fadd_rn(f[a], __fmul_rn(sp.gravity[k][a], m));
        ldn(nd.frc, node, fi);  // the internal forces, summed by the force pass
        for (int a = 0; a < 3; ++a) f[a] = __fadd_rn(f[a], fi[a]);
        stn(nd.frc, node, f);
    }
}
void launch_node_vel(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp, int* err,
                     cudaStream_t s) {
    if (nChunks > 0) { ++g_kernel_launches; k_node_vel<<<nChunks, kNodeThreads, 0, s>>>(nd, grids, chunkBody, sp, err); }
}

// calculateExplicitMomenta (Grid.cpp:634-690) + collisionVelocities (:692-724) + the uniform initial guess
// (:911-947)
__global__ void k_node_explicit(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, StepParams sp, BodySolve* solve,
                                ReduceArrays R, int* err) {
    NodeCtx c = node_ctx(grids, chunkBody);
    double part[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    NODE_LOOP(c) {
        if (l >= c.G) continue;
        float m = nd.mass[node];
        float f[3], ev[3], x[3];
        ldn(nd.frc, node, f);
        ldn(nd.vel, node, ev);
        if (m > 0.f)
            for (int a = 0; a < 3; ++a) ev[a] = __fadd_rn(ev[a], __fdiv_rn(__fmul_rn(sp.dt, f[a]), m));
        node_pos(c, l, sp.h, x);
        int flag = collide(sp.coll, sp.ncoll, ev, x, c.g.fv, false);
        float ps[3] = {__fmul_rn(ev[0], m), __fmul_rn(ev[1], m), __fmul_rn(ev[2], m)};
        if (!isfinite(ps[0] * ps[1] * ps[2])) atomicOr(err, ERR_NAN_MOMENTA);
        stn(nd.pstar, node, ps);
        nd.flag[node] = (signed char)flag;
        float vc[3] = {0.f, 0.f, 0.f};
        if (flag >= 0) {  // collisionVelocities, Grid.cpp:692-724: the object's velocity at the node
            coll_velocity(sp.coll[flag], x, vc);
            for (int a = 0; a < 3; ++a) vc[a] = __fsub_rn(vc[a], c.g.fv[a]);
        }
        stn(nd.vc, node, vc);
        part[0] += m;
        part[1] += ps[0]; part[2] += ps[1]; part[3] += ps[2];
        if (flag >= 0) {
            part[4] += m;
            part[5] += (double)m * vc[0]; part[6] += (double)m * vc[1]; part[7] += (double)m * vc[2];
        }
    }
    double tot[8];
    if (segmented_reduce<8>(part, R, c.b, c.g.ctaBegin, c.g.ctaEnd, tot) && threadIdx.x == 0) {
        BodySolve& S = solve[c.b];
        for (int k = 0; k < 8; ++k) S.guess[k] = tot[k];
        float g[3];
        if (tot[0] == 0.0) g[0] = g[1] = g[2] = 0.f;
        else if (tot[4] == 0.0) for (int a = 0; a < 3; ++a) g[a] = (float)(tot[1 + a] / tot[0]);
        else for (int a = 0; a < 3; ++a) g[a] = (float)(tot[5 + a] / tot[4]);
        S.x0[0] = g[0]; S.x0[1] = g[1]; S.x0[2] = g[2];
        S.done = 0; S.iterations = 0; S.exitReason = 0; S.bzero = 0;
        S.rNorm2 = 0; S.rz = 0; S.ApdPAp = 0; S.alpha = 0; S.beta = 0;
    }
}
void launch_node_explicit(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp,
                          BodySolve* solve, ReduceArrays R, int* err, cudaStream_t s) {
    if (nChunks > 0) { ++g_kernel_launches; k_node_explicit<<<nChunks, kNodeThreads, 0, s>>>(nd, grids, chunkBody, sp, solve, R, err); }
}

// rhs b = p* + dt^2 P DF(vc) (Grid.cpp:983-1002), the Jacobi diagonal (DiagonalPreconditioner, :841-867),
// x = uniform guess, the operator input P x for A x, and |b|^2 (ConjugateResiduals.cpp:32-39)
__global__ void k_node_rhs(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, StepParams sp, BodySolve* solve,
                           ReduceArrays R, int* err, int* ndone) {
    NodeCtx c = node_ctx(grids, chunkBody);
    const float dt2 = sp.dt * sp.dt;
    const float mdt2 = -sp.dt * sp.dt;
    const float* g0 = solve[c.b].x0;
    const float gx[3] = {g0[0], g0[1], g0[2]};
    double part[1] = {0};
    NODE_LOOP(c) {
        if (l >= c.G) continue;
        float x[3], df[3], ps[3], dg[3];
        node_pos(c, l, sp.h, x);
        int flag = nd.flag[node];
        ldn(nd.df, node, df);
        project_node(sp.coll, flag, x, df);
        ldn(nd.pstar, node, ps);
        float b[3] = {ps[0] + dt2 * df[0], ps[1] + dt2 * df[1], ps[2] + dt2 * df[2]};
        if (!isfinite(b[0] * b[1] * b[2])) atomicOr(err, ERR_NAN_MOMENTA);
        stn(nd.b, node, b);
        part[0] += (double)b[0] * b[0] + (double)b[1] * b[1] + (double)b[2] * b[2];
        float m = nd.mass[node];
        ldn(nd.diag, node, dg);
        for (int a = 0; a < 3; ++a) {
            float d = dg[a] * mdt2 + m;
            dg[a] = d == 0.f ? 1.f : d;
        }
        stn(nd.diag, node, dg);
        stn(nd.x, node, gx);
        stn(nd.x0, node, gx);
        float px[3] = {gx[0], gx[1], gx[2]};
        project_node(sp.coll, flag, x, px);
        stn(nd.dxp, node, px);
        const float z[3] = {0.f, 0.f, 0.f};
        stn(nd.df, node, z);
    }
    double tot[1];
    if (segmented_reduce<1>(part, R, c.b, c.g.ctaBegin, c.g.ctaEnd, tot) && threadIdx.x == 0) {
        BodySolve& S = solve[c.b];
        S.bNorm2 = tot[0];
        S.threshold = (double)sp.tol * (double)sp.tol * tot[0];
        if (tot[0] == 0.0) {
            S.bzero = 1; S.done = 1; S.exitReason = 1; S.iterations = 0;
            atomicAdd(ndone, 1);
        }
    }
}
void launch_node_rhs(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp,
                     BodySolve* solve, ReduceArrays R, int* err, cudaStream_t s) {
    if (nChunks > 0) { ++g_kernel_launches; k_node_rhs<<<nChunks, kNodeThreads, 0, s>>>(nd, grids, chunkBody, sp, solve, R, err, R.ndone); }
}

// A x = P(m P x - dt^2 DF(P x)) given dxp = P x and df = DF(P x) — multVector, Grid.cpp:749-771
__device__ __forceinline__ void apply_combine(const NodeCtx& c, const NodeArrays& nd, const StepParams& sp, long long l,
                                              long long node, int flag, float out[3]) {
    float x[3], d[3], f[3];
    ldn(nd.dxp, node, d);
    ldn(nd.df, node, f);
    const float m = nd.mass[node], dt2 = sp.dt * sp.dt;
    for (int a = 0; a < 3; ++a) out[a] = m * d[a] - dt2 * f[a];
    if (flag != -1) {
        node_pos(c, l, sp.h, x);
        project_node(sp.coll, flag, x, out);
    }
}

// CR start (ConjugateResiduals.cpp:50-67): r = b - A x, r_pc = r / diag, p = r_pc, operator input P p
__global__ void k_node_cr_init1(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, StepParams sp,
                                const BodySolve* solve) {
    NodeCtx c = node_ctx(grids, chunkBody);
    if (solve[c.b].done) return;
    NODE_LOOP(c) {
        if (l >= c.G) continue;
        int flag = nd.flag[node];
        float Ax[3], b[3], dg[3], r[3], x[3];
        apply_combine(c, nd, sp, l, node, flag, Ax);
        ldn(nd.b, node, b);
        ldn(nd.diag, node, dg);
        for (int a = 0; a < 3; ++a) r[a] = (b[a] - Ax[a]) / dg[a];
        stn(nd.rpc, node, r);
        stn(nd.p, node, r);
        if (flag != -1) { node_pos(c, l, sp.h, x); project_node(sp.coll, flag, x, r); }
        stn(nd.dxp, node, r);
        const float z[3] = {0.f, 0.f, 0.f};
        stn(nd.df, node, z);
    }
}
void launch_node_cr_init1(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp,
                          BodySolve* solve, cudaStream_t s) {
    if (nChunks > 0) { ++g_kernel_launches; k_node_cr_init1<<<nChunks, kNodeThreads, 0, s>>>(nd, grids, chunkBody, sp, solve); }
}

// CR start (ConjugateResiduals.cpp:69-76): Ap = A p, Ar = Ap (p == r_pc), rz = <r_pc, Ar>; then the loop's
// first <Ap, M^-1 Ap> (:86-102)
__global__ void k_node_cr_init2(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, StepParams sp, BodySolve* solve,
                                ReduceArrays R) {
    NodeCtx c = node_ctx(grids, chunkBody);
    if (solve[c.b].done) return;
    double part[2] = {0, 0};
    NODE_LOOP(c) {
        if (l >= c.G) continue;
        int flag = nd.flag[node];
        float Ap[3], r[3], dg[3];
        apply_combine(c, nd, sp, l, node, flag, Ap);
        stn(nd.Ap, node, Ap);
        stn(nd.Ar, node, Ap);
        ldn(nd.rpc, node, r);
        ldn(nd.diag, node, dg);
        for (int a = 0; a < 3; ++a) {
            part[0] += (double)r[a] * Ap[a];
            part[1] += (double)Ap[a] * (Ap[a] / dg[a]);
        }
    }
    double tot[2];
    if (segmented_reduce<2>(part, R, c.b, c.g.ctaBegin, c.g.ctaEnd, tot) && threadIdx.x == 0) {
        BodySolve& S = solve[c.b];
        S.rz = tot[0];
        S.ApdPAp = tot[1];
        if (tot[1] == 0.0) {
            S.done = 1; S.exitReason = 2; S.iterations = 0;
            atomicAdd(R.ndone, 1);
        } else {
            S.alpha = tot[0] / tot[1];
        }
    }
}
void launch_node_cr_init2(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp,
                          BodySolve* solve, ReduceArrays R, cudaStream_t s) {
    if (nChunks > 0) { ++g_kernel_launches; k_node_cr_init2<<<nChunks, kNodeThreads, 0, s>>>(nd, grids, chunkBody, sp, solve, R); }
}

// CR iteration part 1 (ConjugateResiduals.cpp:104-128): x += alpha p, project x; r_pc -= alpha M^-1 Ap;
// r = M r_pc; termination (SquareMagnitudeTermination.cpp:13-28); operator input P r_pc
__global__ void k_node_cr_update(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, StepParams sp, BodySolve* solve,
                                 ReduceArrays R, int iter) {
    NodeCtx c = node_ctx(grids, chunkBody);
    if (solve[c.b].done) return;
    const float alpha = (float)solve[c.b].alpha;
    double part[1] = {0};
    NODE_LOOP(c) {
        if (l >= c.G) continue;
        int flag = nd.flag[node];
        float xp[3], x[3], p[3], Ap[3], dg[3], r[3];
        if (nd.mass[node] == 0.f) {
            // a node without mass: every particle's weight and weight gradient vanish there, so k_node_cr_init1/2
            // left r = p = Ap = Ar = 0, P r = 0, DF = 0, and no iteration changes them; x += alpha p leaves x
            // alone but for the collider projection, which the first iteration applies
            if (iter == 0 && flag != -1) {
                ldn(nd.x, node, x);
                node_pos(c, l, sp.h, xp);
                project_node(sp.coll, flag, xp, x);
                stn(nd.x, node, x);
            }
            continue;
        }
        ldn(nd.x, node, x);
        ldn(nd.p, node, p);
        for (int a = 0; a < 3; ++a) x[a] = x[a] + alpha * p[a];
        if (flag != -1) { node_pos(c, l, sp.h, xp); project_node(sp.coll, flag, xp, x); }
        stn(nd.x, node, x);
        ldn(nd.Ap, node, Ap);
        ldn(nd.diag, node, dg);
        ldn(nd.rpc, node, r);
        for (int a = 0; a < 3; ++a) {
            r[a] = r[a] - alpha * (Ap[a] / dg[a]);
            float rr = r[a] * dg[a];
            part[0] += (double)rr * rr;
        }
        stn(nd.rpc, node, r);
        if (flag != -1) project_node(sp.coll, flag, xp, r);
        stn(nd.dxp, node, r);
        const float z[3] = {0.f, 0.f, 0.f};
        stn(nd.df, node, z);
    }
    double tot[1];
    if (segmented_reduce<1>(part, R, c.b, c.g.ctaBegin, c.g.ctaEnd, tot) && threadIdx.x == 0) {
        BodySolve& S = solve[c.b];
        S.iterations = iter;
        bool stop = iter >= sp.maxIters;
        if (!stop) {
            S.rNorm2 = tot[0];
            stop = tot[0] < S.threshold;
        }
        if (stop) { S.done = 1; S.exitReason = 0; atomicAdd(R.ndone, 1); }
    }
}
void launch_node_cr_update(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp,
                           BodySolve* solve, ReduceArrays R, int iter, cudaStream_t s) {
    if (nChunks > 0) { ++g_kernel_launches; k_node_cr_update<<<nChunks, kNodeThreads, 0, s>>>(nd, grids, chunkBody, sp, solve, R, iter); }
}

// CR iteration part 2 (ConjugateResiduals.cpp:130-145): Ar = A r_pc, rz = <r_pc, Ar>, beta
__global__ void k_node_cr_ar(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, StepParams sp, BodySolve* solve,
                             ReduceArrays R, int iter) {
    NodeCtx c = node_ctx(grids, chunkBody);
    if (solve[c.b].done) return;
    double part[1] = {0};
    NODE_LOOP(c) {
        if (l >= c.G) continue;
        if (nd.mass[node] == 0.f) continue;  // Ar = 0 and r = 0 there (k_node_cr_update)
        int flag = nd.flag[node];
        float Ar[3], r[3];
        apply_combine(c, nd, sp, l, node, flag, Ar);
        stn(nd.Ar, node, Ar);
        ldn(nd.rpc, node, r);
        part[0] += (double)r[0] * Ar[0] + (double)r[1] * Ar[1] + (double)r[2] * Ar[2];
    }
    double tot[1];
    if (segmented_reduce<1>(part, R, c.b, c.g.ctaBegin, c.g.ctaEnd, tot) && threadIdx.x == 0) {
        BodySolve& S = solve[c.b];
        double rzOld = S.rz;
        S.rz = tot[0];
        if (rzOld == 0.0) { S.done = 1; S.exitReason = 3; atomicAdd(R.ndone, 1); }
        else S.beta = tot[0] / rzOld;
    }
}
void launch_node_cr_ar(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp,
                       BodySolve* solve, ReduceArrays R, int iter, cudaStream_t s) {
    if (nChunks > 0) { ++g_kernel_launches; k_node_cr_ar<<<nChunks, kNodeThreads, 0, s>>>(nd, grids, chunkBody, sp, solve, R, iter); }
}

// CR iteration part 3 (ConjugateResiduals.cpp:147-151, then :86-102 of the next iteration):
// p = r_pc + beta p, Ap = Ar + beta Ap, <Ap, M^-1 Ap>, alpha
__global__ void k_node_cr_p(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, StepParams sp, BodySolve* solve,
                            ReduceArrays R, int iter) {
    NodeCtx c = node_ctx(grids, chunkBody);
    if (solve[c.b].done) return;
    const float beta = (float)solve[c.b].beta;
    double part[1] = {0};
    NODE_LOOP(c) {
        if (l >= c.G) continue;
        if (nd.mass[node] == 0.f) continue;  // p = r + beta p and Ap = Ar + beta Ap stay 0 there (k_node_cr_update)
        float p[3], r[3], Ap[3], Ar[3], dg[3];
        ldn(nd.p, node, p);
        ldn(nd.rpc, node, r);
        ldn(nd.Ap, node, Ap);
        ldn(nd.Ar, node, Ar);
        ldn(nd.diag, node, dg);
        for (int a = 0; a < 3; ++a) {
            p[a] = r[a] + beta * p[a];
            Ap[a] = Ar[a] + beta * Ap[a];
            part[0] += (double)Ap[a] * (Ap[a] / dg[a]);
        }
        stn(nd.p, node, p);
        stn(nd.Ap, node, Ap);
    }
    double tot[1];
    if (segmented_reduce<1>(part, R, c.b, c.g.ctaBegin, c.g.ctaEnd, tot) && threadIdx.x == 0) {
        BodySolve& S = solve[c.b];
        S.ApdPAp = tot[0];
        if (tot[0] == 0.0) { S.done = 1; S.exitReason = 2; S.iterations = iter + 1; atomicAdd(R.ndone, 1); }
        else S.alpha = S.rz / tot[0];
    }
}
void launch_node_cr_p(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp,
                      BodySolve* solve, ReduceArrays R, int iter, cudaStream_t s) {
    if (nChunks > 0) { ++g_kernel_launches; k_node_cr_p<<<nChunks, kNodeThreads, 0, s>>>(nd, grids, chunkBody, sp, solve, R, iter); }
}

// v = x + vc (Grid.cpp:1014); x = 0 when |b| = 0 (ConjugateResiduals.cpp:34-38)
__global__ void k_node_final(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, const BodySolve* solve) {
    NodeCtx c = node_ctx(grids, chunkBody);
    const int bz = solve[c.b].bzero;
    NODE_LOOP(c) {
        if (l >= c.G) continue;
        float x[3], vc[3];
        ldn(nd.x, node, x);
        ldn(nd.vc, node, vc);
        if (bz) { x[0] = x[1] = x[2] = 0.f; stn(nd.x, node, x); }
        float v[3] = {x[0] + vc[0], x[1] + vc[1], x[2] + vc[2]};
        stn(nd.vfin, node, v);
    }
}
void launch_node_final(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const BodySolve* solve,
                       cudaStream_t s) {
    if (nChunks > 0) { ++g_kernel_launches; k_node_final<<<nChunks, kNodeThreads, 0, s>>>(nd, grids, chunkBody, solve); }
}

// inspection helpers
__global__ void k_node_project(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, StepParams sp, const float* in,
                               float* out) {
    NodeCtx c = node_ctx(grids, chunkBody);
    NODE_LOOP(c) {
        if (l >= c.G) continue;
        float v[3], x[3];
        ldn(in, node, v);
        node_pos(c, l, sp.h, x);
        project_node(sp.coll, nd.flag[node], x, v);
        stn(out, node, v);
    }
}
void launch_node_project(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp,
                         const float* in, float* out, cudaStream_t s) {
    if (nChunks > 0) { ++g_kernel_launches; k_node_project<<<nChunks, kNodeThreads, 0, s>>>(nd, grids, chunkBody, sp, in, out); }
}
__global__ void k_node_combine(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, StepParams sp, const float* dxp,
                               const float* df, float* out) {
    NodeCtx c = node_ctx(grids, chunkBody);
    NODE_LOOP(c) {
        if (l >= c.G) continue;
        NodeArrays t = nd;
        t.dxp = const_cast<float*>(dxp);
        t.df = const_cast<float*>(df);
        float o[3];
        apply_combine(c, t, sp, l, node, nd.flag[node], o);
        stn(out, node, o);
    }
}
void launch_node_combine(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp,
                         const float* dxp, const float* df, float* out, cudaStream_t s) {
    if (nChunks > 0) { ++g_kernel_launches; k_node_combine<<<nChunks, kNodeThreads, 0, s>>>(nd, grids, chunkBody, sp, dxp, df, out); }
}

// ---------------------------------------------------------------------------------------------------------
// learned warm start (replaces the uniform guess of Grid.cpp:911-947 for one body)
// ---------------------------------------------------------------------------------------------------------
__global__ void k_ws_features(NodeArrays nd, BodyGrid g, StepParams sp, mpmnn::NnNorm nn, mpmnn::WsHist H,
                              __nv_bfloat16* out) {
    NodeCtx c;
    c.b = 0;
    c.g = g;
    c.G = (long long)g.n[0] * g.n[1] * g.n[2];
    c.l0 = 0;
    const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= c.G) return;
    const long long node = g.nodeOff + l;
    float ps[3], f[3], d[3], hv[3], nrm[3] = {0.f, 0.f, 0.f}, ft[mpmnn::kFeat];
    ldn(nd.pstar, node, ps);
    ldn(nd.frc, node, f);
    ldn(nd.diag, node, d);
    const bool hasHist = mpmnn::hist_at(H, g.n, l, hv);
    const int flag = nd.flag[node];
    if (flag >= 0) {
        float pos[3];
        node_pos(c, l, sp.h, pos);
        coll_normal(sp.coll[flag], pos, nrm);
    }
    mpmnn::node_features(nd.mass[node], ps, f, d, hasHist, hv, nrm, nn, ft);
    __align__(16) __nv_bfloat16 e[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) e[k] = __float2bfloat16(k < mpmnn::kFeat ? ft[k] : 0.f);
    uint4* o = reinterpret_cast<uint4*>(out + l * 16);
    o[0] = reinterpret_cast<const uint4*>(e)[0];
    o[1] = reinterpret_cast<const uint4*>(e)[1];
}
void launch_ws_features(NodeArrays nd, const BodyGrid& g, const StepParams& sp, const mpmnn::NnNorm& nn,
                        const mpmnn::WsHist& H, void* out_bf16, cudaStream_t s) {
    const long long G = (long long)g.n[0] * g.n[1] * g.n[2];
    if (G == 0) return;
    ++g_kernel_launches;
    k_ws_features<<<(unsigned)((G + 255) / 256), 256, 0, s>>>(nd, g, sp, nn, H, (__nv_bfloat16*)out_bf16);
}

__global__ void k_ws_apply(NodeArrays nd, BodyGrid g, StepParams sp, mpmnn::NnNorm nn, mpmnn::WsHist H, mpmnn::WsHist H2,
                           const float* __restrict__ y, int extrapolate) {
    NodeCtx c;
    c.b = 0;
    c.g = g;
    c.G = (long long)g.n[0] * g.n[1] * g.n[2];
    c.l0 = 0;
    const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= c.G) return;
    const long long node = g.nodeOff + l;
    const float m = nd.mass[node];
    float ps[3], hv[3], hv2[3], x[3], yl[3] = {0.f, 0.f, 0.f};
    ldn(nd.pstar, node, ps);
    const bool hasHist = mpmnn::hist_at(H, g.n, l, hv);
    const bool hasHist2 = extrapolate && mpmnn::hist_at(H2, g.n, l, hv2);
    if (y) { yl[0] = y[3 * l]; yl[1] = y[3 * l + 1]; yl[2] = y[3 * l + 2]; }
    mpmnn::node_guess(m, ps, y ? yl : nullptr, hasHist, hv, hasHist2, hv2, extrapolate != 0, nn, x);
    stn(nd.x, node, x);
    stn(nd.x0, node, x);
    const int flag = nd.flag[node];
    if (flag != -1) {
        float pos[3];
        node_pos(c, l, sp.h, pos);
        project_node(sp.coll, flag, pos, x);
    }
    stn(nd.dxp, node, x);
}
void launch_ws_apply(NodeArrays nd, const BodyGrid& g, const StepParams& sp, const mpmnn::NnNorm& nn, const mpmnn::WsHist& H,
                     const mpmnn::WsHist& H2, const float* y, bool extrapolate, cudaStream_t s) {
    const long long G = (long long)g.n[0] * g.n[1] * g.n[2];
    if (G == 0) return;
    ++g_kernel_launches;
    k_ws_apply<<<(unsigned)((G + 255) / 256), 256, 0, s>>>(nd, g, sp, nn, H, H2, y, extrapolate ? 1 : 0);
}


// the history the next step's warm start reads: x - p*/m on heavy nodes, x on light ones, NaN without mass
__global__ void k_ws_record(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, mpmnn::NnNorm nn, float* hist) {
    NodeCtx c = node_ctx(grids, chunkBody);
    NODE_LOOP(c) {
        if (l >= c.G) continue;
        const float m = nd.mass[node];
        float x[3], ps[3], o[3];
        ldn(nd.x, node, x);
        ldn(nd.pstar, node, ps);
        if (!(m > 0.f)) {
            o[0] = o[1] = o[2] = __int_as_float(0x7fc00000);
        } else if (m * nn.inv_mass_unit >= nn.light_mass) {
            for (int a = 0; a < 3; ++a) o[a] = x[a] - ps[a] / m;
        } else {
            for (int a = 0; a < 3; ++a) o[a] = x[a];
        }
        stn(hist, node, o);
    }
}
void launch_ws_record(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const mpmnn::NnNorm& nn,
                      float* hist, cudaStream_t s) {
    if (nChunks > 0) { ++g_kernel_launches; k_ws_record<<<nChunks, kNodeThreads, 0, s>>>(nd, grids, chunkBody, nn, hist); }
}

// =========================================================================================================
// plasticity over all particles (SnowConstitutiveModel::updateParticleData) and advection (Sim.cpp:123-131)
// =========================================================================================================
__global__ void k_plasticity(PartArrays P, int N, StepParams sp, int* fp64Count, int* err) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    float F[9], Fp[9];
    ld9(P.F, N, i, F);
    ld9(P.Fp, N, i, Fp);
    float mu0 = P.mu0 ? P.mu0[i] : sp.mu;
    float lam0 = P.lam0 ? P.lam0[i] : sp.lambda;
    PlasticOut o;
    int used64 = 0;
    snow_plasticity(F, Fp, mu0, lam0, sp.xi, sp.thetaC, sp.thetaS, o, used64);
    if (used64) atomicAdd(fp64Count, 1);
    if (o.bad) atomicOr(err, ERR_HARDNESS);
    st9(P.F, N, i, o.F);
    st9(P.Fp, N, i, o.Fp);
    st9(P.FiT, N, i, o.FiT);
    st9(P.R, N, i, o.R);
    st9(P.Gi, N, i, o.Gi);
    P.J[i] = o.J;
    P.mu[i] = o.mu;
    P.lam[i] = o.lam;
}
void launch_plasticity(const PartArrays& P, int N, const StepParams& sp, int* fp64Count, int* err, cudaStream_t s) {
    if (N > 0) { ++g_kernel_launches; k_plasticity<<<(N + 127) / 128, 128, 0, s>>>(P, N, sp, fp64Count, err); }
}

__global__ void k_advect(PartArrays P, int N, StepParams sp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    float x[3], v[3];
    ld3(P.x, N, i, x);
    ld3(P.v, N, i, v);
    const float zero[3] = {0.f, 0.f, 0.f};
    collide(sp.coll, sp.ncoll, v, x, zero, true);
    for (int a = 0; a < 3; ++a) x[a] = __fadd_rn(x[a], __fmul_rn(v[a], sp.dt));
    st3(P.x, N, i, x);
    st3(P.v, N, i, v);
}
void launch_advect(const PartArrays& P, int N, const StepParams& sp, cudaStream_t s) {
    if (N > 0) { ++g_kernel_launches; k_advect<<<(N + 255) / 256, 256, 0, s>>>(P, N, sp); }
}

// =========================================================================================================
// particle seeding from a sampled signed-distance field — the Houdini SOP's initSim (SOP_MPMSim.cpp:168-214):
// lattice site q = k + nz (j + ny i) (the reference's loop order: i slowest, k fastest) at bbox_min + (i + 0.5) h,
// evaluated as the reference does (double sum, rounded to float), becomes a particle where phi < 0
// =========================================================================================================
__device__ __forceinline__ void seed_site(long long q, const int dims[3], const double bmin[3], double h, float x[3]) {
    const long long k = q % dims[2], r = q / dims[2];
    const long long j = r % dims[1], i = r / dims[1];
    x[0] = (float)(bmin[0] + ((double)i + 0.5) * h);
    x[1] = (float)(bmin[1] + ((double)j + 0.5) * h);
    x[2] = (float)(bmin[2] + ((double)k + 0.5) * h);
}
__global__ void k_seed_flags(DevCollider sdf, SeedLattice L, int* flag) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= L.sites) return;
    float x[3];
    seed_site(q, L.dims, L.bmin, L.h, x);
    flag[q] = coll_phi(sdf, x) < 0.0f ? 1 : 0;
}
__global__ void k_seed_write(DevCollider sdf, SeedLattice L, const int* flag, const int* pos, float mass, float* xo, float* vo,
                             float* mo) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= L.sites || !flag[q]) return;
    float x[3], v[3];
    seed_site(q, L.dims, L.bmin, L.h, x);
    coll_velocity(sdf, x, v);
    const long long p = pos[q];
    for (int a = 0; a < 3; ++a) {
        xo[3 * p + a] = x[a];
        vo[3 * p + a] = v[a];
    }
    mo[p] = mass;
}
void launch_seed(const DevCollider& sdf, const SeedLattice& L, float mass, int* flag, int* pos, int* scanTmp, int* total,
                 float* x, float* v, float* m, bool write, cudaStream_t s) {
    const unsigned nb = (unsigned)((L.sites + 255) / 256);
    if (!write) {
        ++g_kernel_launches; k_seed_flags<<<nb, 256, 0, s>>>(sdf, L, flag);
        scan_exclusive(flag, pos, L.sites, scanTmp, total, s);
        return;
    }
    ++g_kernel_launches; k_seed_write<<<nb, 256, 0, s>>>(sdf, L, flag, pos, mass, x, v, m);
}

// =========================================================================================================
// body segmentation — Sim::calculateBodies (Sim.cpp:136-203): connected components of |x_i - x_j| < h
// (strict, KdTree.inl:188) by lock-free union-find over a hashed cell grid of spacing h; components of one
// particle are ballistic; bodies are numbered by their smallest caller index, the reference's scan order.
// =========================================================================================================
__device__ __forceinline__ unsigned int cell_hash(int x, int y, int z, unsigned int mask) {
    unsigned int h = (unsigned int)x * 73856093u ^ (unsigned int)y * 19349663u ^ (unsigned int)z * 83492791u;
    return h & mask;
}
// The neighbour search's cells, relative to the lower corner o of all particles' bounding box: cells of
// size = max(h (1 + 2^-10), extent / 1024), so that (x - o) / size stays below 1024 and the rounding of the
// subtraction and the division (at most 2^-12 of a cell for two particles together) cannot put two particles
// closer than h two cells apart, however large the scene or far from the origin.
struct SegFrame {
    float o[3];
    float size;
};
__device__ __forceinline__ SegFrame seg_frame(const unsigned int* bbox, float h) {
    SegFrame f;
    float ext = 0.f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        f.o[a] = ordered_to_float(bbox[a]);
        ext = fmaxf(ext, __fsub_ru(ordered_to_float(bbox[3 + a]), f.o[a]));
    }
    f.size = fmaxf(h * (1.f + 1.f / 1024.f), ext * (1.f / 1024.f) * (1.f + 1.f / 1024.f));
    return f;
}
__device__ __forceinline__ void seg_cell(const float x[3], const SegFrame& f, int c[3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) c[a] = (int)floorf(__fdiv_rn(__fsub_rn(x[a], f.o[a]), f.size));
}

// bounding box of all particles (order-preserving unsigned encoding): a grid-stride loop over one wave of CTAs,
// reduced per CTA, then one set of atomics per CTA (per-warp atomics on the same six words serialised in L2)
constexpr int kBboxThreads = 256;
__global__ void __launch_bounds__(kBboxThreads) k_seg_bbox(PartArrays P, int N, unsigned int* bbox) {
    __shared__ unsigned int sh[6][kBboxThreads / 32];
    unsigned int lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, hi[3] = {0u, 0u, 0u};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        float x[3];
        ld3(P.x, N, i, x);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const unsigned int u = float_to_ordered(x[a]);
            lo[a] = min(lo[a], u);
            hi[a] = max(hi[a], u);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            lo[a] = min(lo[a], __shfl_down_sync(0xffffffffu, lo[a], o));
            hi[a] = max(hi[a], __shfl_down_sync(0xffffffffu, hi[a], o));
        }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int a = 0; a < 3; ++a) { sh[a][warp] = lo[a]; sh[3 + a][warp] = hi[a]; }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int a = threadIdx.x;
        unsigned int r = sh[a][0];
        for (int w = 1; w < kBboxThreads / 32; ++w) r = a < 3 ? min(r, sh[a][w]) : max(r, sh[a][w]);
        if (a < 3) atomicMin(&bbox[a], r);
        else atomicMax(&bbox[a], r);
    }
}

__global__ void k_seg_bucket(PartArrays P, int N, float h, const unsigned int* bbox, unsigned int mask, int* count,
                             int* rank, int* err) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    float v[3], x[3];
    ld3(P.v, N, i, v);
    if (!isfinite(v[0] * v[1] * v[2])) atomicOr(err, ERR_NAN_PARTICLE_V);  // Sim.cpp:149-159
    ld3(P.x, N, i, x);
    int c[3];
    seg_cell(x, seg_frame(bbox, h), c);
    unsigned int b = cell_hash(c[0], c[1], c[2], mask);
    rank[i] = atomicAdd(&count[b], 1);
}
__global__ void k_seg_place(PartArrays P, int N, float h, const unsigned int* bbox, unsigned int mask, const int* start,
                            const int* rank, int* sorted, float4* xs, int* parent) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    float x[3];
    ld3(P.x, N, i, x);
    int c[3];
    seg_cell(x, seg_frame(bbox, h), c);
    unsigned int b = cell_hash(c[0], c[1], c[2], mask);
    const int q = start[b] + rank[i];
    sorted[q] = i;
    xs[q] = make_float4(x[0], x[1], x[2], 0.f);
    parent[i] = i;
}
__device__ __forceinline__ int uf_find(int* parent, int x) {
    int p = parent[x];
    while (p != x) {
        int gp = parent[p];
        if (gp != p) parent[x] = gp;  // path halving (benign race)
        x = p;
        p = parent[x];
    }
    return x;
}
// Where a segmentation records its spanning forest: the caller indices of the slots and, per hooked root, the
// pair of particles whose union hooked it (out null: nothing recorded).
struct SegRec {
    const int* orig;
    int2* out;
};
// Hooks the larger root under the smaller.  Each failed compare-and-swap means another thread hooked b first,
// which it can do at most once per root, so the loop ends; the guard turns a loop that would not end into an
// error instead of a wrong partition.  A root is hooked once, so the pair (pi, pj) that hooked it owns its slot
// in rec.out; the pairs of one segmentation are a spanning forest of its components.
__device__ __forceinline__ void uf_union(int* parent, int a, int b, int* err, const SegRec& rec, int pi, int pj) {
    for (int guard = 0; guard < 1 << 20; ++guard) {
        a = uf_find(parent, a);
        b = uf_find(parent, b);
        if (a == b) return;
        if (a > b) { int t = a; a = b; b = t; }
        int old = atomicCAS(&parent[b], b, a);
        if (old == b) {
            if (rec.out) rec.out[b] = make_int2(rec.orig[pi], rec.orig[pj]);
            return;
        }
        b = old;
    }
    atomicOr(err, ERR_SEGMENT);
}
// Connected components of |x_i - x_j| < h in three passes (the sampled-edge scheme of "Afforest", Sutton et al.
// 2018), exact for any input:
//   1. sample: each particle is joined to the first particle within h after it in its own bucket and to the
//      first within h in the +x, +y and +z neighbour buckets — in a body of snow this already links almost
//      every particle into one giant component (sampling one neighbour bucket per particle instead left too
//      many particles outside it at 2 particles per cell, for the finish pass to search in full);
//   2. the giant component's root is the most frequent root of 1024 evenly spaced particles;
//   3. finish: a particle already in the giant component is skipped; every other particle tests every
//      candidate of its 27 neighbour buckets.  An edge with an endpoint outside the giant component at that
//      endpoint's check is thus processed from it, and an edge whose endpoints are both inside joins nothing new.
// Threads walk the particles in bucket order (neighbouring threads query the same cells) and read candidate
// positions from the bucket-ordered copy xs.  Every pair closer than h lies in the same or adjacent cells (the
// cell size is h (1 + 2^-12)); hash collisions only add candidates.  A neighbour whose parent is an ancestor
// already known for i is in i's set: no union-find walk.
__device__ __forceinline__ void seg_join(int* parent, int i, int j, int& ri, int* err, const SegRec& rec) {
    const int pj = parent[j];
    if (pj == ri || pj == i) return;
    ri = uf_find(parent, ri);
    if (uf_find(parent, j) != ri) uf_union(parent, ri, j, err, rec, i, j);
}
__device__ __forceinline__ bool seg_close(const float x[3], const float4 xj, float r2) {
    const float d0 = __fsub_rn(x[0], xj.x), d1 = __fsub_rn(x[1], xj.y), d2 = __fsub_rn(x[2], xj.z);
    const float d2s = __fadd_rn(__fadd_rn(__fmul_rn(d0, d0), __fmul_rn(d1, d1)), __fmul_rn(d2, d2));
    return d2s < r2;
}
__global__ void k_seg_sample(int N, float h, const unsigned int* bbox, unsigned int mask, const int* count, const int* start,
                             const int* sorted, const float4* __restrict__ xs, int* parent, int* err, SegRec rec) {
    const int qi = blockIdx.x * blockDim.x + threadIdx.x;
    if (qi >= N) return;
    const int i = sorted[qi];
    const float4 xi = xs[qi];
    const float x[3] = {xi.x, xi.y, xi.z};
    int c[3];
    seg_cell(x, seg_frame(bbox, h), c);
    const float r2 = h * h;
    int ri = i;
    const int ks[4] = {13, 14, 16, 22};  // own bucket, +x, +y, +z (k = 9 (dz + 1) + 3 (dy + 1) + (dx + 1))
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const int k = ks[t];
        const unsigned int b = cell_hash(c[0] + k % 3 - 1, c[1] + (k / 3) % 3 - 1, c[2] + k / 9 - 1, mask);
        const int e = start[b] + count[b];
        for (int q = (k == 13 ? qi + 1 : start[b]); q < e; ++q)
            if (seg_close(x, xs[q], r2)) {
                seg_join(parent, i, sorted[q], ri, err, rec);
                break;
            }
    }
}
// The links pass of a segmentation that follows another: in place of the sampled neighbour search, the previous
// segmentation's spanning forest (pairs of caller indices, found through slotOf in the current slot order) is
// re-checked against the current positions, and the pairs still closer than h are joined.  While the bodies
// hold together between steps (the common case) this rebuilds them with one union per particle and no search;
// a pair that has come apart joins nothing, and the finish pass searches in full for every particle left
// outside the giant component, so the partition is the same as from the sampled links.
__global__ void k_seg_links(PartArrays P, int N, float h, const int2* __restrict__ edgeIn, const int* __restrict__ slotOf,
                            int* parent, int* err, SegRec rec) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    const int2 e = edgeIn[k];
    if ((unsigned)e.x >= (unsigned)N || (unsigned)e.y >= (unsigned)N) return;  // -1: no pair in this slot
    const int i = slotOf[e.x], j = slotOf[e.y];
    float x[3], y[3];
    ld3(P.x, N, i, x);
    ld3(P.x, N, j, y);
    if (!seg_close(x, make_float4(y[0], y[1], y[2], 0.f), h * h)) return;
    int ri = i;
    seg_join(parent, i, j, ri, err, rec);
}
// the most frequent root among 1024 evenly spaced particles (ties: the smallest); one CTA of 1024 threads
__global__ void __launch_bounds__(1024) k_seg_giant(int N, int* parent, int* giant) {
    __shared__ int roots[1024];
    __shared__ unsigned long long best[32];
    const int ns = min(N, 1024), t = threadIdx.x;
    if (t < ns) roots[t] = uf_find(parent, (int)((long long)t * N / ns));
    __syncthreads();
    unsigned long long key = 0ull;  // (count << 32) | (0x7fffffff - root): max = most frequent, then smallest
    if (t < ns) {
        int cnt = 0;
        for (int k = 0; k < ns; ++k) cnt += roots[k] == roots[t];
        key = ((unsigned long long)cnt << 32) | (unsigned long long)(0x7fffffff - roots[t]);
    }
    for (int o = 16; o; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
        key = other > key ? other : key;
    }
    if ((t & 31) == 0) best[t >> 5] = key;
    __syncthreads();
    if (t < 32) {
        key = best[t];
        for (int o = 16; o; o >>= 1) {
            const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
            key = other > key ? other : key;
        }
        if (t == 0) *giant = 0x7fffffff - (int)(key & 0xffffffffull);
    }
}
__global__ void k_seg_finish(int N, float h, const unsigned int* bbox, unsigned int mask, const int* count, const int* start,
                             const int* sorted, const float4* __restrict__ xs, const int* giant, int* parent, int* err,
                             SegRec rec) {
    const int qi = blockIdx.x * blockDim.x + threadIdx.x;
    if (qi >= N) return;
    const int i = sorted[qi];
    int ri = uf_find(parent, i);
    if (ri == uf_find(parent, *giant)) return;
    const float4 xi = xs[qi];
    const float x[3] = {xi.x, xi.y, xi.z};
    int c[3];
    seg_cell(x, seg_frame(bbox, h), c);
    const float r2 = h * h;
    for (int k = 0; k < 27; ++k) {
        const unsigned int b = cell_hash(c[0] + k % 3 - 1, c[1] + (k / 3) % 3 - 1, c[2] + k / 9 - 1, mask);
        const int s = start[b], e = s + count[b];
        for (int q = s; q < e; ++q)
            if (q != qi && seg_close(x, xs[q], r2)) seg_join(parent, i, sorted[q], ri, err, rec);
    }
}
// component sizes and smallest caller index: one wave of CTAs over contiguous ranges of slots; a thread sums its
// particles per root (flushing with atomics where the root changes), and a CTA whose threads all hold one root
// (the common case: one body) issues one pair of atomics
constexpr int kLabelThreads = 256;
__global__ void __launch_bounds__(kLabelThreads) k_seg_label(PartArrays P, int N, int* parent, int* size, int* minOrig,
                                                             int chunk) {
    __shared__ int sRoot;
    __shared__ int sCnt[kLabelThreads / 32], sMin[kLabelThreads / 32];
    int cur = -1, cnt = 0, mn = 0x7fffffff;
    const int beg = blockIdx.x * chunk, end = min(N, beg + chunk);
    for (int i = beg + threadIdx.x; i < end; i += kLabelThreads) {
        const int r = uf_find(parent, i);
        if (r != cur) {
            if (cnt > 0) {
                atomicAdd(&size[cur], cnt);
                atomicMin(&minOrig[cur], mn);
            }
            cur = r;
            cnt = 0;
            mn = 0x7fffffff;
        }
        ++cnt;
        mn = min(mn, P.orig[i]);
    }
    if (threadIdx.x == 0) sRoot = -1;
    __syncthreads();
    if (cnt > 0) sRoot = cur;  // any one of them
    __syncthreads();
    const int r0 = sRoot;
    const bool uniform = __syncthreads_and(cnt == 0 || cur == r0);
    if (r0 < 0) return;
    if (!uniform) {
        if (cnt > 0) {
            atomicAdd(&size[cur], cnt);
            atomicMin(&minOrig[cur], mn);
        }
        return;
    }
    for (int o = 16; o > 0; o >>= 1) {
        cnt += __shfl_down_sync(0xffffffffu, cnt, o);
        mn = min(mn, __shfl_down_sync(0xffffffffu, mn, o));
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { sCnt[warp] = cnt; sMin[warp] = mn; }
    __syncthreads();
    if (threadIdx.x == 0) {
        int c = 0, m = 0x7fffffff;
        for (int w = 0; w < kLabelThreads / 32; ++w) { c += sCnt[w]; m = min(m, sMin[w]); }
        atomicAdd(&size[r0], c);
        atomicMin(&minOrig[r0], m);
    }
}
__global__ void k_seg_compress(int N, int* parent) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    parent[i] = uf_find(parent, i);
}
__global__ void k_seg_mark(int N, const int* parent, const int* size, const int* minOrig, int* mark) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    if (parent[i] == i && size[i] >= 2) mark[minOrig[i]] = 1;
}
__global__ void k_seg_assign(PartArrays P, int N, const int* parent, const int* size, const int* minOrig, const int* mrank,
                             int* nballistic) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int r = parent[i];
    if (size[r] >= 2) {
        P.body[i] = mrank[minOrig[r]];
    } else {
        P.body[i] = -1;
        atomicAdd(nballistic, 1);
    }
}
__global__ void k_fill_i(int* a, long long n, int v) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

void launch_segment(const PartArrays& P, int N, float h, SegArrays S, int hashBits, int* scanTmp, int* err, cudaStream_t s) {
    if (N <= 0) return;
    const long long HB = 1ll << hashBits;
    const unsigned int mask = (unsigned int)(HB - 1);
    const int nb = (N + 255) / 256;
    cudaMemsetAsync(S.count, 0, sizeof(int) * HB, s);
    cudaMemsetAsync(S.size, 0, sizeof(int) * N, s);
    cudaMemsetAsync(S.mark, 0, sizeof(int) * N, s);
    cudaMemsetAsync(S.nbodies, 0, sizeof(int) * 2, s);
    cudaMemsetAsync(S.bbox, 0xff, sizeof(unsigned int) * 3, s);
    cudaMemsetAsync(S.bbox + 3, 0, sizeof(unsigned int) * 3, s);
    ++g_kernel_launches; k_fill_i<<<nb, 256, 0, s>>>(S.minOrig, N, 0x7fffffff);
    ++g_kernel_launches; k_seg_bbox<<<std::min(nb, 148 * 8), kBboxThreads, 0, s>>>(P, N, S.bbox);
    ++g_kernel_launches; k_seg_bucket<<<nb, 256, 0, s>>>(P, N, h, S.bbox, mask, S.count, S.rank, err);
    scan_exclusive(S.count, S.start, HB, scanTmp, S.nbodies + 2, s);
    ++g_kernel_launches; k_seg_place<<<nb, 256, 0, s>>>(P, N, h, S.bbox, mask, S.start, S.rank, S.sorted, S.xs, S.parent);
    // components: sampled links (or the previous segmentation's forest re-checked), compressed; the giant root
    // (kept in mrank[0], which the scan below overwrites); the full neighbourhoods of the particles outside it.
    // The unions of this segmentation record its own forest in edgeOut (cleared first).
    const SegRec rec{P.orig, S.edgeOut};
    if (S.edgeOut) cudaMemsetAsync(S.edgeOut, 0xff, sizeof(int2) * N, s);
    if (S.useEdges && S.edgeIn && S.slotOf) {
        ++g_kernel_launches; k_seg_links<<<nb, 256, 0, s>>>(P, N, h, S.edgeIn, S.slotOf, S.parent, err, rec);
    } else {
        ++g_kernel_launches;
        k_seg_sample<<<nb, 256, 0, s>>>(N, h, S.bbox, mask, S.count, S.start, S.sorted, S.xs, S.parent, err, rec);
    }
    ++g_kernel_launches; k_seg_compress<<<nb, 256, 0, s>>>(N, S.parent);
    ++g_kernel_launches; k_seg_giant<<<1, 1024, 0, s>>>(N, S.parent, S.mrank);
    ++g_kernel_launches; k_seg_finish<<<nb, 256, 0, s>>>(N, h, S.bbox, mask, S.count, S.start, S.sorted, S.xs, S.mrank, S.parent,
                                                         err, rec);
    {
        const int blocks = std::min(nb, 148 * 8);
        const int per = (N + blocks - 1) / blocks;
        const int chunk = (per + kLabelThreads - 1) / kLabelThreads * kLabelThreads;
        ++g_kernel_launches;
        k_seg_label<<<(N + chunk - 1) / chunk, kLabelThreads, 0, s>>>(P, N, S.parent, S.size, S.minOrig, chunk);
    }
    ++g_kernel_launches; k_seg_compress<<<nb, 256, 0, s>>>(N, S.parent);
    ++g_kernel_launches; k_seg_mark<<<nb, 256, 0, s>>>(N, S.parent, S.size, S.minOrig, S.mark);
    scan_exclusive(S.mark, S.mrank, N, scanTmp, S.nbodies, s);
    ++g_kernel_launches; k_seg_assign<<<nb, 256, 0, s>>>(P, N, S.parent, S.size, S.minOrig, S.mrank, S.nbodies + 1);
}

}  // namespace mpm

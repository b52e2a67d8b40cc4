// BF16 3-D convolution kernels of the learned warm start, on the 5th-generation tensor cores (tcgen05).
//
// Every kernel is an implicit GEMM with one 128-row M tile per CTA, the accumulator in tensor memory (TMEM),
// operands staged by the CTA's threads in shared memory in the UMMA K-major, non-swizzled canonical layout
// (core matrices of 8 rows x 16 bytes; consecutive K chunks LBO bytes apart, consecutive 8-row groups 128 bytes
// apart), and tcgen05.mma issued by one thread.  Two operand buffers alternate; an mbarrier signalled by
// tcgen05.commit tells the CTA when a buffer may be refilled.  Every wait is bounded: on timeout the kernel
// records an error, still waits (bounded) for its own MMAs, frees its TMEM and returns.
//
//   forward       D[v][co]  = sum_{t, ci} X[v + off(t)][ci] W[t][ci][co]          (M = voxels, N = Cout)
//   backward data D[v][ci]  = sum_{t, co} dY[v - off(t)][co] W[t][ci][co]         (M = voxels, N = Cin)
//   weight grad   D[(t,ci)][co] = sum_v X[v + off(t)][ci] dY[v][co]              (M = taps x Cin, N = Cout)
//
// Activations are channels-last bf16 [batch][z][y][x][C] with C padded to 16 or 32; 3x3x3 taps with zero
// padding at the volume border; t = 9 (dz + 1) + 3 (dy + 1) + (dx + 1).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/mpm_gpu.h"
#include "mpm_nn.h"

namespace mpmnn {

constexpr int kM = 128;          // rows per UMMA tile
constexpr int kTaps = 27;
constexpr uint64_t kWaitNs = 1000000000ull;  // 1 s: no MMA group of these kernels takes a millisecond
constexpr int ERR_TIMEOUT = 1;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// UMMA shared-memory descriptor, K-major, no swizzle (layout type 0), sm_100 version bits = 1
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}
// instruction descriptor: kind::f16, A = B = BF16, D = F32, both K-major, M x N
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
// waits for the phase of parity `parity` to complete; gives up after kWaitNs (returns false)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    const uint64_t t0 = global_ns();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (global_ns() - t0 > kWaitNs) return false;
    }
}
__device__ __forceinline__ void tmem_alloc32(uint32_t* dst_smem) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;" ::"r"(smem_u32(dst_smem)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc32(uint32_t taddr) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" ::"r"(taddr));
}
__device__ __forceinline__ void tmem_alloc64(uint32_t* dst_smem) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;" ::"r"(smem_u32(dst_smem)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc64(uint32_t taddr) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" ::"r"(taddr));
}
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
// 16 consecutive fp32 columns of this thread's TMEM lane; the wait is in the same asm statement so no use of the
// destination registers can be scheduled before the load has completed
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&r)[16]) {
    uint32_t u[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7]), "=r"(u[8]),
          "=r"(u[9]), "=r"(u[10]), "=r"(u[11]), "=r"(u[12]), "=r"(u[13]), "=r"(u[14]), "=r"(u[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int k = 0; k < 16; ++k) r[k] = __uint_as_float(u[k]);
}

struct Vol {
    int nx, ny, nz, batch;
    long long nvox;  // nx ny nz batch
};

// ---------------------------------------------------------------------------------------------------------
// weight gradient: rows m = t * CI + ci (27 CI rows, tiles of 128), N = CO (16/32) output channels, K = voxels.
// Each CTA reduces one row tile over a contiguous voxel range in stages of 64 voxels and adds its partial sums
// to dW (fp32 atomics).  Per stage, a table gives each voxel's linear index and a 27-bit mask of the taps whose
// source voxel lies inside the volume; a tap's source is then the voxel's index plus a constant offset.
// ---------------------------------------------------------------------------------------------------------
template <int CI, int CO>
__global__ void __launch_bounds__(128) k_conv_wgrad(const __nv_bfloat16* __restrict__ X, const __nv_bfloat16* __restrict__ dY,
                                                    float* dW, Vol vol, int voxPerCta, int* err) {
    constexpr int KS = 64;      // voxels per stage
    constexpr int KC = KS / 8;  // 16-byte chunks per row per stage
    __shared__ __align__(128) uint4 As[2][KC][kM];
    __shared__ __align__(128) uint4 Bs[2][KC][CO];
    __shared__ uint32_t tapMask[KS];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmemBase;
    __shared__ int abortFlag[2];  // per stage parity: a flag is re-written only after every thread read it
    __shared__ int doneFlag;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int rows = kTaps * CI;
    if (warp == 0) tmem_alloc32(&tmemBase);
    if (tid == 0) {
        abortFlag[0] = abortFlag[1] = 0;
        mbar_init(&mbar[0]);
        mbar_init(&mbar[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmemBase;
    const uint32_t idesc = umma_idesc(kM, CO);
    const int m = blockIdx.y * kM + tid;  // my row of A: tap t, input channel ci
    const bool rowOk = m < rows;
    const int t = rowOk ? m / CI : 0, ci = m % CI;
    const long long tapOff = ((long long)(t / 9 - 1) * vol.ny + (t / 3) % 3 - 1) * vol.nx + t % 3 - 1;
    const long long v0 = (long long)blockIdx.x * voxPerCta;
    const long long v1 = min(vol.nvox, v0 + voxPerCta);
    bool ok = true;
    int stage = 0, last = -1;
    for (long long vs = v0; vs < v1; vs += KS, ++stage) {
        const int buf = stage & 1;
        if (tid < KS) {
            uint32_t mask = 0;
            const long long vv = vs + tid;
            if (vv < v1) {
                long long r = vv;
                const int x = (int)(r % vol.nx); r /= vol.nx;
                const int y = (int)(r % vol.ny); r /= vol.ny;
                const int z = (int)(r % vol.nz);
                for (int tt = 0; tt < kTaps; ++tt) {
                    const int xs = x + tt % 3 - 1, ys = y + (tt / 3) % 3 - 1, zs = z + tt / 9 - 1;
                    if (xs >= 0 && ys >= 0 && zs >= 0 && xs < vol.nx && ys < vol.ny && zs < vol.nz) mask |= 1u << tt;
                }
            }
            tapMask[tid] = mask;
        }
        if (stage >= 2 && !mbar_wait(&mbar[buf], ((stage - 2) >> 1) & 1)) ok = false;
        if (!ok) abortFlag[stage & 1] = 1;
        __syncthreads();
        // A[m][k = voxel vs + j] = X[voxel + off(t)][ci]; 8 consecutive voxels per 16-byte chunk
#pragma unroll 2
        for (int c = 0; c < KC; ++c) {
            __align__(16) __nv_bfloat16 e[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int jj = c * 8 + j;
                e[j] = (rowOk && ((tapMask[jj] >> t) & 1u)) ? X[(vs + jj + tapOff) * CI + ci] : __float2bfloat16(0.f);
            }
            As[buf][c][tid] = *reinterpret_cast<const uint4*>(e);
        }
        // B[k = voxel][n = co]: chunk c, row n holds dY[vs + 8c .. +7][n]
        for (int e2 = tid; e2 < KC * CO; e2 += blockDim.x) {
            const int c = e2 / CO, n = e2 % CO;
            __align__(16) __nv_bfloat16 e[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const long long vv = vs + c * 8 + j;
                e[j] = vv < v1 ? dY[vv * CO + n] : __float2bfloat16(0.f);
            }
            Bs[buf][c][n] = *reinterpret_cast<const uint4*>(e);
        }
        fence_async_smem();
        __syncthreads();
        if (abortFlag[stage & 1]) break;  // uniform: every write of this flag precedes the barriers above
        if (tid == 0) {
            tc_fence_after();
#pragma unroll
            for (int s = 0; s < KC / 2; ++s) {
                const uint64_t ad = umma_desc(smem_u32(&As[buf][2 * s][0]), kM * 16, 128);
                const uint64_t bd = umma_desc(smem_u32(&Bs[buf][2 * s][0]), CO * 16, 128);
                umma_bf16(tmem, ad, bd, idesc, (stage | s) != 0);
            }
            umma_commit(&mbar[buf]);
        }
        last = stage;
    }
    const bool aborted = v0 + (long long)(last + 1) * KS < v1;
    // one thread waits for the last commit; the CTA barrier then releases every warp converged for the
    // .sync.aligned TMEM loads
    if (tid == 0) doneFlag = (last < 0 || mbar_wait(&mbar[last & 1], (last >> 1) & 1)) ? 1 : 0;
    __syncthreads();
    __syncwarp();
    if (!doneFlag || aborted) ok = false;
    if (last >= 0) {
        tc_fence_after();
        float acc[CO];
#pragma unroll
        for (int c0 = 0; c0 < CO; c0 += 16) {
            float r[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
#pragma unroll
            for (int k = 0; k < 16; ++k) acc[c0 + k] = r[k];
        }
        if (rowOk && ok) {
#pragma unroll
            for (int n = 0; n < CO; ++n) atomicAdd(&dW[(size_t)m * CO + n], acc[n]);
        }
    }
    if (!ok) atomicOr(err, ERR_TIMEOUT);
    tc_fence_before();
    __syncthreads();
    __syncwarp();
    if (warp == 0) tmem_dealloc32(tmem);
}

// ---------------------------------------------------------------------------------------------------------
// Halo-tiled convolution, forward or backward data.  CA = channels of the gathered operand (16 or 32), NP = padded
// output channels (16/32); FLIP gathers at v - off(t) (backward data).  Output y = act(acc + bias), with an
// optional mask for backward data through a ReLU (multiply by [maskAct[v][n] > 0]), written as bf16 (ybf,
// stride NP) and/or fp32 (yf, stride yfStride).  Persistent CTAs keep all 27 taps' weights in shared memory and
// walk a list of output blocks of 8 (x) x 16 (y) x 2 (z) voxels: two 128-row M tiles, one per z-plane, with their
// accumulators side by side in TMEM.  Per block the 10 x 18 x 4 input halo is loaded once (each plane's 3-plane
// halo shares two planes with the other's), stored [chunk][z][y][x] in 16-byte units, so that for every tap and
// plane the A operand is the same buffer at a shifted start address: rows m = x + 8 y form core matrices of 8
// consecutive x (128 contiguous bytes), consecutive y are SBO = 10 x 16 bytes apart and the K chunks LBO =
// 720 x 16 bytes apart.  All 2 x 27 x CA/16 MMAs of a block are issued back to back, the planes interleaved, and
// committed once.
// ---------------------------------------------------------------------------------------------------------
constexpr int kTX = 8, kTY = 16, kTZ = 2, kHX = kTX + 2, kHY = kTY + 2, kHZ = kTZ + 2, kHV = kHX * kHY * kHZ;

template <int CA, int NP>
constexpr int tile_smem_bytes() {
    return (kTaps * (CA / 8) * NP + (CA / 8) * kHV) * 16;
}

template <int CA, int NP, bool FLIP>
__global__ void __launch_bounds__(128) k_conv_tile(const __nv_bfloat16* __restrict__ X, const __nv_bfloat16* __restrict__ Wp,
                                                   const float* __restrict__ bias, int nOut, int relu,
                                                   const __nv_bfloat16* __restrict__ maskAct, __nv_bfloat16* ybf,
                                                   float* yf, int yfStride, Vol vol, const int* __restrict__ blockList,
                                                   const int* __restrict__ blockCountDev, int blockCount, int* err) {
    constexpr int KC = CA / 8;
    constexpr int NE = kHV * KC;           // 16-byte chunks in a halo
    constexpr int PER = (NE + 127) / 128;  // per thread
    extern __shared__ __align__(128) uint4 dsm[];
    uint4* Ws = dsm;                       // [27][KC][NP]
    uint4* Hs = dsm + kTaps * KC * NP;     // [KC][kHV]
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmemBase;
    __shared__ int doneFlag;
    const int tid = threadIdx.x, warp = tid >> 5;
    if (warp == 0) tmem_alloc64(&tmemBase);
    if (tid == 0) {
        mbar_init(&mbar);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    const uint4* W4 = reinterpret_cast<const uint4*>(Wp);
    for (int e = tid; e < kTaps * KC * NP; e += blockDim.x) Ws[e] = W4[e];
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmemBase;
    const uint32_t idesc = umma_idesc(kM, NP);
    const int nBlocks = blockCountDev ? *blockCountDev : blockCount;
    const int bxN = (vol.nx + kTX - 1) / kTX, byN = (vol.ny + kTY - 1) / kTY, bzN = (vol.nz + kTZ - 1) / kTZ;
    const uint4* X4 = reinterpret_cast<const uint4*>(X);
    // the halo of a block into registers: every load of the block is in flight at once
    uint4 hreg[PER];
    auto load_halo = [&](int blk) {
        const int bxi = blk % bxN, byi = (blk / bxN) % byN, zz = blk / (bxN * byN);
        const int z = (zz % bzN) * kTZ, bt = zz / bzN;
        const int x0 = bxi * kTX, y0 = byi * kTY;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int e = tid + k * 128;
            uint4 val = make_uint4(0, 0, 0, 0);
            if (e < NE) {
                const int c = e % KC, hv = e / KC;
                const int hx = hv % kHX, hy = (hv / kHX) % kHY, hz = hv / (kHX * kHY);
                const int gx = x0 - 1 + hx, gy = y0 - 1 + hy, gz = z - 1 + hz;
                if (gx >= 0 && gy >= 0 && gz >= 0 && gx < vol.nx && gy < vol.ny && gz < vol.nz)
                    val = X4[((((long long)bt * vol.nz + gz) * vol.ny + gy) * vol.nx + gx) * KC + c];
            }
            hreg[k] = val;
        }
    };
    uint32_t phase = 0;
    bool ok = true;
    int it = blockIdx.x;
    if (it < nBlocks) load_halo(blockList ? blockList[it] : it);
    for (; it < nBlocks; it += gridDim.x) {
        const int blk = blockList ? blockList[it] : it;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int e = tid + k * 128;
            if (e < NE) Hs[(e % KC) * kHV + e / KC] = hreg[k];
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
#pragma unroll 1
            for (int t = 0; t < kTaps; ++t) {
                int dx = t % 3 - 1, dy = (t / 3) % 3 - 1, dz = t / 9 - 1;
                if (FLIP) { dx = -dx; dy = -dy; dz = -dz; }
                const int hoff = ((dz + 1) * kHY + (dy + 1)) * kHX + (dx + 1);
#pragma unroll
                for (int s = 0; s < KC / 2; ++s) {
                    const uint64_t bd = umma_desc(smem_u32(Ws + (t * KC + 2 * s) * NP), NP * 16, 128);
#pragma unroll
                    for (int pz = 0; pz < kTZ; ++pz) {
                        const uint64_t ad =
                            umma_desc(smem_u32(Hs + 2 * s * kHV + hoff + pz * kHX * kHY), kHV * 16, kHX * 16);
                        umma_bf16(tmem + (uint32_t)(pz * 32), ad, bd, idesc, (t | s) != 0);
                    }
                }
            }
            umma_commit(&mbar);
        }
        // the next block's halo loads overlap this block's MMAs and epilogue
        const int nextIt = it + gridDim.x;
        if (nextIt < nBlocks) load_halo(blockList ? blockList[nextIt] : nextIt);
        if (tid == 0) doneFlag = mbar_wait(&mbar, phase) ? 1 : 0;
        __syncthreads();
        __syncwarp();
        phase ^= 1;
        if (!doneFlag) {  // uniform: read after the barrier
            ok = false;
            break;
        }
        tc_fence_after();
        const int bxi = blk % bxN, byi = (blk / bxN) % byN, zz = blk / (bxN * byN);
        const int z0 = (zz % bzN) * kTZ, bt = zz / bzN;
        const int x = bxi * kTX + (tid & 7), y = byi * kTY + (tid >> 3);
#pragma unroll 1
        for (int pz = 0; pz < kTZ; ++pz) {
            float acc[NP];
#pragma unroll
            for (int c0 = 0; c0 < NP; c0 += 16) {
                float r[16];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(pz * 32 + c0), r);
#pragma unroll
                for (int k = 0; k < 16; ++k) acc[c0 + k] = r[k];
            }
            const int z = z0 + pz;
            if (x < vol.nx && y < vol.ny && z < vol.nz) {
                const long long v = (((long long)bt * vol.nz + z) * vol.ny + y) * vol.nx + x;
                __align__(16) __nv_bfloat16 ob[NP];
#pragma unroll
                for (int n = 0; n < NP; ++n) {
                    float val = 0.f;
                    if (n < nOut) {
                        val = acc[n] + (bias ? bias[n] : 0.f);
                        if (relu) val = fmaxf(val, 0.f);
                        if (maskAct && !(__bfloat162float(maskAct[v * NP + n]) > 0.f)) val = 0.f;
                    }
                    ob[n] = __float2bfloat16(val);
                    if (yf && n < nOut) yf[v * yfStride + n] = val;
                }
                if (ybf) {
                    uint4* o = reinterpret_cast<uint4*>(ybf + v * NP);
#pragma unroll
                    for (int q = 0; q < NP / 8; ++q) o[q] = reinterpret_cast<const uint4*>(ob)[q];
                }
            }
        }
        tc_fence_before();
        __syncthreads();  // every warp has read TMEM before the next block's MMAs overwrite it
    }
    if (!ok && tid == 0) atomicOr(err, ERR_TIMEOUT);
    // a timed-out MMA group may still be running: wait for it (bounded) before the TMEM is released
    if (!ok && tid == 0) mbar_wait(&mbar, phase ^ 1);
    tc_fence_before();
    __syncthreads();
    __syncwarp();
    if (warp == 0) tmem_dealloc64(tmem);
}

// master fp32 weights W[t][ci][co] (ci < cin, co < cout) -> forward pack [t][ci_pad/8][co_pad][8] and
// backward-data pack [t][co_pad/8][ci_pad][8]
__global__ void k_pack(const float* W, int cin, int cout, int cinPad, int coutPad, __nv_bfloat16* fwd, __nv_bfloat16* bwd) {
    const int total = kTaps * cinPad * coutPad;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int t = i / (cinPad * coutPad), r = i % (cinPad * coutPad);
    const int ci = r / coutPad, co = r % coutPad;
    const float w = (ci < cin && co < cout) ? W[((size_t)t * cin + ci) * cout + co] : 0.f;
    const __nv_bfloat16 wb = __float2bfloat16(w);
    if (fwd) fwd[(((size_t)t * (cinPad / 8) + ci / 8) * coutPad + co) * 8 + ci % 8] = wb;
    if (bwd) bwd[(((size_t)t * (coutPad / 8) + co / 8) * cinPad + ci) * 8 + co % 8] = wb;
}

// Adam on fp32 master weights
__global__ void k_adam(float* w, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps, float c1,
                       float c2, float wd) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i] + wd * w[i];
    m[i] = b1 * m[i] + (1.f - b1) * gi;
    v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
    w[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
}

// bias gradient: db[n] += sum_v dY[v][n]
__global__ void k_bias_grad(const __nv_bfloat16* dY, int CO, int nOut, long long nvox, float* db) {
    __shared__ float s[32];
    if (threadIdx.x < 32) s[threadIdx.x] = 0.f;
    __syncthreads();
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nvox; v += (long long)gridDim.x * blockDim.x)
        for (int n = 0; n < nOut; ++n) atomicAdd(&s[n], __bfloat162float(dY[v * CO + n]));
    __syncthreads();
    if (threadIdx.x < nOut) atomicAdd(&db[threadIdx.x], s[threadIdx.x]);
}

// training features from captured grid arrays (component-interleaved xyz per node): bf16 [n][16]
__global__ void k_features(const float* mass, const float* pstar, const float* frc, const float* diag, const float* hist,
                           const float* normals, long long n, NnNorm nn, __nv_bfloat16* out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float ps[3] = {pstar[3 * i], pstar[3 * i + 1], pstar[3 * i + 2]};
    const float f[3] = {frc[3 * i], frc[3 * i + 1], frc[3 * i + 2]};
    const float d[3] = {diag[3 * i], diag[3 * i + 1], diag[3 * i + 2]};
    float hv[3] = {0.f, 0.f, 0.f}, nrm[3] = {0.f, 0.f, 0.f};
    bool hasHist = false;
    if (hist) {
        hv[0] = hist[3 * i]; hv[1] = hist[3 * i + 1]; hv[2] = hist[3 * i + 2];
        hasHist = !isnan(hv[0]);
    }
    if (normals) {
        nrm[0] = normals[3 * i]; nrm[1] = normals[3 * i + 1]; nrm[2] = normals[3 * i + 2];
    }
    float ft[kFeat];
    node_features(mass[i], ps, f, d, hasHist, hv, nrm, nn, ft);
    __align__(16) __nv_bfloat16 e[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) e[k] = __float2bfloat16(k < kFeat ? ft[k] : 0.f);
    uint4* o = reinterpret_cast<uint4*>(out + i * 16);
    o[0] = reinterpret_cast<const uint4*>(e)[0];
    o[1] = reinterpret_cast<const uint4*>(e)[1];
}

// weighted squared error over 3 outputs and its gradient: loss += sum_v w_v |y_v - t_v|^2 inv_wsum;
// dy[v][0..2] = 2 w_v (y_v - t_v) inv_wsum (bf16, 16 channels, the padding zero)
__global__ void k_mse(const float* y, int ystride, const float* target, const float* w, long long n, float inv_wsum,
                      __nv_bfloat16* dy, double* loss) {
    __shared__ double red[8];
    double part = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float wi = w[i] * inv_wsum;
        __align__(16) __nv_bfloat16 e[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) e[k] = __float2bfloat16(0.f);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float d = y[i * ystride + a] - target[3 * i + a];
            part += (double)wi * d * d;
            e[a] = __float2bfloat16(2.f * wi * d);
        }
        uint4* o = reinterpret_cast<uint4*>(dy + i * 16);
        o[0] = reinterpret_cast<const uint4*>(e)[0];
        o[1] = reinterpret_cast<const uint4*>(e)[1];
    }
    for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
        atomicAdd(loss, t);
    }
}

cudaError_t pack_weights(const float* w, int cin, int cout, int cin_pad, int cout_pad, void* packed_fwd, void* packed_bwd,
                         cudaStream_t s) {
    const int total = kTaps * cin_pad * cout_pad;
    k_pack<<<(total + 255) / 256, 256, 0, s>>>(w, cin, cout, cin_pad, cout_pad, (__nv_bfloat16*)packed_fwd,
                                               (__nv_bfloat16*)packed_bwd);
    return cudaGetLastError();
}

template <int CA, int NP, bool FL>
cudaError_t launch_tile(const __nv_bfloat16* X, const __nv_bfloat16* W, const float* bias, int cout, int relu,
                        const __nv_bfloat16* M, __nv_bfloat16* Y, float* yf, int yfs, Vol vol, const int* list,
                        const int* countDev, int countHost, int* err, cudaStream_t s) {
    constexpr int smem = tile_smem_bytes<CA, NP>();
    static int configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(k_conv_tile<CA, NP, FL>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(k_conv_tile<CA, NP, FL>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
        if (e != cudaSuccess) return e;
        configured[dev] = 1;
    }
    // resident CTAs per SM: shared memory (1 KB reserved per CTA), registers (allocated per warp in units of 256)
    // and at most 8 (the 512 TMEM columns hold 8 allocations of 64): the grid is one wave of persistent CTAs
    int sms = 0, smemSm = 0, regsSm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&smemSm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&regsSm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    cudaFuncAttributes fa{};
    cudaError_t fe = cudaFuncGetAttributes(&fa, k_conv_tile<CA, NP, FL>);
    if (fe != cudaSuccess) return fe;
    const int regsCta = (fa.numRegs * 32 + 255) / 256 * 256 * (128 / 32);
    const int bySmem = smemSm / (smem + (int)fa.sharedSizeBytes + 1024);
    const int byRegs = regsCta > 0 ? regsSm / regsCta : 8;
    const int perSm = std::max(1, std::min(8, std::min(bySmem, byRegs)));
    const int bxN = (vol.nx + kTX - 1) / kTX, byN = (vol.ny + kTY - 1) / kTY, bzN = (vol.nz + kTZ - 1) / kTZ;
    const long long maxBlocks = (long long)bxN * byN * bzN * vol.batch;
    const long long want = countDev ? maxBlocks : countHost;
    const int grid = (int)std::max<long long>(1, std::min<long long>(want, (long long)std::max(perSm, 1) * sms));
    k_conv_tile<CA, NP, FL><<<grid, 128, smem, s>>>(X, W, bias, cout, relu, M, Y, yf, yfs, vol, list, countDev, countHost, err);
    return cudaGetLastError();
}

cudaError_t conv3d_tiled(const void* x, int cin_pad, const void* packed, const float* bias, int cout, int cout_pad, int relu,
                         int flip, const void* mask_act, void* y_bf16, float* y_f32, int y_f32_stride, int nx, int ny,
                         int nz, int batch, const int* block_list, const int* block_count_dev, int* err, cudaStream_t s) {
    Vol vol{nx, ny, nz, batch, (long long)nx * ny * nz * batch};
    if (vol.nvox == 0) return cudaSuccess;
    const int bxN = (nx + kTX - 1) / kTX, byN = (ny + kTY - 1) / kTY, bzN = (nz + kTZ - 1) / kTZ;
    const int all = bxN * byN * bzN * batch;
    const __nv_bfloat16* X = (const __nv_bfloat16*)x;
    const __nv_bfloat16* W = (const __nv_bfloat16*)packed;
    const __nv_bfloat16* M = (const __nv_bfloat16*)mask_act;
    __nv_bfloat16* Y = (__nv_bfloat16*)y_bf16;
#define MPM_TILE_LAUNCH(CA, NP, FL) \
    return launch_tile<CA, NP, FL>(X, W, bias, cout, relu, M, Y, y_f32, y_f32_stride, vol, block_list, block_count_dev, all, err, s)
    if (cin_pad == 16 && cout_pad == 32) { if (flip) MPM_TILE_LAUNCH(16, 32, true); else MPM_TILE_LAUNCH(16, 32, false); }
    if (cin_pad == 32 && cout_pad == 32) { if (flip) MPM_TILE_LAUNCH(32, 32, true); else MPM_TILE_LAUNCH(32, 32, false); }
    if (cin_pad == 32 && cout_pad == 16) { if (flip) MPM_TILE_LAUNCH(32, 16, true); else MPM_TILE_LAUNCH(32, 16, false); }
    if (flip) MPM_TILE_LAUNCH(16, 16, true);
    MPM_TILE_LAUNCH(16, 16, false);
#undef MPM_TILE_LAUNCH
}

// Per-layer output blocks for the warm start's inference.  Only heavy nodes (mass >= heavy_mass) read the
// network's output, so layer l (of L) is needed only within Chebyshev distance L - 1 - l of a heavy node: the last
// layer at the heavy nodes themselves, layer 0 within L - 1.  Stale values left in the activation buffers outside
// a layer's blocks are never read by a voxel that matters.  The distance to the nearest heavy node, capped at L,
// is built by three separable passes (x, then y, then z) over a byte volume; each output block then goes to the
// lists of the layers whose reach covers its nearest voxel.
__global__ void k_heavy_dist_x(const float* mass, float heavyMass, int nx, int ny, int nz, int R, unsigned char* d) {
    const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= (long long)nx * ny * nz) return;
    const int x = (int)(l % nx);
    int best = R + 1;
    for (int dx = -R; dx <= R; ++dx) {
        const int xx = x + dx, ad = dx < 0 ? -dx : dx;
        if (xx >= 0 && xx < nx && ad < best && mass[l + dx] > 0.f && mass[l + dx] >= heavyMass) best = ad;
    }
    d[l] = (unsigned char)best;
}
// out(v) = min over |k| <= R of max(|k|, in(v + k e_axis)), axis 1 = y, 2 = z
__global__ void k_dist_pass(const unsigned char* in, int nx, int ny, int nz, int R, int axis, unsigned char* out) {
    const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= (long long)nx * ny * nz) return;
    const int c = axis == 1 ? (int)((l / nx) % ny) : (int)(l / ((long long)nx * ny));
    const int n = axis == 1 ? ny : nz;
    const long long stride = axis == 1 ? nx : (long long)nx * ny;
    int best = R + 1;
    for (int k = -R; k <= R; ++k) {
        const int cc = c + k, ak = k < 0 ? -k : k;
        if (cc < 0 || cc >= n) continue;
        const int v = max((int)in[l + k * stride], ak);
        best = min(best, v);
    }
    out[l] = (unsigned char)best;
}
__global__ void k_layer_lists(const unsigned char* d, int nx, int ny, int nz, int L, int* lists, long long listStride,
                              int* counts) {
    const int bxN = (nx + kTX - 1) / kTX, byN = (ny + kTY - 1) / kTY, bzN = (nz + kTZ - 1) / kTZ;
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= bxN * byN * bzN) return;
    const int bx = b % bxN, by = (b / bxN) % byN, bz = b / (bxN * byN);
    int dmin = L;
    for (int z = bz * kTZ; z < min(nz, (bz + 1) * kTZ) && dmin > 0; ++z)
        for (int y = by * kTY; y < min(ny, (by + 1) * kTY) && dmin > 0; ++y)
            for (int x = bx * kTX; x < min(nx, (bx + 1) * kTX); ++x)
                dmin = min(dmin, (int)d[((long long)z * ny + y) * nx + x]);
    for (int l = 0; l < L; ++l)
        if (dmin <= L - 1 - l) lists[l * listStride + atomicAdd(&counts[l], 1)] = b;
}
cudaError_t layer_blocks(const float* mass, float heavy_mass, int nx, int ny, int nz, int layers, unsigned char* scratch,
                         int* lists, long long list_stride, int* counts, cudaStream_t s) {
    const long long G = (long long)nx * ny * nz;
    const long long nb = tile_blocks(nx, ny, nz);
    if (layers < 1 || layers > 200) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(int) * layers, s);
    if (e != cudaSuccess || G == 0) return e;
    const int R = layers - 1;
    unsigned char* a = scratch;
    unsigned char* b = scratch + G;
    const unsigned g = (unsigned)((G + 255) / 256);
    k_heavy_dist_x<<<g, 256, 0, s>>>(mass, heavy_mass, nx, ny, nz, R, a);
    k_dist_pass<<<g, 256, 0, s>>>(a, nx, ny, nz, R, 1, b);
    k_dist_pass<<<g, 256, 0, s>>>(b, nx, ny, nz, R, 2, a);
    k_layer_lists<<<(unsigned)((nb + 255) / 256), 256, 0, s>>>(a, nx, ny, nz, layers, lists, list_stride, counts);
    return cudaGetLastError();
}

long long tile_blocks(int nx, int ny, int nz) {
    return (long long)((nx + kTX - 1) / kTX) * ((ny + kTY - 1) / kTY) * ((nz + kTZ - 1) / kTZ);
}

}  // namespace mpmnn

using namespace mpmnn;

namespace {
bool pad_ok(int c) { return c == 16 || c == 32; }
mpm_status cuda_status(cudaError_t e) { return e == cudaSuccess ? MPM_OK : MPM_ERR_CUDA; }
}  // namespace

extern "C" {

mpm_status mpm_nn_pack_weights(const float* w, int cin, int cout, int cin_pad, int cout_pad, void* packed_fwd,
                               void* packed_bwd, void* stream) {
    if (!w || cin <= 0 || cout <= 0 || cin > cin_pad || cout > cout_pad || !pad_ok(cin_pad) || !pad_ok(cout_pad))
        return MPM_ERR_INVALID_ARGUMENT;
    return cuda_status(pack_weights(w, cin, cout, cin_pad, cout_pad, packed_fwd, packed_bwd, (cudaStream_t)stream));
}

mpm_status mpm_nn_conv3d(const void* x, int cin_pad, const void* packed, const float* bias, int cout, int cout_pad, int relu,
                         int flip, const void* mask_act, void* y_bf16, float* y_f32, int y_f32_stride, int nx, int ny, int nz,
                         int batch, int* err, void* stream) {
    if (!x || !packed || !err || !pad_ok(cin_pad) || !pad_ok(cout_pad) || cout <= 0 || cout > cout_pad || nx < 0 ||
        ny < 0 || nz < 0 || batch < 0 || (!y_bf16 && !y_f32) || (y_f32 && y_f32_stride < cout))
        return MPM_ERR_INVALID_ARGUMENT;
    return cuda_status(conv3d_tiled(x, cin_pad, packed, bias, cout, cout_pad, relu, flip, mask_act, y_bf16, y_f32,
                                    y_f32_stride, nx, ny, nz, batch, nullptr, nullptr, err, (cudaStream_t)stream));
}

mpm_status mpm_nn_conv3d_wgrad(const void* x, int cin_pad, const void* dy, int cout_pad, float* dw, int nx, int ny, int nz,
                               int batch, int* err, void* stream) {
    if (!x || !dy || !dw || !err || !pad_ok(cin_pad) || !pad_ok(cout_pad) || nx < 0 || ny < 0 || nz < 0 || batch < 0)
        return MPM_ERR_INVALID_ARGUMENT;
    Vol vol{nx, ny, nz, batch, (long long)nx * ny * nz * batch};
    if (vol.nvox == 0) return MPM_OK;
    const int voxPerCta = 2048;
    dim3 grid((unsigned)((vol.nvox + voxPerCta - 1) / voxPerCta), (unsigned)((kTaps * cin_pad + kM - 1) / kM));
    cudaStream_t s = (cudaStream_t)stream;
    const __nv_bfloat16* X = (const __nv_bfloat16*)x;
    const __nv_bfloat16* D = (const __nv_bfloat16*)dy;
    if (cin_pad == 16 && cout_pad == 32) k_conv_wgrad<16, 32><<<grid, 128, 0, s>>>(X, D, dw, vol, voxPerCta, err);
    else if (cin_pad == 32 && cout_pad == 32) k_conv_wgrad<32, 32><<<grid, 128, 0, s>>>(X, D, dw, vol, voxPerCta, err);
    else if (cin_pad == 32 && cout_pad == 16) k_conv_wgrad<32, 16><<<grid, 128, 0, s>>>(X, D, dw, vol, voxPerCta, err);
    else k_conv_wgrad<16, 16><<<grid, 128, 0, s>>>(X, D, dw, vol, voxPerCta, err);
    return cuda_status(cudaGetLastError());
}

mpm_status mpm_nn_bias_grad(const void* dy, int cout_pad, int cout, long long nvox, float* db, void* stream) {
    if (!dy || !db || !pad_ok(cout_pad) || cout <= 0 || cout > cout_pad || nvox < 0) return MPM_ERR_INVALID_ARGUMENT;
    if (nvox == 0) return MPM_OK;
    k_bias_grad<<<256, 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)dy, cout_pad, cout, nvox, db);
    return cuda_status(cudaGetLastError());
}

mpm_status mpm_nn_adam(float* w, const float* g, float* m, float* v, int n, float lr, float beta1, float beta2, float eps,
                       int step, float weight_decay, void* stream) {
    if (!w || !g || !m || !v || n <= 0 || step < 1) return MPM_ERR_INVALID_ARGUMENT;
    const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
    k_adam<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(w, g, m, v, n, lr, beta1, beta2, eps, c1, c2, weight_decay);
    return cuda_status(cudaGetLastError());
}

mpm_status mpm_nn_features(const float* mass, const float* pstar, const float* force, const float* diag,
                           const float* history, const float* normals, long long n, float dt, float h, float density,
                           float light_mass, const float* gravity3, const float* feature_scale16, void* out_bf16,
                           void* stream) {
    if (!mass || !pstar || !force || !diag || !out_bf16 || !gravity3 || !feature_scale16 || n < 0 || !(dt > 0.f) ||
        !(h > 0.f) || !(density > 0.f) || !(light_mass >= 0.f))
        return MPM_ERR_INVALID_ARGUMENT;
    if (n == 0) return MPM_OK;
    NnNorm nn{};
    nn.inv_mass_unit = 1.f / (density * h * h * h);
    nn.inv_vel_unit = dt / h;
    nn.vel_unit = h / dt;
    nn.dt = dt;
    for (int a = 0; a < 3; ++a) nn.gdt[a] = dt * gravity3[a];
    for (int k = 0; k < kFeat; ++k) nn.feat_scale[k] = feature_scale16[k];
    nn.out_scale = 1.f;
    nn.light_mass = light_mass;
    k_features<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(mass, pstar, force, diag, history, normals,
                                                                             n, nn, (__nv_bfloat16*)out_bf16);
    return cuda_status(cudaGetLastError());
}

mpm_status mpm_nn_mse(const float* y, int y_stride, const float* target, const float* weight, long long n, float inv_wsum,
                      void* dy_bf16, double* loss, void* stream) {
    if (!y || !target || !weight || !dy_bf16 || !loss || y_stride < 3 || n < 0) return MPM_ERR_INVALID_ARGUMENT;
    if (n == 0) return MPM_OK;
    k_mse<<<592, 256, 0, (cudaStream_t)stream>>>(y, y_stride, target, weight, n, inv_wsum, (__nv_bfloat16*)dy_bf16, loss);
    return cuda_status(cudaGetLastError());
}

}  // extern "C"

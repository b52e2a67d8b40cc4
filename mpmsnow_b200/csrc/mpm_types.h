// Plain-data structures shared by the host orchestration and the kernels of the CUDA MPM step.
#pragma once

#include <stdint.h>

namespace mpm {

constexpr int kMaxColliders = 16;
constexpr int kMaxFields = 8;
constexpr int kTile = 4;                 // tile edge in cells (matches the reference's 4h voxel)
constexpr int kTileCells = kTile * kTile * kTile;
constexpr int kWin = kTile + 3;          // nodes touched by one tile's stencils, per axis
constexpr int kWin3 = kWin * kWin * kWin;
constexpr int kNodeChunk = 1024;         // nodes per reduction CTA; every body's node range is padded to it
constexpr int kNodeThreads = 256;
constexpr int kTileThreads = 128;

struct DevCollider {
    int kind;          // 0 plane, 1 vertical cylinder, 2 sampled signed-distance grid
    float c[4];        // plane coefficients / (cx, cz, radius, unused) / grid (origin x, y, z, spacing)
    float vel[3];      // constant velocity (plane, cylinder)
    float friction;
    int sticky;
    int n[3];          // grid: samples per axis
    const float* phi;  // grid: phi at origin + spacing (i, j, k), x fastest (device memory)
    const float* v;    // grid: velocity, 3 per sample, or null = at rest (device memory)
};

// Everything a kernel needs that is constant over a step; passed by value.
struct StepParams {
    float h;
    float dt;
    float xi, thetaC, thetaS;     // hardening and the clamp [1 - theta_c, 1 + theta_s]
    float mu, lambda;             // scalar Lame parameters of SnowConstitutiveModel
    int ncoll;
    int nfields;
    int maxIters;
    float tol;
    DevCollider coll[kMaxColliders];
    float gravity[kMaxFields][3];
};

// One body's comoving grid (Grid.cpp:171-213), in the concatenated node arrays.
struct BodyGrid {
    float mn[3];          // m_min
    int n[3];             // m_n
    int T[3];             // tiles per axis = ceil(n / 4)
    int tileOff;          // first global tile id
    long long nodeOff;    // first node in the concatenated node arrays
    int ctaBegin, ctaEnd; // node-chunk CTAs [ctaBegin, ctaEnd) covering this body
    float fv[3];          // frame (centre of mass) velocity
};

// Per-body accumulators filled by atomics before the grid is built.
struct BodyAccum {
    double mom[3];
    double mass;
    unsigned int bmin[3];  // order-preserving encoding of float bounds
    unsigned int bmax[3];
    int count;
    int pad;
};

// Per-body solver state (device-resident scalars of ConjugateResiduals).
struct BodySolve {
    double bNorm2, threshold, rz, ApdPAp, alpha, beta, rNorm2;
    double guess[8];      // totalMass, totalMomentum[3], collidedMass, collidedMomentum[3]
    float x0[3];
    int done;             // 0 running, 1 finished
    int iterations;       // iteration index at which the solve returned
    int exitReason;       // 0 termination, 1 b == 0, 2 <Ap, M^-1 Ap> == 0, 3 rz_old == 0
    int bzero;
};

// device error bits (mirrored into mpm_status by the host)
enum : int {
    ERR_NAN_MASSES = 1 << 0,
    ERR_NAN_VELOCITIES = 1 << 1,
    ERR_NAN_MOMENTA = 1 << 2,
    ERR_NAN_STRESS = 1 << 3,
    ERR_HARDNESS = 1 << 4,
    ERR_NAN_PARTICLE_V = 1 << 5,
    ERR_STENCIL_OOB = 1 << 6,
    ERR_SEGMENT = 1 << 7,
};
// the errors the grid phases raise before the solve ends (no particle has moved yet)
constexpr int kGridErrors = ERR_NAN_MASSES | ERR_NAN_VELOCITIES | ERR_NAN_MOMENTA | ERR_NAN_STRESS | ERR_STENCIL_OOB;

// encode a float so that unsigned integer order equals float order (for atomicMin / atomicMax)
__host__ __device__ inline unsigned int float_to_ordered(float f) {
    union { float f; unsigned int u; } x;
    x.f = f;
    return (x.u & 0x80000000u) ? ~x.u : (x.u | 0x80000000u);
}
__host__ __device__ inline float ordered_to_float(unsigned int u) {
    union { float f; unsigned int u; } x;
    x.u = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
    return x.f;
}

}  // namespace mpm

// Launch wrappers of the CUDA MPM step kernels (mpm_kernels.cu).  Host orchestration: mpm_sim.cu.
#pragma once

#include <cuda_runtime.h>

#include "mpm_nn.h"
#include "mpm_types.h"

namespace mpm {

// Particle state, structure of arrays in the current storage (tile-sorted) order; N particles.
// Vectors: component c of particle i at [c * N + i]; matrices: element k (= 3 r + c) at [k * N + i].
struct PartArrays {
    float* x;
    float* v;
    float* F;
    float* Fp;
    float* R;
    float* FiT;
    float* Gi;
    float* m;
    float* vol;
    float* J;
    float* mu;
    float* lam;
    float* mu0;    // nullable: per-particle base Lame parameters
    float* lam0;
    int* orig;     // caller index of the particle in each slot
    int* body;     // body id, -1 = ballistic
};

// The operator's per-particle records for the current step, in storage order, written by the force pass and
// read by the diagonal pass and every CR operator pass of the step, as arrays of float4 over the particles (one
// 16-byte load per group and particle):
//   base[i]       window offset of the particle's stencil (-1 outside the window);
//   w4[g * N + i] its B-spline weights and derivatives, groups wx, dwx, wy, dwy, wz, dwz (4 nodes each; the
//                 same values the other passes of the step use);
//   m4[g * N + i] the upper triangle of the particle's symmetric 9x9 map M from the gathered velocity gradient G
//                 to its force matrix vol A F^T: entry (r, c), r <= c, at position c (c + 1) / 2 + r (columns in
//                 order), 45 entries in 12 groups, the last 3 slots zero.
struct OpRec {
    int* base;
    float4* w4;
    float4* m4;
};
constexpr int kOpRecW4 = 6;
constexpr int kOpRecM = 45;
constexpr int kOpRecM4 = 12;

// Node arrays of all bodies' grids, concatenated; node vectors interleaved [3 * node + c] as the reference's
// VectorXf (Grid.cpp:244).
struct NodeArrays {
    float* mass;
    float* vel;      // P2G velocities (frame-relative)
    float* prev;     // m_prevVelocities
    float* frc;      // forces
    float* pstar;    // explicit momenta
    float* b;        // rhs
    float* vc;       // collision velocities
    float* diag;     // Jacobi preconditioner
    float* x;        // solver iterate
    float* rpc;      // preconditioned residual
    float* p;
    float* Ap;
    float* Ar;
    float* dxp;      // projected operator input
    float* df;       // force-differential accumulator
    float* vfin;     // final grid velocities (x + vc)
    float* x0;       // initial guess (kept for inspection)
    signed char* flag;  // nodeCollided
};

struct TileArrays {
    int* count;      // particles per global tile (+1 bucket for ballistic particles)
    int* start;      // exclusive scan of count
    int* list;       // non-empty tile ids
    int* listBody;   // body of each listed tile
    int* listCount;  // number of listed tiles (device scalar)
    int* sched;      // dynamic tile scheduling: [0] the next list index to take, [1] CTAs finished; both 0 between
                     // launches (the last CTA of a launch resets them)
};

struct ReduceArrays {
    double* partial;     // [numCtas * 8]
    int* counter;        // per body
    int* chunkBody;      // body of each node-chunk CTA
    int* ndone;          // bodies finished (device scalar)
    int* fp64Count;      // particles that took the FP64 SVD
};

struct SegArrays {
    int* count;    // hash buckets
    int* start;
    int* sorted;   // particle slots by bucket
    float4* xs;    // positions in bucket order
    int* rank;
    int* parent;
    int* size;
    int* minOrig;
    int* mark;     // over caller indices
    int* mrank;
    int* nbodies;  // device scalars: [0] bodies, [1] ballistic
    unsigned int* bbox;  // 6 device scalars: the particles' bounding box (order-preserving encoding)
    // The previous segmentation's spanning forest (nullable, with edgeOut null the segmentation records none):
    // every union that joined two components recorded its pair of particles by caller index, one pair per slot
    // of the root it hooked (unused slots -1).  With useEdges the links pass re-checks those pairs against
    // the current positions in place of the sampled neighbour search; the finish pass keeps the result exact.
    const int2* edgeIn;
    int2* edgeOut;
    const int* slotOf;  // caller index -> slot
    int useEdges;
};

// scan: exclusive prefix sum of n ints; tmp must hold scan_tmp_ints(n) ints; total written to *total (device)
size_t scan_tmp_ints(long long n);
void scan_exclusive(const int* in, int* out, long long n, int* tmp, int* total, cudaStream_t s);

void launch_prepare(const PartArrays& P, int N, const StepParams& sp, BodyAccum* acc, int B, int* err, cudaStream_t s);
void launch_keys(const PartArrays& P, int N, const BodyGrid* grids, int totalTiles, float h, int* key, int* rank,
                 int* tileCount, int* err, cudaStream_t s);
// the counting sort's permutation of the whole particle state: each of the n arrays of 32-bit words moves src[i] ->
// dst[tileStart[key[i]] + rank[i]] (gathered through inv, N ints of scratch: inv[d] = i)
constexpr int kPermuteMax = 64;
struct PermuteWords {
    const unsigned int* src[kPermuteMax];
    unsigned int* dst[kPermuteMax];
    int n;
};
void launch_permute_state(const int* key, const int* rank, const int* tileStart, int N, const PermuteWords& w,
                          const int* orig, int* slotOf, int* inv, cudaStream_t s);
void launch_tile_list(const int* tileCount, const BodyGrid* grids, int B, int totalTiles, int* list, int* listBody,
                      int* listCount, cudaStream_t s);
// the tile list reordered by decreasing particle count (tmp / tmpBody: scratch of the list's capacity)
void launch_tile_order(const int* cellStart, int* list, int* listBody, const int* listCount, int* tmp, int* tmpBody,
                       cudaStream_t s);
void launch_gather_user(const float* state, const int* slotOf, float* out, int N, int comps, cudaStream_t s);
void launch_scatter_user(const float* in, const int* slotOf, float* state, int N, int comps, cudaStream_t s);

// tile kernels (grid: persistent over the non-empty tile list)
// node mass and momentum sum_p w m_p (v_p - v_frame) (nd.vel; k_node_vel turns it into the velocity)
void launch_p2g_mass_momentum(const PartArrays& P, int N, const TileArrays& T, int maxTiles, const BodyGrid* grids, float h,
                              NodeArrays nd, int* err, cudaStream_t s);
// internal forces f_i -= sum_p vol P F^T grad(w_ip), added to nd.frc; the dFidXi sums of the Jacobi diagonal added
// to diagOut (nullable); also writes the step's operator records `rec` (the particles must not change between
// this pass and the operator passes that read them); withMass: also the node masses and momenta of
// launch_p2g_mass_momentum, added to nd.mass and nd.vel in the same pass
void launch_p2g_force(const PartArrays& P, int N, const TileArrays& T, int maxTiles, const BodyGrid* grids, float h,
                      NodeArrays nd, float* diagOut, OpRec rec, bool withMass, int* err, cudaStream_t s);
void launch_volumes(const PartArrays& P, int N, const TileArrays& T, int maxTiles, const BodyGrid* grids, float h,
                    NodeArrays nd, cudaStream_t s);
// operator particle pass: out -= sum_p vol A_p F^T grad(w) with A_p = dEdFDifferential(sum_i in_i grad(w_i)^T F),
// through the linear map of the step's operator records `rec`, which the force pass must have written since the
// particles last changed.  Bodies with solve.done are skipped when skipDone; procCount (nullable) accumulates the
// number of particles the launch processed.
void launch_op(const PartArrays& P, int N, const TileArrays& T, int maxTiles, const BodyGrid* grids, float h,
               const float* in, float* out, OpRec rec, const BodySolve* solve, bool skipDone, cudaStream_t s,
               unsigned long long* procCount = nullptr);
// the listed tiles of T whose stencil window holds a collided node, into C.list / C.listBody / *C.listCount
void launch_contact_tiles(const TileArrays& T, int maxTiles, const BodyGrid* grids, const signed char* flag, TileArrays C,
                          cudaStream_t s);
void launch_g2p(const PartArrays& P, int N, const TileArrays& T, int maxTiles, const BodyGrid* grids, float h, float dt,
                NodeArrays nd, cudaStream_t s);

// node kernels (grid: one CTA per node chunk)
void launch_node_mass(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, int* err, cudaStream_t s);
void launch_node_vel(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp, int* err,
                     cudaStream_t s);
void launch_node_explicit(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp,
                          BodySolve* solve, ReduceArrays R, int* err, cudaStream_t s);
void launch_node_rhs(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp,
                     BodySolve* solve, ReduceArrays R, int* err, cudaStream_t s);
void launch_node_cr_init1(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp,
                          BodySolve* solve, cudaStream_t s);
void launch_node_cr_init2(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp,
                          BodySolve* solve, ReduceArrays R, cudaStream_t s);
void launch_node_cr_update(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp,
                           BodySolve* solve, ReduceArrays R, int iter, cudaStream_t s);
void launch_node_cr_ar(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp,
                       BodySolve* solve, ReduceArrays R, int iter, cudaStream_t s);
void launch_node_cr_p(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp,
                      BodySolve* solve, ReduceArrays R, int iter, cudaStream_t s);
void launch_node_final(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const BodySolve* solve,
                       cudaStream_t s);
// debug: out = P(m P in - dt^2 DF(P in)) (op "A") given df accumulated for P in; or project only
void launch_node_project(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp,
                         const float* in, float* out, cudaStream_t s);
void launch_node_combine(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const StepParams& sp,
                         const float* dxp, const float* df, float* out, cudaStream_t s);

// learned warm start of one body's solve: node features (bf16 [G][16]) from the previous solve's history record
// H (h1) and the contact normals of the step's collided nodes, and, from the network output y ([G][3] fp32, null
// without a network), x = x0 = the guess (with the extrapolation h1 - h2 from the record before, H2, when asked)
// and the operator input P x; after the solve, the history for the next step (3 per node, all bodies)
void launch_ws_features(NodeArrays nd, const BodyGrid& g, const StepParams& sp, const mpmnn::NnNorm& nn,
                        const mpmnn::WsHist& H, void* out_bf16, cudaStream_t s);
void launch_ws_apply(NodeArrays nd, const BodyGrid& g, const StepParams& sp, const mpmnn::NnNorm& nn, const mpmnn::WsHist& H,
                     const mpmnn::WsHist& H2, const float* y, bool extrapolate, cudaStream_t s);
void launch_ws_record(NodeArrays nd, const BodyGrid* grids, const int* chunkBody, int nChunks, const mpmnn::NnNorm& nn,
                      float* hist, cudaStream_t s);

// particle kernels
void launch_plasticity(const PartArrays& P, int N, const StepParams& sp, int* fp64Count, int* err, cudaStream_t s);
void launch_advect(const PartArrays& P, int N, const StepParams& sp, cudaStream_t s);

// particle seeding from a sampled signed-distance field (the Houdini SOP's initSim): lattice of `sites` =
// dims[0] dims[1] dims[2] points at bmin + (i + 0.5) h.  Pass 1 (write = false) flags the sites inside (phi < 0)
// and scans them into pos (total: the count); pass 2 writes the particles' positions, velocities (sampled from
// the field's velocity, 0 without one) and masses.
struct SeedLattice {
    int dims[3];
    long long sites;
    double bmin[3];
    double h;
};
void launch_seed(const DevCollider& sdf, const SeedLattice& L, float mass, int* flag, int* pos, int* scanTmp, int* total,
                 float* x, float* v, float* m, bool write, cudaStream_t s);

// body segmentation (Sim::calculateBodies)
void launch_segment(const PartArrays& P, int N, float h, SegArrays S, int hashBits, int* scanTmp, int* err,
                    cudaStream_t s);

}  // namespace mpm

/*
 * mpm_gpu.h — C-ABI of the B200 (sm_100a) implicit MPM snow time step.
 *
 * This is the drop-in boundary below the reference's MpmSim C++ API (davidsminor/mpmsnow).  Each entry point
 * names the reference interface it replaces, by file:line in the reference project.  Plain pointers and sizes
 * only; all arrays are host memory unless a name says _device.  Vectors are 3 floats per particle, matrices
 * 9 floats per particle in row-major order (element (r, c) at 3 r + c).
 *
 * Threading: one host thread drives a handle at a time (the reference's Sim is not re-entrant either).
 * Errors: every call returns an mpm_status; the message that the reference throws as std::runtime_error is
 * available from mpm_last_error().  There is no CPU fallback: without a CUDA device mpm_create fails.
 */
#ifndef MPM_GPU_H
#define MPM_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPM_ABI_VERSION 2

typedef enum mpm_status {
    MPM_OK = 0,
    MPM_ERR_INVALID_ARGUMENT = 1,
    MPM_ERR_CUDA = 2,
    MPM_ERR_NO_DEVICE = 3,
    MPM_ERR_NAN_MASSES = 4,             /* "nans in splatted masses!"            Grid.cpp:239 */
    MPM_ERR_NAN_VELOCITIES = 5,         /* "nans in splatted velocities!"        Grid.cpp:258 */
    MPM_ERR_NAN_MOMENTA = 6,            /* "nan in explicit momenta!"            Grid.cpp:683, 1000 */
    MPM_ERR_NAN_STRESS = 7,             /* "nans in dEnergyDensitydF matrix!"    SnowConstitutiveModel.cpp:212 */
    MPM_ERR_INFINITE_HARDNESS = 8,      /* "infinite hardness!!!"                SnowConstitutiveModel.cpp:109 */
    MPM_ERR_NAN_PARTICLE_VELOCITY = 9,  /* "nans in particle velocity data!"     Sim.cpp:156 */
    MPM_ERR_GRID_TOO_BIG = 10,          /* "grid is too big"                     Grid.cpp:212 */
    MPM_ERR_UNKNOWN_VARIABLE = 11,      /* "Material point data has no variable named '<name>'"  MaterialPointData.inl:23 */
    MPM_ERR_WRONG_SIZE = 12,            /* element count does not match the variable */
    MPM_ERR_UNSUPPORTED = 13,           /* a dimension outside 1-3, another shape function, too many colliders */
    MPM_ERR_CANCELLED = 14,             /* the cancel callback returned non-zero (Sim.cpp:107-111) */
    MPM_ERR_INTERNAL = 15,
    MPM_ERR_OUT_OF_MEMORY = 16,
    MPM_ERR_TOO_MANY_PARTICLES = 17     /* more particles than mpm_calculate_bodies_noalloc_max() */
} mpm_status;

typedef struct mpm_sim mpm_sim;

enum { MPM_COLLIDER_PLANE = 0, MPM_COLLIDER_CYLINDER = 1, MPM_COLLIDER_GRID = 2 };

/* CollisionObject (CollisionObject.h:12-31).  PLANE = CollisionPlane (CollisionPlane.h:12-35):
 * phi = c0 x + c1 y + c2 z + c3, grad = (c0, c1, c2), constant velocity (setV).
 * CYLINDER (no reference counterpart): solid vertical cylinder, coeffs = (cx, cz, radius, 0),
 * phi = |(x - cx, z - cz)| - radius, grad = (x - cx, 0, z - cz).
 * GRID replaces the Houdini plugin's VDBCollisionObject (houdiniPlugin/VDBCollisionObject.cpp:11-37): phi sampled
 * on a dense grid at coeffs[0..2] + coeffs[3] (i, j, k), i < grid_dims[0] (x fastest), and optionally a sampled
 * velocity (3 floats per sample; NULL = at rest).  phi and the velocity are trilinear between samples, grad is
 * the gradient of the trilinear phi; outside the sampled box there is no collider.  The samples are copied to the
 * device when the descriptor is passed (mpm_create, mpm_set_collider). */
typedef struct mpm_collider {
    int kind;
    float coeffs[4];
    float velocity[3];
    float friction;   /* coulombFriction() */
    int sticky;       /* sticky() */
    int grid_dims[3];              /* GRID: samples per axis, each >= 2 */
    const float* grid_phi;         /* GRID: host, grid_dims[0] * grid_dims[1] * grid_dims[2] floats */
    const float* grid_velocity;    /* GRID: host, 3 per sample, or NULL */
} mpm_collider;

/* Arguments of the reference's Sim constructor (Sim.h:32-41) and of SnowConstitutiveModel
 * (SnowConstitutiveModel.h:13-18); gravity fields are GravityField (GravityField.h:10-24), 3 floats each. */
typedef struct mpm_scene_desc {
    float grid_size;
    int dimension;                /* 3, or 2 / 1: grids span axes below it (Grid.cpp:180-207, 1112, 1144-1158) */
    int shape_function;           /* 0 = CubicBsplineShapeFunction */
    float youngs_modulus;
    float poisson_ratio;
    float hardening;
    float compressive_strength;
    float tensile_strength;
    int num_colliders;
    const mpm_collider* colliders;
    int num_gravity_fields;
    const float* gravity;
    int device;                   /* CUDA device ordinal */
} mpm_scene_desc;

/* SquareMagnitudeTermination(maxIters, tolError) (SquareMagnitudeTermination.h:14). */
typedef struct mpm_solve_params {
    int max_iterations;
    float tolerance;
} mpm_solve_params;

typedef struct mpm_step_stats {
    int num_bodies;
    int num_ballistic;
    int max_iterations_used;
    int total_iterations;
    int iterations[64];           /* per body: iteration index at which its solve returned */
    double b_norm2[64];
    double r_norm2[64];
    int exit_reason[64];          /* 0 termination criterion, 1 |b| = 0, 2 <Ap, M^-1 Ap> = 0, 3 rz = 0 */
    int fp64_svd_particles;       /* particles that took the FP64 SVD fallback this step */
    int kernel_launches;          /* kernels launched by this step */
} mpm_step_stats;

/* TerminationCriterion::cancelled (TerminationCriterion.h:15): polled after the grid solve. */
typedef int (*mpm_cancel_fn)(void* ctx);
/* LinearSolver::Debug (LinearSolver.h:17-21): called once per solver iteration with body's iterate x
 * (3 floats per node of that body's grid, frame-relative, projected).  Setting it synchronises every iteration. */
typedef void (*mpm_iterate_fn)(void* ctx, int body, int iteration, const float* x, size_t count);

int mpm_abi_version(void);
const char* mpm_status_string(mpm_status s);
const char* mpm_last_error(const mpm_sim* sim);

/* Sim::Sim (Sim.cpp:17-50): positions x (3n), masses (n); v = 0, F = I, bodies, particle volumes. */
mpm_status mpm_create(const mpm_scene_desc* desc, size_t n, const float* x, const float* masses, mpm_sim** out);
/* ~Sim */
void mpm_destroy(mpm_sim* sim);

/* Sim::advance(dt, SquareMagnitudeTermination) (Sim.cpp:57-134). */
mpm_status mpm_step(mpm_sim* sim, float dt, const mpm_solve_params* solve, mpm_step_stats* stats);
/* Sim::advance with cancellation and the Debug hook.  stop_phase: 0 full step; 1 stop once every body's rhs
 * and preconditioner are built; 2 stop after every body's solve (particles untouched in both). */
mpm_status mpm_step_ex(mpm_sim* sim, float dt, const mpm_solve_params* solve, int stop_phase, mpm_cancel_fn cancel,
                       void* cancel_ctx, mpm_iterate_fn iterate, void* iterate_ctx, mpm_step_stats* stats);

/* Sim::particleData() / MaterialPointData::variable<T>(name) (MaterialPointData.h:20-34).
 * Names: p v (3), F Fp FinvTrans R Ginv (9), m volume J mu lambda (1), and the per-particle base Lame
 * parameters mu0 lambda0 (1; setting them makes the hardening rule scale them instead of the scalars).
 * count is the number of floats; arrays are in the caller's particle order. */
size_t mpm_num_particles(const mpm_sim* sim);
mpm_status mpm_variable_info(const mpm_sim* sim, const char* name, int* components);
mpm_status mpm_get_variable(mpm_sim* sim, const char* name, float* dst, size_t count);
mpm_status mpm_set_variable(mpm_sim* sim, const char* name, const float* src, size_t count);
/* the same with device pointers (no host staging) */
mpm_status mpm_get_variable_device(mpm_sim* sim, const char* name, float* dst_device, size_t count);
mpm_status mpm_set_variable_device(mpm_sim* sim, const char* name, const float* src_device, size_t count);
/* Body partition of Sim::calculateBodies (Sim.cpp:136-203): body id per particle, -1 = ballistic. */
mpm_status mpm_get_bodies(mpm_sim* sim, int* body_of_particle, int* num_bodies, int* num_ballistic);

/* The CUDA stream a handle launches on (a cudaStream_t), for callers that order their own work after a step.
 * A step also uses a second stream of the handle for part of its work and joins it into this one before it
 * returns. */
void* mpm_get_stream(mpm_sim* sim);

/* Replaces collider `index` (of the scene's colliders) between steps: CollisionPlane::setCoeffs / setV
 * (CollisionPlane.cpp:46-56), or a Houdini cook's new collision VDB (SOP_MPMSim.cpp:298-326) as a GRID
 * collider, whose samples are copied to the device here. */
mpm_status mpm_set_collider(mpm_sim* sim, int index, const mpm_collider* collider);
/* Replaces the whole collider set between steps (at most 16): the Houdini SOP rebuilds its collision objects
 * from its inputs at every cook (SOP_MPMSim.cpp:292-326). */
mpm_status mpm_set_colliders(mpm_sim* sim, int num_colliders, const mpm_collider* colliders);

/* The Houdini SOP's particle seeding (SOP_MPMSim.cpp:168-214) on GPU `device`: lattice sites
 * bbox_min + (i + 0.5) h, ceil((bbox_max - bbox_min) / h) per axis, in the SOP's loop order (x slowest, z
 * fastest); a site where the GRID collider descriptor `sdf` has phi < 0 becomes a particle of mass
 * density h^3 with the velocity sampled from sdf's grid_velocity (0 without one).  Writes *count particles to the
 * host arrays x_out, v_out (3 each) and m_out; MPM_ERR_WRONG_SIZE (with *count set) when capacity is smaller. */
mpm_status mpm_seed_particles(const mpm_collider* sdf, const float* bbox_min, const float* bbox_max, float h,
                              float density, int device, float* x_out, float* v_out, float* m_out, size_t capacity,
                              size_t* count);

/* --- measurement (no reference counterpart: the reference has no instrumentation beyond stderr) --------- */
/* Per-phase device time measured with CUDA events recorded on the launching stream around each launch, and
 * the particles / nodes each phase processed.  Enabling clears the record; it adds two event records per
 * launch.  mpm_profile_read fills up to max entries and returns how many phases there are. */
typedef struct mpm_phase_profile {
    char name[32];
    int launches;
    double total_ms;
    double particles;   /* particle visits over all launches (operator launches count only unfinished bodies) */
    double nodes;       /* grid nodes over all launches */
} mpm_phase_profile;
mpm_status mpm_profile_enable(mpm_sim* sim, int enable);
int mpm_profile_read(mpm_sim* sim, mpm_phase_profile* out, int max);

/* --- no-allocation body segmentation -------------------------------------------------------------------- */
/* No counterpart in the reference.  The body segmentation this library runs at the end of every step
 * (connected components of |x_i - x_j| < grid_size, one-particle components ballistic, bodies numbered in the
 * order of their smallest particle index), for callers that cannot allocate device memory when they need it:
 * code recording a CUDA graph (cudaMalloc cannot be captured), hosts that own the GPU's memory through their
 * own pool, latency-critical paths that cannot take cudaMalloc's implicit synchronisation.  It allocates
 * nothing: its working memory is one fixed 16 MB device array in the library image, held by every GPU that
 * loads the library until exit, which limits a call to mpm_calculate_bodies_noalloc_max() = 262,144
 * particles (more return MPM_ERR_TOO_MANY_PARTICLES).
 * x_device: 3 n floats, component-major (all x, then all y, then all z); body_device: n ints, -1 = ballistic;
 * counts_device: 2 ints (bodies, ballistic particles).  All device memory on the current device; the work is
 * queued on `stream` (a cudaStream_t, 0 = legacy default stream) and the outputs are valid once it completes.
 * The first call on a device resolves the array's address on that device; make it before any stream capture.
 * Calls share the array: calls that overlap on the GPU race and must be serialised. */
int mpm_calculate_bodies_noalloc_max(void);
mpm_status mpm_calculate_bodies_noalloc(const float* x_device, size_t n, float grid_size, int* body_device,
                                        int* counts_device, void* stream);

/* --- learned warm start ----------------------------------------------------------------------------------- */
/* No counterpart in the reference: a 4-layer 3x3x3 convolutional network replaces the uniform initial guess of
 * the implicit solve (Grid.cpp:911-947).  Conjugate residuals still runs to the same relative residual from the
 * predicted guess, so a poor prediction costs iterations, never accuracy.
 * Layers (input -> output channels, zero-padded to the widths in brackets): 16 -> 32 ReLU -> 32 ReLU -> 32 ReLU
 * -> 3 [16].  weights: fp32, the four layers back to back, each [27][cin_pad][cout_pad] with tap
 * t = 9 (dz + 1) + 3 (dy + 1) + (dx + 1); biases: fp32 32 + 32 + 32 + 3.
 * Node features: mass / (density h^3) and, on heavy nodes (at least light_mass of that unit), the explicit
 * velocity p* / m and dt (f - m g) / m in units of h/dt, the relative stiffness (d - m) / m of the Jacobi
 * diagonal d, the history h1 (below) in units of h/dt, and the contact normal (the collider's outward normal on
 * a node that the explicit update collided with one object, 0 elsewhere), times feature_scale.
 * History (use_history >= 1): after each solve, per node with mass, x - p* / m (heavy) or x (light); the last two
 * records (h1 of the previous step, h2 of the one before) are mapped onto the current grid by the integer shifts
 * of the grid origins.  The guess on a node with mass is
 *   heavy: p* / m + h1 + (h/dt) y output_scale      light: h1, or p* / m without one
 * and 0 on nodes without mass; y is the network output (0 when weights is NULL: the guess is then p* / m and
 * the history alone).  use_history = 2 without a network adds the linear extrapolation h1 - h2 on heavy nodes. */
typedef struct mpm_warm_start {
    const float* weights;      /* host, MPM_WARM_START_WEIGHTS floats, or NULL (no network) */
    const float* biases;       /* host, MPM_WARM_START_BIASES floats, or NULL with weights */
    float feature_scale[16];
    float output_scale;
    float light_mass;          /* heavy/light threshold, in units of density h^3 */
    float density;             /* kg/m^3 of the mass unit */
    int min_nodes;             /* bodies whose grid has fewer nodes keep the uniform guess */
    int use_history;           /* 0 none; 1 record and use the history; 2 as 1, plus the extrapolation (no network) */
} mpm_warm_start;
#define MPM_WARM_START_WEIGHTS (27 * (16 * 32 + 32 * 32 + 32 * 32 + 32 * 16))
#define MPM_WARM_START_BIASES (32 + 32 + 32 + 3)
/* Installs (copies) the model into the handle and clears the history; NULL turns the warm start off (the
 * reference's guess). */
mpm_status mpm_set_warm_start(mpm_sim* sim, const mpm_warm_start* model);

/* Training kernels of the network (device pointers; work queued on `stream`, a cudaStream_t).
 * Activations are channels-last bf16 [batch][nz][ny][nx][c_pad]; c_pad 16 or 32; zero padding at the volume
 * border.  `err` (device int) gets bit 0 if a tensor-core wait timed out. */
/* fp32 weights [27][cin][cout] -> bf16 packs for the forward ([27][cin_pad/8][cout_pad][8]) and the
 * backward-data ([27][cout_pad/8][cin_pad][8]) convolution; either output may be NULL. */
mpm_status mpm_nn_pack_weights(const float* w, int cin, int cout, int cin_pad, int cout_pad, void* packed_fwd,
                               void* packed_bwd, void* stream);
/* y = act(conv(x) + bias), act = ReLU if relu; channels >= cout are written as 0.  flip = 1: backward data
 * (x = dL/dy of the layer, packed = its backward-data pack, cin_pad/cout_pad = the layer's cout_pad/cin_pad),
 * and mask_act (the layer input's activation, may be NULL) zeroes the outputs where it is not positive.
 * Outputs: y_bf16 [...][cout_pad] and/or y_f32 with row stride y_f32_stride (first cout channels). */
mpm_status mpm_nn_conv3d(const void* x, int cin_pad, const void* packed, const float* bias, int cout, int cout_pad, int relu,
                         int flip, const void* mask_act, void* y_bf16, float* y_f32, int y_f32_stride, int nx, int ny, int nz,
                         int batch, int* err, void* stream);
/* dw[27][cin_pad][cout_pad] += sum over voxels v and taps t of x[v + off(t)][ci] dy[v][co] (fp32, accumulated). */
mpm_status mpm_nn_conv3d_wgrad(const void* x, int cin_pad, const void* dy, int cout_pad, float* dw, int nx, int ny, int nz,
                               int batch, int* err, void* stream);
/* db[c] += sum_v dy[v][c] for c < cout. */
mpm_status mpm_nn_bias_grad(const void* dy, int cout_pad, int cout, long long nvox, float* db, void* stream);
/* Adam (bias-corrected moments, `step` counts from 1) on fp32 weights; the gradient used is g + weight_decay w. */
mpm_status mpm_nn_adam(float* w, const float* g, float* m, float* v, int n, float lr, float beta1, float beta2, float eps,
                       int step, float weight_decay, void* stream);
/* Node features (see above) of n nodes from masses (1 per node), explicit momenta, forces, Jacobi diagonal, the
 * history record h1 and the contact normals (3 per node; mpm_debug_grid_get's "explicitMomenta", "forces",
 * "diag"; the history may be NULL, NaN marks a node without one; normals may be NULL, all 0): bf16 [n][16]. */
mpm_status mpm_nn_features(const float* mass, const float* pstar, const float* force, const float* diag,
                           const float* history, const float* normals, long long n, float dt, float h, float density,
                           float light_mass, const float* gravity3, const float* feature_scale16, void* out_bf16,
                           void* stream);
/* loss += sum_v w_v |y_v - t_v|^2 inv_wsum over the first 3 channels; dy_bf16 [n][16] = its gradient. */
mpm_status mpm_nn_mse(const float* y, int y_stride, const float* target, const float* weight, long long n, float inv_wsum,
                      void* dy_bf16, double* loss, void* stream);

/* --- parity / inspection entry points ------------------------------------------------------------------ */
/* Grid of body b from the last mpm_step(_ex): m_min, m_n (Grid.h:207-210), frame velocity, particle count. */
mpm_status mpm_debug_grid_info(mpm_sim* sim, int body, float* min3, int* n3, float* frame_velocity3, int* num_particles);
/* Node arrays of body b in the reference's node order idx = i + n0 (j + n1 k) (Grid.cpp:1083-1086): masses,
 * nodeCollided (as float) (1 per node); prevVelocities, forces, explicitMomenta, rhs, vc, diag, x0, solution,
 * velocities (3 per node). */
mpm_status mpm_debug_grid_get(mpm_sim* sim, int body, const char* name, float* dst, size_t count);
/* Apply to a node vector of body b: "A" = ImplicitUpdateMatrix::multVector (Grid.cpp:749-771), "DF" =
 * Grid::calculateForceDifferentials (Grid.cpp:620-632).  Valid after a step stopped at phase 1 or 2. */
mpm_status mpm_debug_apply(mpm_sim* sim, int body, const char* op, const float* in, float* out, size_t count, float dt);
/* Per particle (caller order): body id, the stencil's cell int(floor((p - m_min) / h)) (Grid.cpp:1114-1115)
 * and the reference's voxel floor(p / 4h) (Grid.cpp:373-374), from the last step's grids; -1 for ballistic. */
mpm_status mpm_debug_particle_cells(mpm_sim* sim, int* body, int* cell3, int* voxel3);

#ifdef __cplusplus
}
#endif
#endif /* MPM_GPU_H */

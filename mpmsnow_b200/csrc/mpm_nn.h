// The learned warm start's network: a 4-layer 3x3x3 convolution over a body's grid nodes (channels-last bf16
// activations, fp32 accumulation on the tensor cores), shared by the training entry points and the step.
//
// Input channels of a node (16): grid mass in units of density h^3 and, on heavy nodes (mass at least
// light_mass of that unit), the explicit velocity p*/m and the velocity increment of the internal forces
// dt (f - m g)/m, both in units of h/dt, the relative stiffness (d - m)/m of the Jacobi diagonal d of the
// implicit matrix, the previous step's correction h1 and its change since the step before, h1 - h2 (below), in
// units of h/dt; each multiplied by a per-channel scale of the model.  On light nodes (the thin shell the
// B-spline stencil adds around the material) p*/m is dominated by round-off and the solved velocity is barely
// determined, so they get no velocity input and no network correction.
//
// History: after each solve the step records, per node with mass, x - p*/m (heavy) or x (light); the next
// step maps the last two records (h1 of the previous step, h2 of the one before) onto its own grid by the
// integer node shifts between the grids' origins.  The guess is
//   heavy node: p*/m + h1 + (h/dt) out_scale y      light node: h1, or p*/m without one
// (0 where there is no mass), y being the network output (0 without a network); without a network the guess can
// instead extrapolate linearly, p*/m + h1 + (h1 - h2) on heavy nodes.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace mpmnn {

constexpr int kLayers = 4;
constexpr int kCinPad[kLayers] = {16, 32, 32, 32};
constexpr int kCoutPad[kLayers] = {32, 32, 32, 16};
constexpr int kCout[kLayers] = {32, 32, 32, 3};
constexpr int kFeat = 16;

struct NnNorm {
    float inv_mass_unit;   // 1 / (density h^3)
    float inv_vel_unit;    // dt / h
    float vel_unit;        // h / dt
    float dt;
    float gdt[3];          // dt times the sum of the gravity fields
    float feat_scale[kFeat];
    float out_scale;
    float light_mass;      // in units of density h^3
};

inline int layer_weight_count(int l) { return 27 * kCinPad[l] * kCoutPad[l]; }

// the history of the previous solve of one body, mapped onto the current grid
struct WsHist {
    const float* h;      // 3 per node in the previous concatenated layout (NaN = no mass there); null = none
    long long nodeOff;   // the body's first node there
    int n[3];            // the body's previous grid size
    int off[3];          // current node (i, j, k) is previous node (i, j, k) + off
};

// history at current local node l of a grid of size n (false where there is none)
__device__ __forceinline__ bool hist_at(const WsHist& H, const int n[3], long long l, float out[3]) {
    if (!H.h) return false;
    const int i = (int)(l % n[0]);
    const long long r = l / n[0];
    const int j = (int)(r % n[1]), k = (int)(r / n[1]);
    const int pi = i + H.off[0], pj = j + H.off[1], pk = k + H.off[2];
    if (pi < 0 || pj < 0 || pk < 0 || pi >= H.n[0] || pj >= H.n[1] || pk >= H.n[2]) return false;
    const long long q = H.nodeOff + pi + (long long)H.n[0] * (pj + (long long)H.n[1] * pk);
    out[0] = H.h[3 * q];
    out[1] = H.h[3 * q + 1];
    out[2] = H.h[3 * q + 2];
    return !isnan(out[0]);
}

// features of one node from its mass, explicit momentum p*, force f (gravity included), Jacobi diagonal d, the
// history record hv (hasHist) and the contact normal nrm (the collider's outward normal on a node the explicit
// update collided with one object, 0 elsewhere)
__device__ __forceinline__ void node_features(float m, const float ps[3], const float f[3], const float d[3], bool hasHist,
                                              const float hv[3], const float nrm[3], const NnNorm& nn,
                                              float out[kFeat]) {
    for (int k = 0; k < kFeat; ++k) out[k] = 0.f;
    const float mh = m * nn.inv_mass_unit;
    if (m > 0.f) out[0] = mh * nn.feat_scale[0];
    if (m > 0.f && mh >= nn.light_mass) {
        const float inv = 1.f / m;
        for (int a = 0; a < 3; ++a) {
            out[1 + a] = ps[a] * inv * nn.inv_vel_unit * nn.feat_scale[1 + a];
            out[4 + a] = (nn.dt * f[a] * inv - nn.gdt[a]) * nn.inv_vel_unit * nn.feat_scale[4 + a];
            out[7 + a] = (d[a] - m) * inv * nn.feat_scale[7 + a];
            out[10 + a] = hasHist ? hv[a] * nn.inv_vel_unit * nn.feat_scale[10 + a] : 0.f;
            out[13 + a] = nrm[a] * nn.feat_scale[13 + a];
        }
    }
}

// the guess at one node (see the history note above); y may be null (no network); extrapolate adds h1 - h2 on
// heavy nodes
__device__ __forceinline__ void node_guess(float m, const float ps[3], const float* y, bool hasHist, const float hv[3],
                                           bool hasHist2, const float hv2[3], bool extrapolate, const NnNorm& nn,
                                           float x[3]) {
    if (!(m > 0.f)) {
        x[0] = x[1] = x[2] = 0.f;
        return;
    }
    const bool heavy = m * nn.inv_mass_unit >= nn.light_mass;
    const float s = nn.out_scale * nn.vel_unit;
    for (int a = 0; a < 3; ++a) {
        const float base = (heavy || !hasHist) ? ps[a] / m : 0.f;
        const float ext = (heavy && extrapolate && hasHist && hasHist2) ? hv[a] - hv2[a] : 0.f;
        x[a] = base + (hasHist ? hv[a] : 0.f) + ext + ((heavy && y) ? s * y[a] : 0.f);
    }
}

// y = act(conv3x3x3(x) + bias) over nvox = nx ny nz batch voxels (see mpm_nn_conv3d in include/mpm_gpu.h), by the
// halo-tiled kernel over output blocks of 8 x 16 x 1 voxels; block_list (device, may be NULL = every block) with
// its length in block_count_dev restricts the work to those blocks
cudaError_t conv3d_tiled(const void* x, int cin_pad, const void* packed, const float* bias, int cout, int cout_pad, int relu,
                         int flip, const void* mask_act, void* y_bf16, float* y_f32, int y_f32_stride, int nx, int ny,
                         int nz, int batch, const int* block_list, const int* block_count_dev, int* err, cudaStream_t s);
long long tile_blocks(int nx, int ny, int nz);
// per-layer output blocks of the warm start's inference: lists[l * list_stride ...] (counts[l] entries) holds the
// blocks within Chebyshev distance layers - 1 - l of a node whose mass is at least heavy_mass; scratch holds
// 2 nx ny nz bytes; list_stride >= tile_blocks(nx, ny, nz)
cudaError_t layer_blocks(const float* mass, float heavy_mass, int nx, int ny, int nz, int layers, unsigned char* scratch,
                         int* lists, long long list_stride, int* counts, cudaStream_t s);
cudaError_t pack_weights(const float* w, int cin, int cout, int cin_pad, int cout_pad, void* packed_fwd, void* packed_bwd,
                         cudaStream_t s);

}  // namespace mpmnn

// The learned warm start's network: a 4-layer 3x3x3 convolution over a body's grid nodes (channels-last bf16
// activations, fp32 accumulation on the tensor cores), shared by the training entry points and the step.
//
// Input channels of a node (7, padded to 16): grid mass in units of density h^3, the explicit velocity p*/m and
// the velocity increment of the internal forces dt (f - m g)/m, both in units of h/dt; each multiplied by a
// per-channel scale of the model.  Output (3, padded to 16): the implicit correction x - p*/m of the solved
// grid velocity, in units of out_scale h/dt.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace mpmnn {

constexpr int kLayers = 4;
constexpr int kCinPad[kLayers] = {16, 32, 32, 32};
constexpr int kCoutPad[kLayers] = {32, 32, 32, 16};
constexpr int kCout[kLayers] = {32, 32, 32, 3};
constexpr int kFeat = 7;

struct NnNorm {
    float inv_mass_unit;   // 1 / (density h^3)
    float inv_vel_unit;    // dt / h
    float vel_unit;        // h / dt
    float dt;
    float gdt[3];          // dt times the sum of the gravity fields
    float feat_scale[kFeat];
    float out_scale;
};

inline int layer_weight_count(int l) { return 27 * kCinPad[l] * kCoutPad[l]; }

// features of one node from its mass, explicit momentum p* and force f (gravity included): out[0..6]
__device__ __forceinline__ void node_features(float m, const float ps[3], const float f[3], const NnNorm& nn,
                                              float out[kFeat]) {
    if (m > 0.f) {
        const float inv = 1.f / m;
        out[0] = m * nn.inv_mass_unit * nn.feat_scale[0];
        for (int a = 0; a < 3; ++a) {
            out[1 + a] = ps[a] * inv * nn.inv_vel_unit * nn.feat_scale[1 + a];
            out[4 + a] = (nn.dt * f[a] * inv - nn.gdt[a]) * nn.inv_vel_unit * nn.feat_scale[4 + a];
        }
    } else {
        for (int k = 0; k < kFeat; ++k) out[k] = 0.f;
    }
}

// y = act(conv3x3x3(x) + bias) over nvox = nx ny nz batch voxels; see mpm_nn_conv3d in include/mpm_gpu.h
cudaError_t conv3d(const void* x, int cin_pad, const void* packed, const float* bias, int cout, int cout_pad, int relu,
                   int flip, const void* mask_act, void* y_bf16, float* y_f32, int y_f32_stride, int nx, int ny, int nz,
                   int batch, int* err, cudaStream_t s);
cudaError_t pack_weights(const float* w, int cin, int cout, int cin_pad, int cout_pad, void* packed_fwd, void* packed_bwd,
                         cudaStream_t s);

}  // namespace mpmnn

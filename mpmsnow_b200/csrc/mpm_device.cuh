// Device-side math of the implicit MPM snow step: cubic B-spline stencils, collision objects, the snow
// constitutive model and its linearisation, and the per-particle 3x3 SVD / polar plasticity update.
// Matrices are row-major float[9] (element (r, c) at 3 r + c).
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "mpm_types.h"

namespace mpm {

// ------------------------------------------------------------------------------------------------
// Cubic B-spline — CubicBsplineShapeFunction.cpp:11-47, same pieces and branch points.  The outer piece
// (1 <= |x| < 2) is evaluated as (2 - |x|)^3 / 6 rather than the reference's Horner form
// ((-|x| / 6 + 1) |x| - 2) |x| + 4/3: the same polynomial, but the Horner form cancels to within ~1e-7 of zero
// near |x| = 2, so in FP32 the weights of a stencil's tail nodes (true values down to ~1e-10) are rounding noise,
// as are the masses of nodes that only tails reach.  That noise roughly triples the CR iterations to a 1e-5
// residual and is most of the FP32 step's deviation from FP64; 2 - |x| is exact in FP32 (Sterbenz), so the
// form below keeps full relative precision.
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ float bspline_w(float x) {
    float ax = fabsf(x);
    if (ax < 1.0f) return (0.5f * ax - 1.0f) * ax * ax + 2.0f / 3;
    if (ax < 2.0f) {
        const float y = 2.0f - ax;
        return y * y * y * (1.0f / 6);
    }
    return 0.0f;
}
__device__ __forceinline__ float bspline_dw(float x) {
    float s = 1.0f;
    if (x < 0.0f) { x = -x; s = -1.0f; }
    float r;
    if (x < 1.0f) r = x * (1.5f * x - 2.0f);
    else if (x < 2.0f) { float y = x - 2.0f; r = -0.5f * y * y; }
    else r = 0.0f;
    return s * r;
}

// Stencil of one particle in one grid of n nodes per axis — ShapeFunctionIterator::initialize, Grid.cpp:1105-1136.
// The cell index uses separately rounded subtract and divide, so it is bit-identical to the reference's
// int(floor((p - m_min) / h)); `cell` is that index, the stencil's first node is cell - 1.
// An axis with a single node (a grid of dimension < 3, Grid.cpp:203-207) has no stencil along it: the reference's
// iterator visits that axis's node 0 with weight 1 and no derivative (Grid.cpp:1095-1100, 1112, 1144-1158).  Here
// it is cell 0, so node 0 is stencil position 1, with weights (0, 1, 0, 0) and derivatives 0.
struct Stencil {
    int cell[3];
    float w[3][4];
    float dw[3][4];
};
__device__ __forceinline__ void stencil_cells(const float p[3], const float mn[3], const int n[3], float h, int cell[3],
                                              float frac[3]) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (n[d] == 1) {
            cell[d] = 0;
            frac[d] = 0.f;
            continue;
        }
        float f = __fdiv_rn(__fsub_rn(p[d], mn[d]), h);
        float fl = floorf(f);
        cell[d] = (int)fl;
        frac[d] = __fsub_rn(f, (float)cell[d]);
    }
}
// weight and derivative / h of stencil position q (0..3) along an axis, `single` for a one-node axis
__device__ __forceinline__ float stencil_w(bool single, int q, float frac) {
    return single ? (q == 1 ? 1.0f : 0.0f) : bspline_w((float)(q - 1) - frac);
}
__device__ __forceinline__ float stencil_dw(bool single, int q, float frac, float h) {
    return single ? 0.0f : __fdiv_rn(bspline_dw((float)(q - 1) - frac), h);
}
template <bool DERIV>
__device__ __forceinline__ void stencil_eval(const float p[3], const float mn[3], const int n[3], float h, Stencil& s) {
    float frac[3];
    stencil_cells(p, mn, n, h, s.cell, frac);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            s.w[d][i] = stencil_w(n[d] == 1, i, frac[d]);
            if (DERIV) s.dw[d][i] = stencil_dw(n[d] == 1, i, frac[d], h);
        }
    }
}

// ------------------------------------------------------------------------------------------------
// Collision objects — CollisionObject.cpp:19-96, CollisionPlane.cpp:23-56; kind 1 = vertical cylinder; kind 2 =
// a sampled signed-distance grid with an optional sampled velocity (the GPU form of VDBCollisionObject,
// houdiniPlugin/VDBCollisionObject.cpp:11-37: phi, its gradient and the velocity sampled at x).
// phi and the normal use separately rounded operations, as the oracle does, so the in/out decision at a
// grid node is the same bit for bit.
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ float lerp_rn(float a, float b, float t) { return __fadd_rn(a, __fmul_rn(t, __fsub_rn(b, a))); }

// Trilinear sampling of a grid collider at x: the cell (i0, j0, k0) and in-cell fractions t; false outside the
// sampled box (where the collider has no surface: phi is +infinity there).
__device__ __forceinline__ bool grid_cell(const DevCollider& c, const float x[3], int i0[3], float t[3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float u = __fdiv_rn(__fsub_rn(x[a], c.c[a]), c.c[3]);
        if (!(u >= 0.0f) || u > (float)(c.n[a] - 1)) return false;
        const int i = min((int)floorf(u), c.n[a] - 2);
        i0[a] = i;
        t[a] = __fsub_rn(u, (float)i);
    }
    return true;
}
// the 8 corner values of field f (stride comps, component k) around cell i0
__device__ __forceinline__ void grid_corners(const DevCollider& c, const float* f, int comps, int k, const int i0[3], float v[8]) {
    const long long sx = comps, sy = (long long)comps * c.n[0], sz = sy * c.n[1];
    const float* b = f + i0[0] * sx + i0[1] * sy + i0[2] * sz + k;
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = __ldg(b + (q & 1) * sx + ((q >> 1) & 1) * sy + (q >> 2) * sz);
}
// trilinear value: x first, then y, then z
__device__ __forceinline__ float trilinear(const float v[8], const float t[3]) {
    const float x00 = lerp_rn(v[0], v[1], t[0]), x10 = lerp_rn(v[2], v[3], t[0]);
    const float x01 = lerp_rn(v[4], v[5], t[0]), x11 = lerp_rn(v[6], v[7], t[0]);
    return lerp_rn(lerp_rn(x00, x10, t[1]), lerp_rn(x01, x11, t[1]), t[2]);
}
// gradient of the trilinear interpolant (per unit length)
__device__ __forceinline__ void trilinear_grad(const float v[8], const float t[3], float h, float g[3]) {
    const float dx00 = __fsub_rn(v[1], v[0]), dx10 = __fsub_rn(v[3], v[2]), dx01 = __fsub_rn(v[5], v[4]),
                dx11 = __fsub_rn(v[7], v[6]);
    g[0] = __fdiv_rn(lerp_rn(lerp_rn(dx00, dx10, t[1]), lerp_rn(dx01, dx11, t[1]), t[2]), h);
    const float x00 = lerp_rn(v[0], v[1], t[0]), x10 = lerp_rn(v[2], v[3], t[0]);
    const float x01 = lerp_rn(v[4], v[5], t[0]), x11 = lerp_rn(v[6], v[7], t[0]);
    g[1] = __fdiv_rn(lerp_rn(__fsub_rn(x10, x00), __fsub_rn(x11, x01), t[2]), h);
    g[2] = __fdiv_rn(__fsub_rn(lerp_rn(x01, x11, t[1]), lerp_rn(x00, x10, t[1])), h);
}

__device__ __forceinline__ float coll_phi(const DevCollider& c, const float x[3]) {
    if (c.kind == 0)
        return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(c.c[0], x[0]), __fmul_rn(c.c[1], x[1])), __fmul_rn(c.c[2], x[2])),
                         c.c[3]);
    if (c.kind == 2) {
        int i0[3];
        float t[3], v[8];
        if (!grid_cell(c, x, i0, t)) return __int_as_float(0x7f800000);
        grid_corners(c, c.phi, 1, 0, i0, v);
        return trilinear(v, t);
    }
    float dx = __fsub_rn(x[0], c.c[0]), dz = __fsub_rn(x[2], c.c[1]);
    return __fsub_rn(__fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dz, dz))), c.c[2]);
}
__device__ __forceinline__ void coll_normal(const DevCollider& c, const float x[3], float n[3]) {
    float g0, g1, g2;
    if (c.kind == 0) { g0 = c.c[0]; g1 = c.c[1]; g2 = c.c[2]; }
    else if (c.kind == 2) {
        int i0[3];
        float t[3], v[8], g[3] = {0.f, 0.f, 0.f};
        if (grid_cell(c, x, i0, t)) {
            grid_corners(c, c.phi, 1, 0, i0, v);
            trilinear_grad(v, t, c.c[3], g);
        }
        g0 = g[0]; g1 = g[1]; g2 = g[2];
    }
    else { g0 = __fsub_rn(x[0], c.c[0]); g1 = 0.0f; g2 = __fsub_rn(x[2], c.c[1]); }
    // Eigen normalize(): divide by the norm
    float nn = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(g0, g0), __fmul_rn(g1, g1)), __fmul_rn(g2, g2)));
    n[0] = __fdiv_rn(g0, nn);
    n[1] = __fdiv_rn(g1, nn);
    n[2] = __fdiv_rn(g2, nn);
}
// CollisionObject::velocity at x: constant for the analytic kinds, the sampled velocity (or 0) for a grid
__device__ __forceinline__ void coll_velocity(const DevCollider& c, const float x[3], float v[3]) {
    if (c.kind != 2) { v[0] = c.vel[0]; v[1] = c.vel[1]; v[2] = c.vel[2]; return; }
    v[0] = v[1] = v[2] = 0.0f;
    int i0[3];
    float t[3], s[8];
    if (!c.v || !grid_cell(c, x, i0, t)) return;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        grid_corners(c, c.v, 3, k, i0, s);
        v[k] = trilinear(s, t);
    }
}

// CollisionObjectSet::collide.  Returns -1 (none), -2 (several), or the object index.
__device__ __forceinline__ int collide(const DevCollider* objs, int ncoll, float v[3], const float x[3], const float fv[3],
                                       bool addCollisionVelocity) {
    int obj = -1;
    bool hit = false;
    for (int o = 0; o < ncoll; ++o) {
        const DevCollider& c = objs[o];
        if (coll_phi(c, x) <= 0.0f) {
            if (hit) { obj = -2; v[0] = v[1] = v[2] = 0.0f; break; }
            hit = true;
            float vo[3];
            coll_velocity(c, x, vo);
            vo[0] = __fsub_rn(vo[0], fv[0]); vo[1] = __fsub_rn(vo[1], fv[1]); vo[2] = __fsub_rn(vo[2], fv[2]);
            v[0] = __fsub_rn(v[0], vo[0]); v[1] = __fsub_rn(v[1], vo[1]); v[2] = __fsub_rn(v[2], vo[2]);
            float n[3];
            coll_normal(c, x, n);
            float nDotV = __fadd_rn(__fadd_rn(__fmul_rn(n[0], v[0]), __fmul_rn(n[1], v[1])), __fmul_rn(n[2], v[2]));
            if (nDotV < 0.0f) {
                obj = o;
                if (c.sticky) {
                    v[0] = v[1] = v[2] = 0.0f;
                } else {
                    float t0 = __fsub_rn(v[0], __fmul_rn(nDotV, n[0]));
                    float t1 = __fsub_rn(v[1], __fmul_rn(nDotV, n[1]));
                    float t2 = __fsub_rn(v[2], __fmul_rn(nDotV, n[2]));
                    float vt = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(t0, t0), __fmul_rn(t1, t1)), __fmul_rn(t2, t2)));
                    if (vt >= __fmul_rn(-nDotV, c.friction)) {
                        float s = __fadd_rn(1.0f, __fdiv_rn(__fmul_rn(c.friction, nDotV), vt));
                        v[0] = __fmul_rn(t0, s); v[1] = __fmul_rn(t1, s); v[2] = __fmul_rn(t2, s);
                    } else {
                        v[0] = v[1] = v[2] = 0.0f;
                    }
                }
            }
            if (addCollisionVelocity) { v[0] = __fadd_rn(v[0], vo[0]); v[1] = __fadd_rn(v[1], vo[1]); v[2] = __fadd_rn(v[2], vo[2]); }
        }
    }
    return obj;
}

// subspaceProject of one node — Grid.cpp:778-818
__device__ __forceinline__ void project_node(const DevCollider* objs, int flag, const float x[3], float v[3]) {
    if (flag == -1) return;
    if (flag == -2) { v[0] = v[1] = v[2] = 0.0f; return; }
    float n[3];
    coll_normal(objs[flag], x, n);
    float d = n[0] * v[0] + n[1] * v[1] + n[2] * v[2];
    v[0] -= d * n[0]; v[1] -= d * n[1]; v[2] -= d * n[2];
}

// ------------------------------------------------------------------------------------------------
// 3x3 helpers
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void mat_mul(const float* a, const float* b, float* c) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) c[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
}
// c = a * b^T
__device__ __forceinline__ void mat_mul_bt(const float* a, const float* b, float* c) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) c[3 * i + j] = a[3 * i] * b[3 * j] + a[3 * i + 1] * b[3 * j + 1] + a[3 * i + 2] * b[3 * j + 2];
}

// dEnergyDensitydF — SnowConstitutiveModel.cpp:187-216:  P = 2 mu (F - R) + lambda (J - 1) J F^-T
__device__ __forceinline__ void snow_stress(const float* F, const float* R, const float* FiT, float J, float mu, float lam,
                                            float* P) {
    float a = 2.0f * mu, b = lam * (J - 1.0f) * J;
#pragma unroll
    for (int k = 0; k < 9; ++k) P[k] = a * (F[k] - R[k]) + b * FiT[k];
}

// dEdFDifferential — SnowConstitutiveModel.cpp:218-256 with computeRdifferential :266-287
__device__ __forceinline__ void snow_dP(const float* dF, const float* R, const float* FiT, const float* Gi, float J, float mu,
                                        float lam, float* out) {
    float dd = 0.0f;
#pragma unroll
    for (int k = 0; k < 9; ++k) dd += FiT[k] * dF[k];
    float dJ = J * dd;
    // dFInvTrans = -FiT dF^T FiT
    float t[9], dFiT[9];
    mat_mul_bt(FiT, dF, t);  // FiT * dF^T
    mat_mul(t, FiT, dFiT);
    // M = R^T dF (only the antisymmetric part is used)
    float M01 = R[0] * dF[1] + R[3] * dF[4] + R[6] * dF[7];
    float M10 = R[1] * dF[0] + R[4] * dF[3] + R[7] * dF[6];
    float M02 = R[0] * dF[2] + R[3] * dF[5] + R[6] * dF[8];
    float M20 = R[2] * dF[0] + R[5] * dF[3] + R[8] * dF[6];
    float M12 = R[1] * dF[2] + R[4] * dF[5] + R[7] * dF[8];
    float M21 = R[2] * dF[1] + R[5] * dF[4] + R[8] * dF[7];
    float w0 = M01 - M10, w1 = M02 - M20, w2 = M12 - M21;
    float g0 = Gi[0] * w0 + Gi[1] * w1 + Gi[2] * w2;
    float g1 = Gi[3] * w0 + Gi[4] * w1 + Gi[5] * w2;
    float g2 = Gi[6] * w0 + Gi[7] * w1 + Gi[8] * w2;
    // dR = R * [[0, g0, g1], [-g0, 0, g2], [-g1, -g2, 0]]
    float dR[9];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float r0 = R[3 * i], r1 = R[3 * i + 1], r2 = R[3 * i + 2];
        dR[3 * i + 0] = -r1 * g0 - r2 * g1;
        dR[3 * i + 1] = r0 * g0 - r2 * g2;
        dR[3 * i + 2] = r0 * g1 + r1 * g2;
    }
    float a = 2.0f * mu, Jm1 = J - 1.0f;
#pragma unroll
    for (int k = 0; k < 9; ++k)
        out[k] = a * (dF[k] - dR[k]) + lam * (dJ * J * FiT[k] + Jm1 * (dJ * FiT[k] - J * dFiT[k]));
}

// ------------------------------------------------------------------------------------------------
// Snow plasticity — SnowConstitutiveModel::updateParticleData, SnowConstitutiveModel.cpp:39-120.
// SVD by one-sided (Hestenes) Jacobi; every stored quantity (clamped F, Fp, F^-T, R, S -> G^-1, J) is a
// spectral function U f(S) V^T / V f(S) V^T of F, independent of the particular SVD, so this reproduces
// Eigen's JacobiSVD results to round-off.  Runs in T = float, or double for the ill-conditioned fallback.
// ------------------------------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void svd3_jacobi(const float* Fin, T* U, T* s, T* V) {
    T A[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) { A[k] = (T)Fin[k]; V[k] = (k % 4 == 0) ? T(1) : T(0); }
    const T eps = sizeof(T) == 4 ? T(1.1920929e-07) : T(2.220446049250313e-16);
    for (int sweep = 0; sweep < 12; ++sweep) {
        bool rotated = false;
#pragma unroll
        for (int pair = 0; pair < 3; ++pair) {
            const int p = pair == 2 ? 1 : 0, q = pair == 0 ? 1 : 2;
            T al = A[p] * A[p] + A[3 + p] * A[3 + p] + A[6 + p] * A[6 + p];
            T be = A[q] * A[q] + A[3 + q] * A[3 + q] + A[6 + q] * A[6 + q];
            T ga = A[p] * A[q] + A[3 + p] * A[3 + q] + A[6 + p] * A[6 + q];
            if (ga == T(0) || fabs(ga) <= eps * sqrt(al * be)) continue;
            rotated = true;
            T zeta = (be - al) / (T(2) * ga);
            T t = (zeta >= T(0) ? T(1) : T(-1)) / (fabs(zeta) + sqrt(T(1) + zeta * zeta));
            T c = T(1) / sqrt(T(1) + t * t), sn = c * t;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                T ap = A[3 * i + p], aq = A[3 * i + q];
                A[3 * i + p] = c * ap - sn * aq;
                A[3 * i + q] = sn * ap + c * aq;
                T vp = V[3 * i + p], vq = V[3 * i + q];
                V[3 * i + p] = c * vp - sn * vq;
                V[3 * i + q] = sn * vp + c * vq;
            }
        }
        if (!rotated) break;
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        s[j] = sqrt(A[j] * A[j] + A[3 + j] * A[3 + j] + A[6 + j] * A[6 + j]);
        T inv = s[j] > T(0) ? T(1) / s[j] : T(0);
#pragma unroll
        for (int i = 0; i < 3; ++i) U[3 * i + j] = A[3 * i + j] * inv;
    }
    // complete U where a singular value vanished (rank-deficient F)
    if (!(s[0] > T(0)) || !(s[1] > T(0)) || !(s[2] > T(0))) {
        int nz = (s[0] > T(0)) + (s[1] > T(0)) + (s[2] > T(0));
        int a = s[0] > T(0) ? 0 : (s[1] > T(0) ? 1 : 2);
        if (nz == 0) {
#pragma unroll
            for (int k = 0; k < 9; ++k) U[k] = (k % 4 == 0) ? T(1) : T(0);
        } else {
            T u0[3] = {U[a], U[3 + a], U[6 + a]};
            int b = -1;
            for (int j = 0; j < 3; ++j) if (j != a && s[j] > T(0)) b = j;
            T u1[3];
            if (b >= 0) { u1[0] = U[b]; u1[1] = U[3 + b]; u1[2] = U[6 + b]; }
            else {
                T e[3] = {fabs(u0[0]) < T(0.9) ? T(1) : T(0), fabs(u0[0]) < T(0.9) ? T(0) : T(1), T(0)};
                u1[0] = u0[1] * e[2] - u0[2] * e[1]; u1[1] = u0[2] * e[0] - u0[0] * e[2]; u1[2] = u0[0] * e[1] - u0[1] * e[0];
                T nn = sqrt(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
                u1[0] /= nn; u1[1] /= nn; u1[2] /= nn;
                for (int j = 0; j < 3; ++j) if (j != a) { b = j; break; }
                U[b] = u1[0]; U[3 + b] = u1[1]; U[6 + b] = u1[2];
            }
            int c3 = 3 - a - b;
            T u2[3] = {u0[1] * u1[2] - u0[2] * u1[1], u0[2] * u1[0] - u0[0] * u1[2], u0[0] * u1[1] - u0[1] * u1[0]};
            T nn = sqrt(u2[0] * u2[0] + u2[1] * u2[1] + u2[2] * u2[2]);
            U[c3] = u2[0] / nn; U[3 + c3] = u2[1] / nn; U[6 + c3] = u2[2] / nn;
        }
    }
}

struct PlasticOut {
    float F[9], Fp[9], FiT[9], R[9], Gi[9], J, mu, lam;
    int bad;  // non-finite hardening factor
};

template <class T>
__device__ __forceinline__ void snow_plasticity_T(const T* U, const T* s, const T* V, const float* F, const float* Fp, float mu0,
                                                  float lam0, float xi, float thc, float ths, PlasticOut& o) {
    bool modified = false;
    T d[3], di[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        T si = s[i];
        if (si > T(1) + T(ths)) { modified = true; si = T(1) + T(ths); }
        if (si < T(1) - T(thc)) { modified = true; si = T(1) - T(thc); }
        d[i] = si;
        di[i] = T(1) / si;
    }
    // FinvTrans = U diag(1/s) V^T, R = U V^T, F' = U diag(s) V^T
    T FiT[9], R[9], Fn[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            T a = 0, b = 0, c = 0;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                T uv = U[3 * i + k] * V[3 * j + k];
                a += uv * di[k];
                b += uv;
                c += uv * d[k];
            }
            FiT[3 * i + j] = a; R[3 * i + j] = b; Fn[3 * i + j] = c;
        }
    if (modified) {
        // Fp <- V diag(1/s) U^T F Fp = FiT^T (F Fp)
        T FFp[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                FFp[3 * i + j] = (T)F[3 * i] * (T)Fp[j] + (T)F[3 * i + 1] * (T)Fp[3 + j] + (T)F[3 * i + 2] * (T)Fp[6 + j];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                o.Fp[3 * i + j] = (float)(FiT[i] * FFp[j] + FiT[3 + i] * FFp[3 + j] + FiT[6 + i] * FFp[6 + j]);
#pragma unroll
        for (int k = 0; k < 9; ++k) o.F[k] = (float)Fn[k];
    } else {
#pragma unroll
        for (int k = 0; k < 9; ++k) { o.F[k] = F[k]; o.Fp[k] = Fp[k]; }
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) { o.FiT[k] = (float)FiT[k]; o.R[k] = (float)R[k]; }
    // S = V diag(s) V^T; G from S; Ginv = G^-1 (SnowConstitutiveModel.cpp:78-87)
    T S[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) S[3 * i + j] = V[3 * i] * d[0] * V[3 * j] + V[3 * i + 1] * d[1] * V[3 * j + 1] + V[3 * i + 2] * d[2] * V[3 * j + 2];
    T G[9];
    G[0] = S[0] + S[4]; G[4] = S[0] + S[8]; G[8] = S[4] + S[8];
    G[1] = G[3] = S[5]; G[2] = G[6] = -S[2]; G[5] = G[7] = S[1];
    T c00 = G[4] * G[8] - G[5] * G[7], c01 = G[2] * G[7] - G[1] * G[8], c02 = G[1] * G[5] - G[2] * G[4];
    T c10 = G[5] * G[6] - G[3] * G[8], c11 = G[0] * G[8] - G[2] * G[6], c12 = G[2] * G[3] - G[0] * G[5];
    T c20 = G[3] * G[7] - G[4] * G[6], c21 = G[1] * G[6] - G[0] * G[7], c22 = G[0] * G[4] - G[1] * G[3];
    T idet = T(1) / (G[0] * c00 + G[1] * c10 + G[2] * c20);
    o.Gi[0] = (float)(c00 * idet); o.Gi[1] = (float)(c01 * idet); o.Gi[2] = (float)(c02 * idet);
    o.Gi[3] = (float)(c10 * idet); o.Gi[4] = (float)(c11 * idet); o.Gi[5] = (float)(c12 * idet);
    o.Gi[6] = (float)(c20 * idet); o.Gi[7] = (float)(c21 * idet); o.Gi[8] = (float)(c22 * idet);
    o.J = (float)(d[0] * d[1] * d[2]);
    // hardening — :93-114, det(Fp) in float as the reference does
    const float* P = o.Fp;
    float detFp = P[0] * (P[4] * P[8] - P[7] * P[5]) - P[3] * (P[1] * P[8] - P[7] * P[2]) + P[6] * (P[1] * P[5] - P[4] * P[2]);
    float hf = xi * (1.0f - detFp);
    if (hf > 2.0f) hf = 2.0f;
    hf = expf(hf);
    o.bad = !isfinite(hf);
    o.mu = mu0 * hf;
    o.lam = lam0 * hf;
}

// FP32 update with the FP64 fallback for particles whose singular-value ratio exceeds 1e4.
__device__ __forceinline__ void snow_plasticity(const float* F, const float* Fp, float mu0, float lam0, float xi, float thc,
                                                float ths, PlasticOut& o, int& used_fp64) {
    float U[9], V[9], s[3];
    svd3_jacobi<float>(F, U, s, V);
    float smax = fmaxf(s[0], fmaxf(s[1], s[2])), smin = fminf(s[0], fminf(s[1], s[2]));
    if (!(smin > 0.0f) || smax > 1.0e4f * smin || !isfinite(smax)) {
        used_fp64 = 1;
        double Ud[9], Vd[9], sd[3];
        svd3_jacobi<double>(F, Ud, sd, Vd);
        snow_plasticity_T<double>(Ud, sd, Vd, F, Fp, mu0, lam0, xi, thc, ths, o);
    } else {
        used_fp64 = 0;
        snow_plasticity_T<float>(U, s, V, F, Fp, mu0, lam0, xi, thc, ths, o);
    }
}

}  // namespace mpm

// CPU ORACLE — test infrastructure only.
//
// A plain C++ restatement of the implicit MPM snow time step of davidsminor/mpmsnow, templated on the
// floating-point type.  The double instance is the accuracy reference for the CUDA path; the float instance is
// "the reference CPU step" (same order of operations as the reference, FP32 state) and is what the CPU
// baseline times.  Nothing in the product links or calls this file: only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline / reference arm load it, and only as the checker.
//
// Parity status: the reference cannot be built here (Eigen 3.2, TBB, GL, SCons IEBuild and the Houdini HDK
// are absent), and it ships no golden vectors.  This restatement is pinned against every known-answer and
// property test the reference holds for the path (src/tests/*.cpp; see tests/test_oracle_*.py).  Bit-level
// agreement with Eigen's JacobiSVD and with Eigen's SSE reduction order is unpinned.
//
// Each function cites the reference file:line it restates.  Paths are relative to the reference project.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <memory>
#include <queue>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <thread>

namespace mpm_oracle {

// ---------------------------------------------------------------------------------------------------------
// Small fixed-size linear algebra (stand-in for Eigen::Vector3f / Matrix3f).  Row-major a[r][c].
// ---------------------------------------------------------------------------------------------------------
template <class T> struct V3 {
    T v[3];
    V3() : v{T(0), T(0), T(0)} {}
    V3(T a, T b, T c) : v{a, b, c} {}
    T& operator[](int i) { return v[i]; }
    const T& operator[](int i) const { return v[i]; }
    V3 operator+(const V3& o) const { return V3(v[0] + o.v[0], v[1] + o.v[1], v[2] + o.v[2]); }
    V3 operator-(const V3& o) const { return V3(v[0] - o.v[0], v[1] - o.v[1], v[2] - o.v[2]); }
    V3 operator*(T s) const { return V3(v[0] * s, v[1] * s, v[2] * s); }
    V3 operator/(T s) const { return V3(v[0] / s, v[1] / s, v[2] / s); }
    V3& operator+=(const V3& o) { v[0] += o.v[0]; v[1] += o.v[1]; v[2] += o.v[2]; return *this; }
    V3& operator-=(const V3& o) { v[0] -= o.v[0]; v[1] -= o.v[1]; v[2] -= o.v[2]; return *this; }
    T dot(const V3& o) const { return v[0] * o.v[0] + v[1] * o.v[1] + v[2] * o.v[2]; }
    T squaredNorm() const { return v[0] * v[0] + v[1] * v[1] + v[2] * v[2]; }
    T norm() const { return std::sqrt(squaredNorm()); }
    void setZero() { v[0] = v[1] = v[2] = T(0); }
    // Eigen 3.2 MatrixBase::normalize(): *this /= norm() (no zero guard).
    void normalize() { T n = norm(); v[0] /= n; v[1] /= n; v[2] /= n; }
};
template <class T> inline V3<T> operator*(T s, const V3<T>& a) { return a * s; }

template <class T> struct M3 {
    T a[3][3];
    M3() { std::memset(a, 0, sizeof(a)); }
    static M3 Identity() { M3 m; m.a[0][0] = m.a[1][1] = m.a[2][2] = T(1); return m; }
    static M3 Zero() { return M3(); }
    T& operator()(int r, int c) { return a[r][c]; }
    const T& operator()(int r, int c) const { return a[r][c]; }
    M3 operator+(const M3& o) const { M3 m; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) m.a[i][j] = a[i][j] + o.a[i][j]; return m; }
    M3 operator-(const M3& o) const { M3 m; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) m.a[i][j] = a[i][j] - o.a[i][j]; return m; }
    M3 operator*(T s) const { M3 m; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) m.a[i][j] = a[i][j] * s; return m; }
    M3& operator+=(const M3& o) { for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) a[i][j] += o.a[i][j]; return *this; }
    M3 operator*(const M3& o) const {
        M3 m;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) m.a[i][j] = a[i][0] * o.a[0][j] + a[i][1] * o.a[1][j] + a[i][2] * o.a[2][j];
        return m;
    }
    V3<T> operator*(const V3<T>& x) const {
        return V3<T>(a[0][0] * x[0] + a[0][1] * x[1] + a[0][2] * x[2], a[1][0] * x[0] + a[1][1] * x[1] + a[1][2] * x[2],
                     a[2][0] * x[0] + a[2][1] * x[1] + a[2][2] * x[2]);
    }
    M3 transpose() const { M3 m; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) m.a[i][j] = a[j][i]; return m; }
    T determinant() const {
        return a[0][0] * (a[1][1] * a[2][2] - a[2][1] * a[1][2]) - a[1][0] * (a[0][1] * a[2][2] - a[2][1] * a[0][2]) +
               a[2][0] * (a[0][1] * a[1][2] - a[1][1] * a[0][2]);
    }
    // Cofactor inverse (the closed form Eigen uses for 3x3).
    M3 inverse() const {
        M3 c;
        c.a[0][0] = a[1][1] * a[2][2] - a[1][2] * a[2][1];
        c.a[0][1] = a[0][2] * a[2][1] - a[0][1] * a[2][2];
        c.a[0][2] = a[0][1] * a[1][2] - a[0][2] * a[1][1];
        c.a[1][0] = a[1][2] * a[2][0] - a[1][0] * a[2][2];
        c.a[1][1] = a[0][0] * a[2][2] - a[0][2] * a[2][0];
        c.a[1][2] = a[0][2] * a[1][0] - a[0][0] * a[1][2];
        c.a[2][0] = a[1][0] * a[2][1] - a[1][1] * a[2][0];
        c.a[2][1] = a[0][1] * a[2][0] - a[0][0] * a[2][1];
        c.a[2][2] = a[0][0] * a[1][1] - a[0][1] * a[1][0];
        T det = a[0][0] * c.a[0][0] + a[0][1] * c.a[1][0] + a[0][2] * c.a[2][0];
        return c * (T(1) / det);
    }
    T squaredNorm() const { T s = 0; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) s += a[i][j] * a[i][j]; return s; }
    T norm() const { return std::sqrt(squaredNorm()); }
};
// outer product u v^T
template <class T> inline M3<T> outer(const V3<T>& u, const V3<T>& v) {
    M3<T> m;
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) m.a[i][j] = u[i] * v[j];
    return m;
}

template <class T> inline bool finite_(T x) { return std::isfinite(x); }

// ---------------------------------------------------------------------------------------------------------
// Cubic B-spline shape function — src/MpmSim/CubicBsplineShapeFunction.cpp:6-48
// ---------------------------------------------------------------------------------------------------------
template <class T> struct CubicBspline {
    static int supportRadius() { return 2; }  // :6-9
    static T w(T x) {                            // :11-26
        T ax = std::fabs(x);
        if (ax < T(1)) return (T(0.5) * ax - T(1)) * ax * ax + T(2) / T(3);
        else if (ax < T(2)) return ((-ax / T(6) + T(1)) * ax - T(2)) * ax + T(4) / T(3);
        return T(0);
    }
    static T dw(T x) {  // :28-47
        if (x < T(0)) return -dw(-x);
        if (x < T(1)) return x * (T(1.5) * x - T(2));
        else if (x < T(2)) { x -= T(2); return T(-0.5) * x * x; }
        return T(0);
    }
};

// ---------------------------------------------------------------------------------------------------------
// Collision objects — src/CollisionObject.cpp:19-96, src/MpmSim/CollisionPlane.cpp:23-56.
// kind 0: CollisionPlane, phi = c0 x + c1 y + c2 z + c3, grad = c.xyz, constant velocity.
// kind 1: CollisionCylinder (no reference counterpart; the C5 scene's vertical solid cylinder):
//         phi = |(x - cx, z - cz)| - r, grad = (x - cx, 0, z - cz), constant velocity.
// ---------------------------------------------------------------------------------------------------------
template <class T> struct Collider {
    int kind = 0;            // 0 plane, 1 vertical cylinder, 2 sampled signed-distance grid
    T c[4] = {0, 0, 0, 0};   // plane coefficients, (cx, cz, r, unused) for the cylinder, (origin, spacing) for a grid
    V3<T> vel;               // CollisionPlane::setV (CollisionPlane.h:22)
    T friction = T(0.5);
    bool sticky = false;
    // kind 2, the restated VDBCollisionObject (houdiniPlugin/VDBCollisionObject.cpp:11-37) over a dense grid:
    // phi and the velocity sampled at c[0..2] + c[3] (i, j, k), trilinear between samples, grad the gradient of
    // the trilinear phi; no collider outside the sampled box
    int n[3] = {0, 0, 0};
    std::shared_ptr<std::vector<T>> gphi, gvel;

    static T lerp(T a, T b, T t) { return a + t * (b - a); }
    bool cell(const V3<T>& x, int i0[3], T t[3]) const {
        for (int a = 0; a < 3; ++a) {
            const T u = (x[a] - c[a]) / c[3];
            if (!(u >= T(0)) || u > (T)(n[a] - 1)) return false;
            const int i = std::min((int)std::floor(u), n[a] - 2);
            i0[a] = i;
            t[a] = u - (T)i;
        }
        return true;
    }
    void corners(const std::vector<T>& f, int comps, int k, const int i0[3], T v[8]) const {
        const long sx = comps, sy = (long)comps * n[0], sz = sy * n[1];
        const long b = i0[0] * sx + i0[1] * sy + i0[2] * sz + k;
        for (int q = 0; q < 8; ++q) v[q] = f[b + (q & 1) * sx + ((q >> 1) & 1) * sy + (q >> 2) * sz];
    }
    static T trilinear(const T v[8], const T t[3]) {
        const T x00 = lerp(v[0], v[1], t[0]), x10 = lerp(v[2], v[3], t[0]);
        const T x01 = lerp(v[4], v[5], t[0]), x11 = lerp(v[6], v[7], t[0]);
        return lerp(lerp(x00, x10, t[1]), lerp(x01, x11, t[1]), t[2]);
    }

    T phi(const V3<T>& x) const {
        if (kind == 0) return c[0] * x[0] + c[1] * x[1] + c[2] * x[2] + c[3];  // CollisionPlane.cpp:23-26
        if (kind == 2) {
            int i0[3];
            T t[3], v[8];
            if (!cell(x, i0, t)) return std::numeric_limits<T>::infinity();
            corners(*gphi, 1, 0, i0, v);
            return trilinear(v, t);
        }
        T dx = x[0] - c[0], dz = x[2] - c[1];
        return std::sqrt(dx * dx + dz * dz) - c[2];
    }
    V3<T> grad(const V3<T>& x) const {
        if (kind == 0) return V3<T>(c[0], c[1], c[2]);  // CollisionPlane.cpp:28-31
        if (kind == 2) {
            int i0[3];
            T t[3], v[8];
            if (!cell(x, i0, t)) return V3<T>();
            corners(*gphi, 1, 0, i0, v);
            const T h = c[3];
            const T g0 = lerp(lerp(v[1] - v[0], v[3] - v[2], t[1]), lerp(v[5] - v[4], v[7] - v[6], t[1]), t[2]) / h;
            const T x00 = lerp(v[0], v[1], t[0]), x10 = lerp(v[2], v[3], t[0]);
            const T x01 = lerp(v[4], v[5], t[0]), x11 = lerp(v[6], v[7], t[0]);
            const T g1 = lerp(x10 - x00, x11 - x01, t[2]) / h;
            const T g2 = (lerp(x01, x11, t[1]) - lerp(x00, x10, t[1])) / h;
            return V3<T>(g0, g1, g2);
        }
        return V3<T>(x[0] - c[0], T(0), x[2] - c[1]);
    }
    V3<T> velocity(const V3<T>& x) const {  // CollisionPlane.cpp:33-36
        if (kind != 2) return vel;
        V3<T> out;
        int i0[3];
        T t[3], v[8];
        if (!gvel || !cell(x, i0, t)) return out;
        for (int k = 0; k < 3; ++k) {
            corners(*gvel, 3, k, i0, v);
            out[k] = trilinear(v, t);
        }
        return out;
    }
};

// CollisionObjectSet::collide — src/CollisionObject.cpp:19-96
template <class T>
int collide(const std::vector<Collider<T>>& objs, V3<T>& v, const V3<T>& x, const V3<T>& frameVelocity,
            bool addCollisionVelocity) {
    int collisionObject = -1;
    bool intersectedAlready = false;
    for (size_t objIdx = 0; objIdx < objs.size(); ++objIdx) {
        T phi = objs[objIdx].phi(x);
        if (phi <= T(0)) {
            if (intersectedAlready) {  // :33-40
                collisionObject = -2;
                v.setZero();
                break;
            }
            intersectedAlready = true;
            V3<T> vObj = objs[objIdx].velocity(x);
            vObj -= frameVelocity;  // :48
            v -= vObj;              // :51
            V3<T> n = objs[objIdx].grad(x);
            n.normalize();  // :55
            T nDotV = n.dot(v);
            if (nDotV < T(0)) {
                collisionObject = (int)objIdx;
                if (objs[objIdx].sticky) {
                    v.setZero();
                } else {
                    V3<T> vPerp = n * nDotV;
                    V3<T> vTangent = v - vPerp;
                    T vtNorm = vTangent.norm();
                    T mu = objs[objIdx].friction;
                    if (vtNorm >= -nDotV * mu) v = vTangent * (T(1) + mu * nDotV / vTangent.norm());  // :77-80
                    else v.setZero();
                }
            }
            if (addCollisionVelocity) v += vObj;  // :88-91
        }
    }
    return collisionObject;
}

// GravityField::force — src/MpmSim/GravityField.cpp:9-12; ForceFieldSet::force — src/ForceField.cpp:19-25
template <class T> struct Fields {
    std::vector<V3<T>> gravity;
    void force(V3<T>& f, const V3<T>&, T m) const {
        for (auto& g : gravity) f += g * m;
    }
};

// ---------------------------------------------------------------------------------------------------------
// Particle storage — src/MpmSim/MaterialPointData.cpp:8-16 (p, v, F, m, volume) plus the snow model's
// variables created in SnowConstitutiveModel::setParticles (SnowConstitutiveModel.cpp:123-169).
// mu0 / lambda0 hold the per-particle base Lame parameters (the per-particle E0 extension); when empty the
// scalar model values are used, exactly as SnowConstitutiveModel.cpp:113-114 does.
// ---------------------------------------------------------------------------------------------------------
template <class T> struct Particles {
    std::vector<V3<T>> x, v;
    std::vector<M3<T>> F, Fp, FinvTrans, R, Ginv;
    std::vector<T> m, volume, J, mu, lambda, mu0, lambda0;
    size_t size() const { return x.size(); }
};

struct OracleError : std::runtime_error {
    int code;
    OracleError(int c, const std::string& s) : std::runtime_error(s), code(c) {}
};
// status codes shared with the C-ABI (include/mpm_gpu.h)
enum {
    E_OK = 0, E_NAN_MASSES = 4, E_NAN_VELOCITIES = 5, E_NAN_MOMENTA = 6, E_NAN_STRESS = 7, E_HARDNESS = 8,
    E_NAN_PARTICLE_V = 9, E_GRID_TOO_BIG = 10
};

// ---------------------------------------------------------------------------------------------------------
// 3x3 SVD by one-sided (Hestenes) Jacobi.  Eigen's JacobiSVD(F, FullU|FullV) convention: sigma >= 0, U and V
// orthogonal.  Every quantity the snow model derives (U f(S) V^T, V S V^T, products of sigma) is independent
// of the particular SVD, so any convergent SVD with this convention reproduces the reference's values.
// ---------------------------------------------------------------------------------------------------------
template <class T> void svd3(const M3<T>& F, M3<T>& U, V3<T>& sigma, M3<T>& V) {
    M3<T> A = F;
    V = M3<T>::Identity();
    const T eps = std::numeric_limits<T>::epsilon();
    for (int sweep = 0; sweep < 12; ++sweep) {
        bool rotated = false;
        for (int pair = 0; pair < 3; ++pair) {
            int p = pair == 2 ? 1 : 0, q = pair == 0 ? 1 : 2;
            T alpha = 0, beta = 0, gamma = 0;
            for (int i = 0; i < 3; ++i) {
                alpha += A.a[i][p] * A.a[i][p];
                beta += A.a[i][q] * A.a[i][q];
                gamma += A.a[i][p] * A.a[i][q];
            }
            if (std::fabs(gamma) <= eps * std::sqrt(alpha * beta) || gamma == T(0)) continue;
            rotated = true;
            T zeta = (beta - alpha) / (T(2) * gamma);
            T t = (zeta >= T(0) ? T(1) : T(-1)) / (std::fabs(zeta) + std::sqrt(T(1) + zeta * zeta));
            T c = T(1) / std::sqrt(T(1) + t * t), s = c * t;
            for (int i = 0; i < 3; ++i) {
                T ap = A.a[i][p], aq = A.a[i][q];
                A.a[i][p] = c * ap - s * aq;
                A.a[i][q] = s * ap + c * aq;
                T vp = V.a[i][p], vq = V.a[i][q];
                V.a[i][p] = c * vp - s * vq;
                V.a[i][q] = s * vp + c * vq;
            }
        }
        if (!rotated) break;
    }
    // singular values are the column norms; U's columns the normalised columns of A
    int order[3] = {0, 1, 2};
    T nrm[3];
    for (int j = 0; j < 3; ++j) nrm[j] = std::sqrt(A.a[0][j] * A.a[0][j] + A.a[1][j] * A.a[1][j] + A.a[2][j] * A.a[2][j]);
    std::sort(order, order + 3, [&](int a, int b) { return nrm[a] > nrm[b]; });
    M3<T> Vs, As;
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) { Vs.a[i][j] = V.a[i][order[j]]; As.a[i][j] = A.a[i][order[j]]; }
    V = Vs;
    for (int j = 0; j < 3; ++j) sigma[j] = nrm[order[j]];
    // U columns; complete an orthonormal basis where a singular value vanishes
    for (int j = 0; j < 3; ++j) {
        if (sigma[j] > T(0)) {
            for (int i = 0; i < 3; ++i) U.a[i][j] = As.a[i][j] / sigma[j];
        } else {
            for (int i = 0; i < 3; ++i) U.a[i][j] = T(0);
        }
    }
    auto col = [&](int j) { return V3<T>(U.a[0][j], U.a[1][j], U.a[2][j]); };
    auto setcol = [&](int j, const V3<T>& c) { for (int i = 0; i < 3; ++i) U.a[i][j] = c[i]; };
    auto cross = [](const V3<T>& a, const V3<T>& b) {
        return V3<T>(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
    };
    if (!(sigma[0] > T(0))) { setcol(0, V3<T>(1, 0, 0)); }
    if (!(sigma[1] > T(0))) {
        V3<T> u0 = col(0);
        V3<T> e = std::fabs(u0[0]) < T(0.9) ? V3<T>(1, 0, 0) : V3<T>(0, 1, 0);
        V3<T> u1 = cross(u0, e); u1.normalize(); setcol(1, u1);
    }
    if (!(sigma[2] > T(0))) { V3<T> u2 = cross(col(0), col(1)); u2.normalize(); setcol(2, u2); }
}

// ---------------------------------------------------------------------------------------------------------
// Snow constitutive model — src/MpmSim/SnowConstitutiveModel.cpp
// ---------------------------------------------------------------------------------------------------------
template <class T> struct SnowModel {
    T E, nu, xi, thetaC, thetaS, mu, lambda;
    SnowModel(T youngsModulus, T poissonRatio, T hardening, T compressiveStrength, T tensileStrength)
        : E(youngsModulus), nu(poissonRatio), xi(hardening), thetaC(compressiveStrength), thetaS(tensileStrength) {
        mu = (youngsModulus / (T(2) * (T(1) + poissonRatio)));                                               // :23
        lambda = (youngsModulus * poissonRatio / ((T(1) + poissonRatio) * (T(1) - T(2) * poissonRatio)));  // :24
    }

    // setParticles — :123-169
    void setParticles(Particles<T>& p) const {
        size_t n = p.m.size();
        p.Fp.assign(n, M3<T>::Identity());
        p.FinvTrans.assign(n, M3<T>::Identity());
        p.R.assign(n, M3<T>::Identity());
        p.Ginv.assign(n, M3<T>::Identity());
        p.J.assign(n, T(1));
        p.mu.assign(n, mu);
        p.lambda.assign(n, lambda);
    }

    // one particle of updateParticleData — :39-120
    void updateOne(Particles<T>& P, size_t p) const {
        M3<T> U, V;
        V3<T> s;
        svd3(P.F[p], U, s, V);
        M3<T> D, Dinv;
        bool modified = false;
        for (int i = 0; i < 3; ++i) {
            if (s[i] > T(1) + thetaS) { modified = true; s[i] = T(1) + thetaS; }  // :52-56
            if (s[i] < T(1) - thetaC) { modified = true; s[i] = T(1) - thetaC; }  // :59-63
            D.a[i][i] = s[i];
            Dinv.a[i][i] = T(1) / s[i];
        }
        if (modified) {  // :68-73
            M3<T> FNplusOne = P.F[p] * P.Fp[p];
            P.Fp[p] = V * Dinv * U.transpose() * FNplusOne;
            P.F[p] = U * D * V.transpose();
        }
        P.FinvTrans[p] = U * Dinv * V.transpose();  // :75
        P.R[p] = U * V.transpose();                 // :76
        M3<T> S = V * D * V.transpose();            // :78
        M3<T> G;                                    // :79-86
        G.a[0][0] = S.a[0][0] + S.a[1][1];
        G.a[1][1] = S.a[0][0] + S.a[2][2];
        G.a[2][2] = S.a[1][1] + S.a[2][2];
        G.a[0][1] = G.a[1][0] = S.a[1][2];
        G.a[0][2] = G.a[2][0] = -S.a[0][2];
        G.a[1][2] = G.a[2][1] = S.a[0][1];
        P.Ginv[p] = G.inverse();            // :87
        P.J[p] = D.a[0][0] * D.a[1][1] * D.a[2][2];  // :89
        T hardeningFactor = xi * (T(1) - P.Fp[p].determinant());  // :93
        if (hardeningFactor > T(2)) hardeningFactor = T(2);
        hardeningFactor = std::exp(hardeningFactor);
        if (!finite_(hardeningFactor)) throw OracleError(E_HARDNESS, "infinite hardness!!!");
        T m0 = P.mu0.empty() ? mu : P.mu0[p];
        T l0 = P.lambda0.empty() ? lambda : P.lambda0[p];
        P.mu[p] = m0 * hardeningFactor;       // :113
        P.lambda[p] = l0 * hardeningFactor;   // :114
    }
    void updateParticleData(Particles<T>& P) const {
        const long n = (long)P.size();
        for (long p = 0; p < n; ++p) updateOne(P, (size_t)p);  // serial, as :39
    }

    static T doubleDot(const M3<T>& a, const M3<T>& b) {  // :258-264
        return a.a[0][0] * b.a[0][0] + a.a[0][1] * b.a[0][1] + a.a[0][2] * b.a[0][2] + a.a[1][0] * b.a[1][0] +
               a.a[1][1] * b.a[1][1] + a.a[1][2] * b.a[1][2] + a.a[2][0] * b.a[2][0] + a.a[2][1] * b.a[2][1] +
               a.a[2][2] * b.a[2][2];
    }
    T energyDensity(const Particles<T>& P, size_t p) const {  // :171-185
        M3<T> rd = P.F[p] - P.R[p];
        T Jm1 = P.J[p] - T(1);
        return P.mu[p] * doubleDot(rd, rd) + T(0.5) * P.lambda[p] * Jm1 * Jm1;
    }
    M3<T> dEnergyDensitydF(const Particles<T>& P, size_t p) const {  // :187-216
        M3<T> rd = P.F[p] - P.R[p];
        M3<T> ret = rd * (T(2) * P.mu[p]) + P.FinvTrans[p] * (P.lambda[p] * (P.J[p] - T(1)) * P.J[p]);
        if (!finite_(ret.norm())) throw OracleError(E_NAN_STRESS, "nans in dEnergyDensitydF matrix!");
        return ret;
    }
    static M3<T> computeRdifferential(const M3<T>& dF, const M3<T>& R, const M3<T>& Ginv) {  // :266-287
        M3<T> M = R.transpose() * dF;
        V3<T> w(M.a[0][1] - M.a[1][0], M.a[0][2] - M.a[2][0], M.a[1][2] - M.a[2][1]);
        w = Ginv * w;
        M3<T> RtdR;
        RtdR.a[0][1] = w[0]; RtdR.a[1][0] = -w[0];
        RtdR.a[0][2] = w[1]; RtdR.a[2][0] = -w[1];
        RtdR.a[1][2] = w[2]; RtdR.a[2][1] = -w[2];
        return R * RtdR;
    }
    M3<T> dEdFDifferential(const Particles<T>& P, const M3<T>& dFp, size_t p) const {  // :218-256
        T J = P.J[p];
        const M3<T>& FiT = P.FinvTrans[p];
        T dJ = J * doubleDot(FiT, dFp);
        M3<T> dFInvTrans = (FiT * dFp.transpose() * FiT) * T(-1);
        M3<T> dR = computeRdifferential(dFp, P.R[p], P.Ginv[p]);
        return (dFp - dR) * (T(2) * P.mu[p]) +
               (FiT * (dJ * J) + (FiT * dJ + dFInvTrans * J) * (J - T(1))) * P.lambda[p];
    }
};

// ---------------------------------------------------------------------------------------------------------
// Reductions.  Eigen evaluates VectorXf::dot / squaredNorm with SSE packets; the float instance mimics its
// two-accumulator 4-lane scheme (exact agreement with Eigen is unpinned), the double instance sums in order.
// ---------------------------------------------------------------------------------------------------------
template <class T> inline T vdot(const std::vector<T>& a, const std::vector<T>& b) {
    const size_t n = a.size();
    if (sizeof(T) == 4 && n >= 8) {
        T r0[4] = {0, 0, 0, 0}, r1[4] = {0, 0, 0, 0};
        for (int l = 0; l < 4; ++l) { r0[l] = a[l] * b[l]; r1[l] = a[4 + l] * b[4 + l]; }
        size_t end2 = (n / 8) * 8, end = (n / 4) * 4, i = 8;
        for (; i < end2; i += 8)
            for (int l = 0; l < 4; ++l) { r0[l] += a[i + l] * b[i + l]; r1[l] += a[i + 4 + l] * b[i + 4 + l]; }
        for (int l = 0; l < 4; ++l) r0[l] += r1[l];
        if (end > end2) for (int l = 0; l < 4; ++l) r0[l] += a[end2 + l] * b[end2 + l];
        T res = (r0[0] + r0[2]) + (r0[1] + r0[3]);
        for (i = end; i < n; ++i) res += a[i] * b[i];
        return res;
    }
    T s = 0;
    for (size_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}


// ---------------------------------------------------------------------------------------------------------
// A persistent worker pool standing in for the reference's tbb::parallel_for (Grid.inl:13-17).
// ---------------------------------------------------------------------------------------------------------
class WorkerPool {
  public:
    static WorkerPool& instance() { static WorkerPool p; return p; }
    void setThreads(int n) {
        stop();
        nthreads_ = n < 1 ? 1 : n;
        quit_ = false;
        for (int t = 1; t < nthreads_; ++t) workers_.emplace_back([this] { loop(); });
    }
    int threads() const { return nthreads_; }
    // run fn(i) for i in [0, n), chunks handed out dynamically; returns when all are done
    void parallelFor(long n, const std::function<void(long)>& fn) {
        if (nthreads_ <= 1 || n < 2) { for (long i = 0; i < n; ++i) fn(i); return; }
        {
            std::unique_lock<std::mutex> lk(m_);
            job_ = &fn; jobN_ = n; next_.store(0); active_ = nthreads_ - 1; ++gen_;
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [this] { return active_ == 0; });
        job_ = nullptr;
    }
    ~WorkerPool() { stop(); }

  private:
    void work() {
        const long chunk = 4;
        for (;;) {
            long b = next_.fetch_add(chunk);
            if (b >= jobN_) break;
            long e = std::min(jobN_, b + chunk);
            for (long i = b; i < e; ++i) (*job_)(i);
        }
    }
    void loop() {
        unsigned long seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return quit_ || gen_ != seen; });
                if (quit_) return;
                seen = gen_;
            }
            work();
            std::unique_lock<std::mutex> lk(m_);
            if (--active_ == 0) done_.notify_all();
        }
    }
    void stop() {
        { std::unique_lock<std::mutex> lk(m_); quit_ = true; }
        cv_.notify_all();
        for (auto& w : workers_) w.join();
        workers_.clear();
    }
    int nthreads_ = 1;
    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    const std::function<void(long)>* job_ = nullptr;
    long jobN_ = 0;
    std::atomic<long> next_{0};
    int active_ = 0;
    unsigned long gen_ = 0;
    bool quit_ = false;
};

struct SolveStats {
    int iterations = 0;       // iteration index at which termination fired (ConjugateResiduals.cpp:125)
    double bNorm2 = 0, rNorm2 = 0;
    int exitReason = 0;       // 0 converged/maxIters, 1 b==0, 2 ApdPAp==0, 3 rz_old==0
};

using Vec = std::vector<double>;

// ---------------------------------------------------------------------------------------------------------
// Grid — src/MpmSim/Grid.cpp
// ---------------------------------------------------------------------------------------------------------
template <class T> struct Grid {
    using VT = std::vector<T>;
    Particles<T>& d;
    std::vector<int> inds;
    T h;
    V3<T> mmin, mmax;
    int n[3];
    V3<T> frameVelocity;
    VT masses, velocities, prevVelocities;
    std::vector<signed char> nodeCollided;
    // 8 colour partitions: list of [begin,end) index ranges into inds — Grid.h:135-136
    std::vector<std::pair<int, int>> partitions[8];
    // records for tests
    VT rec_explicitMomenta, rec_rhs, rec_vc, rec_diag, rec_x0, rec_solution, rec_forces;
    SolveStats stats;
    bool parallel = false;

    int coordsToIndex(int i, int j, int k) const { return i + n[0] * (j + n[1] * k); }  // Grid.cpp:1083-1086
    long long ncells() const { return (long long)n[0] * n[1] * n[2]; }

    int dim = 3;  // the reference's m_dimension (Grid.cpp:162-169): axes at and above it have one node

    // ShapeFunctionIterator::initialize — Grid.cpp:1105-1136
    struct Stencil {
        int base[3];
        T w[3][4], dw[3][4];
        T weight(int i, int j, int k) const { return w[0][i] * w[1][j] * w[2][k]; }           // :1190-1193
        V3<T> grad(int i, int j, int k) const {                                                 // :1179-1188
            return V3<T>(-dw[0][i] * w[1][j] * w[2][k], -w[0][i] * dw[1][j] * w[2][k], -w[0][i] * w[1][j] * dw[2][k]);
        }
    };
    void stencil(const V3<T>& p, Stencil& s, bool derivs) const {
        const int r = 2;
        // the axes the grid does not span keep the iterator's construction values: base 0, weight 1 at position
        // 0, no derivative (Grid.cpp:1095-1100, m_base.setZero() at :1110)
        for (int a = this->dim; a < 3; ++a) {
            s.base[a] = 0;
            for (int i = 0; i < 4; ++i) { s.w[a][i] = i == 0 ? T(1) : T(0); s.dw[a][i] = T(0); }
        }
        for (int dim = 0; dim < this->dim; ++dim) {
            T frac = (p[dim] - mmin[dim]) / h;
            int dimPos = (int)std::floor(frac);
            frac -= (T)dimPos;
            s.base[dim] = dimPos + 1 - r;
            int j = 1 - r;
            for (int i = 0; i < 4; ++i, ++j) s.w[dim][i] = CubicBspline<T>::w((T)j - frac);
            if (derivs) {
                j = 1 - r;
                for (int i = 0; i < 4; ++i, ++j) s.dw[dim][i] = CubicBspline<T>::dw((T)j - frac) / h;
            }
        }
    }
    // iterate the stencil nodes (64 in 3-D, 16 in 2-D, 4 in 1-D), x fastest — Grid.cpp:1138-1170
    template <class Fn> void forNodes(const Stencil& s, Fn fn) const {
        const int nk = dim >= 3 ? 4 : 1, nj = dim >= 2 ? 4 : 1;
        for (int k = 0; k < nk; ++k)
            for (int j = 0; j < nj; ++j)
                for (int i = 0; i < 4; ++i)
                    fn(coordsToIndex(s.base[0] + i, s.base[1] + j, s.base[2] + k), i, j, k);
    }

    // voxelSort — Grid.cpp:318-352
    static void voxelSort(std::vector<int>::iterator begin, std::vector<int>::iterator end, T voxelSize,
                          const std::vector<V3<T>>& x, int dim = 0) {
        std::sort(begin, end, [&](int a, int b) { return x[a][dim] < x[b][dim]; });
        if (dim == 2) return;
        int currentSlice = (int)std::floor(x[*begin][dim] / voxelSize);
        auto sliceBegin = begin;
        auto sliceEnd = begin + 1;
        for (;; ++sliceEnd) {
            int particleSlice = sliceEnd == end ? currentSlice + 1 : (int)std::floor(x[*sliceEnd][dim] / voxelSize);
            if (particleSlice != currentSlice) {
                voxelSort(sliceBegin, sliceEnd, voxelSize, x, dim + 1);
                if (sliceEnd == end) break;
                sliceBegin = sliceEnd;
                currentSlice = particleSlice;
            }
        }
    }
    // computeProcessingPartitions — Grid.cpp:354-384
    void computeProcessingPartitions() {
        T voxelSize = T(2 * CubicBspline<T>::supportRadius()) * h;
        if (inds.empty()) return;
        voxelSort(inds.begin(), inds.end(), voxelSize, d.x);
        int cur[3] = {0, 0, 0};
        std::pair<int, int>* pend = nullptr;
        for (int it = 0; it < (int)inds.size(); ++it) {
            V3<T> xx = d.x[inds[it]] / voxelSize;
            int vox[3] = {(int)std::floor(xx[0]), (int)std::floor(xx[1]), (int)std::floor(xx[2])};
            if (it == 0 || vox[0] != cur[0] || vox[1] != cur[1] || vox[2] != cur[2]) {
                cur[0] = vox[0]; cur[1] = vox[1]; cur[2] = vox[2];
                int colour = (vox[0] & 1) + 2 * (vox[1] & 1) + 4 * (vox[2] & 1);
                partitions[colour].push_back({it, it});
                pend = &partitions[colour].back();
            }
            ++pend->second;
        }
    }

    // Grid::splat — Grid.inl:10-18.  Colours in order (i&1, (i&2)/2, (i&4)/4); voxels of one colour touch
    // disjoint nodes, so the per-node summation order is the same serial or parallel.
    template <class Fn> void splat(Fn fn) const {
        for (int i = 0; i < 8; ++i) {
            int colour = (i & 1) + 2 * ((i & 2) / 2) + 4 * ((i & 4) / 4);
            const auto& part = partitions[colour];
            const long nv = (long)part.size();
            if (parallel) {
                std::function<void(long)> job = [&](long v) {
                    for (int it = part[v].first; it < part[v].second; ++it) fn(inds[it]);
                };
                WorkerPool::instance().parallelFor(nv, job);
            } else {
                for (long v = 0; v < nv; ++v)
                    for (int it = part[v].first; it < part[v].second; ++it) fn(inds[it]);
            }
        }
    }

    // Grid::Grid — Grid.cpp:156-263
    Grid(Particles<T>& d_, const std::vector<int>& particleInds, T gridSize, V3<T> frameV, bool par = false,
         int dimension = 3)
        : d(d_), inds(particleInds), h(gridSize), frameVelocity(frameV), parallel(par) {
        dim = dimension;
        for (int j = 0; j < 3; ++j) { mmin[j] = T(1.e10); mmax[j] = T(-1.e10); }
        for (int p : inds)
            for (int j = 0; j < dim; ++j) {
                if (d.x[p][j] < mmin[j]) mmin[j] = d.x[p][j];
                if (d.x[p][j] > mmax[j]) mmax[j] = d.x[p][j];
            }
        const int r = CubicBspline<T>::supportRadius();
        for (int j = 0; j < dim; ++j) {  // :194-202
            int cellMin = int(std::floor(mmin[j] / h)) - r - 1;
            int cellMax = int(std::ceil(mmax[j] / h)) + r + 1;
            mmin[j] = (T)cellMin * h;
            mmax[j] = (T)cellMax * h;
            n[j] = cellMax - cellMin;
        }
        for (int j = dim; j < 3; ++j) {  // :203-207
            mmin[j] = mmax[j] = T(0);
            n[j] = 1;
        }
        long long nc = ncells();
        if (nc > 4000000000LL || nc <= 0) throw OracleError(E_GRID_TOO_BIG, "grid is too big");  // :209-213
        computeProcessingPartitions();
        masses.assign((size_t)nc, T(0));
        splat([&](int p) {  // MassSplatter — :73-92
            Stencil s; stencil(d.x[p], s, false);
            forNodes(s, [&](int idx, int i, int j, int k) { masses[idx] += d.m[p] * s.weight(i, j, k); });
        });
        for (auto& mm : masses) {  // :226-241
            if (mm < T(0)) mm = T(0);
            if (!finite_(mm)) throw OracleError(E_NAN_MASSES, "nans in splatted masses!");
        }
        velocities.assign((size_t)nc * 3, T(0));
        splat([&](int p) {  // VelocitySplatter — :116-142
            Stencil s; stencil(d.x[p], s, false);
            V3<T> rel = d.v[p] - frameVelocity;
            forNodes(s, [&](int idx, int i, int j, int k) {
                T gm = masses[idx];
                if (gm > T(0)) {
                    T c = s.weight(i, j, k) * (d.m[p] / gm);
                    for (int a = 0; a < 3; ++a) velocities[3 * idx + a] += c * rel[a];
                }
            });
        });
        for (auto vv : velocities)
            if (!finite_(vv)) throw OracleError(E_NAN_VELOCITIES, "nans in splatted velocities!");
        prevVelocities = velocities;
    }

    // computeParticleVolumes — Grid.cpp:265-292
    void computeParticleVolumes() const {
        T cellVolume = h * h * h;
        for (int p : inds) {
            T density(0);
            Stencil s; stencil(d.x[p], s, false);
            forNodes(s, [&](int idx, int i, int j, int k) { density += s.weight(i, j, k) * masses[idx] / cellVolume; });
            d.volume[p] = d.m[p] / density;
        }
    }

    V3<T> nodePos(int i, int j, int k) const {  // Grid.cpp:668, :454
        return V3<T>(h * (T)i + mmin[0], h * (T)j + mmin[1], h * (T)k + mmin[2]);
    }

    // calculateForces — Grid.cpp:438-463 with ForceSplatter :405-428
    void calculateForces(VT& forces, const SnowModel<T>& model, const Fields<T>& fields) const {
        forces.assign(velocities.size(), T(0));
        for (int i = 0; i < n[0]; ++i)
            for (int j = 0; j < n[1]; ++j)
                for (int k = 0; k < n[2]; ++k) {
                    int idx = coordsToIndex(i, j, k);
                    V3<T> f(forces[3 * idx], forces[3 * idx + 1], forces[3 * idx + 2]);
                    fields.force(f, nodePos(i, j, k), masses[idx]);
                    for (int a = 0; a < 3; ++a) forces[3 * idx + a] = f[a];
                }
        splat([&](int p) {
            M3<T> fm = model.dEnergyDensitydF(d, p) * d.volume[p] * d.F[p].transpose();
            Stencil s; stencil(d.x[p], s, true);
            forNodes(s, [&](int idx, int i, int j, int k) {
                V3<T> g = s.grad(i, j, k);
                V3<T> fg = fm * g;
                for (int a = 0; a < 3; ++a) forces[3 * idx + a] -= fg[a];
            });
        });
    }

    // calculateForceDifferentials — Grid.cpp:620-632 with ForceDifferentialSplatter :569-611
    void calculateForceDifferentials(VT& df, const VT& dx, const SnowModel<T>& model) const {
        df.assign(velocities.size(), T(0));
        splat([&](int p) {
            M3<T> dFp;
            Stencil s; stencil(d.x[p], s, true);
            forNodes(s, [&](int idx, int i, int j, int k) {
                V3<T> g = s.grad(i, j, k);
                V3<T> dxi(dx[3 * idx], dx[3 * idx + 1], dx[3 * idx + 2]);
                dFp += outer(dxi, g) * d.F[p];
            });
            M3<T> fm = model.dEdFDifferential(d, dFp, p) * d.volume[p] * d.F[p].transpose();
            forNodes(s, [&](int idx, int i, int j, int k) {
                V3<T> fg = fm * s.grad(i, j, k);
                for (int a = 0; a < 3; ++a) df[3 * idx + a] -= fg[a];
            });
        });
    }

    // dForceidXi — Grid.cpp:539-546 with dFidXiSplatter :484-531
    void dForceidXi(VT& dfdxi, const SnowModel<T>& model) const {
        dfdxi.assign(velocities.size(), T(0));
        splat([&](int p) {
            Stencil s; stencil(d.x[p], s, true);
            forNodes(s, [&](int idx, int i, int j, int k) {
                V3<T> g = s.grad(i, j, k);
                for (int a = 0; a < 3; ++a) {
                    V3<T> e; e[a] = T(1);
                    M3<T> dFpA = outer(e, g) * d.F[p];
                    M3<T> fm = model.dEdFDifferential(d, dFpA, p) * d.volume[p] * d.F[p].transpose();
                    dfdxi[3 * idx + a] += (fm * g)[a] * T(-1);
                }
            });
        });
    }

    // calculateExplicitMomenta — Grid.cpp:634-690
    void calculateExplicitMomenta(VT& explicitMomenta, std::vector<signed char>& collided, T dt, const SnowModel<T>& model,
                                  const std::vector<Collider<T>>& objs, const Fields<T>& fields) {
        VT forces;
        calculateForces(forces, model, fields);
        rec_forces = forces;
        explicitMomenta.assign(velocities.size(), T(0));
        collided.assign(masses.size(), -1);
        for (int i = 0; i < n[0]; ++i)
            for (int j = 0; j < n[1]; ++j)
                for (int k = 0; k < n[2]; ++k) {
                    int idx = coordsToIndex(i, j, k);
                    V3<T> force(forces[3 * idx], forces[3 * idx + 1], forces[3 * idx + 2]);
                    V3<T> ev(velocities[3 * idx], velocities[3 * idx + 1], velocities[3 * idx + 2]);
                    if (masses[idx] > T(0)) ev += force * dt / masses[idx];
                    collided[idx] = (signed char)collide(objs, ev, nodePos(i, j, k), frameVelocity, false);
                    for (int a = 0; a < 3; ++a) explicitMomenta[3 * idx + a] = ev[a] * masses[idx];
                    T prod = explicitMomenta[3 * idx] * explicitMomenta[3 * idx + 1] * explicitMomenta[3 * idx + 2];
                    if (!finite_(prod)) throw OracleError(E_NAN_MOMENTA, "nan in explicit momenta!");
                }
    }

    // collisionVelocities — Grid.cpp:692-724
    void collisionVelocities(VT& vc, const std::vector<Collider<T>>& objs) const {
        vc.assign(velocities.size(), T(0));
        for (int i = 0; i < n[0]; ++i)
            for (int j = 0; j < n[1]; ++j)
                for (int k = 0; k < n[2]; ++k) {
                    int idx = coordsToIndex(i, j, k);
                    if (nodeCollided[idx] < 0) continue;
                    V3<T> vObj = objs[nodeCollided[idx]].velocity(nodePos(i, j, k)) - frameVelocity;
                    for (int a = 0; a < 3; ++a) vc[3 * idx + a] = vObj[a];
                }
    }

    // ImplicitUpdateMatrix::subspaceProject — Grid.cpp:778-818
    void subspaceProject(VT& v, const std::vector<Collider<T>>& objs) const {
        for (int i = 0; i < n[0]; ++i)
            for (int j = 0; j < n[1]; ++j)
                for (int k = 0; k < n[2]; ++k) {
                    int idx = coordsToIndex(i, j, k);
                    int obj = nodeCollided[idx];
                    if (obj == -1) continue;
                    if (obj == -2) { v[3 * idx] = v[3 * idx + 1] = v[3 * idx + 2] = T(0); continue; }
                    V3<T> vv(v[3 * idx], v[3 * idx + 1], v[3 * idx + 2]);
                    V3<T> nn = objs[obj].grad(nodePos(i, j, k));
                    nn.normalize();
                    T nDotP = nn.dot(vv);
                    vv -= nn * nDotP;
                    for (int a = 0; a < 3; ++a) v[3 * idx + a] = vv[a];
                }
    }
    // ImplicitUpdateMatrix::multVector — Grid.cpp:749-771
    void multVector(const VT& vIn, VT& result, const SnowModel<T>& model, const std::vector<Collider<T>>& objs, T dt) const {
        result = vIn;
        subspaceProject(result, objs);
        VT df;
        calculateForceDifferentials(df, result, model);
        for (size_t idx = 0; idx < masses.size(); ++idx)
            for (int a = 0; a < 3; ++a)
                result[3 * idx + a] = masses[idx] * result[3 * idx + a] - dt * dt * df[3 * idx + a];
        subspaceProject(result, objs);
    }

    // ConjugateResiduals::operator() — ConjugateResiduals.cpp:19-160 with SquareMagnitudeTermination
    // (SquareMagnitudeTermination.cpp:13-28) and DiagonalPreconditioner (Grid.cpp:841-877).
    // iterCb(i, x) is the LinearSolver::Debug hook (ConjugateResiduals.cpp:109-112); cancel() is polled the
    // way TerminationCriterion::cancelled is (Sim.cpp:107).
    void conjugateResiduals(const VT& b, VT& x, const VT& diag, int maxIters, T tol, const SnowModel<T>& model,
                            const std::vector<Collider<T>>& objs, T dt,
                            const std::function<void(int, const VT&)>* iterCb = nullptr) {
        const size_t N = b.size();
        T bNorm2 = vdot(b, b);
        stats = SolveStats();
        stats.bNorm2 = (double)bNorm2;
        if (bNorm2 == T(0)) { std::fill(x.begin(), x.end(), T(0)); stats.exitReason = 1; return; }
        T threshold = tol * tol * bNorm2;
        VT r(N), r_pc(N), Ar(N), p(N), Ap(N), pAp(N), Ax(N);
        multVector(x, Ax, model, objs, dt);
        for (size_t i = 0; i < N; ++i) r[i] = b[i] - Ax[i];
        for (size_t i = 0; i < N; ++i) r_pc[i] = r[i] / diag[i];
        p = r_pc;
        multVector(p, Ap, model, objs, dt);
        Ar = Ap;  // A r_precond is the same product as A p here (p == r_precond), ConjugateResiduals.cpp:70-73
        T rz = vdot(r_pc, Ar);
        for (int i = 0;; ++i) {
            for (size_t q = 0; q < N; ++q) pAp[q] = Ap[q] / diag[q];
            T ApdPAp = vdot(Ap, pAp);
            if (ApdPAp == T(0)) { stats.iterations = i; stats.exitReason = 2; return; }
            T alpha = rz / ApdPAp;
            for (size_t q = 0; q < N; ++q) x[q] = x[q] + alpha * p[q];
            subspaceProject(x, objs);
            if (iterCb) (*iterCb)(i, x);
            for (size_t q = 0; q < N; ++q) r_pc[q] = r_pc[q] - alpha * pAp[q];
            for (size_t q = 0; q < N; ++q) r[q] = r_pc[q] * diag[q];
            // SquareMagnitudeTermination::operator()
            stats.iterations = i;
            if (i >= maxIters) return;
            T rNorm2 = vdot(r, r);
            stats.rNorm2 = (double)rNorm2;
            if (rNorm2 < threshold) return;
            multVector(r_pc, Ar, model, objs, dt);
            T rz_old = rz;
            rz = vdot(r_pc, Ar);
            if (rz_old == T(0)) { stats.exitReason = 3; return; }
            T beta = rz / rz_old;
            for (size_t q = 0; q < N; ++q) p[q] = r_pc[q] + beta * p[q];
            for (size_t q = 0; q < N; ++q) Ap[q] = Ar[q] + beta * Ap[q];
        }
    }

    // updateGridVelocities — Grid.cpp:889-1016.  stopBeforeSolve leaves the grid after the rhs and the
    // preconditioner are built (used by the phase tests).
    void updateGridVelocities(T dt, const SnowModel<T>& model, const std::vector<Collider<T>>& objs,
                              const Fields<T>& fields, int maxIters, T tol, bool stopBeforeSolve = false,
                              const std::function<void(int, const VT&)>* iterCb = nullptr) {
        VT explicitMomenta;
        calculateExplicitMomenta(explicitMomenta, nodeCollided, dt, model, objs, fields);
        rec_explicitMomenta = explicitMomenta;
        VT vc;
        collisionVelocities(vc, objs);
        rec_vc = vc;
        // initial guess — :913-947
        T totalMass = 0, collidedMass = 0;
        V3<T> totalMomentum, collidedMomentum;
        for (size_t idx = 0; idx < masses.size(); ++idx) {
            totalMass += masses[idx];
            totalMomentum += V3<T>(explicitMomenta[3 * idx], explicitMomenta[3 * idx + 1], explicitMomenta[3 * idx + 2]);
            if (nodeCollided[idx] >= 0) {
                collidedMass += masses[idx];
                collidedMomentum += V3<T>(vc[3 * idx], vc[3 * idx + 1], vc[3 * idx + 2]) * masses[idx];
            }
        }
        V3<T> guess;
        if (totalMass == T(0)) guess.setZero();
        else if (collidedMass == T(0)) guess = totalMomentum / totalMass;
        else guess = collidedMomentum / collidedMass;
        for (size_t idx = 0; idx < masses.size(); ++idx)
            for (int a = 0; a < 3; ++a) velocities[3 * idx + a] = guess[a];
        rec_x0 = velocities;
        // rhs — :983-1002
        VT df;
        calculateForceDifferentials(df, vc, model);
        subspaceProject(df, objs);
        for (size_t idx = 0; idx < masses.size(); ++idx) {
            for (int a = 0; a < 3; ++a) explicitMomenta[3 * idx + a] += dt * dt * df[3 * idx + a];
            T prod = explicitMomenta[3 * idx] * explicitMomenta[3 * idx + 1] * explicitMomenta[3 * idx + 2];
            if (!finite_(prod)) throw OracleError(E_NAN_MOMENTA, "nan in explicit momenta!");
        }
        rec_rhs = explicitMomenta;
        // DiagonalPreconditioner — :841-867
        VT diag;
        dForceidXi(diag, model);
        for (auto& dd : diag) dd *= -dt * dt;
        for (size_t i = 0; i < masses.size(); ++i)
            for (int a = 0; a < 3; ++a) {
                diag[3 * i + a] += masses[i];
                if (diag[3 * i + a] == T(0)) diag[3 * i + a] = T(1);
            }
        rec_diag = diag;
        if (stopBeforeSolve) return;
        conjugateResiduals(explicitMomenta, velocities, diag, maxIters, tol, model, objs, dt, iterCb);
        rec_solution = velocities;
        for (size_t i = 0; i < velocities.size(); ++i) velocities[i] += vc[i];  // :1014
    }

    // updateDeformationGradients — Grid.cpp:1018-1047
    void updateDeformationGradients(T dt) {
        for (int p : inds) {
            M3<T> delV;
            Stencil s; stencil(d.x[p], s, true);
            forNodes(s, [&](int idx, int i, int j, int k) {
                V3<T> vi(velocities[3 * idx], velocities[3 * idx + 1], velocities[3 * idx + 2]);
                delV += outer(vi, s.grad(i, j, k));
            });
            d.F[p] = (M3<T>::Identity() + delV * dt) * d.F[p];
        }
    }
    // updateParticleVelocities — Grid.cpp:1049-1081
    void updateParticleVelocities() {
        const T alpha = T(0.95);
        for (int p : inds) {
            V3<T> vFlip = d.v[p], vPic;
            Stencil s; stencil(d.x[p], s, false);
            forNodes(s, [&](int idx, int i, int j, int k) {
                T w = s.weight(i, j, k);
                V3<T> vi(velocities[3 * idx], velocities[3 * idx + 1], velocities[3 * idx + 2]);
                V3<T> pi(prevVelocities[3 * idx], prevVelocities[3 * idx + 1], prevVelocities[3 * idx + 2]);
                vFlip += (vi - pi) * w;
                vPic += (vi + frameVelocity) * w;
            });
            d.v[p] = vFlip * alpha + vPic * (T(1) - alpha);
        }
    }
};

// ---------------------------------------------------------------------------------------------------------
// Exact radius query for body segmentation.  Same neighbour set as KDTree::nearestNeighbours
// (KdTree.inl:166-216): points with squared distance strictly below r*r, the query point included.
// ---------------------------------------------------------------------------------------------------------
template <class T> struct RadiusIndex {
    T cell;
    std::unordered_map<long long, std::vector<int>> bins;
    const std::vector<V3<T>>* x = nullptr;
    static long long key(long long i, long long j, long long k) {
        return ((i & 0x1FFFFF) << 42) | ((j & 0x1FFFFF) << 21) | (k & 0x1FFFFF);
    }
    void build(const std::vector<V3<T>>& pts, T r) {
        x = &pts;
        cell = r;
        bins.clear();
        for (int i = 0; i < (int)pts.size(); ++i)
            bins[key((long long)std::floor(pts[i][0] / cell), (long long)std::floor(pts[i][1] / cell),
                     (long long)std::floor(pts[i][2] / cell))].push_back(i);
    }
    void query(const V3<T>& p, T r, std::vector<int>& out) const {
        out.clear();
        T r2 = r * r;
        long long ci = (long long)std::floor(p[0] / cell), cj = (long long)std::floor(p[1] / cell),
                  ck = (long long)std::floor(p[2] / cell);
        for (long long dk = -1; dk <= 1; ++dk)
            for (long long dj = -1; dj <= 1; ++dj)
                for (long long di = -1; di <= 1; ++di) {
                    auto it = bins.find(key(ci + di, cj + dj, ck + dk));
                    if (it == bins.end()) continue;
                    for (int q : it->second) {
                        V3<T> dd = p - (*x)[q];
                        if (dd.squaredNorm() < r2) out.push_back(q);  // KdTree.inl:186-191
                    }
                }
        std::sort(out.begin(), out.end());
    }
};

// ---------------------------------------------------------------------------------------------------------
// Sim — src/MpmSim/Sim.cpp
// ---------------------------------------------------------------------------------------------------------
struct StepStats {
    int nBodies = 0, nBallistic = 0;
    std::vector<SolveStats> solves;
};

template <class T> struct Sim {
    Particles<T> P;
    T h;
    SnowModel<T> model;
    std::vector<Collider<T>> objs;
    Fields<T> fields;
    std::vector<int> ballistic;
    std::vector<std::vector<int>> bodies;
    bool parallel = false;
    bool recordGrids = false;
    int dimension = 3;  // Sim.h:88-89
    std::vector<Grid<T>*> lastGrids;
    StepStats last;

    ~Sim() { clearGrids(); }
    void clearGrids() { for (auto g : lastGrids) delete g; lastGrids.clear(); }

    // Sim::Sim — Sim.cpp:17-50
    Sim(const std::vector<V3<T>>& x, const std::vector<T>& masses, T gridSize, const SnowModel<T>& m,
        const std::vector<Collider<T>>& colls, const Fields<T>& f, bool par = false,
        const std::vector<T>* mu0 = nullptr, const std::vector<T>* lambda0 = nullptr, int dim = 3)
        : h(gridSize), model(m), objs(colls), fields(f), parallel(par), dimension(dim) {
        const size_t n = x.size();
        P.x = x;
        P.v.assign(n, V3<T>());
        P.F.assign(n, M3<T>::Identity());
        P.m = masses;
        P.volume.assign(n, T(0));
        model.setParticles(P);
        if (mu0 && lambda0 && !mu0->empty()) {
            P.mu0 = *mu0; P.lambda0 = *lambda0;
            P.mu = P.mu0; P.lambda = P.lambda0;  // initial Lame values of the per-particle extension
        }
        calculateBodies();
        for (auto& b : bodies) {
            Grid<T> g(P, b, h, V3<T>(), parallel, dimension);
            g.computeParticleVolumes();
        }
    }

    // Sim::calculateBodies — Sim.cpp:136-203
    void calculateBodies() {
        bodies.clear();
        ballistic.clear();
        const size_t n = P.size();
        RadiusIndex<T> index;
        index.build(P.x, h);
        std::vector<char> processed(n, 0);
        std::vector<int> nn;
        for (size_t i = 0; i < n; ++i) {
            T prod = P.v[i][0] * P.v[i][1] * P.v[i][2];
            if (!finite_(prod)) throw OracleError(E_NAN_PARTICLE_V, "nans in particle velocity data!");
            if (processed[i]) continue;
            index.query(P.x[i], h, nn);
            if (nn.size() == 1) { processed[i] = 1; ballistic.push_back((int)i); continue; }
            bodies.emplace_back();
            auto& b = bodies.back();
            std::queue<int> flood;
            for (int q : nn) flood.push(q);
            while (!flood.empty()) {
                int cur = flood.front();
                flood.pop();
                if (processed[cur]) continue;
                b.push_back(cur);
                processed[cur] = 1;
                index.query(P.x[cur], h, nn);
                for (int q : nn) flood.push(q);
            }
        }
    }

    // Sim::advance — Sim.cpp:57-134.
    // stopPhase (phase tests): 1 = stop after every body's rhs + preconditioner, 2 = stop after every body's
    // solve; the particles are left untouched in both.
    // batched = the CUDA path's schedule: every body's grid is built and solved first, then each body's
    // G2P + F update, then one plasticity pass.  The reference re-runs the plasticity pass over all particles
    // after each body (Sim.cpp:118); that pass is idempotent on particles it already processed, so the two
    // schedules agree up to round-off (tests/test_oracle_sim.py checks this).
    // Returns 1 if cancelled.
    int advance(T dt, int maxIters, T tol, int stopPhase = 0, const std::function<bool()>* cancelled = nullptr,
                const std::function<void(int, int, const std::vector<T>&)>* iterCb = nullptr, bool batched = false) {
        clearGrids();
        last = StepStats();
        last.nBodies = (int)bodies.size();
        last.nBallistic = (int)ballistic.size();
        for (int p : ballistic) {  // :66-73
            V3<T> accn;
            fields.force(accn, P.x[p], P.m[p]);
            accn = accn / P.m[p];
            P.v[p] += accn * dt;
        }
        const bool deferParticles = stopPhase != 0 || batched;
        for (size_t b = 0; b < bodies.size(); ++b) {  // :79-120
            V3<T> comV;
            T mass = 0;
            for (int p : bodies[b]) { comV += P.v[p] * P.m[p]; mass += P.m[p]; }
            comV = comV / mass;
            Grid<T>* g = new Grid<T>(P, bodies[b], h, comV, parallel, dimension);
            lastGrids.push_back(g);
            std::function<void(int, const std::vector<T>&)> cb;
            if (iterCb) cb = [&](int i, const std::vector<T>& xx) { (*iterCb)((int)b, i, xx); };
            g->updateGridVelocities(dt, model, objs, fields, maxIters, tol, stopPhase == 1, iterCb ? &cb : nullptr);
            last.solves.push_back(g->stats);
            if (deferParticles) continue;
            if (cancelled && (*cancelled)()) { calculateBodies(); return 1; }  // :107-111
            g->updateParticleVelocities();
            g->updateDeformationGradients(dt);
            model.updateParticleData(P);
            if (!recordGrids) { delete g; lastGrids.pop_back(); }
        }
        if (stopPhase != 0) return 0;
        if (batched) {
            if (cancelled && (*cancelled)()) { calculateBodies(); return 1; }
            for (auto g : lastGrids) { g->updateParticleVelocities(); g->updateDeformationGradients(dt); }
            if (!bodies.empty()) model.updateParticleData(P);
            if (!recordGrids) clearGrids();
        }
        for (size_t i = 0; i < P.size(); ++i) {  // :123-131
            collide(objs, P.v[i], P.x[i], V3<T>(), true);
            P.x[i] += P.v[i] * dt;
        }
        calculateBodies();
        return 0;
    }
};

}  // namespace mpm_oracle

// The Houdini SOP's cook logic without Houdini (mpmsnow_b200/host/MpmSimSOP.h): particle seeding from a sampled
// SDF on the GPU against a host restatement of SOP_MPMSim.cpp:168-214 (same lattice, same float trilinear
// sampling: positions bit for bit), the initial velocity from the sampled velocity field, cooks that advance by
// sub-steps with a sampled ground as the collider set, and an interrupted cook.  Prints one line per failed check;
// exits 0 when all pass, 1 when any fails, 3 (with "NO_DEVICE") without a CUDA device.
#include <cmath>
#include <cstdio>
#include <string>

#include "MpmSimSOP.h"

using namespace MpmSimHoudini;

static int g_failures = 0;
#define CHECK(c)                                                     \
    do {                                                             \
        if (!(c)) {                                                  \
            std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c); \
            ++g_failures;                                            \
        }                                                            \
    } while (0)

// phi of a sampled field at x, trilinear, as the library evaluates it (separately rounded float operations)
static float lerp(float a, float b, float t) { return a + t * (b - a); }
static bool sample_phi(const SampledField& f, const float x[3], float& phi) {
    int i0[3];
    float t[3];
    for (int a = 0; a < 3; ++a) {
        const float u = (x[a] - f.origin[a]) / f.spacing;
        if (!(u >= 0.f) || u > (float)(f.n[a] - 1)) return false;
        const int i = std::min((int)std::floor(u), f.n[a] - 2);
        i0[a] = i;
        t[a] = u - (float)i;
    }
    float v[8];
    for (int q = 0; q < 8; ++q)
        v[q] = f.phi[(size_t)(i0[0] + (q & 1)) + f.n[0] * ((size_t)(i0[1] + ((q >> 1) & 1)) + f.n[1] * (size_t)(i0[2] + (q >> 2)))];
    const float x00 = lerp(v[0], v[1], t[0]), x10 = lerp(v[2], v[3], t[0]);
    const float x01 = lerp(v[4], v[5], t[0]), x11 = lerp(v[6], v[7], t[0]);
    phi = lerp(lerp(x00, x10, t[1]), lerp(x01, x11, t[1]), t[2]);
    return true;
}

static SampledField sphere_field(float cx, float cy, float cz, float r, float spacing, int n, float vx) {
    SampledField f;
    f.n[0] = f.n[1] = f.n[2] = n;
    f.spacing = spacing;
    const float half = 0.5f * spacing * (n - 1);
    f.origin = MpmSim::Vector3f(cx - half, cy - half, cz - half);
    f.phi.resize((size_t)n * n * n);
    f.velocity.resize(3 * f.phi.size());
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const size_t q = i + (size_t)n * (j + (size_t)n * k);
                const float dx = f.origin[0] + spacing * i - cx, dy = f.origin[1] + spacing * j - cy,
                            dz = f.origin[2] + spacing * k - cz;
                f.phi[q] = std::sqrt(dx * dx + dy * dy + dz * dz) - r;
                f.velocity[3 * q] = vx;
            }
    f.bboxMin = MpmSim::Vector3f(cx - r, cy - r, cz - r);
    f.bboxMax = MpmSim::Vector3f(cx + r, cy + r, cz + r);
    return f;
}

static SampledField ground_field() {  // phi = y over a box below and around the snowball
    SampledField f;
    f.n[0] = 41; f.n[1] = 21; f.n[2] = 41;
    f.spacing = 0.01f;
    f.origin = MpmSim::Vector3f(-0.2f, -0.1f, -0.2f);
    f.phi.resize((size_t)f.n[0] * f.n[1] * f.n[2]);
    for (int k = 0; k < f.n[2]; ++k)
        for (int j = 0; j < f.n[1]; ++j)
            for (int i = 0; i < f.n[0]; ++i) f.phi[i + (size_t)f.n[0] * (j + (size_t)f.n[1] * k)] = f.origin[1] + f.spacing * j;
    return f;
}

int main() {
    const SampledField ball = sphere_field(0.f, 0.06f, 0.f, 0.05f, 0.005f, 31, 0.5f);
    {
        const mpm_collider d = ball.descriptor();
        size_t count = 0;
        if (mpm_seed_particles(&d, ball.bboxMin.data(), ball.bboxMax.data(), 0.005f, 400.f, 0, nullptr, nullptr,
                               nullptr, 0, &count) == MPM_ERR_NO_DEVICE) {
            std::printf("NO_DEVICE\n");
            return 3;
        }
    }
    SopParameters p;
    p.gridSize = 0.01f;
    p.subSteps = 4;
    p.tolerance = 1e-5f;
    // the host restatement of the seeding lattice (SOP_MPMSim.cpp:171-195)
    const float h = p.gridSize / 2;
    std::vector<MpmSim::Vector3f> expect;
    int dims[3];
    for (int a = 0; a < 3; ++a) dims[a] = (int)std::ceil((ball.bboxMax[a] - ball.bboxMin[a]) / h);
    for (int i = 0; i < dims[0]; ++i)
        for (int j = 0; j < dims[1]; ++j)
            for (int k = 0; k < dims[2]; ++k) {
                const float x[3] = {(float)(ball.bboxMin[0] + (i + 0.5) * h), (float)(ball.bboxMin[1] + (j + 0.5) * h),
                                    (float)(ball.bboxMin[2] + (k + 0.5) * h)};
                float phi;
                if (sample_phi(ball, x, phi) && phi < 0.f) expect.emplace_back(x[0], x[1], x[2]);
            }
    try {
        SopSimulation sop;
        sop.initSim(ball, p);
        const std::vector<MpmSim::Vector3f>& x0 = sop.sim()->particleData().variable<MpmSim::Vector3f>("p");
        CHECK(x0.size() == expect.size() && expect.size() > 500);
        bool same = x0.size() == expect.size();
        for (size_t q = 0; same && q < x0.size(); ++q)
            for (int a = 0; a < 3; ++a) same = same && x0[q][a] == expect[q][a];
        CHECK(same);
        const std::vector<float>& m = sop.sim()->particleData().variable<float>("m");
        CHECK(!m.empty() && m[0] == 400.f * h * h * h);
        const std::vector<MpmSim::Vector3f>& v0 = sop.sim()->particleData().variable<MpmSim::Vector3f>("v");
        CHECK(!v0.empty() && std::fabs(v0[0][0] - 0.5f) < 1e-6f && v0[0][1] == 0.f);
        const std::vector<MpmSim::Vector3f> start = x0;
        const std::vector<SampledField> colliders{ground_field()};
        double t = 0.0;
        for (int frame = 1; frame <= 3; ++frame) {
            const double tn = frame / 24.0;
            sop.cook(tn, t, colliders);
            t = tn;
        }
        const std::vector<MpmSim::Vector3f>& x1 = sop.sim()->particleData().variable<MpmSim::Vector3f>("p");
        float ymin = 1e9f, dx = 0.f, dy = 0.f;
        for (size_t q = 0; q < x1.size(); ++q) {
            ymin = std::fmin(ymin, x1[q][1]);
            dx += (x1[q][0] - start[q][0]) / x1.size();
            dy += (x1[q][1] - start[q][1]) / x1.size();
        }
        CHECK(dy < -1e-3f);               // fell
        CHECK(dx > 1e-3f);                // carried by the sampled initial velocity
        CHECK(ymin > -0.5f * p.gridSize);  // stopped by the sampled ground
        // an interrupted cook: the step is cancelled after its solve and leaves the particles where they were
        const std::vector<MpmSim::Vector3f> before = x1;
        sop.cook(t + 1.0 / 24.0, t, colliders, [] { return true; });
        const std::vector<MpmSim::Vector3f>& x2 = sop.sim()->particleData().variable<MpmSim::Vector3f>("p");
        bool unchanged = true;
        for (size_t q = 0; q < x2.size(); ++q)
            for (int a = 0; a < 3; ++a) unchanged = unchanged && x2[q][a] == before[q][a];
        CHECK(unchanged);
    } catch (const MpmSim::Error& e) {
        std::printf("FAIL unexpected error %d: %s\n", (int)e.status, e.what());
        return 1;
    }
    if (g_failures == 0) std::printf("OK\n");
    return g_failures == 0 ? 0 : 1;
}

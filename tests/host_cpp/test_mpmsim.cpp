// The C++ MpmSim API (mpmsnow_b200/host/MpmSim.h) driven the way the reference's tests drive Sim
// (src/tests/TestSimClass.cpp): body partition at construction, the gravity known answer, particle variables,
// the unknown-variable message, cancellation and the Debug hook.  Prints one line per failed check and exits
// 0 when all pass, 1 when any fails, and 3 (with "NO_DEVICE") when there is no CUDA device to run on.
#include <cmath>
#include <cstdio>
#include <string>

#include "MpmSim.h"

using namespace MpmSim;

static int g_failures = 0;
#define CHECK(c)                                                                  \
    do {                                                                          \
        if (!(c)) {                                                               \
            std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c);              \
            ++g_failures;                                                         \
        }                                                                         \
    } while (0)

// The scene of TestSimClass.cpp:120-190: two interleaved 4 x 4 x 4 blocks at half a cell spacing (two bodies)
// and a 4 x 4 x 4 lattice at 1.1 cells (64 ballistic particles), unit masses, h = 0.1, gravity +1 in y.
struct Scene {
    std::vector<Vector3f> x;
    std::vector<float> m;
    float h = 0.1f;
    CubicBsplineShapeFunction shape;
    SnowConstitutiveModel snow{1.4e5f, 0.2f, 0.0f, 1e5f, 1e5f};
    CollisionObject::CollisionObjectSet colliders;
    ForceField::ForceFieldSet fields;
    Scene() {
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j)
                for (int k = 0; k < 4; ++k) {
                    const float a[3] = {0.5f * h * i, 0.5f * h * j, 0.5f * h * k};
                    x.emplace_back(a[0], a[1], a[2]);
                    x.emplace_back(a[0] + 6.f, a[1], a[2]);
                }
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j)
                for (int k = 0; k < 4; ++k) x.emplace_back(20.f + 1.1f * h * i, 1.1f * h * j, 1.1f * h * k);
        m.assign(x.size(), 1.f);
        fields.add(new GravityField(Vector3f(0.f, 1.f, 0.f)));
    }
    Sim make() { return Sim(x, m, h, shape, snow, colliders, fields); }
};

static void test_bodies(Sim& sim) {
    int nb = 0, nbal = 0;
    const std::vector<int> b = sim.bodies(&nb, &nbal);
    CHECK(nb == 2);
    CHECK(nbal == 64);
    CHECK(b[0] == 0 && b[1] == 1 && b[2] == 0 && b[3] == 1);  // bodies numbered by their smallest particle
    CHECK(b[128] == -1 && b[191] == -1);
}

static void test_variables(Sim& sim, const Scene& sc) {
    const std::vector<float>& m = sim.particleData().variable<float>("m");
    CHECK(m.size() == sc.x.size() && m[0] == 1.f);
    const std::vector<Matrix3f>& F = sim.particleData().variable<Matrix3f>("F");
    CHECK(F[5](0, 0) == 1.f && F[5](0, 1) == 0.f && F[5](2, 2) == 1.f);
    const std::vector<Vector3f>& p = sim.particleData().variable<Vector3f>("p");
    CHECK(p[1][0] == sc.x[1][0] && p[1][1] == sc.x[1][1]);
    bool threw = false;
    try {
        sim.particleData().variable<float>("nope");
    } catch (const Error& e) {
        threw = e.status == MPM_ERR_UNKNOWN_VARIABLE &&
                std::string(e.what()) == "Material point data has no variable named 'nope'";
    }
    CHECK(threw);
    bool wrongType = false;
    try {
        sim.particleData().variable<float>("v");
    } catch (const Error& e) {
        wrongType = e.status == MPM_ERR_WRONG_SIZE;
    }
    CHECK(wrongType);
}

static void test_gravity(Sim& sim, size_t n) {
    SquareMagnitudeTermination term(10, 0.f);
    for (int s = 0; s < 3; ++s) sim.advance(0.01f, term);
    const std::vector<Vector3f>& v = sim.particleData().variable<Vector3f>("v");
    double mean[3] = {0, 0, 0};
    for (const Vector3f& a : v)
        for (int c = 0; c < 3; ++c) mean[c] += a[c] / (double)n;
    CHECK(std::fabs(mean[0]) < 1e-6 && std::fabs(mean[2]) < 1e-6);
    CHECK(std::fabs(mean[1] - 0.03) < 1e-5);
}

static void test_reference_lives_across_advance(Sim& sim) {
    // as in the reference, the vector behind variable<T>() lives as long as the Sim: a reference taken before
    // advance() reads the step's new values, and a variable that was only read is not written back
    const std::vector<Vector3f>& p = sim.particleData().variable<Vector3f>("p");
    std::vector<float>& mu = sim.particleData().variable<float>("mu");
    const Vector3f* storage = p.data();
    const float before = p[130][1];
    const float mu0 = mu[0];
    SquareMagnitudeTermination term(10, 1e-5f);
    sim.advance(0.01f, term);
    CHECK(p.data() == storage);
    CHECK(p[130][1] != before);  // a ballistic particle under gravity +1 in y
    CHECK(&sim.particleData().variable<Vector3f>("p") == &p);
    CHECK(mu[0] == mu0);
}

static void test_upload(Sim& sim) {
    // a velocity written through the view is uploaded at the next advance: a ballistic particle moves by v dt
    std::vector<Vector3f>& v = sim.particleData().variable<Vector3f>("v");
    const float x0 = sim.particleData().variable<Vector3f>("p")[150][0];
    v[150] = Vector3f(2.f, 0.f, 0.f);
    SquareMagnitudeTermination term(10, 1e-5f);
    sim.advance(0.01f, term);
    const float x1 = sim.particleData().variable<Vector3f>("p")[150][0];
    CHECK(std::fabs((x1 - x0) - 0.02f) < 1e-5f);
}

struct CancelAll : SquareMagnitudeTermination {
    CancelAll() : SquareMagnitudeTermination(60, 1e-5f) {}
    bool cancelled() const override { return true; }
};

struct CountIterates : LinearSolver::Debug {
    size_t calls = 0, floats = 0;
    void operator()(std::vector<float>& x) override {
        ++calls;
        floats += x.size();
    }
};

static void test_cancel_and_debug(Sim& sim) {
    const std::vector<Vector3f> before = sim.particleData().variable<Vector3f>("p");
    CancelAll cancel;
    sim.advance(0.01f, cancel);
    const std::vector<Vector3f>& after = sim.particleData().variable<Vector3f>("p");
    bool same = true;
    for (size_t i = 0; i < before.size(); ++i)
        for (int c = 0; c < 3; ++c) same = same && before[i][c] == after[i][c];
    CHECK(same);
    CountIterates dbg;
    SquareMagnitudeTermination term(60, 1e-5f);
    sim.advance(0.01f, term, &dbg);
    const mpm_step_stats& st = sim.lastStepStats();
    size_t expect = 0;
    for (int b = 0; b < st.num_bodies; ++b) expect += (size_t)st.iterations[b] + 1;
    CHECK(dbg.calls == expect && dbg.calls > 0 && dbg.floats % 3 == 0);
}

int main() {
    Scene sc;
    try {
        Sim sim = sc.make();
        test_bodies(sim);
        test_variables(sim, sc);
        test_gravity(sim, sc.x.size());
        test_reference_lives_across_advance(sim);
        test_upload(sim);
        test_cancel_and_debug(sim);
    } catch (const Error& e) {
        if (e.status == MPM_ERR_NO_DEVICE) {
            std::printf("NO_DEVICE %s\n", e.what());
            return 3;
        }
        std::printf("FAIL unexpected error %d: %s\n", (int)e.status, e.what());
        return 1;
    }
    if (g_failures == 0) std::printf("OK\n");
    return g_failures == 0 ? 0 : 1;
}

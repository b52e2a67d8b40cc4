// Host-side parts of the C++ MpmSim API (mpmsnow_b200/host/MpmSim.h) that need no device: what the collider
// and force-field objects hand to the C-ABI, the sets' ownership, the termination criterion's parameters, and
// the arguments Sim rejects before it creates anything.  Exits 0 when every check passes.
#include <cstdio>
#include <string>

#include "MpmSim.h"

using namespace MpmSim;

static int g_failures = 0;
#define CHECK(c)                                                     \
    do {                                                             \
        if (!(c)) {                                                  \
            std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c); \
            ++g_failures;                                            \
        }                                                            \
    } while (0)

struct Counted : CollisionPlane {
    static int alive;
    Counted() : CollisionPlane(Vector4f(0.f, 1.f, 0.f, 0.f)) { ++alive; }
    ~Counted() override { --alive; }
};
int Counted::alive = 0;

struct Elastic : ConstitutiveModel {};
struct Never : TerminationCriterion {
    bool cancelled() const override { return false; }
};

int main() {
    // CollisionPlane(c, coulombFriction = 0.5, sticky = false) (CollisionPlane.h:9) as the C-ABI's descriptor
    CollisionPlane plane(Vector4f(-0.5f, 0.866f, 0.f, 0.1f));
    mpm_collider d = plane.descriptor();
    CHECK(d.kind == MPM_COLLIDER_PLANE && d.coeffs[0] == -0.5f && d.coeffs[1] == 0.866f && d.coeffs[3] == 0.1f);
    CHECK(d.friction == 0.5f && d.sticky == 0 && d.velocity[0] == 0.f);
    plane.setV(Vector3f(1.f, 2.f, 3.f));
    plane.setCoeffs(Vector4f(0.f, 1.f, 0.f, -2.f));
    d = plane.descriptor();
    CHECK(d.velocity[2] == 3.f && d.coeffs[3] == -2.f);
    CollisionPlane sticky(Vector4f(1.f, 0.f, 0.f, 0.f), 0.25f, true);
    CHECK(sticky.descriptor().sticky == 1 && sticky.descriptor().friction == 0.25f);

    // CollisionCylinder(cx, cz, radius, coulombFriction = 0.5, sticky = false): the C5 scene's vertical cylinder
    CollisionCylinder cyl(0.4f, 0.5f, 0.1f, 0.3f);
    cyl.setV(Vector3f(0.f, 0.f, -1.f));
    d = cyl.descriptor();
    CHECK(d.kind == MPM_COLLIDER_CYLINDER && d.coeffs[0] == 0.4f && d.coeffs[1] == 0.5f && d.coeffs[2] == 0.1f);
    CHECK(d.coeffs[3] == 0.f && d.friction == 0.3f && d.sticky == 0 && d.velocity[2] == -1.f);

    // GridCollisionObject: samples stay with the object; the descriptor points at them
    std::vector<float> phi(3 * 4 * 5, 1.f);
    GridCollisionObject grid(phi, 3, 4, 5, Vector3f(-1.f, 0.f, 2.f), 0.25f);
    d = grid.descriptor();
    CHECK(d.kind == MPM_COLLIDER_GRID && d.grid_dims[0] == 3 && d.grid_dims[1] == 4 && d.grid_dims[2] == 5);
    CHECK(d.coeffs[0] == -1.f && d.coeffs[2] == 2.f && d.coeffs[3] == 0.25f && d.grid_velocity == nullptr);
    CHECK(d.grid_phi != nullptr && d.grid_phi[59] == 1.f && d.friction == 0.5f && d.sticky == 0);
    bool threw = false;
    try {
        GridCollisionObject bad(std::vector<float>(7, 0.f), 3, 4, 5, Vector3f(), 0.25f);
    } catch (const Error& e) {
        threw = e.status == MPM_ERR_INVALID_ARGUMENT;
    }
    CHECK(threw);

    GravityField g(Vector3f(0.f, -9.81f, 0.f));
    CHECK(g.gravity()[1] == -9.81f);

    // the sets own what is added, as the reference's do
    {
        CollisionObject::CollisionObjectSet set;
        set.add(new Counted());
        set.add(new Counted());
        CHECK(set.numObjects() == 2 && Counted::alive == 2);
    }
    CHECK(Counted::alive == 0);

    SquareMagnitudeTermination t(60, 1e-5f);
    CHECK(t.maxIters() == 60 && t.tolError() == 1e-5f && !t.cancelled());

    // arguments Sim rejects before any device call
    std::vector<Vector3f> x(4, Vector3f(0.f, 0.f, 0.f));
    std::vector<float> m(4, 1.f);
    CubicBsplineShapeFunction shape;
    CollisionObject::CollisionObjectSet none;
    ForceField::ForceFieldSet fields;
    Elastic elastic;
    try {
        Sim s(x, m, 0.01f, shape, elastic, none, fields);
        CHECK(false);
    } catch (const Error& e) {
        CHECK(e.status == MPM_ERR_UNSUPPORTED);
    }
    SnowConstitutiveModel snow(1.4e5f, 0.2f, 10.f, 2.5e-2f, 7.5e-3f);
    std::vector<float> m3(3, 1.f);
    try {
        Sim s(x, m3, 0.01f, shape, snow, none, fields);
        CHECK(false);
    } catch (const Error& e) {
        CHECK(e.status == MPM_ERR_INVALID_ARGUMENT);
    }
    if (g_failures == 0) std::printf("OK\n");
    return g_failures == 0 ? 0 : 1;
}

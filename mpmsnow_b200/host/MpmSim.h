// The reference's MpmSim C++ API (include/MpmSim/*.h of davidsminor/mpmsnow) over this library's C-ABI
// (include/mpm_gpu.h): Sim, MaterialPointData, SnowConstitutiveModel, CubicBsplineShapeFunction, CollisionPlane,
// GravityField, SquareMagnitudeTermination and LinearSolver::Debug keep the reference's names, constructor
// arguments and exception messages, so code written against the reference compiles against this header with
// its Eigen types swapped for the small ones below.  Header-only, C++17; link -lmpmsnow_b200.
//
// Differences from the reference, all forced by the GPU owning the particle state:
//  * Vector3f / Vector4f / Matrix3f are packed floats (Eigen is not a dependency of this library); matrices are
//    row-major, as they cross the C-ABI.
//  * MaterialPointData::variable<T>() returns host vectors that live as long as the Sim, as the reference's do.
//    Sim::advance refreshes every fetched vector with the step's values and, before the step, uploads those
//    whose contents the caller changed.
//  * LinearSolver::Debug receives each body's iterate as a std::vector<float> (3 per grid node).
//  * Only SquareMagnitudeTermination, CollisionPlane, CollisionCylinder (a vertical solid cylinder, which the
//    reference lacks), GridCollisionObject (a sampled collider in place of the Houdini plugin's
//    VDBCollisionObject) and GravityField are translated; other subclasses throw.
//  * The reference's Sim reads its colliders through references each step; here Sim::setCollisionObject passes
//    a changed collider to the device.
#pragma once

#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "mpm_gpu.h"

namespace MpmSim {

struct Vector3f {
    float v[3];
    Vector3f(float x = 0.f, float y = 0.f, float z = 0.f) : v{x, y, z} {}
    float& operator[](int i) { return v[i]; }
    float operator[](int i) const { return v[i]; }
    float* data() { return v; }
    const float* data() const { return v; }
};
struct Vector4f {
    float v[4];
    Vector4f(float a = 0.f, float b = 0.f, float c = 0.f, float d = 0.f) : v{a, b, c, d} {}
    float& operator[](int i) { return v[i]; }
    float operator[](int i) const { return v[i]; }
};
struct Matrix3f {
    float m[9];  // row-major
    Matrix3f() : m{} {}
    float& operator()(int r, int c) { return m[3 * r + c]; }
    float operator()(int r, int c) const { return m[3 * r + c]; }
    static Matrix3f Identity() {
        Matrix3f a;
        a(0, 0) = a(1, 1) = a(2, 2) = 1.f;
        return a;
    }
};
static_assert(sizeof(Vector3f) == 3 * sizeof(float) && sizeof(Matrix3f) == 9 * sizeof(float), "packed floats");

// A C-ABI failure: the reference's exception text, with the status code beside it.
class Error : public std::runtime_error {
public:
    Error(mpm_status s, const std::string& what) : std::runtime_error(what), status(s) {}
    mpm_status status;
};

class ShapeFunction {
public:
    virtual ~ShapeFunction() = default;
    virtual int id() const = 0;  // the C-ABI's shape_function code
};
class CubicBsplineShapeFunction : public ShapeFunction {
public:
    int id() const override { return 0; }
};

class ConstitutiveModel {
public:
    virtual ~ConstitutiveModel() = default;
};
// SnowConstitutiveModel.h:13-18
class SnowConstitutiveModel : public ConstitutiveModel {
public:
    SnowConstitutiveModel(float youngsModulus, float poissonRatio, float hardening, float compressiveStrength,
                          float tensileStrength)
        : youngsModulus(youngsModulus), poissonRatio(poissonRatio), hardening(hardening),
          compressiveStrength(compressiveStrength), tensileStrength(tensileStrength) {}
    float youngsModulus, poissonRatio, hardening, compressiveStrength, tensileStrength;
};

class CollisionObject {
public:
    virtual ~CollisionObject() = default;
    virtual mpm_collider descriptor() const = 0;
    // CollisionObject.h:33-41; the set owns what is added, as the reference's does
    class CollisionObjectSet {
    public:
        CollisionObjectSet() = default;
        CollisionObjectSet(const CollisionObjectSet&) = delete;
        CollisionObjectSet& operator=(const CollisionObjectSet&) = delete;
        void add(CollisionObject* o) { m_objects.emplace_back(o); }
        size_t numObjects() const { return m_objects.size(); }
        const CollisionObject* object(size_t i) const { return m_objects[i].get(); }

    private:
        std::vector<std::unique_ptr<CollisionObject>> m_objects;
    };
};
// CollisionPlane.h:9-18: phi = c0 x + c1 y + c2 z + c3
class CollisionPlane : public CollisionObject {
public:
    explicit CollisionPlane(const Vector4f& c, float coulombFriction = 0.5f, bool sticky = false)
        : m_c(c), m_friction(coulombFriction), m_sticky(sticky) {}
    void setCoeffs(const Vector4f& c) { m_c = c; }
    void setV(const Vector3f& v) { m_v = v; }
    float coulombFriction() const { return m_friction; }
    bool sticky() const { return m_sticky; }
    mpm_collider descriptor() const override {
        mpm_collider d{};
        d.kind = MPM_COLLIDER_PLANE;
        for (int k = 0; k < 4; ++k) d.coeffs[k] = m_c[k];
        for (int k = 0; k < 3; ++k) d.velocity[k] = m_v[k];
        d.friction = m_friction;
        d.sticky = m_sticky ? 1 : 0;
        return d;
    }

private:
    Vector4f m_c;
    Vector3f m_v;
    float m_friction;
    bool m_sticky;
};

// A solid vertical cylinder (axis along y through (cx, cz)), phi = |(x - cx, z - cz)| - radius.  No reference
// counterpart: a CollisionObject subclass with CollisionPlane's friction and sticky arguments.
class CollisionCylinder : public CollisionObject {
public:
    CollisionCylinder(float cx, float cz, float radius, float coulombFriction = 0.5f, bool sticky = false)
        : m_cx(cx), m_cz(cz), m_r(radius), m_friction(coulombFriction), m_sticky(sticky) {}
    void setV(const Vector3f& v) { m_v = v; }
    float coulombFriction() const { return m_friction; }
    bool sticky() const { return m_sticky; }
    mpm_collider descriptor() const override {
        mpm_collider d{};
        d.kind = MPM_COLLIDER_CYLINDER;
        d.coeffs[0] = m_cx;
        d.coeffs[1] = m_cz;
        d.coeffs[2] = m_r;
        for (int k = 0; k < 3; ++k) d.velocity[k] = m_v[k];
        d.friction = m_friction;
        d.sticky = m_sticky ? 1 : 0;
        return d;
    }

private:
    float m_cx, m_cz, m_r;
    Vector3f m_v;
    float m_friction;
    bool m_sticky;
};

// A collider sampled on a dense grid, in place of the Houdini plugin's VDBCollisionObject (VDBCollisionObject.h:
// 14-31, friction 0.5 and not sticky by default as there): phi at origin + spacing (i, j, k), i < nx (x fastest),
// and optionally a sampled velocity (3 per sample).  phi and the velocity are trilinear between samples, grad is
// the gradient of the trilinear phi; outside the sampled box there is no collider.  The samples are copied to
// the device when a Sim is built with it (or given it through Sim::setCollisionObject).
class GridCollisionObject : public CollisionObject {
public:
    GridCollisionObject(std::vector<float> phi, int nx, int ny, int nz, const Vector3f& origin, float spacing,
                        std::vector<float> velocity = {}, float coulombFriction = 0.5f, bool sticky = false)
        : m_phi(std::move(phi)), m_vel(std::move(velocity)), m_n{nx, ny, nz}, m_origin(origin), m_spacing(spacing),
          m_friction(coulombFriction), m_sticky(sticky) {
        const size_t cnt = (size_t)nx * ny * nz;
        if (nx < 2 || ny < 2 || nz < 2 || m_phi.size() != cnt || (!m_vel.empty() && m_vel.size() != 3 * cnt))
            throw Error(MPM_ERR_INVALID_ARGUMENT, "grid collider: phi needs nx ny nz samples (each >= 2), the "
                                                  "velocity 3 per sample or none");
    }
    float coulombFriction() const { return m_friction; }
    bool sticky() const { return m_sticky; }
    mpm_collider descriptor() const override {
        mpm_collider d{};
        d.kind = MPM_COLLIDER_GRID;
        for (int k = 0; k < 3; ++k) d.coeffs[k] = m_origin[k];
        d.coeffs[3] = m_spacing;
        d.friction = m_friction;
        d.sticky = m_sticky ? 1 : 0;
        for (int k = 0; k < 3; ++k) d.grid_dims[k] = m_n[k];
        d.grid_phi = m_phi.data();
        d.grid_velocity = m_vel.empty() ? nullptr : m_vel.data();
        return d;
    }

private:
    std::vector<float> m_phi, m_vel;
    int m_n[3];
    Vector3f m_origin;
    float m_spacing;
    float m_friction;
    bool m_sticky;
};

class ForceField {
public:
    virtual ~ForceField() = default;
    virtual Vector3f gravity() const = 0;
    // ForceField.h:21-30; the set owns what is added
    class ForceFieldSet {
    public:
        ForceFieldSet() = default;
        ForceFieldSet(const ForceFieldSet&) = delete;
        ForceFieldSet& operator=(const ForceFieldSet&) = delete;
        void add(ForceField* f) { m_fields.emplace_back(f); }
        size_t numFields() const { return m_fields.size(); }
        const ForceField* field(size_t i) const { return m_fields[i].get(); }

    private:
        std::vector<std::unique_ptr<ForceField>> m_fields;
    };
};
// GravityField.h:9
class GravityField : public ForceField {
public:
    explicit GravityField(const Vector3f& gravity) : m_g(gravity) {}
    Vector3f gravity() const override { return m_g; }

private:
    Vector3f m_g;
};

// TerminationCriterion.h:7-15: the solve's termination; cancelled() is polled after the grid solve
class TerminationCriterion {
public:
    virtual ~TerminationCriterion() = default;
    virtual bool cancelled() const = 0;
};
// SquareMagnitudeTermination.h:9: |r|^2 < tolError^2 |b|^2 or maxIters iterations
class SquareMagnitudeTermination : public TerminationCriterion {
public:
    SquareMagnitudeTermination(int maxIters, float tolError) : m_maxIters(maxIters), m_tolError(tolError) {}
    int maxIters() const { return m_maxIters; }
    float tolError() const { return m_tolError; }
    bool cancelled() const override { return false; }

private:
    int m_maxIters;
    float m_tolError;
};

// LinearSolver.h:12-16
class LinearSolver {
public:
    class Debug {
    public:
        virtual ~Debug() = default;
        virtual void operator()(std::vector<float>& x) = 0;
    };
};

class Sim;

// MaterialPointData.h:8-20, over the device state of one Sim.  As in the reference, a variable's vector lives
// as long as the Sim: references taken with variable<T>() stay valid across advance(), which refreshes every
// variable the caller has fetched with the step's new values (a device-to-host copy per fetched variable and
// step).  Writes through a reference are uploaded at the next advance(): a variable whose contents differ from
// the values last exchanged with the device goes up, one that was only read does not.
class MaterialPointData {
public:
    template <typename T>
    std::vector<T>& variable(const std::string& name) {
        return *static_cast<std::vector<T>*>(fetch<T>(name).data.get());
    }
    template <typename T>
    const std::vector<T>& variable(const std::string& name) const {
        return *static_cast<const std::vector<T>*>(const_cast<MaterialPointData*>(this)->fetch<T>(name).data.get());
    }
    size_t numParticles() const;

private:
    friend class Sim;
    explicit MaterialPointData(Sim& s) : m_sim(s) {}
    struct Slot {
        std::shared_ptr<void> data;   // the caller's vector, kept for the Sim's lifetime
        std::vector<float> shadow;    // the values last downloaded or uploaded
        size_t floats = 0;
        float* (*ptr)(void*) = nullptr;
    };
    template <typename T>
    Slot& fetch(const std::string& name);
    void download(const std::string& name, Slot& s);
    void flush();    // upload the variables the caller changed
    void refresh();  // the device state moved on: download every fetched variable into its vector
    Sim& m_sim;
    std::map<std::string, Slot> m_slots;
};

// Sim.h:20-52
class Sim {
public:
    Sim(const std::vector<Vector3f>& x, const std::vector<float>& masses, float gridSize,
        const ShapeFunction& shapeFunction, ConstitutiveModel& model,
        const CollisionObject::CollisionObjectSet& collisionObjects, const ForceField::ForceFieldSet& forceFields,
        int dimension = 3, int device = 0)
        : m_data(*this) {
        const SnowConstitutiveModel* snow = dynamic_cast<const SnowConstitutiveModel*>(&model);
        if (!snow) throw Error(MPM_ERR_UNSUPPORTED, "only SnowConstitutiveModel is supported");
        if (x.size() != masses.size()) throw Error(MPM_ERR_INVALID_ARGUMENT, "x and masses differ in length");
        std::vector<mpm_collider> cs;
        for (size_t i = 0; i < collisionObjects.numObjects(); ++i) cs.push_back(collisionObjects.object(i)->descriptor());
        std::vector<float> g;
        for (size_t i = 0; i < forceFields.numFields(); ++i) {
            const Vector3f v = forceFields.field(i)->gravity();
            g.insert(g.end(), v.data(), v.data() + 3);
        }
        mpm_scene_desc d{};
        d.grid_size = gridSize;
        d.dimension = dimension;
        d.shape_function = shapeFunction.id();
        d.youngs_modulus = snow->youngsModulus;
        d.poisson_ratio = snow->poissonRatio;
        d.hardening = snow->hardening;
        d.compressive_strength = snow->compressiveStrength;
        d.tensile_strength = snow->tensileStrength;
        d.num_colliders = (int)cs.size();
        d.colliders = cs.data();
        d.num_gravity_fields = (int)forceFields.numFields();
        d.gravity = g.data();
        d.device = device;
        const float* xp = x.empty() ? nullptr : x[0].data();
        const mpm_status st = mpm_create(&d, x.size(), xp, masses.data(), &m_gpu);
        if (st != MPM_OK) throw Error(st, mpm_status_string(st));
    }
    ~Sim() { mpm_destroy(m_gpu); }
    Sim(const Sim&) = delete;
    Sim& operator=(const Sim&) = delete;

    MaterialPointData& particleData() { return m_data; }

    // Replaces collision object `index` between steps (no reference counterpart: the reference's Sim holds the
    // caller's objects by reference, so a moved CollisionPlane (setCoeffs / setV) or a Houdini cook's new VDB
    // takes effect at the next advance; here the new descriptor is passed to the device).
    void setCollisionObject(int index, const CollisionObject& object) {
        const mpm_collider d = object.descriptor();
        check(mpm_set_collider(m_gpu, index, &d));
    }

    // Sim.cpp:57-134: one implicit step; terminationCriterion.cancelled() is polled after the solve, and a
    // cancelled step leaves the particles where they were
    void advance(float timeStep, TerminationCriterion& terminationCriterion, LinearSolver::Debug* d = nullptr) {
        const SquareMagnitudeTermination* t = dynamic_cast<const SquareMagnitudeTermination*>(&terminationCriterion);
        if (!t) throw Error(MPM_ERR_UNSUPPORTED, "only SquareMagnitudeTermination is supported");
        m_data.flush();
        mpm_solve_params sp{t->maxIters(), t->tolError()};
        const mpm_status st = mpm_step_ex(m_gpu, timeStep, &sp, 0, &Sim::cancelThunk, &terminationCriterion,
                                          d ? &Sim::debugThunk : nullptr, d, &m_stats);
        if (st != MPM_OK && st != MPM_ERR_CANCELLED) check(st);
        m_data.refresh();
    }

    // the body partition of the last calculateBodies (Sim.cpp:136-203): body per particle, -1 = ballistic
    std::vector<int> bodies(int* numBodies = nullptr, int* numBallistic = nullptr) {
        std::vector<int> b(numParticles());
        int nb = 0, nbal = 0;
        check(mpm_get_bodies(m_gpu, b.data(), &nb, &nbal));
        if (numBodies) *numBodies = nb;
        if (numBallistic) *numBallistic = nbal;
        return b;
    }
    size_t numParticles() const { return mpm_num_particles(m_gpu); }
    // solver statistics of the last advance (no reference counterpart)
    const mpm_step_stats& lastStepStats() const { return m_stats; }
    mpm_sim* handle() { return m_gpu; }

    void check(mpm_status st) {
        if (st != MPM_OK) throw Error(st, mpm_last_error(m_gpu));
    }

private:
    static int cancelThunk(void* ctx) { return static_cast<TerminationCriterion*>(ctx)->cancelled() ? 1 : 0; }
    static void debugThunk(void* ctx, int, int, const float* x, size_t count) {
        std::vector<float> v(x, x + count);
        (*static_cast<LinearSolver::Debug*>(ctx))(v);
    }
    mpm_sim* m_gpu = nullptr;
    MaterialPointData m_data;
    mpm_step_stats m_stats{};
};

inline size_t MaterialPointData::numParticles() const { return m_sim.numParticles(); }

template <typename T>
MaterialPointData::Slot& MaterialPointData::fetch(const std::string& name) {
    static_assert(sizeof(T) % sizeof(float) == 0, "variables are made of floats");
    auto it = m_slots.find(name);
    if (it != m_slots.end() && it->second.floats != sizeof(T) / sizeof(float) * numParticles())
        throw Error(MPM_ERR_WRONG_SIZE, "Material point data variable '" + name + "' has another type");
    if (it != m_slots.end()) return it->second;
    int comps = 0;
    const mpm_status st = mpm_variable_info(m_sim.handle(), name.c_str(), &comps);
    if (st == MPM_ERR_UNKNOWN_VARIABLE)  // MaterialPointData.inl:23
        throw Error(st, "Material point data has no variable named '" + name + "'");
    if (st != MPM_OK) throw Error(st, mpm_status_string(st));
    if ((size_t)comps * sizeof(float) != sizeof(T))
        throw Error(MPM_ERR_WRONG_SIZE, "Material point data variable '" + name + "' has " + std::to_string(comps) +
                                            " components");
    auto vec = std::make_shared<std::vector<T>>(numParticles());
    Slot s;
    s.floats = (size_t)comps * vec->size();
    s.ptr = [](void* p) { return reinterpret_cast<float*>(static_cast<std::vector<T>*>(p)->data()); };
    s.data = vec;
    Slot& slot = m_slots.emplace(name, s).first->second;
    download(name, slot);
    return slot;
}

inline void MaterialPointData::download(const std::string& name, Slot& s) {
    float* dst = s.ptr(s.data.get());
    m_sim.check(mpm_get_variable(m_sim.handle(), name.c_str(), dst, s.floats));
    s.shadow.assign(dst, dst + s.floats);
}

inline void MaterialPointData::flush() {
    for (auto& kv : m_slots) {
        Slot& s = kv.second;
        const float* cur = s.ptr(s.data.get());
        if (s.floats == 0 || std::memcmp(cur, s.shadow.data(), s.floats * sizeof(float)) == 0) continue;
        m_sim.check(mpm_set_variable(m_sim.handle(), kv.first.c_str(), cur, s.floats));
        s.shadow.assign(cur, cur + s.floats);
    }
}

inline void MaterialPointData::refresh() {
    for (auto& kv : m_slots) download(kv.first, kv.second);
}

}  // namespace MpmSim

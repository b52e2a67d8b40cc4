// The Houdini plugin's simulation SOP (src/houdiniPlugin/SOP_MPMSim.cpp of davidsminor/mpmsnow) without Houdini:
// its cook logic over this library's C++ API (MpmSim.h), with the HDK types replaced by plain sampled fields.
// A SOP built with the HDK keeps its parameter templates, input locking and geometry output, and forwards to
// SopSimulation:
//   * initSim (SOP_MPMSim.cpp:138-222): the input VDBs sampled onto a dense grid (phi, and velocity "v" when the
//     input has one) become a GridCollisionObject-style SampledField; the particles are seeded from it on the GPU
//     (mpm_seed_particles: lattice at half the grid size inside phi < 0, density 400, the sampled velocity);
//   * cookMySop (SOP_MPMSim.cpp:224-372): a cook at the start frame restarts the simulation; other cooks advance
//     it by subSteps steps of (t - previous cook time) / subSteps, with the collision VDBs of inputs 1.. as the
//     collider set, a termination whose cancelled() is the UT_Interrupt (HoudiniSolveTermination.cpp:13-26), and
//     return the particle positions for the SOP to write out.
// The gravity field (0, -9.8, 0) and the initial density 400 are the SOP's constants (SOP_MPMSim.cpp:161, 182).
#pragma once

#include <cmath>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "MpmSim.h"

namespace MpmSimHoudini {

// A field sampled on a dense grid: phi (nx ny nz values, x fastest) at origin + spacing (i, j, k) and optionally a
// velocity (3 per sample) — what the SOP reads from a GEO_PrimVDB pair (SOP_MPMSim.cpp:113-136), resampled.
struct SampledField {
    std::vector<float> phi, velocity;
    int n[3] = {0, 0, 0};
    MpmSim::Vector3f origin;
    float spacing = 0.f;
    MpmSim::Vector3f bboxMin, bboxMax;  // the bounding box of the field's active region (GEO_PrimVDB::getBBox)

    mpm_collider descriptor() const {
        mpm_collider d{};
        d.kind = MPM_COLLIDER_GRID;
        for (int k = 0; k < 3; ++k) d.coeffs[k] = origin[k];
        d.coeffs[3] = spacing;
        d.friction = 0.5f;  // VDBCollisionObject::coulombFriction (VDBCollisionObject.cpp:39-42)
        d.sticky = 0;       // VDBCollisionObject::sticky (:44-47)
        for (int k = 0; k < 3; ++k) d.grid_dims[k] = n[k];
        d.grid_phi = phi.data();
        d.grid_velocity = velocity.empty() ? nullptr : velocity.data();
        return d;
    }
};

// The SOP's parameters (SOP_MPMSim.cpp:37-90) and their defaults.
struct SopParameters {
    float gridSize = 0.1f;
    int subSteps = 1;
    float tolerance = 1e-4f;
    int maxIterations = 60;
    float youngsModulus = 1.4e5f;
    float poissonRatio = 0.2f;
    float hardening = 10.f;
    float compressiveStrength = 2.5e-2f;
    float tensileStrength = 7.5e-3f;
};

// HoudiniSolveTermination (HoudiniSolveTermination.h): SquareMagnitudeTermination whose cancelled() polls the
// host's interrupt.
class HoudiniSolveTermination : public MpmSim::SquareMagnitudeTermination {
public:
    HoudiniSolveTermination(int maxIters, float tolError, std::function<bool()> interrupted)
        : SquareMagnitudeTermination(maxIters, tolError), m_interrupted(std::move(interrupted)) {}
    bool cancelled() const override { return m_interrupted && m_interrupted(); }

private:
    std::function<bool()> m_interrupted;
};

// A collider set rebuilt from sampled fields at every cook.
class SampledCollisionObject : public MpmSim::CollisionObject {
public:
    explicit SampledCollisionObject(const SampledField& f) : m_field(f) {}
    mpm_collider descriptor() const override { return m_field.descriptor(); }

private:
    const SampledField& m_field;
};

class SopSimulation {
public:
    // SOP_MPMSim::initSim: seeds particles inside `initialState` and builds the Sim (no colliders until a cook).
    void initSim(const SampledField& initialState, const SopParameters& p, int device = 0) {
        m_sim.reset();
        m_params = p;
        const float h = p.gridSize / 2;  // SOP_MPMSim.cpp:171
        const mpm_collider sdf = initialState.descriptor();
        size_t count = 0;
        mpm_status st = mpm_seed_particles(&sdf, initialState.bboxMin.data(), initialState.bboxMax.data(), h, 400.f,
                                           device, nullptr, nullptr, nullptr, 0, &count);
        if (st != MPM_OK && st != MPM_ERR_WRONG_SIZE) throw MpmSim::Error(st, mpm_status_string(st));
        m_x.assign(count, MpmSim::Vector3f());
        std::vector<MpmSim::Vector3f> v(count);
        std::vector<float> m(count);
        if (count > 0) {
            st = mpm_seed_particles(&sdf, initialState.bboxMin.data(), initialState.bboxMax.data(), h, 400.f, device,
                                    m_x[0].data(), v[0].data(), m.data(), count, &count);
            if (st != MPM_OK) throw MpmSim::Error(st, mpm_status_string(st));
        }
        m_model.reset(new MpmSim::SnowConstitutiveModel(p.youngsModulus, p.poissonRatio, p.hardening,
                                                        p.compressiveStrength, p.tensileStrength));
        m_fields.reset(new MpmSim::ForceField::ForceFieldSet());
        m_fields->add(new MpmSim::GravityField(MpmSim::Vector3f(0.f, -9.8f, 0.f)));
        m_colliders.reset(new MpmSim::CollisionObject::CollisionObjectSet());
        m_sim.reset(new MpmSim::Sim(m_x, m, p.gridSize, m_shape, *m_model, *m_colliders, *m_fields, 3, device));
        if (!initialState.velocity.empty())  // SOP_MPMSim.cpp:202-214
            m_sim->particleData().variable<MpmSim::Vector3f>("v") = v;
    }

    bool initialised() const { return (bool)m_sim; }

    // SOP_MPMSim::cookMySop from the second cook on: advances from the previous cook time to t in subSteps
    // steps with `colliders` as the collider set; a step that throws is reported to `log` and the cook goes on,
    // as the SOP does (SOP_MPMSim.cpp:346-353).  Returns the particle positions.
    const std::vector<MpmSim::Vector3f>& cook(double t, double prevCookTime, const std::vector<SampledField>& colliders,
                                              const std::function<bool()>& interrupted = {},
                                              const std::function<void(const std::string&)>& log = {}) {
        if (!m_sim) throw MpmSim::Error(MPM_ERR_INVALID_ARGUMENT, "no particles!");
        const int steps = m_params.subSteps;
        const float dt = float(t - prevCookTime) / steps;
        std::vector<mpm_collider> cs;
        for (const SampledField& f : colliders) cs.push_back(f.descriptor());
        m_sim->check(mpm_set_colliders(m_sim->handle(), (int)cs.size(), cs.empty() ? nullptr : cs.data()));
        for (int i = 0; i < steps; ++i) {
            try {
                HoudiniSolveTermination term(m_params.maxIterations, m_params.tolerance, interrupted);
                m_sim->advance(dt, term);
                if (interrupted && interrupted()) break;
            } catch (const std::exception& e) {
                if (log) log(e.what());
            }
        }
        m_x = m_sim->particleData().variable<MpmSim::Vector3f>("p");
        return m_x;
    }

    MpmSim::Sim* sim() { return m_sim.get(); }

private:
    SopParameters m_params;
    MpmSim::CubicBsplineShapeFunction m_shape;
    std::unique_ptr<MpmSim::SnowConstitutiveModel> m_model;
    std::unique_ptr<MpmSim::ForceField::ForceFieldSet> m_fields;
    std::unique_ptr<MpmSim::CollisionObject::CollisionObjectSet> m_colliders;
    std::unique_ptr<MpmSim::Sim> m_sim;
    std::vector<MpmSim::Vector3f> m_x;
};

}  // namespace MpmSimHoudini

// CPU ORACLE — test infrastructure only.  extern "C" entry points over mpm_oracle.hpp so that tests/ and
// bench.py's CPU arm can drive the restatement through ctypes.  All arrays cross this boundary as double
// (converted to/from the instance's type T on entry/exit); matrices are row-major 3x3.
#include "mpm_oracle.hpp"

#include <chrono>
#include <cstdio>
#include <memory>

using namespace mpm_oracle;

extern "C" {

typedef struct {
    int kind;          // 0 plane, 1 vertical cylinder, 2 sampled signed-distance grid
    double c[4];       // plane coefficients / (cx, cz, radius, unused) / grid (origin x, y, z, spacing)
    double vel[3];
    double friction;
    int sticky;
    int dims[3];           // grid: samples per axis
    const double* phi;     // grid: dims product values, x fastest
    const double* gvel;    // grid: 3 per sample, or null
} orc_collider;

typedef struct {
    int nBodies, nBallistic;
    int iterations[64];
    double bNorm2[64], rNorm2[64];
    int exitReason[64];
} orc_step_stats;
}

namespace {

struct Base {
    virtual ~Base() {}
    int prec = 32;
    std::string err;
};

template <class T> struct Impl : Base {
    std::unique_ptr<Sim<T>> sim;
};

template <class T> Collider<T> toCollider(const orc_collider& c) {
    Collider<T> o;
    o.kind = c.kind;
    for (int i = 0; i < 4; ++i) o.c[i] = (T)c.c[i];
    for (int i = 0; i < 3; ++i) o.vel[i] = (T)c.vel[i];
    o.friction = (T)c.friction;
    o.sticky = c.sticky != 0;
    if (c.kind == 2) {
        const long cnt = (long)c.dims[0] * c.dims[1] * c.dims[2];
        for (int i = 0; i < 3; ++i) o.n[i] = c.dims[i];
        o.gphi = std::make_shared<std::vector<T>>(cnt);
        for (long i = 0; i < cnt; ++i) (*o.gphi)[i] = (T)c.phi[i];
        if (c.gvel) {
            o.gvel = std::make_shared<std::vector<T>>(3 * cnt);
            for (long i = 0; i < 3 * cnt; ++i) (*o.gvel)[i] = (T)c.gvel[i];
        }
    }
    return o;
}

template <class T> void getVar(const Particles<T>& P, const std::string& name, double* dst, int& ok) {
    ok = 1;
    size_t n = P.size();
    auto v3 = [&](const std::vector<V3<T>>& a) { for (size_t i = 0; i < n; ++i) for (int k = 0; k < 3; ++k) dst[3 * i + k] = (double)a[i][k]; };
    auto m3 = [&](const std::vector<M3<T>>& a) {
        for (size_t i = 0; i < n; ++i) for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) dst[9 * i + 3 * r + c] = (double)a[i].a[r][c];
    };
    auto s1 = [&](const std::vector<T>& a) { for (size_t i = 0; i < n; ++i) dst[i] = (double)a[i]; };
    if (name == "p") v3(P.x);
    else if (name == "v") v3(P.v);
    else if (name == "F") m3(P.F);
    else if (name == "Fp") m3(P.Fp);
    else if (name == "FinvTrans") m3(P.FinvTrans);
    else if (name == "R") m3(P.R);
    else if (name == "Ginv") m3(P.Ginv);
    else if (name == "m") s1(P.m);
    else if (name == "volume") s1(P.volume);
    else if (name == "J") s1(P.J);
    else if (name == "mu") s1(P.mu);
    else if (name == "lambda") s1(P.lambda);
    else ok = 0;
}
template <class T> void setVar(Particles<T>& P, const std::string& name, const double* src, int& ok) {
    ok = 1;
    size_t n = P.size();
    auto v3 = [&](std::vector<V3<T>>& a) { for (size_t i = 0; i < n; ++i) for (int k = 0; k < 3; ++k) a[i][k] = (T)src[3 * i + k]; };
    auto m3 = [&](std::vector<M3<T>>& a) {
        for (size_t i = 0; i < n; ++i) for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) a[i].a[r][c] = (T)src[9 * i + 3 * r + c];
    };
    auto s1 = [&](std::vector<T>& a) { for (size_t i = 0; i < n; ++i) a[i] = (T)src[i]; };
    if (name == "p") v3(P.x);
    else if (name == "v") v3(P.v);
    else if (name == "F") m3(P.F);
    else if (name == "Fp") m3(P.Fp);
    else if (name == "FinvTrans") m3(P.FinvTrans);
    else if (name == "R") m3(P.R);
    else if (name == "Ginv") m3(P.Ginv);
    else if (name == "m") s1(P.m);
    else if (name == "volume") s1(P.volume);
    else if (name == "J") s1(P.J);
    else if (name == "mu") s1(P.mu);
    else if (name == "lambda") s1(P.lambda);
    else ok = 0;
}

template <class T> Impl<T>* as(void* h) { return static_cast<Impl<T>*>(static_cast<Base*>(h)); }

void copyMsg(char* msg, const std::string& s) {
    if (msg) { std::snprintf(msg, 256, "%s", s.c_str()); }
}

template <class T>
Base* create(long n, const double* x, const double* m, const double* mu0, const double* lambda0, double h, const double* snow,
             int ncoll, const orc_collider* colls, int ngrav, const double* grav, int threads, int dim, int& status,
             char* msg) {
    std::vector<V3<T>> X(n);
    std::vector<T> M(n), MU0, LA0;
    for (long i = 0; i < n; ++i) {
        X[i] = V3<T>((T)x[3 * i], (T)x[3 * i + 1], (T)x[3 * i + 2]);
        M[i] = (T)m[i];
    }
    if (mu0 && lambda0) {
        MU0.resize(n); LA0.resize(n);
        for (long i = 0; i < n; ++i) { MU0[i] = (T)mu0[i]; LA0[i] = (T)lambda0[i]; }
    }
    SnowModel<T> model((T)snow[0], (T)snow[1], (T)snow[2], (T)snow[3], (T)snow[4]);
    std::vector<Collider<T>> objs;
    for (int i = 0; i < ncoll; ++i) objs.push_back(toCollider<T>(colls[i]));
    Fields<T> fields;
    for (int i = 0; i < ngrav; ++i) fields.gravity.push_back(V3<T>((T)grav[3 * i], (T)grav[3 * i + 1], (T)grav[3 * i + 2]));
    if (threads > 0 && WorkerPool::instance().threads() != threads) WorkerPool::instance().setThreads(threads);
    auto* impl = new Impl<T>();
    impl->prec = sizeof(T) == 4 ? 32 : 64;
    try {
        impl->sim.reset(new Sim<T>(X, M, (T)h, model, objs, fields, threads > 1, MU0.empty() ? nullptr : &MU0,
                                   LA0.empty() ? nullptr : &LA0, dim));
        impl->sim->recordGrids = true;
        status = 0;
    } catch (OracleError& e) {
        status = e.code;
        copyMsg(msg, e.what());
        delete impl;
        return nullptr;
    }
    return impl;
}

template <class T> int advance(Base* b, double dt, int maxIters, double tol, int stopPhase, int batched, orc_step_stats* st, char* msg) {
    auto* impl = static_cast<Impl<T>*>(b);
    try {
        impl->sim->advance((T)dt, maxIters, (T)tol, stopPhase, nullptr, nullptr, batched != 0);
    } catch (OracleError& e) {
        copyMsg(msg, e.what());
        return e.code;
    }
    if (st) {
        auto& L = impl->sim->last;
        st->nBodies = L.nBodies;
        st->nBallistic = L.nBallistic;
        for (int i = 0; i < 64 && i < (int)L.solves.size(); ++i) {
            st->iterations[i] = L.solves[i].iterations;
            st->bNorm2[i] = L.solves[i].bNorm2;
            st->rNorm2[i] = L.solves[i].rNorm2;
            st->exitReason[i] = L.solves[i].exitReason;
        }
    }
    return 0;
}

template <class T> Grid<T>* gridOf(Base* b, int g) {
    auto* impl = static_cast<Impl<T>*>(b);
    if (g < 0 || g >= (int)impl->sim->lastGrids.size()) return nullptr;
    return impl->sim->lastGrids[g];
}

template <class T> int gridGet(Base* b, int gi, const std::string& name, double* dst) {
    Grid<T>* g = gridOf<T>(b, gi);
    if (!g) return 1;
    const std::vector<T>* src = nullptr;
    if (name == "masses") src = &g->masses;
    else if (name == "velocities") src = &g->velocities;
    else if (name == "prevVelocities") src = &g->prevVelocities;
    else if (name == "explicitMomenta") src = &g->rec_explicitMomenta;
    else if (name == "rhs") src = &g->rec_rhs;
    else if (name == "vc") src = &g->rec_vc;
    else if (name == "diag") src = &g->rec_diag;
    else if (name == "x0") src = &g->rec_x0;
    else if (name == "solution") src = &g->rec_solution;
    else if (name == "forces") src = &g->rec_forces;
    else if (name == "nodeCollided") {
        for (size_t i = 0; i < g->nodeCollided.size(); ++i) dst[i] = g->nodeCollided[i];
        return 0;
    }
    if (!src) return 2;
    for (size_t i = 0; i < src->size(); ++i) dst[i] = (double)(*src)[i];
    return 0;
}

template <class T> int gridApply(Base* b, int gi, const std::string& op, const double* in, double* out, double dt) {
    auto* impl = static_cast<Impl<T>*>(b);
    Grid<T>* g = gridOf<T>(b, gi);
    if (!g) return 1;
    std::vector<T> x(g->velocities.size()), y;
    for (size_t i = 0; i < x.size(); ++i) x[i] = (T)in[i];
    try {
        if (op == "A") g->multVector(x, y, impl->sim->model, impl->sim->objs, (T)dt);
        else if (op == "DF") g->calculateForceDifferentials(y, x, impl->sim->model);
        else if (op == "dFidXi") g->dForceidXi(y, impl->sim->model);
        else return 2;
    } catch (OracleError& e) {
        return e.code;
    }
    for (size_t i = 0; i < y.size(); ++i) out[i] = (double)y[i];
    return 0;
}

}  // namespace

extern "C" {

void* orc_create(int prec, long n, const double* x, const double* m, const double* mu0, const double* lambda0, double h,
                 const double* snow, int ncoll, const orc_collider* colls, int ngrav, const double* grav, int threads,
                 int dim, int* status, char* msg) {
    int st = 0;
    if (dim < 1 || dim > 3) {
        if (status) *status = 1;
        copyMsg(msg, "dimension must be 1, 2 or 3");
        return nullptr;
    }
    Base* b = prec == 64 ? create<double>(n, x, m, mu0, lambda0, h, snow, ncoll, colls, ngrav, grav, threads, dim, st, msg)
                         : create<float>(n, x, m, mu0, lambda0, h, snow, ncoll, colls, ngrav, grav, threads, dim, st, msg);
    if (status) *status = st;
    return b;
}

void orc_destroy(void* h) { delete static_cast<Base*>(h); }

int orc_advance(void* h, double dt, int maxIters, double tol, int stopPhase, int batched, orc_step_stats* st, char* msg) {
    Base* b = static_cast<Base*>(h);
    return b->prec == 64 ? advance<double>(b, dt, maxIters, tol, stopPhase, batched, st, msg)
                         : advance<float>(b, dt, maxIters, tol, stopPhase, batched, st, msg);
}

long orc_num_particles(void* h) {
    Base* b = static_cast<Base*>(h);
    return b->prec == 64 ? (long)as<double>(h)->sim->P.size() : (long)as<float>(h)->sim->P.size();
}

int orc_get(void* h, const char* name, double* dst) {
    Base* b = static_cast<Base*>(h);
    int ok = 0;
    if (b->prec == 64) getVar<double>(as<double>(h)->sim->P, name, dst, ok);
    else getVar<float>(as<float>(h)->sim->P, name, dst, ok);
    return ok ? 0 : 1;
}

int orc_set(void* h, const char* name, const double* src) {
    Base* b = static_cast<Base*>(h);
    int ok = 0;
    if (b->prec == 64) setVar<double>(as<double>(h)->sim->P, name, src, ok);
    else setVar<float>(as<float>(h)->sim->P, name, src, ok);
    return ok ? 0 : 1;
}

// body id per particle (-1 = ballistic), in the reference's body order
int orc_bodies(void* h, int* bodyOf, int* nBodies, int* nBallistic) {
    Base* b = static_cast<Base*>(h);
    auto fill = [&](auto* sim) {
        const size_t n = sim->P.size();
        for (size_t i = 0; i < n; ++i) bodyOf[i] = -1;
        for (size_t k = 0; k < sim->bodies.size(); ++k)
            for (int p : sim->bodies[k]) bodyOf[p] = (int)k;
        *nBodies = (int)sim->bodies.size();
        *nBallistic = (int)sim->ballistic.size();
    };
    if (b->prec == 64) fill(as<double>(h)->sim.get());
    else fill(as<float>(h)->sim.get());
    return 0;
}

int orc_num_grids(void* h) {
    Base* b = static_cast<Base*>(h);
    return b->prec == 64 ? (int)as<double>(h)->sim->lastGrids.size() : (int)as<float>(h)->sim->lastGrids.size();
}

int orc_grid_info(void* h, int g, double* min3, int* n3, double* frameV3, int* nParticles) {
    Base* b = static_cast<Base*>(h);
    auto fill = [&](auto* gr) {
        if (!gr) return 1;
        for (int k = 0; k < 3; ++k) { min3[k] = (double)gr->mmin[k]; n3[k] = gr->n[k]; frameV3[k] = (double)gr->frameVelocity[k]; }
        *nParticles = (int)gr->inds.size();
        return 0;
    };
    return b->prec == 64 ? fill(gridOf<double>(b, g)) : fill(gridOf<float>(b, g));
}

int orc_grid_get(void* h, int g, const char* name, double* dst) {
    Base* b = static_cast<Base*>(h);
    return b->prec == 64 ? gridGet<double>(b, g, name, dst) : gridGet<float>(b, g, name, dst);
}

int orc_grid_apply(void* h, int g, const char* op, const double* in, double* out, double dt) {
    Base* b = static_cast<Base*>(h);
    return b->prec == 64 ? gridApply<double>(b, g, op, in, out, dt) : gridApply<float>(b, g, op, in, out, dt);
}

// Particles of grid g in the grid's voxel-sorted order, with each particle's stencil base node
// (ShapeFunctionIterator::initialize, Grid.cpp:1114-1119), its voxel (Grid.cpp:373-374) and colour.
int orc_grid_particles(void* h, int g, int* inds, int* base3, int* voxel3, int* colour) {
    Base* b = static_cast<Base*>(h);
    auto fill = [&](auto* gr) {
        if (!gr) return 1;
        using TT = std::remove_reference_t<decltype(gr->h)>;
        TT voxelSize = TT(4) * gr->h;
        for (size_t q = 0; q < gr->inds.size(); ++q) {
            int p = gr->inds[q];
            inds[q] = p;
            typename std::remove_pointer_t<decltype(gr)>::Stencil s;
            gr->stencil(gr->d.x[p], s, false);
            int vx[3];
            for (int k = 0; k < 3; ++k) {
                base3[3 * q + k] = s.base[k];
                vx[k] = (int)std::floor(gr->d.x[p][k] / voxelSize);
                voxel3[3 * q + k] = vx[k];
            }
            colour[q] = (vx[0] & 1) + 2 * (vx[1] & 1) + 4 * (vx[2] & 1);
        }
        return 0;
    };
    return b->prec == 64 ? fill(gridOf<double>(b, g)) : fill(gridOf<float>(b, g));
}

// --- pure functions ----------------------------------------------------------------------------------
void orc_bspline(int prec, long n, const double* x, double* w, double* dw) {
    for (long i = 0; i < n; ++i) {
        if (prec == 64) { w[i] = CubicBspline<double>::w(x[i]); dw[i] = CubicBspline<double>::dw(x[i]); }
        else { w[i] = CubicBspline<float>::w((float)x[i]); dw[i] = CubicBspline<float>::dw((float)x[i]); }
    }
}

int orc_collide(int prec, int ncoll, const orc_collider* colls, double* v, const double* x, const double* frameV, int addCV) {
    auto run = [&](auto zero) {
        using T = decltype(zero);
        std::vector<Collider<T>> objs;
        for (int i = 0; i < ncoll; ++i) objs.push_back(toCollider<T>(colls[i]));
        V3<T> vv((T)v[0], (T)v[1], (T)v[2]), xx((T)x[0], (T)x[1], (T)x[2]), fv((T)frameV[0], (T)frameV[1], (T)frameV[2]);
        int r = collide(objs, vv, xx, fv, addCV != 0);
        for (int k = 0; k < 3; ++k) v[k] = (double)vv[k];
        return r;
    };
    return prec == 64 ? run(0.0) : run(0.0f);
}

// SnowConstitutiveModel::updateParticleData over n particles held in the caller's arrays (row-major 3x3).
int orc_snow_update(int prec, const double* snow, long n, double* F, double* Fp, double* FinvTrans, double* R, double* Ginv,
                    double* J, double* mu, double* lambda) {
    auto run = [&](auto zero) {
        using T = decltype(zero);
        SnowModel<T> model((T)snow[0], (T)snow[1], (T)snow[2], (T)snow[3], (T)snow[4]);
        Particles<T> P;
        P.m.assign(n, T(1));
        P.x.assign(n, V3<T>());
        model.setParticles(P);
        P.F.resize(n);
        int ok;
        setVar<T>(P, "F", F, ok);
        setVar<T>(P, "Fp", Fp, ok);
        try { model.updateParticleData(P); } catch (OracleError& e) { return e.code; }
        getVar<T>(P, "F", F, ok); getVar<T>(P, "Fp", Fp, ok); getVar<T>(P, "FinvTrans", FinvTrans, ok);
        getVar<T>(P, "R", R, ok); getVar<T>(P, "Ginv", Ginv, ok); getVar<T>(P, "J", J, ok);
        getVar<T>(P, "mu", mu, ok); getVar<T>(P, "lambda", lambda, ok);
        return 0;
    };
    return prec == 64 ? run(0.0) : run(0.0f);
}

// energyDensity, dEnergyDensitydF and dEdFDifferential(dF) of one particle state.
int orc_snow_eval(int prec, const double* snow, const double* F, const double* R, const double* FinvTrans, const double* Ginv,
                  double J, double mu, double lambda, const double* dF, double* energy, double* dEdF, double* dEdFdiff) {
    auto run = [&](auto zero) {
        using T = decltype(zero);
        SnowModel<T> model((T)snow[0], (T)snow[1], (T)snow[2], (T)snow[3], (T)snow[4]);
        Particles<T> P;
        P.m.assign(1, T(1));
        P.x.assign(1, V3<T>());
        model.setParticles(P);
        P.F.resize(1);
        int ok;
        setVar<T>(P, "F", F, ok); setVar<T>(P, "R", R, ok); setVar<T>(P, "FinvTrans", FinvTrans, ok);
        setVar<T>(P, "Ginv", Ginv, ok);
        P.J[0] = (T)J; P.mu[0] = (T)mu; P.lambda[0] = (T)lambda;
        M3<T> dFm;
        for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) dFm.a[r][c] = (T)dF[3 * r + c];
        try {
            *energy = (double)model.energyDensity(P, 0);
            M3<T> a = model.dEnergyDensitydF(P, 0), b = model.dEdFDifferential(P, dFm, 0);
            for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) { dEdF[3 * r + c] = a.a[r][c]; dEdFdiff[3 * r + c] = b.a[r][c]; }
        } catch (OracleError& e) { return e.code; }
        return 0;
    };
    return prec == 64 ? run(0.0) : run(0.0f);
}

// Dense conjugate residuals on a caller matrix (TestConjugateResiduals.cpp:14-38 / :43-102).  Returns the
// per-iteration residuals and search directions (the solver's m_log record) when the buffers are given.
int orc_cr_dense(int prec, int n, const double* A, const double* b, double* x, int maxIters, double tol, double* residuals,
                 double* directions, int* nrec) {
    auto run = [&](auto zero) {
        using T = decltype(zero);
        std::vector<T> AA(n * n), bb(n), xx(n, T(0));
        for (int i = 0; i < n * n; ++i) AA[i] = (T)A[i];
        for (int i = 0; i < n; ++i) bb[i] = (T)b[i];
        auto mult = [&](const std::vector<T>& v, std::vector<T>& out) {
            out.assign(n, T(0));
            for (int i = 0; i < n; ++i) { T s = 0; for (int j = 0; j < n; ++j) s += AA[i * n + j] * v[j]; out[i] = s; }
        };
        int rec = 0;
        auto log = [&](const std::vector<T>& r, const std::vector<T>& p) {
            if (residuals) for (int i = 0; i < n; ++i) residuals[rec * n + i] = (double)r[i];
            if (directions) for (int i = 0; i < n; ++i) directions[rec * n + i] = (double)p[i];
            ++rec;
        };
        // ConjugateResiduals.cpp:19-160 without preconditioner, SquareMagnitudeTermination(maxIters, tol)
        T bNorm2 = vdot(bb, bb);
        if (bNorm2 == T(0)) { for (int i = 0; i < n; ++i) x[i] = 0; *nrec = 0; return 0; }
        T threshold = (T)tol * (T)tol * bNorm2;
        std::vector<T> r(n), Ar(n), p(n), Ap(n), Ax(n);
        mult(xx, Ax);
        for (int i = 0; i < n; ++i) r[i] = bb[i] - Ax[i];
        p = r;
        mult(p, Ap);
        Ar = Ap;
        T rz = vdot(r, Ar);
        log(r, p);
        for (int i = 0;; ++i) {
            T ApdPAp = vdot(Ap, Ap);
            if (ApdPAp == T(0)) break;
            T alpha = rz / ApdPAp;
            for (int q = 0; q < n; ++q) xx[q] += alpha * p[q];
            for (int q = 0; q < n; ++q) r[q] -= alpha * Ap[q];
            if (i >= maxIters) break;
            if (vdot(r, r) < threshold) break;
            mult(r, Ar);
            T rz_old = rz;
            rz = vdot(r, Ar);
            if (rz_old == T(0)) break;
            T beta = rz / rz_old;
            for (int q = 0; q < n; ++q) p[q] = r[q] + beta * p[q];
            for (int q = 0; q < n; ++q) Ap[q] = Ar[q] + beta * Ap[q];
            log(r, p);
        }
        for (int i = 0; i < n; ++i) x[i] = (double)xx[i];
        *nrec = rec;
        return 0;
    };
    return prec == 64 ? run(0.0) : run(0.0f);
}

double orc_wall_seconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------------------
// Grid sessions: a Grid over caller-given particles, driven the way the reference's TestGrid drives
// MpmSim::Grid through its friend access (src/tests/TestGrid.cpp).
// ---------------------------------------------------------------------------------------------------------
namespace {
struct GBase {
    virtual ~GBase() {}
    int prec = 32;
};
template <class T> struct GImpl : GBase {
    Particles<T> P;
    std::unique_ptr<SnowModel<T>> model;
    std::unique_ptr<Grid<T>> grid;
    std::vector<Collider<T>> objs;
    Fields<T> fields;
};
template <class T> GImpl<T>* gs(void* h) { return static_cast<GImpl<T>*>(static_cast<GBase*>(h)); }

template <class T>
GBase* gcreate(long n, const double* x, const double* v, const double* m, const double* volume, const double* F,
               const double* snow, int updateModel, double h, const double* frameV, const int* inds, long ninds,
               int ncoll, const orc_collider* colls, int ngrav, const double* grav, int& status) {
    auto* g = new GImpl<T>();
    g->prec = sizeof(T) == 4 ? 32 : 64;
    g->P.x.resize(n); g->P.v.resize(n); g->P.F.resize(n); g->P.m.resize(n); g->P.volume.resize(n);
    int ok;
    setVar<T>(g->P, "p", x, ok);
    setVar<T>(g->P, "v", v, ok);
    setVar<T>(g->P, "m", m, ok);
    setVar<T>(g->P, "volume", volume, ok);
    setVar<T>(g->P, "F", F, ok);
    g->model.reset(new SnowModel<T>((T)snow[0], (T)snow[1], (T)snow[2], (T)snow[3], (T)snow[4]));
    g->model->setParticles(g->P);
    for (int i = 0; i < ncoll; ++i) g->objs.push_back(toCollider<T>(colls[i]));
    for (int i = 0; i < ngrav; ++i) g->fields.gravity.push_back(V3<T>((T)grav[3 * i], (T)grav[3 * i + 1], (T)grav[3 * i + 2]));
    std::vector<int> I(inds, inds + ninds);
    try {
        if (updateModel) g->model->updateParticleData(g->P);
        g->grid.reset(new Grid<T>(g->P, I, (T)h, V3<T>((T)frameV[0], (T)frameV[1], (T)frameV[2])));
    } catch (OracleError& e) {
        status = e.code;
        delete g;
        return nullptr;
    }
    status = 0;
    return g;
}

template <class T> int gcall(GImpl<T>* g, const std::string& op, const double* in, double* out, double dt, int maxIters, double tol) {
    auto& G = *g->grid;
    std::vector<T> a, b;
    auto load = [&](size_t k) { a.resize(k); for (size_t i = 0; i < k; ++i) a[i] = (T)in[i]; };
    auto store = [&](const std::vector<T>& y) { for (size_t i = 0; i < y.size(); ++i) out[i] = (double)y[i]; };
    try {
        if (op == "forces") { G.calculateForces(b, *g->model, g->fields); store(b); }
        else if (op == "DF") { load(G.velocities.size()); G.calculateForceDifferentials(b, a, *g->model); store(b); }
        else if (op == "dFidXi") { G.dForceidXi(b, *g->model); store(b); }
        else if (op == "explicit") {
            std::vector<T> em;
            G.calculateExplicitMomenta(em, G.nodeCollided, (T)dt, *g->model, g->objs, g->fields);
            store(em);
        }
        else if (op == "A") { load(G.velocities.size()); G.multVector(a, b, *g->model, g->objs, (T)dt); store(b); }
        else if (op == "solve") { G.updateGridVelocities((T)dt, *g->model, g->objs, g->fields, maxIters, (T)tol); }
        else if (op == "updateF") G.updateDeformationGradients((T)dt);
        else if (op == "updateV") G.updateParticleVelocities();
        else if (op == "volumes") G.computeParticleVolumes();
        else if (op == "model") g->model->updateParticleData(g->P);
        else if (op == "setVelocities") { load(G.velocities.size()); G.velocities = a; }
        else if (op == "vc") { G.collisionVelocities(b, g->objs); store(b); }
        else if (op == "energy") {
            for (size_t i = 0; i < g->P.size(); ++i) out[i] = (double)g->model->energyDensity(g->P, i);
        }
        else return -1;
    } catch (OracleError& e) {
        return e.code;
    }
    return 0;
}
}  // namespace

extern "C" {

void* orc_grid_create(int prec, long n, const double* x, const double* v, const double* m, const double* volume, const double* F,
                      const double* snow, int updateModel, double h, const double* frameV, const int* inds, long ninds,
                      int ncoll, const orc_collider* colls, int ngrav, const double* grav, int* status) {
    int st = 0;
    GBase* g = prec == 64 ? gcreate<double>(n, x, v, m, volume, F, snow, updateModel, h, frameV, inds, ninds, ncoll, colls, ngrav, grav, st)
                          : gcreate<float>(n, x, v, m, volume, F, snow, updateModel, h, frameV, inds, ninds, ncoll, colls, ngrav, grav, st);
    if (status) *status = st;
    return g;
}
void orc_grid_destroy(void* h) { delete static_cast<GBase*>(h); }

int orc_grid_call(void* h, const char* op, const double* in, double* out, double dt, int maxIters, double tol) {
    GBase* b = static_cast<GBase*>(h);
    return b->prec == 64 ? gcall<double>(gs<double>(h), op, in, out, dt, maxIters, tol)
                         : gcall<float>(gs<float>(h), op, in, out, dt, maxIters, tol);
}

int orc_grid_sinfo(void* h, double* min3, int* n3) {
    GBase* b = static_cast<GBase*>(h);
    auto fill = [&](auto* g) { for (int k = 0; k < 3; ++k) { min3[k] = (double)g->grid->mmin[k]; n3[k] = g->grid->n[k]; } };
    if (b->prec == 64) fill(gs<double>(h)); else fill(gs<float>(h));
    return 0;
}

int orc_grid_sget(void* h, const char* name, double* dst) {
    GBase* b = static_cast<GBase*>(h);
    auto run = [&](auto* g) -> int {
        std::string nm(name);
        auto& G = *g->grid;
        if (nm == "masses") { for (size_t i = 0; i < G.masses.size(); ++i) dst[i] = (double)G.masses[i]; return 0; }
        if (nm == "velocities") { for (size_t i = 0; i < G.velocities.size(); ++i) dst[i] = (double)G.velocities[i]; return 0; }
        if (nm == "prevVelocities") { for (size_t i = 0; i < G.prevVelocities.size(); ++i) dst[i] = (double)G.prevVelocities[i]; return 0; }
        if (nm == "nodeCollided") { for (size_t i = 0; i < G.nodeCollided.size(); ++i) dst[i] = G.nodeCollided[i]; return 0; }
        if (nm == "rhs") { for (size_t i = 0; i < G.rec_rhs.size(); ++i) dst[i] = (double)G.rec_rhs[i]; return 0; }
        if (nm == "explicitMomenta") { for (size_t i = 0; i < G.rec_explicitMomenta.size(); ++i) dst[i] = (double)G.rec_explicitMomenta[i]; return 0; }
        if (nm == "diag") { for (size_t i = 0; i < G.rec_diag.size(); ++i) dst[i] = (double)G.rec_diag[i]; return 0; }
        if (nm == "vc") { for (size_t i = 0; i < G.rec_vc.size(); ++i) dst[i] = (double)G.rec_vc[i]; return 0; }
        if (nm == "inds") { for (size_t i = 0; i < G.inds.size(); ++i) dst[i] = G.inds[i]; return 0; }
        int ok;
        getVar(g->P, nm, dst, ok);
        return ok ? 0 : 1;
    };
    return b->prec == 64 ? run(gs<double>(h)) : run(gs<float>(h));
}

int orc_grid_sset(void* h, const char* name, const double* src) {
    GBase* b = static_cast<GBase*>(h);
    auto run = [&](auto* g) -> int { int ok; setVar(g->P, name, src, ok); return ok ? 0 : 1; };
    return b->prec == 64 ? run(gs<double>(h)) : run(gs<float>(h));
}

int orc_grid_sstats(void* h, int* iters, double* bNorm2, double* rNorm2) {
    GBase* b = static_cast<GBase*>(h);
    auto run = [&](auto* g) { *iters = g->grid->stats.iterations; *bNorm2 = g->grid->stats.bNorm2; *rNorm2 = g->grid->stats.rNorm2; };
    if (b->prec == 64) run(gs<double>(h)); else run(gs<float>(h));
    return 0;
}

// ShapeFunctionIterator of the grid built around one particle at `origin` with spacing h, evaluated at point p
// (TestShapeFunction.cpp:44-156): the grid's m_min, the base node, 64 weights and weight gradients in
// iteration order (x fastest).
void orc_stencil(int prec, double h, const double* origin, const double* p, double* min3, int* base3, double* w64, double* g64) {
    auto run = [&](auto zero) {
        using T = decltype(zero);
        Particles<T> P;
        P.x.assign(1, V3<T>((T)origin[0], (T)origin[1], (T)origin[2]));
        P.m.assign(1, T(1));
        P.v.assign(1, V3<T>());
        Grid<T> G(P, std::vector<int>{0}, (T)h, V3<T>());
        typename Grid<T>::Stencil s;
        G.stencil(V3<T>((T)p[0], (T)p[1], (T)p[2]), s, true);
        int q = 0;
        for (int k = 0; k < 4; ++k) for (int j = 0; j < 4; ++j) for (int i = 0; i < 4; ++i, ++q) {
            w64[q] = (double)s.weight(i, j, k);
            V3<T> g = s.grad(i, j, k);
            for (int a = 0; a < 3; ++a) g64[3 * q + a] = (double)g[a];
        }
        for (int a = 0; a < 3; ++a) { base3[a] = s.base[a]; min3[a] = (double)G.mmin[a]; }
    };
    if (prec == 64) run(0.0); else run(0.0f);
}

}  // extern "C"

// C entry points over the UNMODIFIED reference sources (gdeskos/DVMpp src/*.cpp),
// compiled by oracle/Makefile into oracle/_ref/libdvmref.so.
//
// TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
// reference / cpu_baseline legs load this library as the checker or as the timed
// CPU baseline.  The product path (dvmpp_b200/) never links or calls it.
//
// The time loop below is DVMBase::solve (src/DVMBase.cpp:67-84) minus
// write_outputs(); each step calls the reference's own increment_step() and
// compute_step() (src/DVMBase.cpp:86-133, 145-149).  Private members are
// reached by compiling this one translation unit with `private` redefined as
// `public` after every system header has been included; the reference classes
// themselves are compiled unchanged in their own translation units.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <memory>
#include <random>
#include <sstream>
#include <string>
#include <tuple>
#include <unordered_map>
#include <vector>
#include <cassert>
#include <armadillo>
#include "pugiconfig.hpp"
#include "pugixml.hpp"

#define private public
#include "DVMBase.hpp"
#include "VelocityKernel.hpp"
#undef private

namespace {
thread_local std::string g_err;
struct NullBuf : std::streambuf {
    int overflow(int c) override { return c; }
};
NullBuf g_null;

struct RefSim {
    XmlHandler xml;
    std::unique_ptr<DVMBase> base;
};

struct CoutSilencer {
    std::streambuf* old = nullptr;
    explicit CoutSilencer(bool on) {
        if (on) old = std::cout.rdbuf(&g_null);
    }
    ~CoutSilencer() {
        if (old) std::cout.rdbuf(old);
    }
};
}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

// ---- VelocityKernel (src/VelocityKernel.cpp:30-109) -----------------------
int ref_direct_self(const double* x, const double* z, const double* circ, const double* sigma,
                    size_t n, double* u, double* w) {
    try {
        auto k = dvm::VelocityKernel::create("direct");
        std::vector<dvm::VortexParticle> p(n);
        for (size_t i = 0; i < n; ++i) p[i] = {x[i], z[i], circ[i], sigma[i]};
        std::vector<dvm::VelocityResult> v;
        k->computeSelfInduced(p, v);
        for (size_t i = 0; i < n; ++i) { u[i] = v[i].u; w[i] = v[i].w; }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

int ref_direct_at(const double* x, const double* z, const double* circ, const double* sigma,
                  size_t ns, const double* tx, const double* tz, size_t nt, double* u, double* w) {
    try {
        auto k = dvm::VelocityKernel::create("direct");
        std::vector<dvm::VortexParticle> p(ns);
        for (size_t i = 0; i < ns; ++i) p[i] = {x[i], z[i], circ[i], sigma[i]};
        std::vector<double> vx(tx, tx + nt), vz(tz, tz + nt);
        std::vector<dvm::VelocityResult> v;
        k->computeInducedAt(p, vx, vz, v);
        for (size_t i = 0; i < nt; ++i) { u[i] = v[i].u; w[i] = v[i].w; }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// ---- VortexBlobs::merge_blobs (src/VortexBlobs.cpp:110-209) ---------------
// In/out arrays of length n (8 SoA arrays + ids); returns the merge count, the
// new length in *n_out.
int ref_merge_blobs(double* x, double* z, double* circ, double* sigma, double* u, double* w,
                    double* uvs, double* wvs, unsigned* id, size_t n, double threshold,
                    size_t* n_out, unsigned* merged) {
    try {
        VortexBlobs b((unsigned)n);
        for (size_t i = 0; i < n; ++i) {
            b.m_ID[i] = id[i];
            b.m_x(i) = x[i]; b.m_z(i) = z[i]; b.m_circ(i) = circ[i]; b.m_sigma(i) = sigma[i];
            b.m_u(i) = u[i]; b.m_w(i) = w[i]; b.m_uvs(i) = uvs[i]; b.m_wvs(i) = wvs[i];
        }
        *merged = b.merge_blobs(threshold);
        const size_t m = b.size();
        for (size_t i = 0; i < m; ++i) {
            id[i] = b.m_ID[i];
            x[i] = b.m_x(i); z[i] = b.m_z(i); circ[i] = b.m_circ(i); sigma[i] = b.m_sigma(i);
            u[i] = b.m_u(i); w[i] = b.m_w(i); uvs[i] = b.m_uvs(i); wvs[i] = b.m_wvs(i);
        }
        *n_out = m;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// ---- Random (src/Random.cpp) ------------------------------------------------
void ref_random_stream(int seed, size_t n, double* out) {
    Random r;
    r.seed(seed);
    for (size_t i = 0; i < n; ++i) out[i] = r.rand();
}

// ---- full simulation (DVMBase) ---------------------------------------------
void* ref_sim_create(const char* xml_path, const char* stamp, int quiet) {
    CoutSilencer s(quiet != 0);
    try {
        auto* sim = new RefSim{XmlHandler(xml_path), nullptr};
        sim->base = std::make_unique<DVMBase>(sim->xml, stamp);
        return sim;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void ref_sim_destroy(void* h) { delete static_cast<RefSim*>(h); }

// One full reference step: DVMBase::increment_step + compute_step.
int ref_sim_step(void* h, int nsteps, int quiet) {
    CoutSilencer s(quiet != 0);
    try {
        auto& b = *static_cast<RefSim*>(h)->base;
        for (int k = 0; k < nsteps; ++k) {
            b.increment_step();
            b.compute_step();
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// Individual phases of compute_step, in its order (src/DVMBase.cpp:86-133).
//  0 biotsavart   1 solvevortexsheet   2 vortexsheetbc   3 convect (whole)
//  4 diffusion    5 release+append     6 surface crossing (per XML)
//  7 compute_loads                    8 increment_step
//  9 reflect      10 delete_inside
int ref_sim_phase(void* h, int phase, int quiet) {
    CoutSilencer s(quiet != 0);
    try {
        auto& b = *static_cast<RefSim*>(h)->base;
        switch (phase) {
            case 0: b.m_vortex.biotsavart(); break;
            case 1: b.m_vortsheet.solvevortexsheet(b.m_vortex); break;
            case 2: b.m_vortsheet.vortexsheetbc(b.m_vortex); break;
            case 3: b.convect(); break;
            case 4: b.m_vortex.diffusion_random_walk(b.m_rand, b.m_nu, b.m_dt); break;
            case 5: {
                VortexBlobs nv = b.m_vortsheet.release_nascent_vortices_rw(b.m_rand);
                b.m_vortex.append_vortices(nv);
                break;
            }
            case 6:
                switch (b.m_surfcross) {
                    case SurfaceCross::Delete: b.m_vortsheet.delete_inside(b.m_vortex); break;
                    case SurfaceCross::Absorb: b.m_vortsheet.reflect(b.m_vortex); break;
                    case SurfaceCross::Reflect: b.m_vortsheet.reflect(b.m_vortex); break;
                }
                break;
            case 7: b.m_vortsheet.compute_loads(b.m_Ur); break;
            case 8: b.increment_step(); break;
            case 9: b.m_vortsheet.reflect(b.m_vortex); break;
            case 10: b.m_vortsheet.delete_inside(b.m_vortex); break;
            default: g_err = "bad phase"; return 2;
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// DVMBase::write_outputs (src/DVMBase.cpp:151-158): the per-step text files.
int ref_sim_write(void* h) {
    try {
        static_cast<RefSim*>(h)->base->write_outputs();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

size_t ref_sim_nblobs(void* h) { return static_cast<RefSim*>(h)->base->m_vortex.size(); }
int ref_sim_npanels(void* h) { return static_cast<int>(static_cast<RefSim*>(h)->base->m_vortsheet.size()); }

void ref_sim_get_blobs(void* h, double* x, double* z, double* circ, double* sigma, double* u,
                       double* w, double* uvs, double* wvs, unsigned* id) {
    auto& v = static_cast<RefSim*>(h)->base->m_vortex;
    const size_t n = v.size();
    for (size_t i = 0; i < n; ++i) {
        if (x) x[i] = v.m_x(i);
        if (z) z[i] = v.m_z(i);
        if (circ) circ[i] = v.m_circ(i);
        if (sigma) sigma[i] = v.m_sigma(i);
        if (u) u[i] = v.m_u(i);
        if (w) w[i] = v.m_w(i);
        if (uvs) uvs[i] = v.m_uvs(i);
        if (wvs) wvs[i] = v.m_wvs(i);
        if (id) id[i] = v.m_ID[i];
    }
}

void ref_sim_set_blobs(void* h, size_t n, const double* x, const double* z, const double* circ,
                       const double* sigma) {
    auto& v = static_cast<RefSim*>(h)->base->m_vortex;
    VortexBlobs nb(static_cast<unsigned>(n));
    for (size_t i = 0; i < n; ++i) {
        nb.m_ID[i] = static_cast<unsigned>(i);
        nb.m_x(i) = x[i];
        nb.m_z(i) = z[i];
        nb.m_circ(i) = circ[i];
        nb.m_sigma(i) = sigma[i];
        nb.m_u(i) = 0.0;
        nb.m_w(i) = 0.0;
        nb.m_uvs(i) = 0.0;
        nb.m_wvs(i) = 0.0;
    }
    nb.copyOutputConfig(v);
    v = std::move(nb);
}

// Panel geometry and strengths (src/VortexSheet.hpp:24-38).
void ref_sim_get_sheet(void* h, double* gamma, double* xc, double* zc, double* ds, double* theta,
                       double* enx, double* enz, double* x, double* z) {
    auto& s = static_cast<RefSim*>(h)->base->m_vortsheet;
    const size_t np = s.size();
    for (size_t i = 0; i < np; ++i) {
        if (gamma) gamma[i] = s.m_gamma(i);
        if (xc) xc[i] = s.m_xc(i);
        if (zc) zc[i] = s.m_zc(i);
        if (ds) ds[i] = s.m_ds(i);
        if (theta) theta[i] = s.m_theta(i);
        if (enx) enx[i] = s.m_enx(i);
        if (enz) enz[i] = s.m_enz(i);
    }
    for (size_t i = 0; i <= np; ++i) {
        if (x) x[i] = s.m_x(i);
        if (z) z[i] = s.m_z(i);
    }
}

void ref_sim_set_gamma(void* h, const double* gamma) {
    auto& s = static_cast<RefSim*>(h)->base->m_vortsheet;
    for (size_t i = 0; i < s.size(); ++i) s.m_gamma(i) = gamma[i];
}

// Influence matrix, (Np+1) x Np, column-major (src/VortexSheet.cpp:104-165).
void ref_sim_get_infm(void* h, double* a) {
    auto& s = static_cast<RefSim*>(h)->base->m_vortsheet;
    std::memcpy(a, s.m_infM.mem.data(), sizeof(double) * s.m_infM.n_elem);
}

void ref_sim_get_forces(void* h, double* fx, double* fz, double* area) {
    auto& s = static_cast<RefSim*>(h)->base->m_vortsheet;
    *fx = s.m_fx;
    *fz = s.m_fz;
    if (area) *area = s.m_A;
}

int ref_sim_inside(void* h, double x, double z) {
    return static_cast<RefSim*>(h)->base->m_vortsheet.inside_body(x, z) ? 1 : 0;
}

unsigned ref_sim_stepno(void* h) { return static_cast<RefSim*>(h)->base->m_step; }

}  // extern "C"

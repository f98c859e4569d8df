#include "DVMBase.hpp"

#include <cmath>
#include <iostream>
#include <vector>

#include "Device.hpp"

DVMBase::DVMBase(XmlHandler& xml, const std::string& stamp)
    : m_vortex(xml, stamp), m_vortsheet(xml, stamp), m_probe(xml, stamp), m_xml(xml),
      m_mesh(xml) {
    m_nu = xml.getValueAttribute("constants", "nu");
    m_dt = xml.getValueAttribute("time", "dt");
    m_steps = static_cast<unsigned>(xml.getValueAttribute("time", "steps"));
    m_Ux = xml.getValueAttribute("flow", "ux");
    m_Uz = xml.getValueAttribute("flow", "uz");
    m_Ur = std::sqrt(m_Ux * m_Ux + m_Uz * m_Uz);
    const int seed = xml.getIntAttribute("constants", "seed");
    m_rand.seed(seed);
    const std::string scheme = xml.getStringAttribute("time", "scheme");
    m_scheme = scheme == "RK3" ? Scheme::RK3 : Scheme::Euler;
    const std::string sc = xml.getStringAttribute("algorithms", "surface_crossing");
    m_surfcross = sc == "DELETE" ? SurfaceCross::Delete
                                 : (sc == "ABSORB" ? SurfaceCross::Absorb : SurfaceCross::Reflect);
    if (xml.has("algorithms", "velocity_kernel")) {
        const std::string k = xml.getStringAttribute("algorithms", "velocity_kernel");
        m_precision = (k == "cuda") ? DVM_F32 : DVM_F64;
        m_vortex.setKernelType(k == "fmm" ? "direct" : k);
    }
    if (xml.has("algorithms", "diffusion_rng"))
        m_rng_mode = xml.getStringAttribute("algorithms", "diffusion_rng") == "philox"
                         ? DVM_RNG_PHILOX
                         : DVM_RNG_INJECT;
    // src/DVMBase.cpp:51-64
    if (xml.has("algorithms", "merge_threshold") && xml.has("algorithms", "merge_frequency")) {
        m_merge_threshold = xml.getValueAttribute("algorithms", "merge_threshold");
        m_merge_frequency = static_cast<unsigned>(xml.getIntAttribute("algorithms", "merge_frequency"));
    }
    if (m_merge_frequency > 0 && m_merge_threshold > 0)
        std::cout << "Vortex merging enabled: threshold = " << m_merge_threshold
                  << ", frequency = " << m_merge_frequency << std::endl;
    if (m_mesh.is_enabled())  // as src/DVMBase.cpp:61-64 reports merging
        std::cout << "Remeshing enabled: " << m_mesh.nx() << " x " << m_mesh.nz()
                  << " mesh nodes" << std::endl;
    const int cross = m_surfcross == SurfaceCross::Delete
                          ? DVM_DELETE
                          : (m_surfcross == SurfaceCross::Absorb ? DVM_ABSORB : DVM_REFLECT);
    m_vortsheet.set_params(m_precision, m_rng_mode,
                           m_scheme == Scheme::RK3 ? DVM_RK3 : DVM_EULER, cross, seed);
    m_sim = m_vortsheet.device(0);
}

unsigned DVMBase::get_steps() const { return m_steps; }
double DVMBase::get_time() const { return m_time; }

void DVMBase::increment_step() {
    m_step++;
    m_time = m_step * m_dt;
}

void DVMBase::supply_uniforms() {
    // Inject mode: keep at least this step's draws on the device -- 2N for the
    // walk plus the release -- as the next values of the reference's stream.
    if (m_rng_mode != DVM_RNG_INJECT) return;
    uint64_t n = 0, consumed = 0, avail = 0;
    dvm::check_status(dvm_sim_num_blobs(m_sim, &n), "DVMBase");
    dvm::check_status(dvm_sim_rng_position(m_sim, &consumed, &avail), "DVMBase");
    const uint64_t need = 2 * n + m_vortsheet.max_release();
    if (avail >= need) return;
    std::vector<double> u(need - avail + 2 * n + 4096);  // a little ahead
    for (auto& v : u) v = m_rand.rand();
    dvm::check_status(dvm_sim_push_uniforms(m_sim, u.data(), u.size()), "DVMBase");
}

void DVMBase::compute_step() {
    // Grow the device simulation when the next releases might not fit: copy
    // the state out, rebuild with twice the room, and restore it (including the
    // not-yet-consumed part of the random stream).
    uint64_t n = 0;
    dvm::check_status(dvm_sim_num_blobs(m_sim, &n), "DVMBase");
    const bool remesh_now = m_mesh.should_remesh(m_step);
    // a remesh can turn the blobs into as many blobs as there are mesh nodes
    const uint64_t need = n + m_vortsheet.max_release() +
                          (remesh_now ? (uint64_t)m_mesh.nx() * m_mesh.nz() : 0);
    if (need > m_vortsheet.capacity()) {
        std::vector<double> pending;
        if (m_rng_mode == DVM_RNG_INJECT) {
            uint64_t np = 0;
            dvm::check_status(dvm_sim_pending_uniforms(m_sim, nullptr, 0, &np), "DVMBase");
            pending.resize(np);
            if (np)
                dvm::check_status(dvm_sim_pending_uniforms(m_sim, pending.data(), np, &np),
                                  "DVMBase");
        }
        sync_to_host();
        m_sim = m_vortsheet.device(need);
        dvm::check_status(dvm_sim_set_blobs(m_sim, m_vortex.size(), dvm::vec_ptr(m_vortex.m_x),
                                            dvm::vec_ptr(m_vortex.m_z),
                                            dvm::vec_ptr(m_vortex.m_circ),
                                            dvm::vec_ptr(m_vortex.m_sigma)),
                          "DVMBase");
        dvm::check_status(dvm_sim_set_step(m_sim, m_step - 1), "DVMBase");
        if (!pending.empty())
            dvm::check_status(dvm_sim_push_uniforms(m_sim, pending.data(), pending.size()),
                              "DVMBase");
    }
    supply_uniforms();
    if (!remesh_now) {
        // convect (Euler or RK3), diffusion, release + append, surface
        // crossing, loads: src/DVMBase.cpp:86-133, one batched sequence
        dvm::check_status(dvm_sim_step(m_sim, 1), "DVMBase::compute_step");
    } else {
        // the same step phase by phase, with the remesh after convection
        // (src/DVMBase.cpp:88-92)
        for (int ph : {DVM_PHASE_INCREMENT, DVM_PHASE_CONVECT})
            dvm::check_status(dvm_sim_phase(m_sim, ph), "DVMBase::compute_step");
        dvm::check_status(dvm_sim_remesh(m_sim, &m_mesh.params(), nullptr), "DVMBase::remesh");
        supply_uniforms();  // the walk draws 2 per blob of the remeshed set
        for (int ph : {DVM_PHASE_DIFFUSE, DVM_PHASE_RELEASE, DVM_PHASE_CROSS, DVM_PHASE_LOADS})
            dvm::check_status(dvm_sim_phase(m_sim, ph), "DVMBase::compute_step");
    }
    dvm::check_status(dvm_sim_status(m_sim), "DVMBase::compute_step");
    // merge after the loads (src/DVMBase.cpp:124-132), on the device
    if (m_merge_frequency > 0 && m_merge_threshold > 0 && m_step % m_merge_frequency == 0) {
        uint64_t merged = 0;
        dvm::check_status(dvm_sim_merge(m_sim, m_merge_threshold, &merged), "DVMBase merge");
        if (merged > 0) std::cout << "Merged " << merged << " vortex pairs" << std::endl;
    }
}

void DVMBase::convect() { dvm::check_status(dvm_sim_phase(m_sim, DVM_PHASE_CONVECT), "convect"); }

void DVMBase::remesh() {
    if (m_mesh.should_remesh(m_step))
        dvm::check_status(dvm_sim_remesh(m_sim, &m_mesh.params(), nullptr), "DVMBase::remesh");
}

// full: every blob array (what a caller reads after run()); otherwise only
// what the output files need (positions, circulations, the sheet and loads).
void DVMBase::sync_to_host(bool full) {
    uint64_t n = 0;
    dvm::check_status(dvm_sim_num_blobs(m_sim, &n), "DVMBase");
    m_vortex.resize((unsigned)n);
    if (full) {
        std::vector<uint32_t> ids(n);
        dvm::check_status(
            dvm_sim_get_blobs(m_sim, n, &n, dvm::vec_ptr(m_vortex.m_x), dvm::vec_ptr(m_vortex.m_z),
                              dvm::vec_ptr(m_vortex.m_circ), dvm::vec_ptr(m_vortex.m_sigma),
                              dvm::vec_ptr(m_vortex.m_u), dvm::vec_ptr(m_vortex.m_w),
                              dvm::vec_ptr(m_vortex.m_uvs), dvm::vec_ptr(m_vortex.m_wvs),
                              ids.data()),
            "DVMBase");
        for (uint64_t i = 0; i < n; ++i) m_vortex.m_ID[i] = ids[i];
    } else {
        dvm::check_status(dvm_sim_get_blobs(m_sim, n, &n, dvm::vec_ptr(m_vortex.m_x),
                                            dvm::vec_ptr(m_vortex.m_z),
                                            dvm::vec_ptr(m_vortex.m_circ), nullptr, nullptr,
                                            nullptr, nullptr, nullptr, nullptr),
                          "DVMBase");
    }
    m_vortsheet.pull_from_device();
}

void DVMBase::write_outputs() {
    if (m_probe.size())  // velocities at the probe points from the device-resident state
        dvm::check_status(dvm_sim_probe(m_sim, dvm::vec_ptr(m_probe.m_x),
                                        dvm::vec_ptr(m_probe.m_z), m_probe.size(),
                                        dvm::vec_ptr(m_probe.m_u), dvm::vec_ptr(m_probe.m_w),
                                        dvm::vec_ptr(m_probe.m_uvs), dvm::vec_ptr(m_probe.m_wvs)),
                          "DVMBase probes");
    // one job per step, so the files are appended step by step in order
    m_writer.submit([a = m_vortex.write_step_job(m_time, m_step),
                     b = m_vortsheet.write_step_job(m_time), c = m_probe.write_step_job(m_time)] {
        a();
        b();
        c();
    });
}

void DVMBase::run(unsigned steps, bool write, bool quiet) {
    m_quiet = quiet;
    for (unsigned j = 1; j <= steps; j++) {
        increment_step();
        compute_step();
        if (j == steps) sync_to_host(true);
        else if (write || !quiet) sync_to_host(false);
        if (write) write_outputs();
        if (!quiet) {
            double fx = 0, fz = 0, cd = 0, cl = 0;
            dvm_sim_get_loads(m_sim, &fx, &fz, &cd, &cl);
            std::cout << "C_D = " << cd << "\tC_L = " << cl << std::endl;
            std::cout << "Simulation time          = " << get_time() << "\tStep " << j << "/"
                      << steps << std::endl;
            std::cout << "Number of vortex blobs   = " << m_vortex.size() << std::endl;
        }
    }
    m_writer.flush();  // every file complete on return
}

void DVMBase::solve() { run(get_steps(), true, false); }

unsigned DVMBase::num_blobs() const { return m_vortex.size(); }

std::tuple<double, double> DVMBase::forces() const { return m_vortsheet.get_forces(); }

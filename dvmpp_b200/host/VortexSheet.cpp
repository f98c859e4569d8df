#include "VortexSheet.hpp"

#include "OutputWriter.hpp"
#include "Probe.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <filesystem>
#include <iostream>
#include <vector>

#include "Device.hpp"

namespace fs = std::filesystem;

VortexSheet::VortexSheet() = default;

VortexSheet::VortexSheet(const XmlHandler& xml, const std::string& stamp) {
    m_rho = xml.getValueAttribute("constants", "density");
    m_nu = xml.getValueAttribute("constants", "nu");
    m_dt = xml.getValueAttribute("time", "dt");
    m_Ux = xml.getValueAttribute("flow", "ux");
    m_Uz = xml.getValueAttribute("flow", "uz");
    m_maxNumPanelVort = static_cast<unsigned>(xml.getValueAttribute("constants", "max_NumPanelVort"));
    m_cutoff_exp = xml.getValueAttribute("constants", "cutoff_exp");
    const fs::path inpath(xml.getStringAttribute("io", "input_dir"));
    read_input_coord((inpath / xml.getStringAttribute("io", "domain_file")).string());

    m_params.rho = m_rho;
    m_params.nu = m_nu;
    m_params.dt = m_dt;
    m_params.ux = m_Ux;
    m_params.uz = m_Uz;
    m_params.cutoff_exp = m_cutoff_exp;
    m_params.max_numpanelvort = m_maxNumPanelVort;
    m_params.scheme = DVM_EULER;
    m_params.surface_cross = DVM_REFLECT;
    m_params.rng = DVM_RNG_INJECT;
    m_params.precision = DVM_F64;
    m_params.seed = 0;
    const double steps = xml.getValueAttribute("time", "steps");
    const double npanels = (double)m_x.n_elem - 1.0;
    build_device((uint64_t)(steps * 2.0 * (m_maxNumPanelVort + 1) * npanels) + 4096);

    const std::string outdir = xml.getStringAttribute("io", "output_dir", true);
    m_gammapath = (fs::path(outdir) / (stamp + "_gamma.dat")).string();
    std::ofstream gammafile(m_gammapath);
    if (!gammafile) throw dvm::FileIOException::cannotOpen(m_gammapath);
    // headers of src/VortexSheet.cpp:43-53
    gammafile << m_xc.n_elem << " # Number of collocation points\n"
              << m_dt << " # Time Step\n"
              << steps << " # Steps\n"
              << "Time [s] Gamma - Vortex sheet strength\n";
    m_forcepath = (fs::path(outdir) / (stamp + "_loads.dat")).string();
    std::ofstream forcefile(m_forcepath);
    if (!forcefile) throw dvm::FileIOException::cannotOpen(m_forcepath);
    forcefile << "Time [s]\tF_x [-]\tF_z [s]\n";
}

VortexSheet::~VortexSheet() {
    if (m_sim) dvm_sim_destroy(m_sim);
}

void VortexSheet::read_input_coord(const std::string& file) {
    // two numbers per line, blank lines ignored (the reference's raw_ascii load)
    std::ifstream f(file);
    if (!f) throw dvm::FileIOException::cannotRead(file);
    std::vector<double> xs, zs;
    std::string line;
    while (std::getline(f, line)) {
        // whitespace-separated numbers (strtod: nan and inf included, so they
        // reach the finiteness check); a token that is not a number fails
        std::istringstream s(line);
        std::vector<double> v;
        std::string tok;
        while (s >> tok) {
            char* end = nullptr;
            const double d = std::strtod(tok.c_str(), &end);
            if (end == tok.c_str() || *end != '\0') throw dvm::FileIOException::cannotRead(file);
            v.push_back(d);
        }
        if (v.empty()) continue;
        if (v.size() != 2) throw dvm::FileIOException::cannotRead(file);
        xs.push_back(v[0]);
        zs.push_back(v[1]);
    }
    if (xs.size() < 3) throw dvm::FileIOException::cannotRead(file);
    // The panel method needs a closed contour of finite points, at least 3
    // panels, none of zero length; the reference loads any two-column file, so
    // these checks add a clear error where it would build a singular system.
    const size_t npts = xs.size();
    double L = 0.0;
    for (size_t i = 0; i < npts; ++i) {
        if (!std::isfinite(xs[i]) || !std::isfinite(zs[i]))
            throw dvm::FileIOException("Invalid body contour in " + file + ": point " +
                                       std::to_string(i) + " is not finite");
        L = std::max({L, std::fabs(xs[i] - xs[0]), std::fabs(zs[i] - zs[0])});
    }
    if (npts < 4)
        throw dvm::FileIOException("Invalid body contour in " + file +
                                   ": a closed body needs at least 3 panels (4 points, the "
                                   "first repeated last)");
    const double tol = 1e-12 * L;
    if (!(L > 0) || std::fabs(xs[npts - 1] - xs[0]) > tol || std::fabs(zs[npts - 1] - zs[0]) > tol)
        throw dvm::FileIOException("Invalid body contour in " + file +
                                   ": not closed (the last point must repeat the first)");
    for (size_t i = 0; i + 1 < npts; ++i)
        if (std::hypot(xs[i + 1] - xs[i], zs[i + 1] - zs[i]) <= tol)
            throw dvm::FileIOException("Invalid body contour in " + file + ": panel " +
                                       std::to_string(i) + " has zero length (repeated point)");
    m_x = Vector(xs);
    m_z = Vector(zs);
    std::cout << "Successfully loaded coordinate file with " << m_x.n_elem << " points."
              << std::endl;
    m_A = *std::max_element(xs.begin(), xs.end()) - *std::min_element(xs.begin(), xs.end());
    std::cout << "A = " << m_A << " (assuming cylinder)\n";
}

void VortexSheet::build_device(uint64_t capacity) {
    if (m_sim) {
        dvm_sim_destroy(m_sim);
        m_sim = nullptr;
    }
    const size_t npts = m_x.n_elem, np = npts - 1;
    m_params.capacity = std::max<uint64_t>(capacity, 1024);
    m_params.rng_capacity = 2 * m_params.capacity + 64ull * (m_maxNumPanelVort + 1) * np + 4096;
    dvm::check_status(dvm_sim_create(dvm::device_context(), &m_params, dvm::vec_ptr(m_x),
                                     dvm::vec_ptr(m_z), (int)npts, &m_sim),
                      "VortexSheet");
    // panel geometry, as the reference forms it (src/VortexSheet.cpp:78-102)
    m_xc.set_size(np);
    m_zc.set_size(np);
    m_ds.set_size(np);
    m_theta.set_size(np);
    m_enx.set_size(np);
    m_enz.set_size(np);
    m_etx.set_size(np);
    m_etz.set_size(np);
    dvm::check_status(dvm_sim_get_panels(m_sim, dvm::vec_ptr(m_xc), dvm::vec_ptr(m_zc),
                                         dvm::vec_ptr(m_ds), dvm::vec_ptr(m_theta),
                                         dvm::vec_ptr(m_enx), dvm::vec_ptr(m_enz)),
                      "VortexSheet");
    for (size_t i = 0; i < np; ++i) {
        m_etx(i) = -m_enz(i);
        m_etz(i) = m_enx(i);
    }
    if (m_gamma.n_elem != np) {
        m_gamma.set_size(np);
        m_gamma.zeros();
    }
    dvm::check_status(dvm_sim_set_gamma(m_sim, dvm::vec_ptr(m_gamma)), "VortexSheet");
}

void VortexSheet::set_params(int precision, int rng, int scheme, int cross, int64_t seed) {
    m_params.precision = precision;
    m_params.rng = rng;
    m_params.scheme = scheme;
    m_params.surface_cross = cross;
    m_params.seed = seed;
    build_device(m_params.capacity);
}

dvm_sim* VortexSheet::device(uint64_t capacity) {
    if (!m_sim || capacity > m_params.capacity) build_device(std::max(capacity, 2 * m_params.capacity));
    return m_sim;
}

unsigned VortexSheet::max_release() const {
    return 16u * (m_maxNumPanelVort + 1) * size() + 1024u;
}

void VortexSheet::upload(const VortexBlobs& b) {
    const unsigned n = b.size();
    device((uint64_t)n + max_release());
    dvm::check_status(dvm_sim_set_blobs(m_sim, n, dvm::vec_ptr(b.m_x), dvm::vec_ptr(b.m_z),
                                        dvm::vec_ptr(b.m_circ), dvm::vec_ptr(b.m_sigma)),
                      "VortexSheet upload");
    dvm::check_status(dvm_sim_set_gamma(m_sim, dvm::vec_ptr(m_gamma)), "VortexSheet upload");
}

void VortexSheet::pull_from_device() {
    dvm::check_status(dvm_sim_get_gamma(m_sim, dvm::vec_ptr(m_gamma)), "VortexSheet");
    double cd = 0, cl = 0;
    dvm::check_status(dvm_sim_get_loads(m_sim, &m_fx, &m_fz, &cd, &cl), "VortexSheet");
}

void VortexSheet::solvevortexsheet(VortexBlobs& blobs) {
    upload(blobs);
    dvm::check_status(dvm_sim_phase(m_sim, DVM_PHASE_SOLVE), "solvevortexsheet");
    dvm::check_status(dvm_sim_get_gamma(m_sim, dvm::vec_ptr(m_gamma)), "solvevortexsheet");
}

void VortexSheet::vortexsheetbc(VortexBlobs& blobs) {
    upload(blobs);
    dvm::check_status(dvm_sim_phase(m_sim, DVM_PHASE_SHEETBC), "vortexsheetbc");
    uint64_t n = 0;
    dvm::check_status(dvm_sim_get_blobs(m_sim, blobs.size(), &n, nullptr, nullptr, nullptr,
                                        nullptr, nullptr, nullptr, dvm::vec_ptr(blobs.m_uvs),
                                        dvm::vec_ptr(blobs.m_wvs), nullptr),
                      "vortexsheetbc");
}

VortexBlobs VortexSheet::release_nascent_vortices_rw(Random& rng) {
    // Run the release on an empty blob set with the next values of the
    // caller's stream, then consume exactly as many as the release drew.
    device(max_release());
    dvm::check_status(dvm_sim_set_blobs(m_sim, 0, nullptr, nullptr, nullptr, nullptr), "release");
    dvm::check_status(dvm_sim_set_gamma(m_sim, dvm::vec_ptr(m_gamma)), "release");
    if (m_params.rng == DVM_RNG_INJECT) {
        std::vector<double> u;
        rng.peek(max_release(), u);
        dvm::check_status(dvm_sim_clear_uniforms(m_sim), "release");
        dvm::check_status(dvm_sim_push_uniforms(m_sim, u.data(), u.size()), "release");
    }
    dvm::check_status(dvm_sim_phase(m_sim, DVM_PHASE_RELEASE), "release_nascent_vortices_rw");
    dvm::check_status(dvm_sim_status(m_sim), "release_nascent_vortices_rw");
    uint64_t n = 0;
    dvm::check_status(dvm_sim_num_blobs(m_sim, &n), "release");
    VortexBlobs nv((unsigned)n);
    std::vector<uint32_t> ids(n);
    dvm::check_status(dvm_sim_get_blobs(m_sim, n, &n, dvm::vec_ptr(nv.m_x), dvm::vec_ptr(nv.m_z),
                                        dvm::vec_ptr(nv.m_circ), dvm::vec_ptr(nv.m_sigma),
                                        dvm::vec_ptr(nv.m_u), dvm::vec_ptr(nv.m_w),
                                        dvm::vec_ptr(nv.m_uvs), dvm::vec_ptr(nv.m_wvs), ids.data()),
                      "release");
    for (uint64_t i = 0; i < n; ++i) nv.m_ID[i] = 0;  // nascent IDs are 0 (src/VortexSheet.cpp:300)
    if (m_params.rng == DVM_RNG_INJECT) rng.discard(n);  // one draw per nascent blob
    return nv;
}

void VortexSheet::reflect(VortexBlobs& v) {
    upload(v);
    dvm::check_status(dvm_sim_phase(m_sim, DVM_PHASE_REFLECT), "reflect");
    uint64_t n = 0;
    dvm::check_status(dvm_sim_get_blobs(m_sim, v.size(), &n, dvm::vec_ptr(v.m_x),
                                        dvm::vec_ptr(v.m_z), nullptr, nullptr, nullptr, nullptr,
                                        nullptr, nullptr, nullptr),
                      "reflect");
}

void VortexSheet::delete_inside(VortexBlobs& v) {
    const unsigned n0 = v.size();
    upload(v);
    // keep the velocities too: the reference's compaction copies them
    std::vector<double> u(v.m_u.memptr(), v.m_u.memptr() + n0), w(v.m_w.memptr(), v.m_w.memptr() + n0);
    dvm::check_status(dvm_sim_phase(m_sim, DVM_PHASE_DELETE), "delete_inside");
    uint64_t n = 0;
    dvm::check_status(dvm_sim_num_blobs(m_sim, &n), "delete_inside");
    if (n == n0) return;  // nothing deleted: IDs unchanged (src/VortexSheet.cpp:420-422)
    VortexBlobs nv((unsigned)n);
    std::vector<uint32_t> ids(n);
    dvm::check_status(dvm_sim_get_blobs(m_sim, n, &n, dvm::vec_ptr(nv.m_x), dvm::vec_ptr(nv.m_z),
                                        dvm::vec_ptr(nv.m_circ), dvm::vec_ptr(nv.m_sigma),
                                        nullptr, nullptr, nullptr, nullptr, ids.data()),
                      "delete_inside");
    // u, w, uvs, wvs follow the kept blobs in order (kept = outside the body)
    size_t k = 0;
    for (unsigned i = 0; i < n0 && k < n; ++i) {
        if (v.m_x(i) != nv.m_x(k) || v.m_z(i) != nv.m_z(k)) continue;
        nv.m_u(k) = v.m_u(i);
        nv.m_w(k) = v.m_w(i);
        nv.m_uvs(k) = v.m_uvs(i);
        nv.m_wvs(k) = v.m_wvs(i);
        ++k;
    }
    for (uint64_t i = 0; i < n; ++i) nv.m_ID[i] = ids[i];
    nv.copyOutputConfig(v);
    const unsigned deleted = n0 - (unsigned)n;
    v = std::move(nv);
    std::cout << "Deleted " << deleted << " vortices inside body" << std::endl;
}

void VortexSheet::compute_loads(double Ur) {
    (void)Ur;  // the device uses |U| from ux, uz: the same value DVMBase passes
    dvm::check_status(dvm_sim_set_gamma(m_sim, dvm::vec_ptr(m_gamma)), "compute_loads");
    dvm::check_status(dvm_sim_phase(m_sim, DVM_PHASE_LOADS), "compute_loads");
    double cd = 0, cl = 0;
    dvm::check_status(dvm_sim_get_loads(m_sim, &m_fx, &m_fz, &cd, &cl), "compute_loads");
    std::cout << "C_D = " << cd << "\t" << "C_L = " << cl << std::endl;
}

unsigned VortexSheet::size() const {
    const size_t n = m_gamma.n_elem;
    if (n != m_xc.n_elem || n != m_zc.n_elem || n + 1 != m_x.n_elem || n + 1 != m_z.n_elem ||
        n != m_ds.n_elem || n != m_theta.n_elem || n != m_enx.n_elem || n != m_enz.n_elem ||
        n != m_etx.n_elem || n != m_etz.n_elem)
        throw dvm::SizeMismatchException("VortexSheet");
    return static_cast<unsigned>(n);
}

void VortexSheet::print_collocation() const {
    for (unsigned i = 0; i < size(); ++i)
        std::cout << "(xc,zc) = (" << m_xc(i) << "," << m_zc(i) << ")" << std::endl;
}

void VortexSheet::print_unit_vectors() const {
    for (unsigned i = 0; i < size(); ++i)
        std::cout << "For panel No " << i << " the normal vectors are en = (" << m_enx(i) << ","
                  << m_enz(i) << ") and et = (" << m_etx(i) << "," << m_etz(i) << ")" << std::endl;
}

void VortexSheet::print_gamma() const {
    for (size_t i = 0; i < m_gamma.n_elem; ++i) std::cout << "   " << m_gamma(i) << "\n";
}

void VortexSheet::write_step(double time) { write_step_job(time)(); }

std::function<void()> VortexSheet::write_step_job(double time) const {
    // formats of src/VortexSheet.cpp:335-343
    if (m_gammapath.empty() || m_forcepath.empty())
        throw dvm::FileIOException("VortexSheet::write_step: no output files were set up");
    std::string g, f;
    for (size_t i = 0; i < m_xc.n_elem; ++i) {
        dvm::append_g(g, time);
        g += "\t ";
        dvm::append_g(g, m_xc(i));
        g += '\t';
        dvm::append_g(g, m_zc(i));
        g += '\t';
        dvm::append_g(g, m_gamma(i));
        g += '\t';
        dvm::append_g(g, m_ds(i));
        g += '\n';
    }
    dvm::append_g(f, time);
    f += '\t';
    dvm::append_g(f, m_fx);
    f += '\t';
    dvm::append_g(f, m_fz);
    f += '\n';
    return [g = std::move(g), f = std::move(f), gp = m_gammapath, fp = m_forcepath] {
        dvm::append_file(gp, g);
        dvm::append_file(fp, f);
    };
}

std::tuple<double, double> VortexSheet::get_forces() const { return std::make_tuple(m_fx, m_fz); }

void VortexSheet::probe_velocities(const VortexBlobs& blobs, Probe& probe) {
    // The intended formula of src/VortexSheet.cpp:559-646 (blob sum over all
    // blobs, sheet sum over all panels, free stream), on the GPU.
    upload(blobs);
    const unsigned n = probe.size();
    for (Vector* v : {&probe.m_u, &probe.m_w, &probe.m_uvs, &probe.m_wvs}) v->set_size(n);
    dvm::check_status(dvm_sim_probe(m_sim, dvm::vec_ptr(probe.m_x), dvm::vec_ptr(probe.m_z), n,
                                    dvm::vec_ptr(probe.m_u), dvm::vec_ptr(probe.m_w),
                                    dvm::vec_ptr(probe.m_uvs), dvm::vec_ptr(probe.m_wvs)),
                      "VortexSheet::probe_velocities");
}

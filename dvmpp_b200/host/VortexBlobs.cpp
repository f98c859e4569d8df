#include "VortexBlobs.hpp"

#include <filesystem>
#include <fstream>
#include <iostream>
#include <thread>

#include "Device.hpp"
#include "OutputWriter.hpp"
#include "VelocityKernel.hpp"

namespace fs = std::filesystem;

VortexBlobs::VortexBlobs() : m_kernel(dvm::VelocityKernel::create("direct")) {}

VortexBlobs::VortexBlobs(const XmlHandler& xml, const std::string& stamp)
    : m_kernel(dvm::VelocityKernel::create("direct")) {
    const std::string outdir = xml.getStringAttribute("io", "output_dir", true);
    const double dt = xml.getValueAttribute("time", "dt");
    const double steps = xml.getValueAttribute("time", "steps");
    m_blobsfile = (fs::path(outdir) / (stamp + "_vortex.dat")).string();
    std::ofstream bf(m_blobsfile);
    if (!bf) throw dvm::FileIOException::cannotOpen(m_blobsfile);
    // header of src/VortexBlobs.cpp:24-27
    bf << size() << " # Number of nodes\n"
       << dt << " # Time step\n"
       << steps << " # Steps\n"
       << "Time [s]\tx-position [m]\tz-position [m]\tcirculation\n";
    m_numfile = (fs::path(outdir) / (stamp + "_vortex_num.dat")).string();
    std::ofstream nf(m_numfile);
    if (!nf) throw dvm::FileIOException::cannotOpen(m_numfile);
    nf << "Time [s]\tNumber of vortices\n";
}

VortexBlobs::VortexBlobs(unsigned N) : m_kernel(dvm::VelocityKernel::create("direct")) {
    resize(N);
}

VortexBlobs::~VortexBlobs() = default;
VortexBlobs::VortexBlobs(VortexBlobs&& o) noexcept = default;
VortexBlobs& VortexBlobs::operator=(VortexBlobs&& o) noexcept = default;

VortexBlobs::VortexBlobs(const VortexBlobs& o)
    : m_ID(o.m_ID), m_x(o.m_x), m_z(o.m_z), m_circ(o.m_circ), m_sigma(o.m_sigma), m_u(o.m_u),
      m_w(o.m_w), m_uvs(o.m_uvs), m_wvs(o.m_wvs), m_blobsfile(o.m_blobsfile),
      m_numfile(o.m_numfile),
      m_kernel(dvm::VelocityKernel::create(o.m_kernel ? o.m_kernel->name() : "direct")) {}

VortexBlobs& VortexBlobs::operator=(const VortexBlobs& o) {
    if (this != &o) {
        m_ID = o.m_ID;
        m_x = o.m_x;
        m_z = o.m_z;
        m_circ = o.m_circ;
        m_sigma = o.m_sigma;
        m_u = o.m_u;
        m_w = o.m_w;
        m_uvs = o.m_uvs;
        m_wvs = o.m_wvs;
        m_blobsfile = o.m_blobsfile;
        m_numfile = o.m_numfile;
        m_kernel = dvm::VelocityKernel::create(o.m_kernel ? o.m_kernel->name() : "direct");
    }
    return *this;
}

void VortexBlobs::resize(unsigned n) {
    m_ID.resize(n);
    m_x.set_size(n);
    m_z.set_size(n);
    m_circ.set_size(n);
    m_sigma.set_size(n);
    m_u.set_size(n);
    m_w.set_size(n);
    m_uvs.set_size(n);
    m_wvs.set_size(n);
}

void VortexBlobs::setKernelType(const std::string& type) {
    m_kernel = dvm::VelocityKernel::create(type);
}

std::string VortexBlobs::kernelType() const { return m_kernel ? m_kernel->name() : "direct"; }

void VortexBlobs::copyOutputConfig(const VortexBlobs& o) {
    m_blobsfile = o.m_blobsfile;
    m_numfile = o.m_numfile;
}

unsigned VortexBlobs::merge_blobs(double threshold) {
    // src/VortexBlobs.cpp:110-209 on the GPU (dvm_merge_blobs): the same greedy
    // order and arithmetic, so the same merged set, bit for bit
    const uint64_t n = size();
    if (n < 2) return 0;
    Vector* const arr[8] = {&m_x, &m_z, &m_circ, &m_sigma, &m_u, &m_w, &m_uvs, &m_wvs};
    std::vector<std::vector<double>> v(8);
    for (int k = 0; k < 8; ++k) v[k].assign(arr[k]->memptr(), arr[k]->memptr() + n);
    std::vector<uint32_t> ids(n);
    for (uint64_t i = 0; i < n; ++i) ids[i] = m_ID[i];
    uint64_t m = n, merged = 0;
    dvm::check_status(dvm_merge_blobs(dvm::device_context(), v[0].data(), v[1].data(),
                                      v[2].data(), v[3].data(), v[4].data(), v[5].data(),
                                      v[6].data(), v[7].data(), ids.data(), n, threshold, &m,
                                      &merged),
                      "VortexBlobs::merge_blobs");
    if (merged == 0) return 0;
    resize((unsigned)m);
    for (int k = 0; k < 8; ++k)
        for (uint64_t i = 0; i < m; ++i) (*arr[k])(i) = v[k][i];
    for (uint64_t i = 0; i < m; ++i) m_ID[i] = ids[i];
    return (unsigned)merged;
}

void VortexBlobs::append_vortices(VortexBlobs& nb) {
    // IDs of appended blobs are shifted by the old count (src/VortexBlobs.cpp:211-217)
    const unsigned nold = size(), nnew = nb.size();
    for (unsigned i = 0; i < nnew; ++i) m_ID.push_back(nold + nb.m_ID[i]);
    m_x.insert_rows(m_x.n_elem, nb.m_x);
    m_z.insert_rows(m_z.n_elem, nb.m_z);
    m_circ.insert_rows(m_circ.n_elem, nb.m_circ);
    m_sigma.insert_rows(m_sigma.n_elem, nb.m_sigma);
    m_u.insert_rows(m_u.n_elem, nb.m_u);
    m_w.insert_rows(m_w.n_elem, nb.m_w);
    m_uvs.insert_rows(m_uvs.n_elem, nb.m_uvs);
    m_wvs.insert_rows(m_wvs.n_elem, nb.m_wvs);
}

void VortexBlobs::biotsavart() {
    const unsigned n = size();
    if (n == 0) return;
    std::vector<dvm::VortexParticle> p(n);
    for (unsigned i = 0; i < n; ++i) p[i] = {m_x(i), m_z(i), m_circ(i), m_sigma(i)};
    std::vector<dvm::VelocityResult> v;
    m_kernel->computeSelfInduced(p, v);
    for (unsigned i = 0; i < n; ++i) {
        m_u(i) = v[i].u;
        m_w(i) = v[i].w;
    }
}

void VortexBlobs::diffusion_random_walk(Random& rng, double nu, double dt) {
    const unsigned n = size();
    if (n == 0) return;
    std::vector<double> R(2 * (size_t)n);
    for (auto& r : R) r = rng.rand();  // R1, R2 per blob, in blob order
    dvm::check_status(dvm_random_walk(dvm::device_context(), dvm::vec_ptr(m_x),
                                      dvm::vec_ptr(m_z), n, R.data(), nu, dt),
                      "diffusion_random_walk");
}

double VortexBlobs::totalcirc() const {
    double s = 0.0;
    for (size_t i = 0; i < m_circ.n_elem; ++i) s += m_circ(i);
    return s;
}

unsigned VortexBlobs::size() const {
    const size_t n = m_ID.size();
    if (n != m_x.size() || n != m_z.size() || n != m_circ.size() || n != m_sigma.size() ||
        n != m_u.size() || n != m_w.size() || n != m_uvs.size() || n != m_wvs.size())
        throw dvm::SizeMismatchException("VortexBlobs");
    return static_cast<unsigned>(n);
}

void VortexBlobs::print_location() const {
    for (unsigned i = 0; i < size(); ++i)
        std::cout << " The location of Vortex Blob " << m_ID[i] << " is (x,z) = (" << m_x(i)
                  << "," << m_z(i) << ")" << std::endl;
}

void VortexBlobs::print_velocity() const {
    for (unsigned i = 0; i < size(); ++i)
        std::cout << "(u,w) = (" << m_u(i) << "," << m_w(i) << ")" << std::endl;
}

void VortexBlobs::print_circulation() const {
    for (unsigned i = 0; i < size(); ++i) std::cout << " circ = " << m_circ(i) << std::endl;
}

void VortexBlobs::write_step(double time, unsigned step) { write_step_job(time, step)(); }

std::function<void()> VortexBlobs::write_step_job(double time, unsigned step) const {
    // formats of src/VortexBlobs.cpp:310-332: one "t x z circ" row per blob,
    // then "step n" in the count file
    if (m_blobsfile.empty() || m_numfile.empty())
        throw dvm::FileIOException("VortexBlobs::write_step: must set filenames before writing");
    const size_t n = size();
    std::vector<double> x(m_x.memptr(), m_x.memptr() + n), z(m_z.memptr(), m_z.memptr() + n),
        c(m_circ.memptr(), m_circ.memptr() + n);
    return [time, step, n, x = std::move(x), z = std::move(z), c = std::move(c),
            bfile = m_blobsfile, nfile = m_numfile] {
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency() / 2);
        dvm::append_file(bfile, dvm::format_rows4(time, x.data(), z.data(), c.data(), n, hw));
        std::string line;
        dvm::append_u(line, step);
        line += '\t';
        dvm::append_u(line, n);
        line += '\n';
        dvm::append_file(nfile, line);
    };
}

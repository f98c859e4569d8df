#include "Probe.hpp"

#include <filesystem>
#include <fstream>

#include "Exceptions.hpp"
#include "OutputWriter.hpp"

namespace fs = std::filesystem;

Probe::Probe() = default;

Probe::Probe(const XmlHandler& xml, const std::string& stamp) {
    m_x = Vector(xml.getList("probe", "x"));
    m_z = Vector(xml.getList("probe", "z"));
    const size_t n = m_x.n_elem;
    for (Vector* v : {&m_u, &m_w, &m_uvs, &m_wvs}) {
        v->set_size(n);
        v->zeros();
    }
    const std::string outdir = xml.getStringAttribute("io", "output_dir", true);
    m_outfile = (fs::path(outdir) / (stamp + "_probe.dat")).string();
    std::ofstream of(m_outfile);
    if (!of) throw dvm::FileIOException::cannotOpen(m_outfile);
    // header of src/Probe.cpp:28-30
    of << xml.getValueAttribute("time", "dt") << " # Time step\n"
       << xml.getValueAttribute("time", "steps") << " # Steps\n"
       << "Time [s]\tu [m/s]\tw [m/s]\n";
}

unsigned Probe::size() const { return static_cast<unsigned>(m_x.n_elem); }

void Probe::write_step(double time) { write_step_job(time)(); }

std::function<void()> Probe::write_step_job(double time) const {
    // format of src/Probe.cpp:43-55: "t u w" per probe point
    std::string s;
    for (unsigned i = 0; i < size(); ++i) {
        dvm::append_g(s, time);
        s += '\t';
        dvm::append_g(s, m_u(i));
        s += '\t';
        dvm::append_g(s, m_w(i));
        s += '\n';
    }
    return [s = std::move(s), path = m_outfile] { dvm::append_file(path, s); };
}

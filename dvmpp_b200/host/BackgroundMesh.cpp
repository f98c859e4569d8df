#include "BackgroundMesh.hpp"

#include <vector>

#include "Device.hpp"
#include "Exceptions.hpp"

BackgroundMesh::BackgroundMesh() = default;

BackgroundMesh::BackgroundMesh(const XmlHandler& xml) {
    if (!xml.has("remesh", "frequency")) return;
    const double f = xml.getValueAttribute("remesh", "frequency");
    if (!(f >= 1.0)) return;
    m_frequency = (unsigned)f;
    m_p.xmin = xml.getValueAttribute("remesh", "xmin");
    m_p.xmax = xml.getValueAttribute("remesh", "xmax");
    m_p.zmin = xml.getValueAttribute("remesh", "zmin");
    m_p.zmax = xml.getValueAttribute("remesh", "zmax");
    m_p.dx = xml.getValueAttribute("remesh", "dx");
    m_p.dz = xml.getValueAttribute("remesh", "dz");
    m_p.sigma = xml.getValueAttribute("remesh", "sigma");
    m_p.circ_threshold =
        xml.has("remesh", "circ_threshold") ? xml.getValueAttribute("remesh", "circ_threshold") : 0.0;
    const std::string k =
        xml.has("remesh", "kernel") ? xml.getStringAttribute("remesh", "kernel") : "M4prime";
    if (k == "M4prime") m_p.kernel = DVM_REMESH_M4PRIME;
    else if (k == "M6") m_p.kernel = DVM_REMESH_M6;
    else if (k == "gaussian") m_p.kernel = DVM_REMESH_GAUSSIAN;
    else throw dvm::AlgorithmException("remesh/kernel: unknown kernel " + k);
    uint32_t nx = 0, nz = 0;
    dvm::check_status(dvm_remesh_grid(&m_p, &nx, &nz), "BackgroundMesh");
    m_nx = nx;
    m_nz = nz;
    m_enabled = true;
}

VortexBlobs BackgroundMesh::remesh(const VortexBlobs& blobs) const {
    if (!m_enabled) return blobs;  // a disabled mesh returns a copy
    const unsigned n = blobs.size();
    std::vector<dvm_particle> in(n);
    for (unsigned i = 0; i < n; ++i)
        in[i] = dvm_particle{blobs.m_x(i), blobs.m_z(i), blobs.m_circ(i), blobs.m_sigma(i)};
    std::vector<dvm_particle> out((size_t)m_nx * m_nz + n);
    uint64_t m = 0;
    dvm::check_status(dvm_remesh(dvm::device_context(), in.data(), n, &m_p, out.data(),
                                 out.size(), &m),
                      "BackgroundMesh::remesh");
    VortexBlobs r((unsigned)m);
    for (unsigned i = 0; i < (unsigned)m; ++i) {
        r.m_ID[i] = i;
        r.m_x(i) = out[i].x;
        r.m_z(i) = out[i].z;
        r.m_circ(i) = out[i].circ;
        r.m_sigma(i) = out[i].sigma;
        r.m_u(i) = r.m_w(i) = r.m_uvs(i) = r.m_wvs(i) = 0.0;
    }
    r.copyOutputConfig(blobs);
    return r;
}

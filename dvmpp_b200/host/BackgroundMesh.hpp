// The reference's BackgroundMesh (declared in src/DVMBase.hpp:51, used at
// src/DVMBase.cpp:91-92, 160-164; options src/XmlHandler.cpp:191-201).  Its
// source is not part of the reference; the behaviour follows the reference's
// tests (tests/unit/test_BackgroundMesh.cpp): a default-constructed mesh is
// disabled (should_remesh false, nx = nz = 0, remesh returns a copy); an
// enabled one remeshes every `frequency` steps onto nodes xmin + i dx,
// zmin + j dz with the M4', M6 or truncated-Gaussian tensor-product kernel,
// on the GPU (dvm_remesh / dvm_sim_remesh).
#ifndef DVMPP_B200_BACKGROUNDMESH_HPP
#define DVMPP_B200_BACKGROUNDMESH_HPP

#include "VortexBlobs.hpp"
#include "XmlHandler.hpp"
#include "dvm_cuda.h"

class BackgroundMesh
{
  public:
    BackgroundMesh();
    // Enabled when remesh/frequency > 0; a case without a <remesh> section
    // gives a disabled mesh.
    explicit BackgroundMesh(const XmlHandler& xml);

    [[nodiscard]] bool is_enabled() const { return m_enabled; }
    [[nodiscard]] bool should_remesh(unsigned step) const {
        return m_enabled && m_frequency > 0 && step % m_frequency == 0;
    }
    [[nodiscard]] unsigned nx() const { return m_nx; }
    [[nodiscard]] unsigned nz() const { return m_nz; }
    [[nodiscard]] const dvm_remesh_params& params() const { return m_p; }

    // A new blob set: mesh-node blobs (|circulation| > circ_threshold), then
    // the blobs whose kernel support leaves the mesh, unchanged.
    [[nodiscard]] VortexBlobs remesh(const VortexBlobs& blobs) const;

  private:
    bool m_enabled = false;
    unsigned m_frequency = 0, m_nx = 0, m_nz = 0;
    dvm_remesh_params m_p{};
};

#endif

// Disabled stand-in for the reference's BackgroundMesh class, whose source
// (src/BackgroundMesh.{hpp,cpp}) is referenced by src/DVMBase.hpp:4,51 but is
// absent from the reference tree.  Test infrastructure only: remeshing is not
// on the hot path, and this stub keeps it permanently off so that DVMBase
// compiles.  API per tests/unit/test_BackgroundMesh.cpp:14-18.
#ifndef DVM_REFSHIM_BACKGROUNDMESH
#define DVM_REFSHIM_BACKGROUNDMESH

#include "VortexBlobs.hpp"
#include "XmlHandler.hpp"

class BackgroundMesh
{
  public:
    BackgroundMesh() = default;
    explicit BackgroundMesh(const XmlHandler&) {}
    bool is_enabled() const { return false; }
    bool should_remesh(unsigned) const { return false; }
    VortexBlobs remesh(const VortexBlobs& v) const { return v; }
    unsigned nx() const { return 0; }
    unsigned nz() const { return 0; }
};

#endif

// The reference's solver class (src/DVMBase.hpp:43-105): DVMBase(xml, stamp)
// and solve().  The time loop keeps every blob and the sheet on the GPU
// (one device-resident simulation, one batched kernel sequence per step) and
// copies state back only for the per-step output files, which keep the
// reference's formats and are written by a background thread (the files are
// complete when solve() / run() return).  The random walk uses the reference's stream
// (constants/seed through std::mt19937) unless algorithms/diffusion_rng is
// "philox".  algorithms/velocity_kernel selects the pair arithmetic:
// "direct" (default, FP64) or "cuda" (FP32 with compensated sums).
#ifndef DVMPP_B200_DVMBASE_HPP
#define DVMPP_B200_DVMBASE_HPP

#include <string>

#include "BackgroundMesh.hpp"
#include "BaseTypes.hpp"
#include "Exceptions.hpp"
#include "OutputWriter.hpp"
#include "Probe.hpp"
#include "Random.hpp"
#include "VortexBlobs.hpp"
#include "VortexSheet.hpp"
#include "XmlHandler.hpp"

enum class Scheme { Euler, RK3 };
enum class SurfaceCross { Delete, Absorb, Reflect };

class DVMBase
{
  private:
    VortexBlobs m_vortex;
    VortexSheet m_vortsheet;
    Probe m_probe;
    Random m_rand;
    XmlHandler m_xml;
    BackgroundMesh m_mesh;
    double m_nu = 0, m_Ux = 0, m_Uz = 0, m_Ur = 0, m_dt = 0, m_time = 0;
    unsigned m_step = 0, m_steps = 0;
    double m_merge_threshold = 0.0;  // algorithms/merge_threshold
    unsigned m_merge_frequency = 0;  // algorithms/merge_frequency
    Scheme m_scheme = Scheme::Euler;
    SurfaceCross m_surfcross = SurfaceCross::Reflect;
    int m_rng_mode = DVM_RNG_INJECT;
    int m_precision = DVM_F64;
    bool m_quiet = false;
    dvm_sim* m_sim = nullptr;  // owned by m_vortsheet
    // Output files are formatted and appended on a background thread while
    // the GPU runs the next step (declared last: destroyed, i.e. drained,
    // before the objects its jobs were copied from).
    dvm::AsyncWriter m_writer{2};

    void compute_step();
    void increment_step();
    [[nodiscard]] unsigned get_steps() const;
    [[nodiscard]] double get_time() const;
    void convect();
    void remesh();
    void write_outputs();
    void sync_to_host(bool full = true);
    void supply_uniforms();

  public:
    DVMBase(XmlHandler& xml, const std::string& timestamp);
    void solve();
    // solve() without the per-step files (`write` false) or console lines.
    void run(unsigned steps, bool write, bool quiet);
    [[nodiscard]] unsigned num_blobs() const;
    [[nodiscard]] std::tuple<double, double> forces() const;
    VortexBlobs& blobs() { return m_vortex; }
};

#endif

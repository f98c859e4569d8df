// The reference's VortexSheet (src/VortexSheet.hpp:21-127), same public
// methods, backed by a device-resident simulation (dvm_sim): the body, its
// influence matrix and least-squares pseudo-inverse live in HBM.  The methods
// that take a VortexBlobs container upload its state, run the matching GPU
// phase and copy the results back -- a drop-in for code that calls them one by
// one; DVMBase instead keeps the blobs on the device for the whole run.
#ifndef DVMPP_B200_VORTEXSHEET_HPP
#define DVMPP_B200_VORTEXSHEET_HPP

#include <fstream>
#include <functional>
#include <string>
#include <tuple>

#include "BaseTypes.hpp"
#include "Exceptions.hpp"
#include "Random.hpp"
#include "VortexBlobs.hpp"
#include "XmlHandler.hpp"
#include "dvm_cuda.h"

class Probe;

class VortexSheet
{
  private:
    Vector m_gamma, m_x, m_z, m_xc, m_zc, m_theta, m_ds, m_enx, m_enz, m_etx, m_etz;
    double m_A = 0.0;
    double m_rho = 1.0, m_nu = 0.0, m_dt = 0.0;
    unsigned m_maxNumPanelVort = 0;
    double m_cutoff_exp = 0.0;
    double m_fx = 0.0, m_fz = 0.0;
    double m_Ux = 0.0, m_Uz = 0.0;
    std::string m_gammapath, m_forcepath;  // output files (headers written at set-up)
    // device side
    dvm_sim_params m_params{};
    dvm_sim* m_sim = nullptr;

    void read_input_coord(const std::string& domain);
    void build_device(uint64_t capacity);
    void upload(const VortexBlobs& blobs);

  public:
    VortexSheet();
    VortexSheet(const XmlHandler& xml, const std::string& timestamp);
    ~VortexSheet();
    VortexSheet(const VortexSheet&) = delete;
    VortexSheet& operator=(const VortexSheet&) = delete;

    void vortexsheetbc(VortexBlobs& blobs);
    void solvevortexsheet(VortexBlobs& blobs);
    [[nodiscard]] VortexBlobs release_nascent_vortices_rw(Random& _rand);
    void reflect(VortexBlobs& vortex);
    void delete_inside(VortexBlobs& vortex);
    void compute_loads(double Urel);
    [[nodiscard]] unsigned size() const;
    void print_collocation() const;
    void print_unit_vectors() const;
    void print_gamma() const;
    void write_step(double time);
    // The same output as a job owning copies of what it writes.
    [[nodiscard]] std::function<void()> write_step_job(double time) const;
    [[nodiscard]] std::tuple<double, double> get_forces() const;
    // Not provided: the reference never calls it and its formula is not the
    // intended one; throws dvm::AlgorithmException.
    void probe_velocities(const VortexBlobs& blobs, Probe& probe);

    // ---- device access for DVMBase ----
    // The simulation holding this body, with room for at least `capacity` blobs.
    dvm_sim* device(uint64_t capacity);
    void set_params(int precision, int rng, int scheme, int surface_cross, int64_t seed);
    // Pull gamma and the loads of the last step from the device.
    void pull_from_device();
    [[nodiscard]] unsigned max_release() const;
    [[nodiscard]] uint64_t capacity() const { return m_params.capacity; }
};

#endif

// The reference's Probe (src/Probe.hpp:13-37): probe points from the XML
// lists <probe><x string=...>/<z string=...> and the per-step _probe.dat
// writer.  The reference's loop never computes probe velocities (its file
// holds whatever the vectors were initialised to); the drop-in DVMBase fills
// them from the device at every written step (dvm_sim_probe).
#ifndef DVMPP_B200_PROBE_HPP
#define DVMPP_B200_PROBE_HPP

#include <functional>
#include <string>

#include "BaseTypes.hpp"
#include "XmlHandler.hpp"

class Probe
{
  public:
    Vector m_x, m_z, m_u, m_w, m_uvs, m_wvs;

  private:
    std::string m_outfile;

  public:
    Probe();
    Probe(const XmlHandler& xml, const std::string& stamp);
    [[nodiscard]] unsigned size() const;
    void write_step(double time);
    [[nodiscard]] std::function<void()> write_step_job(double time) const;
};

#endif

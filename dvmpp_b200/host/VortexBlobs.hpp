// The reference's VortexBlobs container (src/VortexBlobs.hpp:21-109), same
// public members and methods.  Its compute methods run on the GPU:
// biotsavart() through the velocity-kernel plugin (dvm::DirectKernel by
// default, FP64) and diffusion_random_walk() through dvm_random_walk with the
// caller's Random stream.  Inside DVMBase the blob state lives on the device and
// these host arrays are refreshed only for output.
#ifndef DVMPP_B200_VORTEXBLOBS_HPP
#define DVMPP_B200_VORTEXBLOBS_HPP

#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "BaseTypes.hpp"
#include "Exceptions.hpp"
#include "Random.hpp"
#include "XmlHandler.hpp"

namespace dvm {
class VelocityKernel;
}

class VortexBlobs
{
  public:
    std::vector<unsigned> m_ID;
    Vector m_x;
    Vector m_z;
    Vector m_circ;
    Vector m_sigma;
    Vector m_u;
    Vector m_w;
    Vector m_uvs;
    Vector m_wvs;

  private:
    std::string m_blobsfile;
    std::string m_numfile;
    std::unique_ptr<dvm::VelocityKernel> m_kernel;

  public:
    VortexBlobs();
    VortexBlobs(const XmlHandler& xml, const std::string& stamp);
    explicit VortexBlobs(unsigned N);
    ~VortexBlobs();
    VortexBlobs(VortexBlobs&& other) noexcept;
    VortexBlobs& operator=(VortexBlobs&& other) noexcept;
    VortexBlobs(const VortexBlobs& other);
    VortexBlobs& operator=(const VortexBlobs& other);

    void append_vortices(VortexBlobs& NewVortBlobs);
    void biotsavart();
    void diffusion_random_walk(Random& _rand, double nu, double dt);
    [[nodiscard]] double totalcirc() const;
    [[nodiscard]] unsigned size() const;
    void print_location() const;
    void print_velocity() const;
    void print_circulation() const;
    void write_step(double time, unsigned step);
    // The same output as a job that owns copies of what it writes (for a
    // background writer; files are appended when the job runs).
    [[nodiscard]] std::function<void()> write_step_job(double time, unsigned step) const;
    void setKernelType(const std::string& type);
    [[nodiscard]] std::string kernelType() const;
    void copyOutputConfig(const VortexBlobs& other);
    // Greedy vortex merging (src/VortexBlobs.cpp:110-209) on the GPU through
    // dvm_merge_blobs: the reference's index order and FP64 arithmetic, so the
    // merged set is bit-identical; returns the merge count.
    unsigned merge_blobs(double threshold = 1e-5);
    // Resize every array to n (values of new entries unspecified, as set_size).
    void resize(unsigned n);
};

#endif

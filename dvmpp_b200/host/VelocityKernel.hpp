// The reference's velocity-kernel plugin seam (src/VelocityKernel.hpp:12-62)
// with GPU implementations behind it:
//   create("direct")  DirectKernel -- the reference's direct O(N^2) sum,
//                     FP64 on the GPU (same operation order)
//   create("cuda")    CudaKernel   -- FP32 pair sums with compensated
//                     accumulation on the GPU
//   create("cuda64")  CudaKernel in FP64
// Unknown names throw dvm::AlgorithmException, as the reference's factory does.
#ifndef DVMPP_B200_VELOCITYKERNEL_HPP
#define DVMPP_B200_VELOCITYKERNEL_HPP

#include <memory>
#include <string>
#include <vector>

#include "BaseTypes.hpp"

namespace dvm {

struct VelocityResult {
    double u = 0.0;
    double w = 0.0;
};

struct VortexParticle {
    double x;
    double z;
    double circ;
    double sigma;
};

class VelocityKernel {
  public:
    virtual ~VelocityKernel() = default;
    virtual void computeSelfInduced(const std::vector<VortexParticle>& particles,
                                    std::vector<VelocityResult>& velocities) = 0;
    virtual void computeInducedAt(const std::vector<VortexParticle>& sources,
                                  const std::vector<double>& target_x,
                                  const std::vector<double>& target_z,
                                  std::vector<VelocityResult>& velocities) = 0;
    [[nodiscard]] static std::unique_ptr<VelocityKernel> create(const std::string& type);
    [[nodiscard]] virtual std::string name() const = 0;
    // DVM_F64 or DVM_F32: the arithmetic of the pair sums.
    [[nodiscard]] virtual int precision() const = 0;
};

class CudaKernel : public VelocityKernel {
  public:
    explicit CudaKernel(int precision, std::string name);
    void computeSelfInduced(const std::vector<VortexParticle>& particles,
                            std::vector<VelocityResult>& velocities) override;
    void computeInducedAt(const std::vector<VortexParticle>& sources,
                          const std::vector<double>& target_x,
                          const std::vector<double>& target_z,
                          std::vector<VelocityResult>& velocities) override;
    [[nodiscard]] std::string name() const override { return m_name; }
    [[nodiscard]] int precision() const override { return m_precision; }

  private:
    int m_precision;
    std::string m_name;
};

// The direct method under its reference name: FP64 on the GPU.
class DirectKernel : public CudaKernel {
  public:
    DirectKernel();
};

}  // namespace dvm

#endif

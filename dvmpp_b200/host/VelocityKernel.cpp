#include "VelocityKernel.hpp"

#include "Device.hpp"
#include "Exceptions.hpp"

static_assert(sizeof(dvm::VortexParticle) == sizeof(dvm_particle), "particle layout");
static_assert(sizeof(dvm::VelocityResult) == sizeof(dvm_velocity), "velocity layout");

namespace dvm {

std::unique_ptr<VelocityKernel> VelocityKernel::create(const std::string& type) {
    if (type == "direct") return std::make_unique<DirectKernel>();
    if (type == "cuda") return std::make_unique<CudaKernel>(DVM_F32, "cuda");
    if (type == "cuda64") return std::make_unique<CudaKernel>(DVM_F64, "cuda64");
    throw AlgorithmException("Unknown velocity kernel type: " + type +
                             ". Available: direct, cuda, cuda64");
}

CudaKernel::CudaKernel(int precision, std::string name)
    : m_precision(precision), m_name(std::move(name)) {}

DirectKernel::DirectKernel() : CudaKernel(DVM_F64, "direct") {}

void CudaKernel::computeSelfInduced(const std::vector<VortexParticle>& p,
                                    std::vector<VelocityResult>& v) {
    v.resize(p.size());  // the callee sizes the output, as the reference does
    if (p.empty()) return;
    check_status(dvm_biot_savart_self(device_context(),
                                      reinterpret_cast<const dvm_particle*>(p.data()), p.size(),
                                      reinterpret_cast<dvm_velocity*>(v.data()), m_precision),
                 "computeSelfInduced");
}

void CudaKernel::computeInducedAt(const std::vector<VortexParticle>& s,
                                  const std::vector<double>& tx, const std::vector<double>& tz,
                                  std::vector<VelocityResult>& v) {
    if (tx.size() != tz.size()) throw SizeMismatchException("computeInducedAt targets");
    v.resize(tx.size());
    if (tx.empty()) return;
    check_status(dvm_biot_savart_at(device_context(),
                                    reinterpret_cast<const dvm_particle*>(s.data()), s.size(),
                                    tx.data(), tz.data(), tx.size(),
                                    reinterpret_cast<dvm_velocity*>(v.data()), m_precision),
                 "computeInducedAt");
}

}  // namespace dvm

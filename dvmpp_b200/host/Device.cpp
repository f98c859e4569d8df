#include "Device.hpp"

#include <cstdlib>
#include <mutex>
#include <string>

#include "Exceptions.hpp"

namespace dvm {

void check_status(int status, const char* where) {
    if (status == DVM_OK) return;
    const std::string msg = std::string(where) + ": " + dvm_last_error();
    switch (status) {
        case DVM_ERR_ARG: throw SizeMismatchException(msg);
        case DVM_ERR_RELEASE: throw VortexException(msg);
        case DVM_ERR_CAPACITY:
        case DVM_ERR_RNG:
        case DVM_ERR_STATE: throw AlgorithmException(msg);
        default: throw DVMException(msg);
    }
}

dvm_ctx* device_context() {
    static std::once_flag once;
    static dvm_ctx* ctx = nullptr;
    static int status = DVM_OK;
    std::call_once(once, [] {
        const char* d = std::getenv("DVMPP_DEVICE");
        status = dvm_ctx_create(d ? std::atoi(d) : 0, 0, &ctx);
    });
    check_status(status, "device context");
    return ctx;
}

}  // namespace dvm

// Process-wide device context of the drop-in host library: one dvm_ctx on the
// device named by $DVMPP_DEVICE (default 0), created on first use.
#ifndef DVMPP_B200_DEVICE_HPP
#define DVMPP_B200_DEVICE_HPP

#include "dvm_cuda.h"

namespace dvm {
dvm_ctx* device_context();
}

#endif

// C entry points of libdvmpp_host.so, for hosts without a C++ binding.
#include <cstring>
#include <exception>
#include <iostream>
#include <sstream>
#include <string>

#include "DVMBase.hpp"
#include "XmlHandler.hpp"

namespace {
thread_local std::string g_host_err;
}

extern "C" {

const char* dvmpp_host_last_error() { return g_host_err.c_str(); }

// DVMBase(xml, stamp) then `steps` steps (0: the XML's time/steps), writing the
// reference's per-step output files when `write` != 0.  Returns 0, or 1 with
// dvmpp_host_last_error() set.  nblobs / fx / fz (optional) get the final state.
int dvmpp_host_run_xml(const char* xml_path, const char* stamp, unsigned steps, int write,
                       int quiet, unsigned long long* nblobs, double* fx, double* fz) {
    std::streambuf* old = nullptr;
    std::ostringstream sink;
    if (quiet) old = std::cout.rdbuf(sink.rdbuf());
    int rc = 0;
    try {
        XmlHandler xml(xml_path);
        DVMBase dvm(xml, stamp);
        const unsigned n = steps ? steps : (unsigned)xml.getValueAttribute("time", "steps");
        dvm.run(n, write != 0, quiet != 0);
        if (nblobs) *nblobs = dvm.num_blobs();
        auto f = dvm.forces();
        if (fx) *fx = std::get<0>(f);
        if (fz) *fz = std::get<1>(f);
    } catch (const std::exception& e) {
        g_host_err = e.what();
        rc = 1;
    }
    if (old) std::cout.rdbuf(old);
    return rc;
}

}  // extern "C"

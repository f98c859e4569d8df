// Checks dvm::append_g / format_rows4 against std::ostream's default double
// formatting (the reference's writers) and AsyncWriter's ordering / errors.
// Built and run by tests/test_output_writer.py; prints "ok" or the first mismatch.
#include <cmath>
#include <cstdio>
#include <limits>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "Exceptions.hpp"
#include "OutputWriter.hpp"

static std::string ostream_g(double v) {
    std::ostringstream o;
    o << v;
    return o.str();
}

int main(int argc, char** argv) {
    const std::string dir = argc > 1 ? argv[1] : ".";
    std::vector<double> vals = {0.0, -0.0, 1.0, -1.0, 0.1, 1e-5, 1e-4, 123456.0, 1234567.0,
                                999999.5, 9999995.0, 1e21, 1e-300, 5e-324, 2.5, 0.5, 1.0 / 3.0,
                                std::numeric_limits<double>::max(),
                                std::numeric_limits<double>::min(),
                                std::numeric_limits<double>::infinity(),
                                -std::numeric_limits<double>::infinity(), 0.005, 0.0049999999};
    std::mt19937_64 g(7);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    std::uniform_int_distribution<int> e(-40, 40);
    for (int i = 0; i < 2000000; ++i) vals.push_back(u(g) * std::pow(10.0, e(g)));
    for (int i = 0; i < 200000; ++i) vals.push_back(std::round(u(g) * 1e7) / 1e3);
    for (double v : vals) {
        std::string s;
        dvm::append_g(s, v);
        if (s != ostream_g(v)) {
            std::printf("mismatch %.17g: to_chars '%s' ostream '%s'\n", v, s.c_str(),
                        ostream_g(v).c_str());
            return 1;
        }
    }
    // rows, multi-threaded, equal to a plain ostream loop
    const size_t n = 300000;
    std::vector<double> x(n), z(n), c(n);
    for (size_t i = 0; i < n; ++i) {
        x[i] = u(g) * 20;
        z[i] = u(g);
        c[i] = u(g) * 1e-3;
    }
    std::ostringstream ref;
    for (size_t i = 0; i < n; ++i) ref << 0.125 << "\t" << x[i] << "\t" << z[i] << "\t" << c[i] << "\n";
    if (dvm::format_rows4(0.125, x.data(), z.data(), c.data(), n, 8) != ref.str()) {
        std::printf("format_rows4 differs from the ostream rows\n");
        return 1;
    }
    // ordered background appends, then an error surfaces on flush
    const std::string path = dir + "/order.txt";
    std::remove(path.c_str());
    {
        dvm::AsyncWriter w(2);
        for (int k = 0; k < 200; ++k)
            w.submit([k, path] { dvm::append_file(path, std::to_string(k) + "\n"); });
        w.flush();
        std::string expect;
        for (int k = 0; k < 200; ++k) expect += std::to_string(k) + "\n";
        std::FILE* f = std::fopen(path.c_str(), "rb");
        std::string got(expect.size() + 16, '\0');
        got.resize(std::fread(&got[0], 1, got.size(), f));
        std::fclose(f);
        if (got != expect) {
            std::printf("background appends out of order\n");
            return 1;
        }
        w.submit([dir] { dvm::append_file(dir + "/no/such/dir/x.txt", "x"); });
        bool threw = false;
        try {
            w.flush();
        } catch (const dvm::FileIOException&) {
            threw = true;
        }
        if (!threw) {
            std::printf("a failed append did not surface\n");
            return 1;
        }
        w.submit([] {});  // usable again after the error was reported
        w.flush();
    }
    std::printf("ok\n");
    return 0;
}

// Basic types of the drop-in host library (the reference's src/BaseTypes.hpp:
// Vector / Matrix / Vector_un aliases and the math constants).
//
// Where Armadillo is available the aliases are Armadillo's, exactly as in the
// reference; otherwise Vector is a small column vector with the subset of
// Armadillo's interface that the DVM classes and their users touch
// (operator(), n_elem, size, set_size, copy_size, insert_rows, memptr, zeros).
#ifndef DVMPP_B200_BASETYPES_HPP
#define DVMPP_B200_BASETYPES_HPP

#include <cstddef>
#include <vector>

#if defined(DVMPP_USE_ARMADILLO) || __has_include(<armadillo>)
#include <armadillo>
using Matrix = arma::mat;
using Vector = arma::vec;
using Vector_un = arma::Col<unsigned>;
#define DVMPP_HAVE_ARMADILLO 1
#else
namespace dvm {
// Column vector of doubles with Armadillo-style accessors.
class HostVector {
  public:
    std::vector<double> mem;
    std::size_t n_elem = 0;
    HostVector() = default;
    explicit HostVector(std::size_t n) : mem(n, 0.0), n_elem(n) {}
    HostVector(const std::vector<double>& v) : mem(v), n_elem(v.size()) {}
    double& operator()(std::size_t i) { return mem[i]; }
    double operator()(std::size_t i) const { return mem[i]; }
    double& operator[](std::size_t i) { return mem[i]; }
    double operator[](std::size_t i) const { return mem[i]; }
    std::size_t size() const { return n_elem; }
    void set_size(std::size_t n) {
        mem.resize(n);
        n_elem = n;
    }
    void copy_size(const HostVector& o) { set_size(o.n_elem); }
    void zeros() {
        for (auto& v : mem) v = 0.0;
    }
    void insert_rows(std::size_t at, const HostVector& o) {
        mem.insert(mem.begin() + (std::ptrdiff_t)at, o.mem.begin(), o.mem.end());
        n_elem = mem.size();
    }
    double* memptr() { return mem.data(); }
    const double* memptr() const { return mem.data(); }
};
}  // namespace dvm
using Vector = dvm::HostVector;
#endif

namespace math {
inline constexpr double pi = 3.14159265358979323846;
inline constexpr double rpi2 = 1.0 / (2.0 * 3.14159265358979323846);
template <typename T>
constexpr T sqr(T x) noexcept {
    return x * x;
}
}  // namespace math

namespace dvm {
inline double* vec_ptr(Vector& v) { return v.memptr(); }
inline const double* vec_ptr(const Vector& v) { return v.memptr(); }
}  // namespace dvm

#endif

// Random numbers of the drop-in host library: the reference's Random class
// (src/Random.hpp, src/Random.cpp) -- std::mt19937 with
// std::uniform_real_distribution<double> on [0, 1), seeded from
// std::random_device unless seed(s) is called with s >= 0.  Using the same
// standard-library engine and distribution reproduces the reference's stream,
// which the device consumes in inject mode.
#ifndef DVMPP_B200_RANDOM_HPP
#define DVMPP_B200_RANDOM_HPP

#include <cstdint>
#include <random>
#include <vector>

class Random
{
  private:
    std::uniform_real_distribution<> m_dist;
    std::mt19937 m_re;

  public:
    Random();
    double rand();
    void seed(int seed);
    // The next n values of the stream without consuming them.
    void peek(std::size_t n, std::vector<double>& out) const;
    // Consume n values.
    void discard(std::size_t n);
};

#endif

#include "Random.hpp"

Random::Random() : m_dist(0.0, 1.0) {
    std::random_device rd;
    m_re.seed(rd());
}

double Random::rand() { return m_dist(m_re); }

void Random::seed(int s) {
    if (s >= 0) m_re.seed(static_cast<std::mt19937::result_type>(s));
}

void Random::peek(std::size_t n, std::vector<double>& out) const {
    std::mt19937 e = m_re;
    std::uniform_real_distribution<> d(0.0, 1.0);
    out.resize(n);
    for (std::size_t i = 0; i < n; ++i) out[i] = d(e);
}

void Random::discard(std::size_t n) {
    for (std::size_t i = 0; i < n; ++i) (void)m_dist(m_re);
}

#include "OutputWriter.hpp"

#include <algorithm>
#include <charconv>
#include <cstdio>
#include <vector>

#include "Exceptions.hpp"

namespace dvm {

void append_g(std::string& out, double v) {
    char buf[64];
    // std::to_chars with chars_format::general and a precision is specified
    // as printf's %g with that precision in the "C" locale -- what a default
    // std::ostream prints for a double (precision 6, no showpoint).
    const auto r = std::to_chars(buf, buf + sizeof(buf), v, std::chars_format::general, 6);
    out.append(buf, r.ptr);
}

void append_u(std::string& out, uint64_t v) {
    char buf[32];
    const auto r = std::to_chars(buf, buf + sizeof(buf), v);
    out.append(buf, r.ptr);
}

static void rows4(std::string& s, double t, const double* x, const double* z, const double* c,
                  size_t i0, size_t i1) {
    std::string ts;
    append_g(ts, t);
    s.reserve(s.size() + (i1 - i0) * (ts.size() + 40));
    for (size_t i = i0; i < i1; ++i) {
        s += ts;
        s += '\t';
        append_g(s, x[i]);
        s += '\t';
        append_g(s, z[i]);
        s += '\t';
        append_g(s, c[i]);
        s += '\n';
    }
}

std::string format_rows4(double t, const double* x, const double* z, const double* c, size_t n,
                         unsigned threads) {
    constexpr size_t kPerThread = 1u << 16;  // below this, one thread is faster
    const size_t parts = std::max<size_t>(1, std::min<size_t>(threads, n / kPerThread));
    std::vector<std::string> chunks(parts);
    std::vector<std::thread> pool;
    for (size_t p = 1; p < parts; ++p)
        pool.emplace_back([&, p] {
            rows4(chunks[p], t, x, z, c, n * p / parts, n * (p + 1) / parts);
        });
    rows4(chunks[0], t, x, z, c, 0, n / parts);
    for (auto& th : pool) th.join();
    if (parts == 1) return std::move(chunks[0]);
    size_t total = 0;
    for (auto& s : chunks) total += s.size();
    std::string out;
    out.reserve(total);
    for (auto& s : chunks) out += s;
    return out;
}

void append_file(const std::string& path, const std::string& data) {
    std::FILE* f = std::fopen(path.c_str(), "ab");
    if (!f) throw FileIOException::cannotWrite(path);
    const size_t w = data.empty() ? 0 : std::fwrite(data.data(), 1, data.size(), f);
    const int rc = std::fclose(f);
    if (w != data.size() || rc != 0) throw FileIOException::cannotWrite(path);
}

AsyncWriter::AsyncWriter(size_t max_pending)
    : m_max(std::max<size_t>(1, max_pending)), m_thread([this] { loop(); }) {}

AsyncWriter::~AsyncWriter() {
    {
        std::lock_guard<std::mutex> lk(m_mu);
        m_stop = true;
    }
    m_cv.notify_all();
    m_thread.join();  // runs what is queued first
}

void AsyncWriter::rethrow_locked(std::unique_lock<std::mutex>& lk) {
    if (!m_err) return;
    std::exception_ptr e = m_err;
    m_err = nullptr;
    lk.unlock();
    std::rethrow_exception(e);
}

void AsyncWriter::submit(std::function<void()> job) {
    std::unique_lock<std::mutex> lk(m_mu);
    m_cv.wait(lk, [&] { return m_q.size() < m_max || m_err; });
    rethrow_locked(lk);
    m_q.push_back(std::move(job));
    lk.unlock();
    m_cv.notify_all();
}

void AsyncWriter::flush() {
    std::unique_lock<std::mutex> lk(m_mu);
    m_cv.wait(lk, [&] { return (m_q.empty() && !m_busy) || m_err; });
    rethrow_locked(lk);
}

void AsyncWriter::loop() {
    std::unique_lock<std::mutex> lk(m_mu);
    for (;;) {
        m_cv.wait(lk, [&] { return !m_q.empty() || m_stop; });
        if (m_q.empty()) return;  // stopping, nothing left
        std::function<void()> job = std::move(m_q.front());
        m_q.pop_front();
        m_busy = true;
        lk.unlock();
        m_cv.notify_all();
        std::exception_ptr err;
        try {
            job();
        } catch (...) {
            err = std::current_exception();
        }
        lk.lock();
        if (err) {
            m_err = err;
            m_q.clear();  // later jobs would leave the files out of order
        }
        m_busy = false;
        m_cv.notify_all();
    }
}

}  // namespace dvm

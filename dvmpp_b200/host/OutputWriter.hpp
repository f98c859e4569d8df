// Output files in the reference's text formats, off the time loop.
//
// The reference writes every blob at every step through std::ostream
// (src/VortexBlobs.cpp:310-332, src/VortexSheet.cpp:335-343, src/Probe.cpp);
// once the step itself runs on the GPU, formatting millions of numbers a step
// on the calling thread is the bottleneck.  Here:
//   * append_g formats a double exactly as `std::ostream << double` does with
//     default flags (printf "%g", precision 6) but through std::to_chars,
//     several times faster and locale-free;
//   * AsyncWriter runs file jobs on one background thread in submission order
//     (so every file is byte-identical to the synchronous writer's), with a
//     bounded queue: a producer that runs ahead of the disk waits.
#ifndef DVMPP_B200_OUTPUTWRITER_HPP
#define DVMPP_B200_OUTPUTWRITER_HPP

#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <deque>
#include <exception>
#include <functional>
#include <mutex>
#include <string>
#include <thread>

namespace dvm {

// `out << v` for a default-formatted std::ostream, appended to `out`.
void append_g(std::string& out, double v);
void append_u(std::string& out, uint64_t v);

// Rows "t\tx\tz\tc\n" for i < n, formatted on up to `threads` threads (chunks
// concatenated in order).
std::string format_rows4(double t, const double* x, const double* z, const double* c, size_t n,
                         unsigned threads);

// Append `data` to the file at `path` (binary, no reformatting); throws
// dvm::FileIOException when the file cannot be written.
void append_file(const std::string& path, const std::string& data);

class AsyncWriter
{
  public:
    explicit AsyncWriter(size_t max_pending = 2);
    ~AsyncWriter();
    AsyncWriter(const AsyncWriter&) = delete;
    AsyncWriter& operator=(const AsyncWriter&) = delete;

    // Queue a job; blocks while max_pending jobs are already waiting.  If an
    // earlier job threw, its exception is rethrown here (and the job dropped).
    void submit(std::function<void()> job);
    // Wait until every queued job has run; rethrows a job's exception.
    void flush();

  private:
    void loop();
    void rethrow_locked(std::unique_lock<std::mutex>& lk);

    size_t m_max;
    std::mutex m_mu;
    std::condition_variable m_cv;
    std::deque<std::function<void()>> m_q;
    bool m_busy = false;
    bool m_stop = false;
    std::exception_ptr m_err;
    std::thread m_thread;
};

}  // namespace dvm

#endif

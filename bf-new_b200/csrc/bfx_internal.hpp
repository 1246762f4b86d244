// Internal plumbing shared by the host builders and the CUDA engine: error
// capture for the C ABI (every extern "C" entry point converts exceptions to
// a status code plus a thread-local message) and a small host thread pool.
#pragma once

#include "bfx.h"

#include <cstdint>
#include <exception>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace bfx {

// Exception carrying a bfx status code; std exceptions map by type the way
// the reference's exception types map to the codes in bfx.h.
class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
  [[nodiscard]] int code() const noexcept { return code_; }

 private:
  int code_;
};

void set_last_error(const std::string& message);

template <typename F>
int guarded(F&& f) noexcept {
  try {
    f();
    set_last_error("");
    return BFX_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code();
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return BFX_ERR_OUT_OF_MEMORY;
  } catch (const std::out_of_range& e) {
    set_last_error(e.what());
    return BFX_ERR_OUT_OF_RANGE;
  } catch (const std::overflow_error& e) {
    set_last_error(e.what());
    return BFX_ERR_OVERFLOW;
  } catch (const std::length_error& e) {
    set_last_error(e.what());
    return BFX_ERR_OVERFLOW;
  } catch (const std::invalid_argument& e) {
    set_last_error(e.what());
    return BFX_ERR_INVALID_ARGUMENT;
  } catch (const std::logic_error& e) {
    set_last_error(e.what());
    return BFX_ERR_STATE;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return BFX_ERR_STATE;
  } catch (...) {
    set_last_error("unknown exception");
    return BFX_ERR_STATE;
  }
}

inline void require(bool ok, const char* message) {
  if (!ok) throw std::invalid_argument(message);
}

// Splits [0, n) into contiguous chunks over `threads` host threads.
template <typename F>
void parallel_for(std::uint64_t n, unsigned threads, F&& body) {
  if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
  if (n < 4096 || threads <= 1) {
    body(std::uint64_t{0}, n);
    return;
  }
  const std::uint64_t chunk = (n + threads - 1) / threads;
  std::vector<std::thread> pool;
  std::vector<std::exception_ptr> errors(threads);
  for (unsigned t = 0; t < threads; ++t) {
    const std::uint64_t b = std::min<std::uint64_t>(n, t * chunk);
    const std::uint64_t e = std::min<std::uint64_t>(n, b + chunk);
    if (b >= e) break;
    pool.emplace_back([&, b, e, t] {
      try {
        body(b, e);
      } catch (...) {
        errors[t] = std::current_exception();
      }
    });
  }
  for (auto& th : pool) th.join();
  for (auto& err : errors) {
    if (err) std::rethrow_exception(err);
  }
}

}  // namespace bfx

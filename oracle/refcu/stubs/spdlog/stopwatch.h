// spdlog/stopwatch.h (stub) -- TEST INFRASTRUCTURE ONLY: the reference's
// compute_step times its kernels with spdlog::stopwatch for its debug log.
#pragma once
#include <chrono>
namespace spdlog {
struct stopwatch {
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    std::chrono::duration<double> elapsed() const { return std::chrono::steady_clock::now() - t0; }
};
}  // namespace spdlog

// spdlog/spdlog.h (stub) -- TEST INFRASTRUCTURE ONLY: the log calls that the
// reference's solver headers make are no-ops.
#pragma once
namespace spdlog {
template <class... A> void critical(A &&...) {}
template <class... A> void debug(A &&...) {}
template <class... A> void info(A &&...) {}
template <class... A> void warn(A &&...) {}
}  // namespace spdlog

// Stand-in for spdlog (Core/include/Core/timer.h includes it): logging is dropped.
#pragma once
namespace spdlog {
template <class... A> void info(A&&...) {}
template <class... A> void warn(A&&...) {}
template <class... A> void error(A&&...) {}
}  // namespace spdlog

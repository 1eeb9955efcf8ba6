// spdlog/spdlog.h stub for building the reference's frontend on the host: the logging calls of
// SceneManager.cpp print their format string to stderr (arguments are not formatted). Test
// infrastructure only.
#pragma once
#include <cstdio>
namespace spdlog {
template <class... A> void info(const char *fmt, A &&...) { std::fprintf(stderr, "[info] %s\n", fmt); }
template <class... A> void warn(const char *fmt, A &&...) { std::fprintf(stderr, "[warn] %s\n", fmt); }
template <class... A> void error(const char *fmt, A &&...) { std::fprintf(stderr, "[error] %s\n", fmt); }
}  // namespace spdlog

// Included before every translation unit of the reference's frontend built on the host
// (test infrastructure only). SceneManager.cpp throws std::exception("") for unsupported pbrt
// types, a constructor only MSVC's standard library has; the standard headers are included
// first, then the name is pointed at a type with that constructor for the reference's code.
#pragma once
#include <algorithm>
#include <array>
#include <cassert>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <limits>
#include <map>
#include <new>
#include <optional>
#include <source_location>
#include <tuple>
#include <typeinfo>
#include <unordered_map>
#include <utility>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <fstream>
#include <iostream>
#include <iterator>
#include <memory>
#include <span>
#include <sstream>
#include <stdexcept>
#include <string>
#include <string_view>
#include <vector>
namespace std {
struct wl_msvc_exception : exception {
    wl_msvc_exception() = default;
    explicit wl_msvc_exception(const char *) {}
};
}  // namespace std
#define exception wl_msvc_exception

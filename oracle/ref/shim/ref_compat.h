// Force-included ahead of the reference's own headers by oracle/ref/build_ref.py
// (TEST INFRASTRUCTURE ONLY). The reference compiles against the fmt library
// through spdlog; with spdlog's std::format backend (SPDLOG_USE_STD_FORMAT) it
// needs fmt::format spelled as std::format, a formatter for the cudaError_t
// values one of its assertions logs, and two standard headers it uses
// without including.
#pragma once
#include <cuda_runtime.h>

#include <format>
#include <map>
#include <set>

template <>
struct std::formatter<cudaError_t> : std::formatter<int> {
    auto format(cudaError_t e, std::format_context &ctx) const { return std::formatter<int>::format((int)e, ctx); }
};

namespace fmt {
using std::format;
}

// Minimal stand-in for the {fmt} header, written for building the reference
// engine as a test oracle only. The engine's join path never formats text; the
// contest headers merely declare `fmt::formatter` specialisations, so only the
// names they mention need to exist. Calling any of these at run time throws.
#pragma once
#include <stdexcept>
#include <string>
#include <utility>

namespace fmt {
template <typename T, typename Char = char, typename Enable = void>
struct formatter;

template <typename Out, typename... Args>
Out format_to(Out out, const char*, Args&&...) {
    throw std::runtime_error("fmt stub: formatting is not available in the oracle build");
    return out;
}

template <typename... Args>
std::string format(const char*, Args&&...) {
    throw std::runtime_error("fmt stub: formatting is not available in the oracle build");
}

template <typename... Args>
void print(const char*, Args&&...) {}
} // namespace fmt

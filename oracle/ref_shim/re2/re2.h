// Minimal stand-in for RE2, written for building the reference engine as a
// test oracle only. The contest's SQL LIKE filter (the only RE2 user) runs at
// table-load time, never inside the join path, so the oracle never calls it.
#pragma once
#include <stdexcept>
#include <string>
#include <string_view>

namespace re2 {
class RE2 {
    public:
    struct Options {
        void set_dot_nl(bool) {}
        void set_log_errors(bool) {}
        void set_case_sensitive(bool) {}
        void set_posix_syntax(bool) {}
        void set_longest_match(bool) {}
        void set_encoding(int) {}
    };
    enum Encoding { EncodingUTF8 = 1, EncodingLatin1 };
    RE2(const std::string&, const Options&) {}
    explicit RE2(const std::string&) {}
    bool ok() const { return true; }
    template <typename... A>
    static bool FullMatch(std::string_view, const RE2&, A&&...) {
        throw std::runtime_error("re2 stub: regex matching is not available in the oracle build");
    }
};
} // namespace re2
using re2::RE2;

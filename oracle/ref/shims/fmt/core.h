// Stand-in for the one fmt call the compiled reference sources make
// (fmt::format with "{}" placeholders in CompatibilityReport::log_issues).
// Test infrastructure for the oracle build only.
#pragma once

#include <sstream>
#include <string>

namespace fmt {

    inline void format_rest(std::ostringstream& out, const char* f) { out << f; }

    template <typename T, typename... Rest>
    void format_rest(std::ostringstream& out, const char* f, const T& v, const Rest&... rest) {
        while (*f) {
            if (f[0] == '{' && f[1] == '}') {
                out << v;
                format_rest(out, f + 2, rest...);
                return;
            }
            out << *f++;
        }
    }

    template <typename... Args>
    std::string format(const char* f, const Args&... args) {
        std::ostringstream out;
        format_rest(out, f, args...);
        return out.str();
    }

} // namespace fmt

// Replacement for libFluid's helpers/Log.cpp in the oracle build (the
// original needs fmt's chrono/color headers, which are absent here). Log is
// not on the simulation path; messages go to stderr. Test infrastructure only.
#include "helpers/Log.hpp"

#include <iostream>

namespace LibFluid {
    bool Log::print_to_console = false;
    std::vector<Log::Entry> Log::entries;
    std::mutex Log::mutex;

    std::string Log::type_to_string(Type type) {
        return type == TYPE_ERROR ? "ERROR" : (type == TYPE_WARNING ? "WARNING" : "MESSAGE");
    }
    std::string Log::Entry::human_readable() const { return "[" + type_to_string(type) + "] " + message; }
    void Log::log(Type type, const std::string& message) {
        std::lock_guard<std::mutex> lock(mutex);
        entries.push_back({message, std::chrono::system_clock::now(), type});
        if (print_to_console) std::cerr << entries.back().human_readable() << std::endl;
    }
    void Log::message(const std::string& m) { log(TYPE_MESSAGE, m); }
    void Log::warning(const std::string& m) { log(TYPE_WARNING, m); }
    void Log::error(const std::string& m) { log(TYPE_ERROR, m); }
    std::vector<Log::Entry> Log::get_entries() {
        std::lock_guard<std::mutex> lock(mutex);
        return entries;
    }
    void Log::print_entry_to_console(const Entry& entry) { std::cerr << entry.human_readable() << std::endl; }
} // namespace LibFluid

// Stand-in for the one fmt chrono call the reference's sensor base makes
// (SensorBase.hpp: fmt::gmtime of the time point for a JSON timestamp).
// Test infrastructure for the oracle build only: the oracle computes sensor
// values and never writes sensor files, so the time stamp is a plain count
// of seconds.
#pragma once

#include <chrono>
#include <ostream>

#include "core.h"

namespace fmt {

    struct gm_time {
        long long seconds;
    };

    inline gm_time gmtime(std::chrono::time_point<std::chrono::system_clock> t) {
        return {(long long)std::chrono::duration_cast<std::chrono::seconds>(t.time_since_epoch()).count()};
    }

    inline std::ostream& operator<<(std::ostream& o, const gm_time& g) { return o << g.seconds; }

} // namespace fmt

// "Reference, threaded" variant of libFluid's StdParallelForEach
// (parallelization/StdParallelForEach.cpp:64-128): the same 16-particle chunks,
// distributed over all host cores with an OpenMP dynamic schedule instead of
// std::execution::par (which GCC runs serially when TBB is absent). Everything
// else in the oracle build is the reference's own code. Used only to time the
// reference CPU path on all cores; results of the IISPH L1 loop may differ run
// to run here exactly as they would under the reference's own parallel backend
// (it reads neighbor densities while writing them).
#include "parallelization/StdParallelForEach.hpp"

#include <algorithm>
#include <limits>

namespace LibFluid {

    void StdParallelForEach::loop_for(size_t from, size_t to, const std::function<void(size_t i)>& fn) {
        if (to <= from) return;
        const long long chunks = (long long)((to - from + chunk_size - 1) / chunk_size);
#pragma omp parallel for schedule(dynamic, 4)
        for (long long c = 0; c < chunks; c++) {
            size_t base = from + (size_t)c * chunk_size;
            size_t end = std::min(base + chunk_size, to);
            for (size_t i = base; i < end; i++) fn(i);
        }
    }

    void StdParallelForEach::loop_for(size_t from, size_t to, size_t step, const std::function<void(size_t i)>& fn) {
        if (to <= from) return;
        const long long steps = (long long)(((to - 1) - from) / step + 1);
#pragma omp parallel for schedule(dynamic, 64)
        for (long long i = 0; i < steps; i++) fn(from + (size_t)i * step);
    }

    float StdParallelForEach::loop_for_max(size_t from, size_t to, const std::function<float(size_t)>& fn) {
        float result = std::numeric_limits<float>::lowest();
        if (to <= from) return result;
        const long long chunks = (long long)((to - from + chunk_size - 1) / chunk_size);
#pragma omp parallel for schedule(dynamic, 4) reduction(max : result)
        for (long long c = 0; c < chunks; c++) {
            size_t base = from + (size_t)c * chunk_size;
            size_t end = std::min(base + chunk_size, to);
            for (size_t i = base; i < end; i++) result = std::max(result, fn(i));
        }
        return result;
    }

} // namespace LibFluid

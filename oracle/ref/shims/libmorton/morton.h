// Stand-in for libmorton's 3D 64-bit Morton encoder (test infrastructure for
// the oracle build). Interleaves the low 21 bits of x, y and z with x in bit 0,
// y in bit 1 and z in bit 2 of every triple, which is the layout the published
// libmorton encoder produces. The neighbor SETS of the reference searches do not
// depend on the layout; only the order in which the reference re-sorts its
// particle collection does, and the parity tests compare in tag space.
#pragma once

#include <cstdint>

namespace libmorton {

    inline uint64_t morton_split_by_3(uint32_t a) {
        uint64_t x = a & 0x1fffffu;
        x = (x | (x << 32)) & 0x1f00000000ffffull;
        x = (x | (x << 16)) & 0x1f0000ff0000ffull;
        x = (x | (x << 8)) & 0x100f00f00f00f00full;
        x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
        x = (x | (x << 2)) & 0x1249249249249249ull;
        return x;
    }

    inline uint64_t morton3D_64_encode(uint32_t x, uint32_t y, uint32_t z) {
        return morton_split_by_3(x) | (morton_split_by_3(y) << 1) | (morton_split_by_3(z) << 2);
    }

} // namespace libmorton

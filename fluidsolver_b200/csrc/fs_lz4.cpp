// LZ4 frame and block coding and XXH32 (see fs_lz4.hpp for the formats).
#include "fs_lz4.hpp"

#include <cstring>

namespace fsio {

namespace {

constexpr uint32_t kFrameMagic = 0x184D2204u;
constexpr uint32_t kSkippableMagic = 0x184D2A50u;   // .. 0x184D2A5F
constexpr size_t kBlockMax = 64 * 1024;             // the encoder's block size (BD code 4)
constexpr size_t kMinMatch = 4;
constexpr size_t kLastLiterals = 5;                 // a block ends with at least 5 literals
constexpr size_t kMatchFindLimit = 12;              // no match starts in the last 12 bytes
constexpr int kHashLog = 14;

uint32_t rd32(const uint8_t* p) { return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24; }
void wr32(std::vector<uint8_t>& v, uint32_t x) {
    for (int i = 0; i < 4; i++) v.push_back((uint8_t)(x >> (8 * i)));
}
uint32_t rotl(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

// length extension bytes: 255 while at least 255 remain, then the rest
uint8_t* put_length(uint8_t* op, size_t n) {
    while (n >= 255) {
        *op++ = 255;
        n -= 255;
    }
    *op++ = (uint8_t)n;
    return op;
}

}  // namespace

uint32_t xxh32(const uint8_t* p, size_t len, uint32_t seed) {
    const uint32_t P1 = 2654435761u, P2 = 2246822519u, P3 = 3266489917u, P4 = 668265263u, P5 = 374761393u;
    const uint8_t* const end = p + len;
    uint32_t h;
    if (len >= 16) {
        uint32_t v1 = seed + P1 + P2, v2 = seed + P2, v3 = seed, v4 = seed - P1;
        const uint8_t* const limit = end - 16;
        do {
            v1 = rotl(v1 + rd32(p) * P2, 13) * P1;
            v2 = rotl(v2 + rd32(p + 4) * P2, 13) * P1;
            v3 = rotl(v3 + rd32(p + 8) * P2, 13) * P1;
            v4 = rotl(v4 + rd32(p + 12) * P2, 13) * P1;
            p += 16;
        } while (p <= limit);
        h = rotl(v1, 1) + rotl(v2, 7) + rotl(v3, 12) + rotl(v4, 18);
    } else {
        h = seed + P5;
    }
    h += (uint32_t)len;
    for (; p + 4 <= end; p += 4) h = rotl(h + rd32(p) * P3, 17) * P4;
    for (; p < end; p++) h = rotl(h + (*p) * P5, 11) * P1;
    h ^= h >> 15;
    h *= P2;
    h ^= h >> 13;
    h *= P3;
    h ^= h >> 16;
    return h;
}

size_t lz4_block_bound(size_t len) { return len + len / 255 + 16; }

size_t lz4_block_compress(const uint8_t* src, size_t len, uint8_t* dst) {
    uint8_t* op = dst;
    size_t anchor = 0;
    if (len > kMatchFindLimit) {
        std::vector<uint32_t> table((size_t)1 << kHashLog, 0xffffffffu);   // last position of each hash
        const size_t find_limit = len - kMatchFindLimit;   // matches start before this
        const size_t match_limit = len - kLastLiterals;    // and end at or before this
        size_t ip = 0;
        while (ip < find_limit) {
            const uint32_t seq = rd32(src + ip);
            const uint32_t h = (seq * 2654435761u) >> (32 - kHashLog);
            const uint32_t ref = table[h];
            table[h] = (uint32_t)ip;
            if (ref == 0xffffffffu || ip - ref > 65535 || rd32(src + ref) != seq) {
                ip++;
                continue;
            }
            size_t m = ip, r = ref;
            // extend backwards over pending literals, then forwards
            while (m > anchor && r > 0 && src[m - 1] == src[r - 1]) {
                m--;
                r--;
            }
            size_t ml = (ip - m) + kMinMatch;
            while (m + ml < match_limit && src[r + ml] == src[m + ml]) ml++;
            // sequence: token, literal length, literals, offset, match length
            const size_t lit = m - anchor;
            uint8_t* token = op++;
            *token = (uint8_t)((lit >= 15 ? 15 : lit) << 4);
            if (lit >= 15) op = put_length(op, lit - 15);
            std::memcpy(op, src + anchor, lit);
            op += lit;
            const size_t off = m - r;
            *op++ = (uint8_t)(off & 0xff);
            *op++ = (uint8_t)(off >> 8);
            const size_t mc = ml - kMinMatch;
            *token |= (uint8_t)(mc >= 15 ? 15 : mc);
            if (mc >= 15) op = put_length(op, mc - 15);
            ip = m + ml;
            anchor = ip;
            if (ip >= 2 && ip - 2 < find_limit)   // keep the table fresh inside long matches
                table[(rd32(src + ip - 2) * 2654435761u) >> (32 - kHashLog)] = (uint32_t)(ip - 2);
        }
    }
    // the last literals
    const size_t lit = len - anchor;
    *op++ = (uint8_t)((lit >= 15 ? 15 : lit) << 4);
    if (lit >= 15) op = put_length(op, lit - 15);
    std::memcpy(op, src + anchor, lit);
    op += lit;
    return (size_t)(op - dst);
}

long long lz4_block_decompress(const uint8_t* src, size_t len, uint8_t* dst, size_t cap, const uint8_t* history_begin) {
    const uint8_t* ip = src;
    const uint8_t* const iend = src + len;
    uint8_t* op = dst;
    uint8_t* const oend = dst + cap;
    auto get_length = [&](size_t base, size_t& n) -> bool {
        n = base;
        if (base != 15) return true;
        for (;;) {
            if (ip >= iend) return false;
            const uint8_t b = *ip++;
            n += b;
            if (b != 255) return true;
        }
    };
    while (ip < iend) {
        const uint8_t token = *ip++;
        size_t lit;
        if (!get_length(token >> 4, lit)) return -1;
        if ((size_t)(iend - ip) < lit || (size_t)(oend - op) < lit) return -1;
        std::memcpy(op, ip, lit);
        ip += lit;
        op += lit;
        if (ip == iend) break;   // the last sequence has no match
        if (iend - ip < 2) return -1;
        const size_t off = (size_t)ip[0] | (size_t)ip[1] << 8;
        ip += 2;
        size_t ml;
        if (!get_length(token & 15, ml)) return -1;
        ml += kMinMatch;
        if (off == 0 || (size_t)(op - history_begin) < off || (size_t)(oend - op) < ml) return -1;
        const uint8_t* match = op - off;
        if (off >= ml) {
            std::memcpy(op, match, ml);
            op += ml;
        } else {
            for (size_t i = 0; i < ml; i++) *op++ = *match++;   // overlapping: repeats the last off bytes
        }
    }
    return (long long)(op - dst);
}

std::string lz4_frame_decode(const uint8_t* in, size_t len, std::vector<uint8_t>& out) {
    size_t pos = 0;
    while (pos < len) {
        if (len - pos < 4) return "truncated frame header";
        const uint32_t magic = rd32(in + pos);
        if ((magic & 0xfffffff0u) == kSkippableMagic) {
            if (len - pos < 8) return "truncated skippable frame";
            const size_t n = rd32(in + pos + 4);
            if (len - pos - 8 < n) return "truncated skippable frame";
            pos += 8 + n;
            continue;
        }
        if (magic != kFrameMagic) return "not an LZ4 frame";
        if (len - pos < 7) return "truncated frame header";
        const uint8_t flg = in[pos + 4], bd = in[pos + 5];
        if ((flg >> 6) != 1) return "unsupported LZ4 frame version";
        if ((flg & 0x02) || (bd & 0x8f)) return "reserved bits set in the frame descriptor";
        const bool indep = flg & 0x20, block_sum = flg & 0x10, has_size = flg & 0x08, content_sum = flg & 0x04,
                   has_dict = flg & 0x01;
        const int code = (bd >> 4) & 7;
        if (code < 4) return "invalid block maximum size";
        const size_t block_max = (size_t)1 << (8 + 2 * code);
        const size_t desc = 2 + (has_size ? 8 : 0) + (has_dict ? 4 : 0);
        if (len - pos < 4 + desc + 1) return "truncated frame header";
        if (((xxh32(in + pos + 4, desc, 0) >> 8) & 0xff) != in[pos + 4 + desc]) return "frame header checksum mismatch";
        uint64_t content_size = 0;
        if (has_size)
            for (int i = 0; i < 8; i++) content_size |= (uint64_t)in[pos + 6 + i] << (8 * i);
        if (has_dict) return "frames with a dictionary are not supported";
        pos += 4 + desc + 1;
        const size_t frame_start = out.size();
        for (;;) {
            if (len - pos < 4) return "truncated block";
            const uint32_t word = rd32(in + pos);
            pos += 4;
            if (word == 0) break;   // end mark
            const bool raw = word & 0x80000000u;
            const size_t n = word & 0x7fffffffu;
            if (n > block_max) return "block larger than the frame's maximum";
            if (len - pos < n + (block_sum ? 4 : 0)) return "truncated block";
            if (block_sum && xxh32(in + pos, n, 0) != rd32(in + pos + n)) return "block checksum mismatch";
            const size_t old = out.size();
            if (raw) {
                out.insert(out.end(), in + pos, in + pos + n);
            } else {
                out.resize(old + block_max);
                const long long got = lz4_block_decompress(in + pos, n, out.data() + old, block_max,
                                                           indep ? out.data() + old : out.data() + frame_start);
                if (got < 0) return "corrupt LZ4 block";
                out.resize(old + (size_t)got);
            }
            pos += n + (block_sum ? 4 : 0);
        }
        if (content_sum) {
            if (len - pos < 4) return "truncated content checksum";
            if (xxh32(out.data() + frame_start, out.size() - frame_start, 0) != rd32(in + pos))
                return "content checksum mismatch";
            pos += 4;
        }
        if (has_size && content_size != out.size() - frame_start) return "content size mismatch";
    }
    return std::string();
}

std::vector<uint8_t> lz4_frame_encode(const uint8_t* data, size_t len) {
    std::vector<uint8_t> out;
    out.reserve(lz4_block_bound(len) + 64);
    wr32(out, kFrameMagic);
    const uint8_t desc[2] = {0x60, 0x40};   // version 01, independent blocks; 64 KB blocks
    out.push_back(desc[0]);
    out.push_back(desc[1]);
    out.push_back((uint8_t)((xxh32(desc, 2, 0) >> 8) & 0xff));
    std::vector<uint8_t> tmp(lz4_block_bound(kBlockMax));
    for (size_t at = 0; at < len; at += kBlockMax) {
        const size_t n = len - at < kBlockMax ? len - at : kBlockMax;
        const size_t c = lz4_block_compress(data + at, n, tmp.data());
        if (c < n) {
            wr32(out, (uint32_t)c);
            out.insert(out.end(), tmp.begin(), tmp.begin() + (long)c);
        } else {   // incompressible: stored
            wr32(out, (uint32_t)n | 0x80000000u);
            out.insert(out.end(), data + at, data + at + n);
        }
    }
    wr32(out, 0);   // end mark
    return out;
}

}  // namespace fsio

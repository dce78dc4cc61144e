// container.cu - a self-describing container for volume bit streams (host
// code).  The reference's example writes a stream as raw concatenated u32
// words with nothing else (examples.cpp:527-536), so the reader must know the
// codec, levels, sizes and steps out of band; this container stores them.
//
// Layout (little-endian; all offsets in bytes from the start):
//   header (48 bytes)
//     0  u32  magic 0x32424343 ("CCB2")
//     4  u32  version (1)
//     8  u32  codec: 0 float (compressVolumeFloat), 1 quant-first
//             (compressVolumeFloatQuantFirst), 2 heightfield
//    12  u32  flags (CC_VOLUME_RLE_ONLY_LEVEL0)
//    16  u32  levels
//    20  u32  coding block size
//    24  u32  log2 of the Huffman symbol count bound
//    28  u32  entry count n
//    32  u64  total bytes of the container
//    40  u64  reserved (0)
//   n entries (32 bytes each)
//     0  u32  size x, y, z (12 bytes)
//    12  f32  quantization step (level 0 step, or the quant-first step)
//    16  u64  bit size of the stream
//    24  u64  byte offset of the stream's first word
//   the streams' words, each starting 8-byte aligned.
#include <cstring>

#include "capi_internal.cuh"

namespace {

constexpr uint32_t kMagic = 0x32424343u;
constexpr uint32_t kVersion = 1u;
constexpr uint64_t kHeaderBytes = 48, kEntryBytes = 32;

uint64_t wordsOf(uint64_t bits) { return (bits + 31) / 32; }
uint64_t align8(uint64_t v) { return (v + 7) & ~uint64_t(7); }

template <class T>
void put(unsigned char* p, T v) { std::memcpy(p, &v, sizeof(T)); }
template <class T>
T get(const unsigned char* p) {
    T v;
    std::memcpy(&v, p, sizeof(T));
    return v;
}

}  // namespace

using namespace ccb;

extern "C" {

uint64_t cc_container_bytes(uint32_t count, const uint64_t* bit_sizes) {
    uint64_t at = kHeaderBytes + uint64_t(count) * kEntryBytes;
    for (uint32_t i = 0; i < count; ++i) at = align8(at) + wordsOf(bit_sizes ? bit_sizes[i] : 0) * 4;
    return align8(at);
}

int cc_container_write(void* dst, uint64_t capacity, const cc_container_info* info, const cc_container_entry* entries,
                       uint32_t count, uint64_t* written) {
    if (!dst || !info || (count && !entries)) { setError("cc_container_write: null argument"); return CC_ERR_INVALID_ARGUMENT; }
    if (info->codec > 2) { setError("cc_container_write: unknown codec %u", info->codec); return CC_ERR_INVALID_ARGUMENT; }
    std::vector<uint64_t> bits(count);
    for (uint32_t i = 0; i < count; ++i) {
        if (entries[i].bit_size && !entries[i].words) { setError("cc_container_write: entry %u has no words", i); return CC_ERR_INVALID_ARGUMENT; }
        bits[i] = entries[i].bit_size;
    }
    const uint64_t total = cc_container_bytes(count, bits.data());
    if (total > capacity) { setError("cc_container_write: needs %llu bytes", (unsigned long long)total); return CC_ERR_CAPACITY; }
    unsigned char* p = static_cast<unsigned char*>(dst);
    std::memset(p, 0, total);
    put<uint32_t>(p + 0, kMagic);
    put<uint32_t>(p + 4, kVersion);
    put<uint32_t>(p + 8, info->codec);
    put<uint32_t>(p + 12, info->flags);
    put<uint32_t>(p + 16, info->levels);
    put<uint32_t>(p + 20, info->coding_block_size);
    put<uint32_t>(p + 24, info->log2_symbol_count);
    put<uint32_t>(p + 28, count);
    put<uint64_t>(p + 32, total);
    uint64_t at = kHeaderBytes + uint64_t(count) * kEntryBytes;
    for (uint32_t i = 0; i < count; ++i) {
        unsigned char* e = p + kHeaderBytes + uint64_t(i) * kEntryBytes;
        at = align8(at);
        put<uint32_t>(e + 0, entries[i].size_x);
        put<uint32_t>(e + 4, entries[i].size_y);
        put<uint32_t>(e + 8, entries[i].size_z);
        put<float>(e + 12, entries[i].quant_step);
        put<uint64_t>(e + 16, entries[i].bit_size);
        put<uint64_t>(e + 24, at);
        const uint64_t nb = wordsOf(entries[i].bit_size) * 4;
        if (nb) std::memcpy(p + at, entries[i].words, nb);
        at += nb;
    }
    if (written) *written = total;
    return CC_OK;
}

int cc_container_read(const void* src, uint64_t bytes, cc_container_info* info, cc_container_entry* entries,
                      uint32_t capacity, uint32_t* count) {
    if (!src || !info || !count) { setError("cc_container_read: null argument"); return CC_ERR_INVALID_ARGUMENT; }
    const unsigned char* p = static_cast<const unsigned char*>(src);
    if (bytes < kHeaderBytes || get<uint32_t>(p) != kMagic) { setError("cc_container_read: not a container"); return CC_ERR_CORRUPT_STREAM; }
    if (get<uint32_t>(p + 4) != kVersion) { setError("cc_container_read: version %u", get<uint32_t>(p + 4)); return CC_ERR_CORRUPT_STREAM; }
    const uint32_t n = get<uint32_t>(p + 28);
    const uint64_t total = get<uint64_t>(p + 32);
    if (total > bytes || kHeaderBytes + uint64_t(n) * kEntryBytes > total) {
        setError("cc_container_read: truncated (%llu of %llu bytes)", (unsigned long long)bytes, (unsigned long long)total);
        return CC_ERR_CORRUPT_STREAM;
    }
    info->codec = get<uint32_t>(p + 8);
    info->flags = get<uint32_t>(p + 12);
    info->levels = get<uint32_t>(p + 16);
    info->coding_block_size = get<uint32_t>(p + 20);
    info->log2_symbol_count = get<uint32_t>(p + 24);
    *count = n;
    if (!entries) return CC_OK;   // count query
    if (capacity < n) { setError("cc_container_read: %u entries, room for %u", n, capacity); return CC_ERR_CAPACITY; }
    for (uint32_t i = 0; i < n; ++i) {
        const unsigned char* e = p + kHeaderBytes + uint64_t(i) * kEntryBytes;
        cc_container_entry& o = entries[i];
        o.size_x = get<uint32_t>(e + 0);
        o.size_y = get<uint32_t>(e + 4);
        o.size_z = get<uint32_t>(e + 8);
        o.quant_step = get<float>(e + 12);
        o.bit_size = get<uint64_t>(e + 16);
        const uint64_t off = get<uint64_t>(e + 24);
        if (off % 4 || off > total || wordsOf(o.bit_size) * 4 > total - off) {
            setError("cc_container_read: entry %u out of bounds", i);
            return CC_ERR_CORRUPT_STREAM;
        }
        o.words = reinterpret_cast<const uint32_t*>(p + off);
    }
    return CC_OK;
}

}  // extern "C"

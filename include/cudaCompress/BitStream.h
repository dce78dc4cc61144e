// BitStream.h - host bit stream over 32-bit words (drop-in for the
// reference's include/cudaCompress/BitStream.h; same class names, members
// and semantics, implemented independently).
//
// Format rules the coder relies on:
// - bits are written MSB first inside each 32-bit word (bit position p lives
//   in word p/32 at bit 31 - p%32);
// - *Aligned transfers align the position to 4 bytes, then to sizeof(T),
//   copy raw little-endian bytes, and align to 4 bytes again;
// - writeAlign moves the position (and grows the stream) without touching
//   the skipped bits.
#ifndef CUDACOMPRESS_B200_BIT_STREAM_H
#define CUDACOMPRESS_B200_BIT_STREAM_H

#include <algorithm>
#include <cassert>
#include <cstring>
#include <vector>

#include <cudaCompress/global.h>

namespace cudaCompress {

struct BitStreamAccess;

class BitStreamReadOnly {
public:
    BitStreamReadOnly(const uint* pBuffer, uint bitSize) : m_pBuffer(pBuffer), m_bitSize(bitSize), m_bufferPos(0), m_bitPos(0) {}
    BitStreamReadOnly(BitStreamReadOnly&& other)
        : m_pBuffer(other.m_pBuffer), m_bitSize(other.m_bitSize), m_bufferPos(other.m_bufferPos), m_bitPos(other.m_bitPos) {
        other.m_pBuffer = nullptr;
        other.m_bitSize = other.m_bufferPos = other.m_bitPos = 0;
    }
    virtual ~BitStreamReadOnly() {}

    uint getBitPosition() const { return m_bufferPos * 32 + m_bitPos; }
    // false (and position at the end) if bitPos is beyond the stream
    bool setBitPosition(uint bitPos) {
        bool ok = bitPos <= m_bitSize;
        if (!ok) bitPos = m_bitSize;
        m_bufferPos = bitPos / 32;
        m_bitPos = bitPos % 32;
        return ok;
    }
    uint getBitSize() const { return m_bitSize; }

    // next bit into the lsb of data; returns bits read (0 at the end)
    uint readBit(uint& data) {
        if (getBitPosition() == m_bitSize) return 0;
        data = (data & ~1u) | ((m_pBuffer[m_bufferPos] >> (31 - m_bitPos)) & 1u);
        advance(1);
        return 1;
    }
    // next bitCount (<= 32) bits into the low bits of data, the other bits of
    // data unchanged; returns the bits actually read (fewer at the end)
    uint readBits(uint& data, uint bitCount) {
        assert(bitCount <= 32);
        const uint n = std::min(bitCount, m_bitSize - getBitPosition());
        if (n == 0) return 0;
        const uint w = m_bufferPos;
        const unsigned long long hi = m_pBuffer[w];
        const unsigned long long lo = (m_bitPos + n > 32) ? m_pBuffer[w + 1] : 0ull;
        const unsigned long long window = (hi << 32) | lo;
        const uint value = uint((window << m_bitPos) >> (64 - n));
        const uint mask = n == 32 ? ~0u : ((1u << n) - 1u);
        data = (data & ~mask) | value;
        advance(n);
        return n;
    }
    uint skipBits(uint bitCount) {
        const uint n = std::min(bitCount, m_bitSize - getBitPosition());
        advance(n);
        return n;
    }

    template <typename T>
    uint readAligned(T* pTarget, uint count) {
        align<uint>();
        align<T>();
        const uint avail = (m_bitSize - getBitPosition()) / 8 / uint(sizeof(T));
        const uint n = std::min(avail, count);
        std::memcpy(pTarget, reinterpret_cast<const byte*>(m_pBuffer + m_bufferPos) + m_bitPos / 8, size_t(n) * sizeof(T));
        advance(n * uint(sizeof(T)) * 8);
        align<uint>();
        return n;
    }
    template <typename T>
    uint skipAligned(uint count) {
        align<uint>();
        align<T>();
        const uint avail = (m_bitSize - getBitPosition()) / 8 / uint(sizeof(T));
        const uint n = std::min(avail, count);
        advance(n * uint(sizeof(T)) * 8);
        align<uint>();
        return n;
    }
    template <typename T>
    const T* getAlignedPointer() {
        align<uint>();
        align<T>();
        const T* p = reinterpret_cast<const T*>(getRaw()) + getBitPosition() / (8 * sizeof(T));
        align<uint>();
        return p;
    }

    template <typename T>
    bool align() { return align(uint(sizeof(T))); }
    // align to byteCount bytes; false (position unchanged if already at the
    // end) when that would leave the stream
    bool align(uint byteCount) {
        const uint unit = byteCount * 8;
        uint off = m_bitPos % unit;
        const uint room = m_bitSize - getBitPosition();
        bool ok = true;
        if (off > room) { off = room; ok = false; }
        if (off != 0) advance(unit - off);
        return ok;
    }

    const uint* getRaw() const { return m_pBuffer; }
    uint getRawSizeUInts() const { return (m_bitSize + 31) / 32; }
    uint getRawSizeBytes() const { return (m_bitSize + 7) / 8; }

protected:
    friend struct BitStreamAccess;
    void advance(uint bits) {
        const uint p = m_bitPos + bits;
        m_bufferPos += p / 32;
        m_bitPos = p % 32;
    }

    const uint* m_pBuffer;
    uint m_bitSize;
    uint m_bufferPos;
    uint m_bitPos;

private:
    BitStreamReadOnly(const BitStreamReadOnly&);
    BitStreamReadOnly& operator=(const BitStreamReadOnly&);
};

class BitStream : public BitStreamReadOnly {
public:
    // with pVector == nullptr the stream owns its storage
    BitStream(std::vector<uint>* pVector = nullptr) : BitStreamReadOnly(nullptr, 0) {
        m_ownBuffer = pVector == nullptr;
        m_pVector = m_ownBuffer ? new std::vector<uint> : pVector;
        m_bitSize = uint(m_pVector->size()) * 32;
        m_pBuffer = m_pVector->data();
    }
    BitStream(BitStream&& other) : BitStreamReadOnly(std::move(other)), m_pVector(other.m_pVector), m_ownBuffer(other.m_ownBuffer) {
        other.m_pVector = nullptr;
        other.m_ownBuffer = false;
    }
    virtual ~BitStream() {
        if (m_ownBuffer) delete m_pVector;
    }

    void setBitSize(uint bitSize) {
        m_bitSize = bitSize;
        resizeVector((bitSize + 31) / 32);
        setBitPosition(std::min(getBitPosition(), m_bitSize));
    }
    void reserveBitSize(uint bitSize) { m_pVector->reserve((bitSize + 31) / 32); }

    // bitCount (<= 32) low bits of data, most significant first
    void writeBits(uint data, uint bitCount) {
        assert(bitCount <= 32);
        grow(getBitPosition() + bitCount);
        while (bitCount > 0) {
            const uint n = std::min(bitCount, 32 - m_bitPos);
            const uint mask = n == 32 ? ~0u : ((1u << n) - 1u);
            const uint value = (data >> (bitCount - n)) & mask;
            const uint shift = 32 - n - m_bitPos;
            uint& word = (*m_pVector)[m_bufferPos];
            word = (word & ~(mask << shift)) | (value << shift);
            advance(n);
            bitCount -= n;
        }
    }

    template <typename T>
    void writeAligned(const T* pSource, uint count) {
        writeAlign<uint>();
        writeAlign<T>();
        if (count == 0) return;
        const uint start = getBitPosition();
        grow(start + count * uint(sizeof(T)) * 8);
        std::memcpy(reinterpret_cast<byte*>(m_pVector->data()) + start / 8, pSource, size_t(count) * sizeof(T));
        advance(count * uint(sizeof(T)) * 8);
        writeAlign<uint>();
    }

    template <typename T>
    void writeAlign() { writeAlign(uint(sizeof(T))); }
    // align to byteCount bytes, growing the stream if needed (new bits zero)
    void writeAlign(uint byteCount) {
        const uint unit = byteCount * 8;
        const uint off = m_bitPos % unit;
        if (off != 0) advance(unit - off);
        grow(getBitPosition());
    }

    uint* getRaw() { return m_pVector->data(); }

private:
    friend struct BitStreamAccess;
    void grow(uint bitEnd) {
        if (bitEnd > m_bitSize) {
            m_bitSize = bitEnd;
            const uint words = (bitEnd + 31) / 32;
            if (words > m_pVector->size()) resizeVector(words);
        }
    }
    void resizeVector(uint words) {
        m_pVector->resize(words, 0u);
        m_pBuffer = m_pVector->data();
    }

    std::vector<uint>* m_pVector;
    bool m_ownBuffer;

    BitStream(const BitStream&);
    BitStream& operator=(const BitStream&);
};

}

#endif

// hgx/wxf.hpp -- a streaming writer of the Wolfram Exchange Format (WXF), header only.
//
// Emits the binary form the reference's worker replies in (paclet_source/hg_gpu_backend.cpp,
// through wxf/wxf.cpp): the "8:" header, then expressions -- integers in the narrowest of the
// 8/16/32/64-bit little-endian forms ('C', 'j', 'i', 'L'), strings ('S', varint length + UTF-8),
// lists as List[...] ('f', varint argument count, then the head as a symbol 's'), associations
// ('A', varint rule count, then '-' key value per rule). Booleans are written as the integers
// 1 / 0, as the reference's writer stores them. Counts precede contents in this format, so every
// list and association is opened with its final length.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace hgx {
namespace wxf {

class Writer {
public:
    Writer() { buf_ = {'8', ':'}; }

    void integer(int64_t v) {
        if (v >= INT8_MIN && v <= INT8_MAX) {
            buf_.push_back('C');
            put_le(static_cast<uint64_t>(v), 1);
        } else if (v >= INT16_MIN && v <= INT16_MAX) {
            buf_.push_back('j');
            put_le(static_cast<uint64_t>(v), 2);
        } else if (v >= INT32_MIN && v <= INT32_MAX) {
            buf_.push_back('i');
            put_le(static_cast<uint64_t>(v), 4);
        } else {
            buf_.push_back('L');
            put_le(static_cast<uint64_t>(v), 8);
        }
    }
    void boolean(bool b) { integer(b ? 1 : 0); }
    void string(const std::string& s) { text('S', s); }
    void symbol(const std::string& s) { text('s', s); }
    // List[...] of n elements; the n elements follow.
    void list(size_t n) {
        buf_.push_back('f');
        varint(n);
        symbol("List");
    }
    // <| ... |> of n rules; each rule is key() (or rule() + a key expression) then a value.
    void association(size_t n) {
        buf_.push_back('A');
        varint(n);
    }
    void rule() { buf_.push_back('-'); }
    void key(const std::string& k) {
        rule();
        string(k);
    }
    void int_key(int64_t k) {
        rule();
        integer(k);
    }

    size_t size() const { return buf_.size(); }
    const std::vector<uint8_t>& data() const { return buf_; }
    std::vector<uint8_t> take() { return std::move(buf_); }

private:
    void varint(uint64_t v) {
        while (v >= 0x80) {
            buf_.push_back(static_cast<uint8_t>((v & 0x7F) | 0x80));
            v >>= 7;
        }
        buf_.push_back(static_cast<uint8_t>(v));
    }
    void put_le(uint64_t v, int bytes) {
        for (int i = 0; i < bytes; ++i) buf_.push_back(static_cast<uint8_t>(v >> (8 * i)));
    }
    void text(uint8_t tok, const std::string& s) {
        buf_.push_back(tok);
        varint(s.size());
        buf_.insert(buf_.end(), s.begin(), s.end());
    }

    std::vector<uint8_t> buf_;
};

}  // namespace wxf
}  // namespace hgx

// Sequential unformatted Fortran records as gfortran writes them (the format of the reference's
// checkpoints, src/io/mod_checkpoint_io.f90: `open(..., form='unformatted', access='sequential')`).
// A record is a 4-byte length marker, the payload and the same marker again.  A payload longer than
// the largest positive 32-bit marker is split into subrecords: each carries its own pair of
// markers, the leading one negated when more subrecords follow and the trailing one negated when a
// subrecord precedes it.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

namespace dpm {
namespace frec {

constexpr int64_t kMaxSub = 2147483639;  // largest subrecord payload gfortran writes

inline bool write_marker(std::FILE* f, int32_t m) { return std::fwrite(&m, 4, 1, f) == 1; }

inline bool write_record(std::FILE* f, const void* data, int64_t bytes, int64_t max_sub = kMaxSub) {
  const char* p = static_cast<const char*>(data);
  int64_t left = bytes;
  bool first = true;
  do {
    const int64_t len = left > max_sub ? max_sub : left;
    const bool more = left > len;
    if (!write_marker(f, more ? -(int32_t)len : (int32_t)len)) return false;
    if (len && std::fwrite(p, 1, (size_t)len, f) != (size_t)len) return false;
    if (!write_marker(f, first ? (int32_t)len : -(int32_t)len)) return false;
    p += len;
    left -= len;
    first = false;
  } while (left > 0);
  return true;
}

// Reads one whole record (all its subrecords) into out; false on a malformed or short file.
inline bool read_record(std::FILE* f, std::vector<char>& out) {
  out.clear();
  bool first = true;
  for (;;) {
    int32_t head = 0, tail = 0;
    if (std::fread(&head, 4, 1, f) != 1) return false;
    const bool more = head < 0;
    const int64_t len = more ? -(int64_t)head : (int64_t)head;
    const size_t at = out.size();
    out.resize(at + (size_t)len);
    if (len && std::fread(out.data() + at, 1, (size_t)len, f) != (size_t)len) return false;
    if (std::fread(&tail, 4, 1, f) != 1) return false;
    const int64_t tlen = tail < 0 ? -(int64_t)tail : (int64_t)tail;
    if (tlen != len || (tail < 0) == first) return false;
    first = false;
    if (!more) return true;
  }
}

// Reads a record whose payload must be exactly `bytes` long into dst.
inline bool read_record_into(std::FILE* f, void* dst, int64_t bytes) {
  std::vector<char> buf;
  if (!read_record(f, buf) || (int64_t)buf.size() != bytes) return false;
  if (bytes) std::memcpy(dst, buf.data(), (size_t)bytes);
  return true;
}

}  // namespace frec
}  // namespace dpm

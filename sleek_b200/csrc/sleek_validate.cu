// sleek_validate.cu -- host-side parser and checker of the stream format
// (int64 original size | uint16 csize[chunks] | payloads, a compressed payload
// being 32 x uint8 bit width | packed bits | int16 byte count).  The rules are the
// ones the device decoders enforce (sleek_kernels.cu), checked in stream order so
// that the first malformed chunk is the one reported.
#include <cstdint>
#include <cstring>

#include "../../include/sleek_capi.h"
#include "sleek_launch.h"

namespace {

constexpr long long CS = 16384;

void fail(sleek_stream_info* info, int reason, long long chunk)
{
  info->reason = reason;
  info->bad_chunk = chunk;
}

}  // namespace

extern "C" {

const char* sleek_stream_reason_string(int reason)
{
  switch (reason) {
    case SLEEK_STREAM_OK: return "valid";
    case SLEEK_STREAM_SHORT_HEADER: return "stream shorter than its 8-byte header";
    case SLEEK_STREAM_BAD_SIZE: return "original size negative or not a multiple of the element size";
    case SLEEK_STREAM_SHORT_TABLE: return "size table runs past the end of the stream";
    case SLEEK_STREAM_BAD_CHUNK_SIZE: return "chunk size out of range";
    case SLEEK_STREAM_SHORT_PAYLOAD: return "chunk payload runs past the end of the stream";
    case SLEEK_STREAM_BAD_WIDTH: return "subchunk bit width above the element width";
    case SLEEK_STREAM_SIZE_MISMATCH: return "bit widths do not add up to the chunk size";
    case SLEEK_STREAM_BAD_TRAILER: return "chunk trailer differs from the chunk's byte count";
    default: return "unknown reason";
  }
}

int sleek_validate_stream(const unsigned char* s, long long len, int elem_bytes, sleek_stream_info* info)
{
  return sleek::validate_stream(s, len, elem_bytes, info, true);
}

}  // extern "C"

int sleek::validate_stream(const unsigned char* s, long long len, int elem_bytes, sleek_stream_info* info,
                           bool payloads)
{
  if (!info || (!s && len > 0) || len < 0 || (elem_bytes != 4 && elem_bytes != 8)) return SLEEK_ERR_INVALID_ARG;
  std::memset(info, 0, sizeof(*info));
  info->insize = -1;
  info->bad_chunk = -1;
  if (len < 8) {
    fail(info, SLEEK_STREAM_SHORT_HEADER, -1);
    return SLEEK_ERR_CORRUPT_STREAM;
  }
  long long insize;
  std::memcpy(&insize, s, 8);
  info->insize = insize;
  if (insize < 0 || insize % elem_bytes != 0) {
    fail(info, SLEEK_STREAM_BAD_SIZE, -1);
    return SLEEK_ERR_CORRUPT_STREAM;
  }
  const long long chunks = (insize + CS - 1) / CS;
  info->chunks = chunks;
  if (chunks > (len - 8) / 2) {
    fail(info, SLEEK_STREAM_SHORT_TABLE, -1);
    return SLEEK_ERR_CORRUPT_STREAM;
  }
  const long long base = 8 + 2 * chunks;
  const int vps = elem_bytes == 4 ? 128 : 64;  // values per subchunk
  const int tb = 8 * elem_bytes;
  long long off = base;
  info->stream_bytes = base;
  for (long long c = 0; c < chunks; ++c) {
    uint16_t cs;
    std::memcpy(&cs, s + 8 + 2 * c, 2);
    const int os = static_cast<int>(insize - c * CS < CS ? insize - c * CS : CS);
    if (cs == 0 || cs > os || (cs < os && cs < 34)) {
      fail(info, SLEEK_STREAM_BAD_CHUNK_SIZE, c);
      return SLEEK_ERR_CORRUPT_STREAM;
    }
    if (off + cs > len) {
      fail(info, SLEEK_STREAM_SHORT_PAYLOAD, c);
      return SLEEK_ERR_CORRUPT_STREAM;
    }
    const unsigned char* p = s + off;
    if (cs == os) {
      info->raw_chunks++;
    } else if (payloads) {
      long long bits = 0;
      for (int i = 0; i < 32; ++i) {
        if (p[i] > tb) {
          fail(info, SLEEK_STREAM_BAD_WIDTH, c);
          return SLEEK_ERR_CORRUPT_STREAM;
        }
        bits += static_cast<long long>(p[i]) * vps;
      }
      if (34 + bits / 8 != cs) {
        fail(info, SLEEK_STREAM_SIZE_MISMATCH, c);
        return SLEEK_ERR_CORRUPT_STREAM;
      }
      int16_t tr;
      std::memcpy(&tr, p + cs - 2, 2);
      if (tr != os) {
        fail(info, SLEEK_STREAM_BAD_TRAILER, c);
        return SLEEK_ERR_CORRUPT_STREAM;
      }
    }
    off += cs;
    info->stream_bytes = off;
  }
  return SLEEK_OK;
}



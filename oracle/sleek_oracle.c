/*
 * sleek_oracle.c -- CPU restatement of SLEEK's chunk codec, used ONLY as the
 * parity checker by tests/, __graft_entry__.smoke() and the cpu_baseline leg of
 * bench.py.  It is test infrastructure, never the product path: the library in
 * sleek_b200/ has no CPU fallback and never links this file.
 *
 * Parity pin: tests/test_oracle.py checks this restatement byte-for-byte
 * against the reference's own CPU code (include/sleek_common_cpu.h, compiled
 * from the reference sources by oracle/Makefile into oracle/_ref/) and against
 * the committed golden fixtures in tests/golden/ that were produced by that
 * reference build.
 *
 * Sequential by design (one chunk after another, running byte offset) so the
 * output placement is obviously the exclusive prefix sum of chunk sizes.
 *
 * Reference map (paths inside the SLEEK project):
 *   lossless forward transform   include/sleek_common_cpu.h:152-170
 *   lossless inverse transform   include/sleek_common_cpu.h:317-335
 *   quantize                     include/sleek_common_cpu.h:393-419
 *   deQuantize                   include/sleek_common_cpu.h:559-591
 *   h_encode (format, fallback)  include/sleek_common_cpu.h:101-256, 422-556
 *   h_decode                     include/sleek_common_cpu.h:259-385, 594-685
 *   sleek_error_bound            include/sleek_lossy_cpu.h:56-71
 *   sleek_upper_bound_size       include/sleek_common_cpu.h:67-71
 */
#include <stdint.h>
#include <string.h>
#include <stdlib.h>

#define CS 16384   /* chunk bytes, fixed by the format */
#define SC 32      /* subchunks per chunk */

enum { OR_OK = 0, OR_ERR_ARG = 1, OR_ERR_CORRUPT = 5, OR_ERR_EB = 4 };

long long oracle_upper_bound_size(long long insize)
{
  const long long chunks = (insize + CS - 1) / CS;
  return 12 + chunks * 2 + chunks * CS;
}

/* ---- per-value transforms, 32-bit ------------------------------------- */

static uint32_t fwd32(uint32_t v)  /* sleek_common_cpu.h:153-160 */
{
  v = (v << 1) | (v >> 31);
  if (v & 0xff000000u) {
    v -= 0x80000000u;
    if (((v & 0xff000000u) == 0) || (v >= 0x80000000u)) v -= 0x01000000u;
  }
  return (v << 1) ^ (uint32_t)(((int32_t)v) >> 31);
}

static uint32_t inv32(uint32_t v)  /* sleek_common_cpu.h:318-325 */
{
  v = (v >> 1) ^ (uint32_t)(((int32_t)(v << 31)) >> 31);
  if (v & 0xff000000u) {
    if (v >= 0x80000000u) v += 0x01000000u;
    v += 0x80000000u;
  }
  return (v << 31) | (v >> 1);
}

static uint32_t quant32(uint32_t val, int eb_e, int thr_e, uint32_t offs)  /* :393-419 */
{
  const uint32_t a = val & 0x7fffffffu;
  const int val_e = (int)(a >> 23);
  uint32_t enc = 0;
  if (val_e >= thr_e) {
    enc = a - offs;
  } else if (val_e >= eb_e) {
    const int shift = thr_e - val_e;
    uint32_t mant = (val & 0x007fffffu) | 0x00800000u;
    mant += 1u << (shift - 1);
    enc = mant >> shift;
  }
  enc = (enc << 1) | ((~val) >> 31);
  if (enc != 0) enc--;
  return enc;
}

static uint32_t dequant32(uint32_t enc, int thr_e, uint32_t offs)  /* :559-591 */
{
  uint32_t dec = 0;
  if (enc != 0) {
    const uint32_t a = (enc + 1u) >> 1;
    if (a >= (1u << 23)) {
      dec = a + offs;
    } else if (a > 0) {
      const int shift = __builtin_clz(a) - 8;
      dec = (a << shift) & 0x007fffffu;
      dec |= (uint32_t)(thr_e - shift) << 23;
    }
    dec |= enc << 31;
  }
  return dec;
}

/* ---- per-value transforms, 64-bit ------------------------------------- */

static uint64_t fwd64(uint64_t v)  /* sleek_common_cpu.h:162-169 */
{
  v = (v << 1) | (v >> 63);
  if (v & 0xffe0000000000000ull) {
    v -= 0x8000000000000000ull;
    if (((v & 0xffe0000000000000ull) == 0) || (v >= 0x8000000000000000ull)) v -= 0x0020000000000000ull;
  }
  return (v << 1) ^ (uint64_t)(((int64_t)v) >> 63);
}

static uint64_t inv64(uint64_t v)  /* sleek_common_cpu.h:327-334 */
{
  v = (v >> 1) ^ (uint64_t)(((int64_t)(v << 63)) >> 63);
  if (v & 0xffe0000000000000ull) {
    if (v >= 0x8000000000000000ull) v += 0x0020000000000000ull;
    v += 0x8000000000000000ull;
  }
  return (v << 63) | (v >> 1);
}

static uint64_t quant64(uint64_t val, int eb_e, int thr_e, uint64_t offs)
{
  const uint64_t a = val & 0x7fffffffffffffffull;
  const int val_e = (int)(a >> 52);
  uint64_t enc = 0;
  if (val_e >= thr_e) {
    enc = a - offs;
  } else if (val_e >= eb_e) {
    const int shift = thr_e - val_e;
    uint64_t mant = (val & 0x000fffffffffffffull) | 0x0010000000000000ull;
    mant += 1ull << (shift - 1);
    enc = mant >> shift;
  }
  enc = (enc << 1) | ((~val) >> 63);
  if (enc != 0) enc--;
  return enc;
}

static uint64_t dequant64(uint64_t enc, int thr_e, uint64_t offs)
{
  uint64_t dec = 0;
  if (enc != 0) {
    const uint64_t a = (enc + 1u) >> 1;
    if (a >= (1ull << 52)) {
      dec = a + offs;
    } else if (a > 0) {
      const int shift = __builtin_clzll(a) - 11;
      dec = (a << shift) & 0x000fffffffffffffull;
      dec |= (uint64_t)(thr_e - shift) << 52;
    }
    dec |= enc << 63;
  }
  return dec;
}

/* ---- error bound (sleek_lossy_cpu.h:56-71) ----------------------------- */

int oracle_error_bound_f32(float eb, int* eb_e, int* thr_e, uint32_t* offs)
{
  uint32_t bits;
  memcpy(&bits, &eb, 4);
  const int e = (int)((bits >> 23) & 0xff);
  const int t = e + 24;
  if (t >= 255) return OR_ERR_EB;
  *eb_e = e; *thr_e = t; *offs = ((uint32_t)t << 23) - (1u << 23);
  return OR_OK;
}

int oracle_error_bound_f64(double eb, int* eb_e, int* thr_e, uint64_t* offs)
{
  uint64_t bits;
  memcpy(&bits, &eb, 8);
  const int e = (int)((bits >> 52) & 0x7ff);
  const int t = e + 53;
  if (t >= 2047) return OR_ERR_EB;
  *eb_e = e; *thr_e = t; *offs = ((uint64_t)t << 52) - (1ull << 52);
  return OR_OK;
}

/* ---- chunk codec ------------------------------------------------------- */

/* Bit k of the packed stream is bit (k % 8) of byte k / 8 (little-endian words,
 * LSB first), identical for 32- and 64-bit words. */
static void put_bits(uint8_t* dst, long long bitpos, uint64_t v, int n)
{
  const long long byte = bitpos >> 3;
  const int sh = (int)(bitpos & 7);
  const unsigned __int128 x = (unsigned __int128)v << sh;   /* v < 2^n, dst pre-zeroed */
  const int nb = (sh + n + 7) / 8;
  for (int i = 0; i < nb; i++) dst[byte + i] |= (uint8_t)(x >> (8 * i));
}

static uint64_t get_bits(const uint8_t* src, long long bitpos, int n)
{
  const long long byte = bitpos >> 3;
  const int sh = (int)(bitpos & 7);
  const int nb = (sh + n + 7) / 8;
  unsigned __int128 x = 0;
  for (int i = 0; i < nb; i++) x |= (unsigned __int128)src[byte + i] << (8 * i);
  x >>= sh;
  return (n == 64) ? (uint64_t)x : ((uint64_t)x & ((1ull << n) - 1));
}

/* width: 4 or 8 bytes; mode: 0 lossless, 1 lossy */
static long long encode_any(int width, int mode, const uint8_t* in, long long insize, uint8_t* out,
                            int eb_e, int thr_e, uint64_t offs)
{
  const long long chunks = (insize + CS - 1) / CS;
  const int TB = width * 8;
  const int vpc = CS / width;
  const int vps = vpc / SC;
  memcpy(out, &insize, 8);
  uint8_t* size_out = out + 8;
  uint8_t* data_out = out + 8 + 2 * chunks;
  long long off = 0;
  uint8_t buf[CS];
  uint64_t tv[CS / 4];
  uint8_t enc[CS];
  for (long long c = 0; c < chunks; c++) {
    const long long base = c * CS;
    const int osize = (int)((insize - base) < CS ? (insize - base) : CS);
    memset(buf, 0, CS);                         /* zero-pad the last chunk (:135-139) */
    memcpy(buf, in + base, osize);
    int ln[SC];
    long long bits = 0;
    for (int i = 0; i < SC; i++) {
      uint64_t mx = 0;
      for (int j = i * vps; j < (i + 1) * vps; j++) {
        uint64_t t;
        if (width == 4) {
          uint32_t v; memcpy(&v, buf + 4 * j, 4);
          t = mode ? quant32(v, eb_e, thr_e, (uint32_t)offs) : fwd32(v);
        } else {
          uint64_t v; memcpy(&v, buf + 8 * j, 8);
          t = mode ? quant64(v, eb_e, thr_e, offs) : fwd64(v);
        }
        tv[j] = t;
        if (t > mx) mx = t;
      }
      ln[i] = mx ? TB - (width == 4 ? __builtin_clz((uint32_t)mx) : __builtin_clzll(mx)) : 0;
      bits += (long long)ln[i] * vps;
    }
    const int newsize = (int)((SC * 8 + bits + 16) / 8);   /* :184 */
    int csize;
    if (newsize < CS && newsize < osize) {                 /* :198 */
      memset(enc, 0, CS);
      for (int i = 0; i < SC; i++) enc[i] = (uint8_t)ln[i];
      long long pos = SC * 8;
      for (int i = 0; i < SC; i++) {
        for (int j = i * vps; j < (i + 1) * vps; j++) {
          put_bits(enc, pos, tv[j], ln[i]);
          pos += ln[i];
        }
      }
      const int16_t tr = (int16_t)osize;                  /* trailer (:238) */
      memcpy(enc + newsize - 2, &tr, 2);
      memcpy(data_out + off, enc, newsize);
      csize = newsize;
    } else {
      memcpy(data_out + off, in + base, osize);            /* raw fallback (:246) */
      csize = osize;
    }
    const uint16_t cs16 = (uint16_t)csize;
    memcpy(size_out + 2 * c, &cs16, 2);
    off += csize;
  }
  return 8 + 2 * chunks + off;
}

/* Returns 0 or OR_ERR_CORRUPT.  stream_len bounds every read of the stream. */
static int decode_any(int width, int mode, const uint8_t* in, long long stream_len, uint8_t* out,
                      long long out_cap, long long* outsize, int thr_e, uint64_t offs)
{
  if (stream_len < 8) return OR_ERR_CORRUPT;
  long long insize;
  memcpy(&insize, in, 8);
  *outsize = insize;
  if (insize < 0 || insize > out_cap) return OR_ERR_CORRUPT;
  const long long chunks = (insize + CS - 1) / CS;
  if (8 + 2 * chunks > stream_len) return OR_ERR_CORRUPT;
  const int TB = width * 8;
  const int vpc = CS / width;
  const int vps = vpc / SC;
  const uint8_t* size_in = in + 8;
  const uint8_t* data_in = in + 8 + 2 * chunks;
  const long long payload_len = stream_len - 8 - 2 * chunks;
  long long off = 0;
  int status = OR_OK;
  uint8_t dec[CS];
  for (long long c = 0; c < chunks; c++) {
    const long long base = c * CS;
    const int osize = (int)((insize - base) < CS ? (insize - base) : CS);
    uint16_t cs16; memcpy(&cs16, size_in + 2 * c, 2);
    const int csize = cs16;
    if (off + csize > payload_len) return OR_ERR_CORRUPT;
    const uint8_t* src = data_in + off;
    if (csize == osize) {                                  /* :296-298 */
      memcpy(out + base, src, osize);
    } else {
      if (csize < SC + 2) return OR_ERR_CORRUPT;
      long long bits = 0;
      for (int i = 0; i < SC; i++) {
        if (src[i] > TB) return OR_ERR_CORRUPT;
        bits += (long long)src[i] * vps;
      }
      if ((SC * 8 + bits + 16) / 8 > csize) return OR_ERR_CORRUPT;
      long long pos = SC * 8;
      for (int i = 0; i < SC; i++) {
        const int l = src[i];
        for (int j = i * vps; j < (i + 1) * vps; j++) {
          const uint64_t t = l ? get_bits(src, pos, l) : 0;
          pos += l;
          if (width == 4) {
            const uint32_t v = mode ? dequant32((uint32_t)t, thr_e, (uint32_t)offs) : (l ? inv32((uint32_t)t) : 0u);
            memcpy(dec + 4 * j, &v, 4);
          } else {
            const uint64_t v = mode ? dequant64(t, thr_e, offs) : (l ? inv64(t) : 0ull);
            memcpy(dec + 8 * j, &v, 8);
          }
        }
      }
      int16_t tr; memcpy(&tr, src + csize - 2, 2);        /* trailer check (:376-378) */
      if (tr != osize) status = OR_ERR_CORRUPT;
      memcpy(out + base, dec, osize);
    }
    off += csize;
  }
  return status;
}

/* ---- exported entry points -------------------------------------------- */

long long oracle_encode(int width, int mode, const void* in, long long insize, void* out,
                        int eb_e, int thr_e, unsigned long long offs)
{
  if ((width != 4 && width != 8) || insize < 0 || (insize % width) != 0) return -OR_ERR_ARG;
  return encode_any(width, mode, (const uint8_t*)in, insize, (uint8_t*)out, eb_e, thr_e, offs);
}

int oracle_decode(int width, int mode, const void* in, long long stream_len, void* out,
                  long long out_cap, long long* outsize, int thr_e, unsigned long long offs)
{
  if (width != 4 && width != 8) return OR_ERR_ARG;
  return decode_any(width, mode, (const uint8_t*)in, stream_len, (uint8_t*)out, out_cap, outsize, thr_e, offs);
}

/* Element-wise transforms exposed for unit tests of the oracle itself. */
unsigned int oracle_fwd32(unsigned int v) { return fwd32(v); }
unsigned int oracle_inv32(unsigned int v) { return inv32(v); }
unsigned long long oracle_fwd64(unsigned long long v) { return fwd64(v); }
unsigned long long oracle_inv64(unsigned long long v) { return inv64(v); }
unsigned int oracle_quant32(unsigned int v, int eb_e, int thr_e, unsigned int offs) { return quant32(v, eb_e, thr_e, offs); }
unsigned int oracle_dequant32(unsigned int v, int thr_e, unsigned int offs) { return dequant32(v, thr_e, offs); }
unsigned long long oracle_quant64(unsigned long long v, int eb_e, int thr_e, unsigned long long offs) { return quant64(v, eb_e, thr_e, offs); }
unsigned long long oracle_dequant64(unsigned long long v, int thr_e, unsigned long long offs) { return dequant64(v, thr_e, offs); }

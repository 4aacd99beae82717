// sleek_device.cuh -- device building blocks of the sm_100a SLEEK codec.
//
// Everything here is integer / bit arithmetic.  The value transforms restate the
// reference's arithmetic exactly (that is what makes the byte stream identical);
// the data movement (TMA bulk loads into shared memory, gather-form bit packing,
// bounded decoupled look-back, 16-byte shifted stores) is this project's own.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "sleek_launch.h"

namespace sleek {

constexpr int CS = 16384;          // chunk bytes; fixed by the stream format
constexpr int SC = 32;             // subchunks per chunk; fixed by the stream format
constexpr int STAGE_BYTES = CS + 64;  // one chunk plus room for a 16-byte misaligned window

// status codes shared with the C ABI (include/sleek_capi.h)
constexpr unsigned ST_CORRUPT = 5;
constexpr unsigned ST_TIMEOUT = 6;
constexpr unsigned ST_CAPACITY = 9;

// Workspace: 32 header words (u64 each), then the look-back flags.  Words 0 and
// 1 are the launch's ticket and done counters; two blocks of per-launch results
// (status, total, error position, flags used) follow at words 0-7 and 8-15 (the
// first block shares its first two words with the counters), then the launch
// epoch (word 16) and words the range reduction uses (24-26).  Single-buffer
// launches alternate between the blocks and between two flag regions by epoch
// parity (see WsPhase below); batched launches use block 0 and the first region
// of a workspace cleared before each run.
enum WsWord {
  WS_TICKET = 0, WS_DONE = 1,                                   // counters (words 0, 1)
  WS_STATUS = 2, WS_TOTAL = 3, WS_ERRPOS = 4, WS_USED = 5,      // within a block
  WS_BLOCK = 8,       // words per block
  WS_EPOCH = 16,      // launches completed on this workspace
  WS_MINMAX = 24,     // three words for the range reduction (cleared by its own call)
  WS_HDR_WORDS = 32
};

// look-back flag: state in bits 62-63, value in bits 0-61
constexpr uint64_t FLAG_AGG = 1ull << 62;
constexpr uint64_t FLAG_INC = 2ull << 62;
constexpr uint64_t FLAG_VAL = (1ull << 62) - 1;

constexpr unsigned long long SPIN_TIMEOUT_NS = 4000000000ull;  // 4 s of wall time per wait

// ----------------------------------------------------------------------------
// value traits
// ----------------------------------------------------------------------------
template <typename T> struct VT;
template <> struct VT<uint32_t> {
  static constexpr int TB = 32;            // bits per value
  static constexpr int VPC = CS / 4;       // values per chunk
  static constexpr int VPS = VPC / SC;     // values per subchunk (128)
  static constexpr int WPS_PER_LN = 2;     // packed u64 words per subchunk per bit of width
};
template <> struct VT<uint64_t> {
  static constexpr int TB = 64;
  static constexpr int VPC = CS / 8;
  static constexpr int VPS = VPC / SC;     // 64
  static constexpr int WPS_PER_LN = 1;
};

// ----------------------------------------------------------------------------
// PTX helpers
// ----------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init()
{
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Tests the phase with the given parity; a thread whose phase is not complete
// is suspended until it completes (or about 0.5 ms pass), so waiting warps do
// not spin on issue slots.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(500000u)
      : "memory");
  return ok != 0;
}

// Waits for the phase with the given parity; gives up after `limit_ns`.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  unsigned long long limit_ns = SPIN_TIMEOUT_NS)
{
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (globaltimer_ns() - t0 > limit_ns) return false;
  }
  return true;
}

// 1-D bulk copy global -> shared (no multicast); completion counted on `bar`.
__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ uint64_t ld_acquire_u64(const uint64_t* p)
{
  uint64_t v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release_u64(uint64_t* p, uint64_t v)
{
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Flags carry their own value, so publishing one needs no ordering against the
// thread's earlier stores (a release would wait for the chunk stores in flight).
__device__ __forceinline__ void st_relaxed_u64(uint64_t* p, uint64_t v)
{
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t* p)
{
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// records the first error in a counter block; later errors keep the first code
__device__ __forceinline__ void set_status(uint64_t* hdr, unsigned code, long long pos)
{
  if (atomicCAS(reinterpret_cast<unsigned long long*>(&hdr[WS_STATUS]), 0ull, (unsigned long long)code) == 0ull) {
    atomicExch(reinterpret_cast<unsigned long long*>(&hdr[WS_ERRPOS]), (unsigned long long)pos);
  }
}

// ----------------------------------------------------------------------------
// Self-resetting workspace of the single-buffer kernels.  A launch works in
// result block and flag region p = epoch & 1 (both clean when it starts), and
// leaves the other parity clean for the next launch: every CTA clears its share
// of the flags the previous launch used there, and the last CTA resets that
// block and the ticket and done counters, records how many flags this launch
// used, then advances the epoch.  The counters do not depend on the epoch, so a
// CTA takes its first ticket without waiting for the epoch's load.  A workspace
// that starts zeroed therefore needs no clearing between launches on one stream;
// a workspace cleared before every launch (epoch 0) behaves the same.  flag_cap
// is the size of one flag region.
// ----------------------------------------------------------------------------
struct WsPhase {
  uint64_t* hdr;        // this launch's counter block
  uint64_t* hdr_other;  // the other block (the previous launch's)
  uint64_t* flags;      // this launch's flag region
  uint64_t* flags_other;
  uint64_t epoch;
  long long used_other;  // flags the previous launch left in the other region

  // The epoch and the other block's flag count were written by an earlier launch
  // and do not change before every CTA of this one has read them, so they are
  // plain loads, free to overlap the kernel's other start-up loads (a volatile
  // load would order them first: measured -7 % on 26 MB decodes).
  __device__ static WsPhase of(uint64_t* ws, long long flag_cap)
  {
    WsPhase w;
    w.epoch = ws[WS_EPOCH];
    const int p = static_cast<int>(w.epoch & 1u);
    w.hdr = ws + WS_BLOCK * p;
    w.hdr_other = ws + WS_BLOCK * (1 - p);
    w.flags = ws + WS_HDR_WORDS + flag_cap * p;
    w.flags_other = ws + WS_HDR_WORDS + flag_cap * (1 - p);
    w.used_other = static_cast<long long>(w.hdr_other[WS_USED]);
    return w;
  }

  // block 0 and the first flag region, nothing to clear (a workspace cleared
  // before each launch, as the batched launches use it)
  __device__ static WsPhase fixed(uint64_t* ws)
  {
    WsPhase w;
    w.epoch = 0;
    w.hdr = ws;
    w.hdr_other = ws + WS_BLOCK;
    w.flags = ws + WS_HDR_WORDS;
    w.flags_other = w.flags;
    w.used_other = 0;
    return w;
  }

  // this CTA's share of the other region's flags, by the calling warp
  __device__ void clear_other_share(int lane) const
  {
    const long long per = (used_other + gridDim.x - 1) / gridDim.x;
    const long long b = per * blockIdx.x;
    const long long e = min(b + per, used_other);
    for (long long i = b + lane; i < e; i += 32) flags_other[i] = 0ull;
  }

  // the last CTA, one thread, after every CTA has counted itself done (so no
  // ticket or done atomic of this launch is still to come)
  __device__ void finish(uint64_t* ws, long long used) const
  {
    hdr[WS_USED] = static_cast<uint64_t>(used);
#pragma unroll
    for (int i = WS_STATUS; i < WS_BLOCK; ++i) hdr_other[i] = 0ull;
    ws[WS_TICKET] = 0ull;
    ws[WS_DONE] = 0ull;
    __threadfence();
    ws[WS_EPOCH] = epoch + 1u;
  }
};

// ----------------------------------------------------------------------------
// value transforms (restated from include/sleek_common_gpu.h of the reference:
// lossless forward :356-374, inverse :614-632, quantize :776-802, deQuantize
// :1077-1108).  Bit-exactness of the stream depends on these being identical.
// ----------------------------------------------------------------------------
// The reference's forward step, on the rotated word v with exponent field
// E = v >> 24: if E != 0, subtract 2^31, then subtract one more exponent unit if
// the field became 0 or the top bit is set.  Case by case that adds 0 (E = 0),
// 2^31 - 2^24 (1 <= E <= 0x80) or 2^31 (E > 0x80) mod 2^32, which is how it is
// computed here (equal on all 2^32 inputs).
__device__ __forceinline__ uint32_t fwd(uint32_t v)
{
  v = (v << 1) | (v >> 31);
  v += v < 0x01000000u ? 0u : (v < 0x81000000u ? 0x7f000000u : 0x80000000u);
  return (v << 1) ^ static_cast<uint32_t>(static_cast<int32_t>(v) >> 31);
}

// 64-bit lossless forward transform on 32-bit halves: the exponent test and
// both subtractions touch only the high word (no borrow crosses into the low
// word), the rotate and the final shift are funnel shifts.
__device__ __forceinline__ uint64_t fwd(uint64_t v)
{
  const uint32_t h = static_cast<uint32_t>(v >> 32);
  const uint32_t l = static_cast<uint32_t>(v);
  uint32_t nh = __funnelshift_l(l, h, 1);        // rotate left by 1
  const uint32_t nl = __funnelshift_l(h, l, 1);
  // the same step on the 11-bit field: adds 0, 2^31 - 2^21 or 2^31
  nh += nh < 0x00200000u ? 0u : (nh < 0x80200000u ? 0x7fe00000u : 0x80000000u);
  const uint32_t sg = static_cast<uint32_t>(static_cast<int32_t>(nh) >> 31);
  const uint32_t oh = __funnelshift_l(nl, nh, 1) ^ sg;  // (v << 1) ^ (v >> 63 arithmetic)
  const uint32_t ol = (nl << 1) ^ sg;
  return (static_cast<uint64_t>(oh) << 32) | ol;
}

__device__ __forceinline__ uint32_t inv(uint32_t v)
{
  v = (v >> 1) ^ static_cast<uint32_t>(static_cast<int32_t>(v << 31) >> 31);
  if (v & 0xff000000u) {
    if (v >= 0x80000000u) v += 0x01000000u;
    v += 0x80000000u;
  }
  return (v << 31) | (v >> 1);
}

__device__ __forceinline__ uint64_t inv(uint64_t v)
{
  const uint32_t h = static_cast<uint32_t>(v >> 32);
  const uint32_t l = static_cast<uint32_t>(v);
  const uint32_t sg = 0u - (l & 1u);                       // (v << 63) >> 63 arithmetic
  uint32_t nh = (h >> 1) ^ sg;
  const uint32_t nl = __funnelshift_r(l, h, 1) ^ sg;
  if (nh & 0xffe00000u) {
    if (nh >= 0x80000000u) nh += 0x00200000u;
    nh += 0x80000000u;
  }
  const uint32_t oh = __funnelshift_r(nh, nl, 1);          // rotate right by 1
  const uint32_t ol = __funnelshift_r(nl, nh, 1);
  return (static_cast<uint64_t>(oh) << 32) | ol;
}

__device__ __forceinline__ uint32_t quant(uint32_t val, const QParams& q)
{
  const uint32_t a = val & 0x7fffffffu;
  const int ve = static_cast<int>(a >> 23);
  uint32_t enc = 0;
  if (ve >= q.thr_e) {
    enc = a - static_cast<uint32_t>(q.offs);
  } else if (ve >= q.eb_e) {
    const int sh = q.thr_e - ve;
    const uint32_t mant = ((val & 0x007fffffu) | 0x00800000u) + (1u << (sh - 1));
    enc = mant >> sh;
  }
  enc = (enc << 1) | ((~val) >> 31);
  return enc ? enc - 1u : 0u;
}

// 64-bit quantize on 32-bit halves (same arithmetic as the 64-bit form: the
// rounding add carries into the high word, the shift is a funnel shift).
__device__ __forceinline__ uint64_t quant(uint64_t val, const QParams& q)
{
  const uint32_t h = static_cast<uint32_t>(val >> 32);
  const uint32_t l = static_cast<uint32_t>(val);
  const uint32_t ah = h & 0x7fffffffu;
  const int ve = static_cast<int>(ah >> 20);
  uint32_t eh = 0, el = 0;
  if (ve >= q.thr_e) {
    const uint32_t oh = static_cast<uint32_t>(q.offs >> 32);
    const uint32_t ol = static_cast<uint32_t>(q.offs);
    el = l - ol;
    eh = ah - oh - (l < ol ? 1u : 0u);
  } else if (ve >= q.eb_e) {
    const int sh = q.thr_e - ve;  // 1 .. 53
    uint32_t mh = (h & 0x000fffffu) | 0x00100000u;
    uint32_t ml = l;
    const int b = sh - 1;
    if (b < 32) {
      const uint32_t add = 1u << b;
      ml += add;
      mh += ml < add ? 1u : 0u;
    } else {
      mh += 1u << (b - 32);
    }
    if (sh < 32) {
      el = __funnelshift_r(ml, mh, sh);
      eh = mh >> sh;
    } else {
      el = mh >> (sh - 32);
    }
  }
  uint32_t rh = __funnelshift_l(el, eh, 1);
  uint32_t rl = (el << 1) | ((h >> 31) ^ 1u);
  if (rh | rl) {
    rh -= rl == 0u ? 1u : 0u;
    rl -= 1u;
  }
  return (static_cast<uint64_t>(rh) << 32) | rl;
}

__device__ __forceinline__ uint32_t dequant(uint32_t enc, const QParams& q)
{
  if (enc == 0u) return 0u;
  const uint32_t a = (enc + 1u) >> 1;
  uint32_t dec = 0;
  if (a >= (1u << 23)) {
    dec = a + static_cast<uint32_t>(q.offs);
  } else if (a > 0u) {
    const int sh = __clz(a) - 8;
    dec = ((a << sh) & 0x007fffffu) | (static_cast<uint32_t>(q.thr_e - sh) << 23);
  }
  return dec | (enc << 31);
}

// 64-bit dequantize on 32-bit halves.
__device__ __forceinline__ uint64_t dequant(uint64_t enc, const QParams& q)
{
  const uint32_t eh = static_cast<uint32_t>(enc >> 32);
  const uint32_t el = static_cast<uint32_t>(enc);
  if ((eh | el) == 0u) return 0ull;
  const uint32_t tl = el + 1u;                      // (enc + 1) >> 1, wrapping like the 64-bit form
  const uint32_t th = eh + (tl == 0u ? 1u : 0u);
  const uint32_t ah = th >> 1;
  const uint32_t al = __funnelshift_r(tl, th, 1);
  uint32_t dh = 0, dl = 0;
  if (ah >= (1u << 20)) {                            // a >= 2^52: stored losslessly
    const uint32_t oh = static_cast<uint32_t>(q.offs >> 32);
    const uint32_t ol = static_cast<uint32_t>(q.offs);
    dl = al + ol;
    dh = ah + oh + (dl < ol ? 1u : 0u);
  } else if ((ah | al) != 0u) {
    const int lz = ah ? __clz(ah) : 32 + __clz(al);
    const int sh = lz - 11;                          // normalise the leading 1 to bit 52
    if (sh < 32) {
      dh = __funnelshift_l(al, ah, sh);
      dl = al << sh;
    } else {
      dh = al << (sh - 32);
    }
    dh = (dh & 0x000fffffu) | (static_cast<uint32_t>(q.thr_e - sh) << 20);
  }
  dh |= el << 31;                                    // sign from the lowest bit
  return (static_cast<uint64_t>(dh) << 32) | dl;
}

// ----------------------------------------------------------------------------
// The same quantize / dequantize with the rounding division done in floating
// point (the integer forms above stay the definition; these are exact rewrites).
//
// Dequantize: for 0 < a < 2^m the integer form normalises a and sets the
// exponent to thr_e - shift, which is the IEEE value a * 2^(thr_e - bias - m):
// the int -> float conversion of a is exact (a < 2^m) and the power-of-two
// product is exact and normal (its exponent field is at least thr_e - m >= 1).
//
// Quantize: for eb_e <= e < thr_e the integer form computes
// floor((M + 2^(sh-1)) / 2^sh), M the significand with its implicit bit and
// sh = thr_e - e.  With y = |v| * 2^(bias + m - thr_e) = M / 2^sh (exact: a
// power-of-two scaling of a normal number with a normal result, y >= 1/2),
// that is floor(y + 1/2).  y + 1/2 = N / 2^sh with N < 2^(m+2) is exact unless
// N needs m + 2 bits and is odd; then rounding toward minus infinity yields
// (N - 1) / 2^sh, and N odd with sh >= 1 means floor((N - 1) / 2^sh) =
// floor(N / 2^sh).  So trunc(round_down(y + 1/2)) is exact.  Denormal values
// (e = 0) are quantized only when eb_e = 0, where the integer form still adds
// the implicit bit; that case keeps the integer form.
//
// Below eb_e the integer form gives 0, and so does eq without a test: e < eb_e
// means |v| < 2^(eb_e - bias), so y < 2^(eb_e + m - thr_e) = 1/2 (thr_e =
// eb_e + m + 1), y + 1/2 < 1 and its round-down truncates to 0 (a product that
// underflows is rounded, but far below 1/2).
//
// The sign step `e2 = (enc << 1) | !sign; e2 ? e2 - 1 : 0` is written as
// `(enc << 1) - (enc ? sign : 0)`: for enc > 0 both are 2 enc - sign, and for
// enc = 0 both are 0 (e2 is 1 - sign there).
// ----------------------------------------------------------------------------
__device__ __forceinline__ uint32_t quant_fp(uint32_t val, const QParams& q)
{
  if (q.eb_e == 0) return quant(val, q);
  const uint32_t a = val & 0x7fffffffu;
  const int ve = static_cast<int>(a >> 23);
  const float inv_scale = __uint_as_float(static_cast<uint32_t>(277 - q.thr_e) << 23);  // 2^(150 - thr_e)
  const uint32_t eq = __float2uint_rz(__fadd_rd(__fmul_rn(__uint_as_float(a), inv_scale), 0.5f));
  const uint32_t enc = ve >= q.thr_e ? a - static_cast<uint32_t>(q.offs) : eq;
  return (enc << 1) - (enc ? (val >> 31) : 0u);
}

__device__ __forceinline__ uint64_t quant_fp(uint64_t val, const QParams& q)
{
  if (q.eb_e == 0) return quant(val, q);
  const uint64_t a = val & 0x7fffffffffffffffull;
  const int ve = static_cast<int>(a >> 52);
  const double inv_scale = __longlong_as_double(static_cast<long long>(2098 - q.thr_e) << 52);  // 2^(1075 - thr_e)
  const uint64_t eq = __double2ull_rz(__dadd_rd(__dmul_rn(__longlong_as_double(static_cast<long long>(a)), inv_scale), 0.5));
  const uint64_t enc = ve >= q.thr_e ? a - q.offs : eq;
  return (enc << 1) - (enc ? (val >> 63) : 0ull);
}

__device__ __forceinline__ uint32_t dequant_fp(uint32_t enc, const QParams& q)
{
  if (enc == 0u) return 0u;
  const uint32_t a = (enc + 1u) >> 1;
  const float scale = __uint_as_float(static_cast<uint32_t>(q.thr_e - 23) << 23);  // 2^(thr_e - 150)
  const uint32_t dec = a >= (1u << 23) ? a + static_cast<uint32_t>(q.offs)
                                       : __float_as_uint(__fmul_rn(__uint2float_rn(a), scale));
  return dec | (enc << 31);
}

__device__ __forceinline__ uint64_t dequant_fp(uint64_t enc, const QParams& q)
{
  if (enc == 0ull) return 0ull;
  const uint64_t a = (enc + 1ull) >> 1;
  const double scale = __longlong_as_double(static_cast<long long>(q.thr_e - 52) << 52);  // 2^(thr_e - 1075)
  const uint64_t dec = a >= (1ull << 52) ? a + q.offs
                                         : static_cast<uint64_t>(__double_as_longlong(__dmul_rn(__ull2double_rn(a), scale)));
  return dec | (enc << 63);
}

// dequant_fp of a 64-bit code below 2^32 (a chunk whose widths are all at most
// 32): a = ceil(enc / 2) < 2^31 never reaches the 2^52 escape, and the u32 ->
// f64 conversion is exact, so the result equals dequant_fp's.
__device__ __forceinline__ uint64_t dequant_fp_narrow(uint32_t enc, const QParams& q)
{
  if (enc == 0u) return 0ull;
  const uint32_t a = (enc >> 1) + (enc & 1u);
  const double scale = __longlong_as_double(static_cast<long long>(q.thr_e - 52) << 52);
  const uint64_t dec = static_cast<uint64_t>(__double_as_longlong(__dmul_rn(__uint2double_rn(a), scale)));
  return dec | (static_cast<uint64_t>(enc & 1u) << 63);
}

template <bool LOSSY, typename T>
__device__ __forceinline__ T encode_value(T v, const QParams& q)
{
  if constexpr (LOSSY) return quant_fp(v, q);
  else return fwd(v);
}

template <bool LOSSY, typename T>
__device__ __forceinline__ T decode_value(T v, const QParams& q)
{
  if constexpr (LOSSY) return dequant_fp(v, q);
  else return inv(v);
}

__device__ __forceinline__ int bit_width(uint32_t m) { return m ? 32 - __clz(m) : 0; }
__device__ __forceinline__ int bit_width(uint64_t m) { return m ? 64 - __clzll(m) : 0; }

__device__ __forceinline__ uint32_t warp_max(uint32_t v) { return __reduce_max_sync(0xffffffffu, v); }
__device__ __forceinline__ uint64_t warp_max(uint64_t v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const uint64_t w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

// bit width of the largest value held by the warp, from the OR of all values
__device__ __forceinline__ int warp_bit_width(uint32_t v)
{
  return bit_width(__reduce_or_sync(0xffffffffu, v));
}
__device__ __forceinline__ int warp_bit_width(uint64_t v)
{
  const uint32_t hi = __reduce_or_sync(0xffffffffu, static_cast<uint32_t>(v >> 32));
  const uint32_t lo = __reduce_or_sync(0xffffffffu, static_cast<uint32_t>(v));
  return hi ? 64 - __clz(hi) : bit_width(lo);
}

__device__ __forceinline__ long long warp_sum(long long v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ----------------------------------------------------------------------------
// Decoupled look-back over flag words.  Called by one whole warp for item
// `idx` whose segment starts at `seg_begin` (items before the segment count as
// an inclusive prefix of 0).  Each poll reads the 32 nearest unresolved flags
// (one load per lane), sums the run of aggregates up to the
// nearest inclusive prefix, and slides past runs of aggregates; it only waits
// when the nearest unresolved flag is not published yet.  Returns the exclusive
// prefix, or -1 when a wait exceeded `limit_ns` or another CTA already
// reported an error in the counter block `hdr`.
// ----------------------------------------------------------------------------
__device__ __forceinline__ long long lookback(const uint64_t* flags, long long idx, long long seg_begin,
                                              const uint64_t* hdr, unsigned long long limit_ns = SPIN_TIMEOUT_NS)
{
  constexpr int PER = 1;  // polls of 32 flags: measured against 64 and 128, encode +2 % and +4-9 %
  const int lane = threadIdx.x & 31;
  long long excl = 0;
  long long end = idx - 1;
  unsigned long long t0 = 0;
  unsigned sleep_ns = 256;
  int polls = 0;
  while (true) {
    uint64_t f[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const long long j = end - lane - 32 * k;
      f[k] = (j >= seg_begin) ? ld_relaxed_u64(&flags[j]) : FLAG_INC;
    }
    int z = 32 * PER;  // distance of the nearest unpublished flag
    int p = 32 * PER;  // distance of the nearest inclusive prefix
#pragma unroll
    for (int k = PER - 1; k >= 0; --k) {
      const unsigned nr = __ballot_sync(0xffffffffu, (f[k] >> 62) == 0ull);
      const unsigned inc = __ballot_sync(0xffffffffu, (f[k] >> 62) == 2ull);
      if (nr) z = 32 * k + __ffs(nr) - 1;
      if (inc) p = 32 * k + __ffs(inc) - 1;
    }
    if (p < z) {
      long long s = 0;
#pragma unroll
      for (int k = 0; k < PER; ++k)
        if (lane + 32 * k <= p) s += static_cast<long long>(f[k] & FLAG_VAL);
      return excl + warp_sum(s);
    }
    if (z > 0) {
      long long s = 0;
#pragma unroll
      for (int k = 0; k < PER; ++k)
        if (lane + 32 * k < z) s += static_cast<long long>(f[k] & FLAG_VAL);
      excl += warp_sum(s);
      end -= z;
      continue;
    }
    // the nearest predecessor has not published yet: back off, bounded in time
    if (++polls == 64) {
      t0 = globaltimer_ns();
    } else if (polls > 64 && (polls & 63) == 0) {
      const bool late = globaltimer_ns() - t0 > limit_ns;
      const bool failed = ld_relaxed_u64(&hdr[WS_STATUS]) != 0ull;
      if (__any_sync(0xffffffffu, late || failed)) return -1;
    }
    // sleeping from the first miss keeps hundreds of waiting warps from flooding
    // the L2 with polls (measured: decode +3-8 %, encode unchanged)
    __nanosleep(sleep_ns);
    if (sleep_ns < 2048) sleep_ns <<= 1;
  }
}

// ----------------------------------------------------------------------------
// Shifted store: writes `len` bytes from 16-byte aligned shared memory `src`
// to the arbitrary global byte address `dst`.  Whole aligned 16-byte granules
// get one vector store each, funnel-shifted from two aligned shared loads; the
// at most two granules shared with neighbouring chunks are written byte by
// byte.  Called by NT threads with tid = 0 .. NT-1 (the encoder: its producer
// warp, NT = 32).
// ----------------------------------------------------------------------------
template <int WQ>
__device__ __forceinline__ uint4 shifted_granule(const uint4 x, const uint4 y, int bb8)
{
  // output granule from source granules x = j - 1 and y = j
  const uint32_t w[8] = {x.x, x.y, x.z, x.w, y.x, y.y, y.z, y.w};
  uint4 o;
  o.x = __funnelshift_r(w[WQ + 0], w[WQ + 1], bb8);
  o.y = __funnelshift_r(w[WQ + 1], w[WQ + 2], bb8);
  o.z = __funnelshift_r(w[WQ + 2], w[WQ + 3], bb8);
  o.w = __funnelshift_r(w[WQ + 3], w[WQ + 4], bb8);
  return o;
}

// Granules jf .. jl-1, consecutive lanes on consecutive granules (so a warp's
// loads hit every bank once and its stores fill whole sectors), two granules in
// flight per thread.
template <int WQ, int NT>
__device__ __forceinline__ void shifted_run(uint4* out, const uint4* s4, int jf, int jl, int bb8, int t)
{
  for (int j = jf + t; j < jl; j += 2 * NT) {
    const bool two = j + NT < jl;
    const uint4 x0 = s4[j - 1], y0 = s4[j];
    uint4 x1 = x0, y1 = y0;
    if (two) {
      x1 = s4[j + NT - 1];
      y1 = s4[j + NT];
    }
    out[j] = shifted_granule<WQ>(x0, y0, bb8);
    if (two) out[j + NT] = shifted_granule<WQ>(x1, y1, bb8);
  }
}

template <int NT>
__device__ __forceinline__ void store_shifted(uint8_t* dst, const uint8_t* src, int len, int tid)
{
  const uintptr_t d = reinterpret_cast<uintptr_t>(dst);
  const int sft = static_cast<int>(d & 15u);
  uint8_t* const a0 = dst - sft;
  uint4* const out = reinterpret_cast<uint4*>(a0);
  const uint4* const s4 = reinterpret_cast<const uint4*>(src);
  const int nunits = (sft + len + 15) >> 4;
  const int jf = sft ? 1 : 0;              // first granule entirely inside the chunk
  const int jl = (sft + len) >> 4;         // one past the last such granule
  if (sft == 0) {
    for (int j = tid; j < jl; j += NT) out[j] = s4[j];
  } else {
    const int bo = 16 - sft;
    const int bb8 = (bo & 3) * 8;
    switch (bo >> 2) {
      case 0: shifted_run<0, NT>(out, s4, jf, jl, bb8, tid); break;
      case 1: shifted_run<1, NT>(out, s4, jf, jl, bb8, tid); break;
      case 2: shifted_run<2, NT>(out, s4, jf, jl, bb8, tid); break;
      default: shifted_run<3, NT>(out, s4, jf, jl, bb8, tid); break;
    }
  }
  // edge granules (shared with the neighbouring chunks): one byte per lane of
  // the first warp, lanes 0-15 the first granule, lanes 16-31 the last
  if (tid < 32) {
    int e = -1;
    if (tid < 16) {
      if (sft != 0) e = 0;
    } else {
      const int last = nunits - 1;
      if (last >= jl && !(last == 0 && sft != 0)) e = last;
    }
    if (e >= 0) {
      const int r = 16 * e - sft + (tid & 15);  // source byte of this lane
      if (r >= 0 && r < len) a0[16 * e + (tid & 15)] = src[r];
    }
  }
}

// Reads the u32 word starting at an arbitrary byte offset of 16-byte aligned
// shared memory (the two aligned words around it, funnel-shifted).
__device__ __forceinline__ uint32_t lds_u32_at_byte(const uint8_t* base, int byte_off)
{
  const uint32_t* w = reinterpret_cast<const uint32_t*>(base);
  const int wi = byte_off >> 2;
  const int sh = (byte_off & 3) * 8;
  return __funnelshift_r(w[wi], w[wi + 1], sh);
}

// Extracts `ln` bits (1 <= ln <= 64) starting at bit `pos` of 16-byte aligned
// shared memory, LSB-first little-endian (the stream's bit order).
__device__ __forceinline__ uint32_t extract_bits32(const uint32_t* w, int pos, int ln)
{
  const int wi = pos >> 5;
  const uint32_t v = __funnelshift_r(w[wi], w[wi + 1], pos & 31);
  return ln >= 32 ? v : (v & ((1u << ln) - 1u));
}

__device__ __forceinline__ uint64_t extract_bits64(const uint32_t* w, int pos, int ln)
{
  const int wi = pos >> 5;
  const int sh = pos & 31;
  const uint32_t w0 = w[wi], w1 = w[wi + 1], w2 = w[wi + 2];
  const uint32_t lo = __funnelshift_r(w0, w1, sh);
  const uint32_t hi = __funnelshift_r(w1, w2, sh);
  const uint64_t v = (static_cast<uint64_t>(hi) << 32) | lo;
  return ln >= 64 ? v : (v & ((1ull << ln) - 1ull));
}

}  // namespace sleek

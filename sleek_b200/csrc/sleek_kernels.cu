// sleek_kernels.cu -- sm_100a encode / decode kernels (one buffer, and batches).
//
// Encode (replaces d_encode, include/sleek_common_gpu.h:474-559, 989-1074 of the
// reference): persistent CTAs of 8 compute warps, a producer warp and a scanner
// warp, 3 per SM.  The producer takes a chunk ticket (atomic, just in time) and
// copies the 16 KB chunk into one of four shared-memory stages with a 1-D TMA bulk
// copy, two chunks ahead.  Each compute warp loads 4 subchunks into registers,
// transforms or quantizes them (value arithmetic restated from the reference) and
// ORs them into bit widths; after the compute warps' one barrier per chunk every
// warp derives the offsets it needs by warp reductions, thread 0 publishes the
// chunk's size, and each warp packs its subchunks from registers into the stage
// (funnel-shifted runs with one neighbour exchange; short runs by shared OR).  The
// scanner looks back over the chunk flags as soon as the chunk has landed and
// records its payload offset; the producer stores the packed chunk to the stream
// (16-byte vector stores, consecutive lanes on consecutive granules) right before
// it refills that stage, so the compute warps never wait for an offset.  A chunk
// whose encoding is not smaller than its input is stored raw straight from the
// staged copy (never re-read from HBM).
//
// Decode (replaces d_decode, :688-768, 1199-1279): CTAs take contiguous chunk
// ranges in ticket order, sum their ranges' compressed sizes, look back over the
// preceding ranges once, then stream their chunks through a two-stage TMA
// pipeline (each copy is the 16-byte aligned superset of the chunk's bytes); every
// warp checks each chunk itself and unpacks its own subchunks straight into
// coalesced global stores, with no CTA barrier per chunk.  Malformed streams set
// an error status instead of trapping; every wait is bounded in time.
#include "sleek_device.cuh"
#include "sleek_launch.h"

namespace sleek {

// Launch shape of the encode kernel: CW compute warps (each takes SC / CW
// subchunks of a chunk) and ST shared-memory stages of one chunk each.  The
// producer copies chunk k once the compute warps have sized chunk k - AHEAD, right
// after storing the stage's previous chunk, k - ST (whose look-back thereby gets
// ST - AHEAD chunks of compute time).  MINB is the CTAs per SM the registers are
// budgeted for.  Every shape writes the same bytes.
template <int CW_, int ST_, int MINB_>
struct EncShape {
  static constexpr int CW = CW_;
  static constexpr int ST = ST_;
  // the copy of chunk seq is issued once the compute warps have sized chunk seq - AHEAD
  static constexpr int AHEAD = 2;
  static constexpr int MINB = MINB_;
  static constexpr int NT = (CW + 2) * 32;  // + a producer warp and a scanner warp
  static constexpr int SPW = SC / CW;       // subchunks per compute warp
  static_assert(SC % CW == 0 && AHEAD < ST, "shape");
};
// the shapes the library is built with (index = the C ABI's shape number)
using EncShape0 = EncShape<8, 4, 3>;   // default: 10 warps, 66 KB, 3 CTAs per SM
using EncShape1 = EncShape<16, 4, 2>;  // 18 warps, 66 KB, 2 CTAs per SM
using EncShape2 = EncShape<4, 4, 3>;   // 6 warps, 66 KB, 3 CTAs per SM
using EncShape3 = EncShape<8, 3, 3>;   // 10 warps, 3 stages (50 KB), 3 CTAs per SM
using EncShape4 = EncShape<8, 5, 2>;   // 10 warps, 5 stages (83 KB), 2 CTAs per SM
constexpr int ENC_SHAPES = 5;
constexpr long long NO_CHUNK = 0x7fffffffffffffffll;

// What the producer tells the compute and scanner warps about the chunk in a stage.
struct EncMeta {
  long long g;          // look-back flag index (chunk id across the launch), or NO_CHUNK
  long long c;          // chunk index within its buffer
  long long seg;        // flag index of the buffer's first chunk
  long long chunks;     // chunks of the buffer
  long long insize;     // bytes of the buffer
  uint8_t* out;         // the buffer's stream
  long long* outsize;   // the buffer's size output
  long long excl;       // payload offset of the chunk (scanner), -1 after an error
  QParams q;            // the buffer's quantizer parameters
  int kind;             // bit 0: 64-bit values, bit 1: lossy
  int osize;
  int csize;
  int comp;
};

template <int ST>
struct EncMisc {
  uint64_t full[ST];    // chunk bytes landed (TMA tx count)
  uint64_t sized[ST];   // compressed size of the stage's chunk known (compute warps past phase A)
  uint64_t placed[ST];  // payload offset of the stage's chunk known
  uint64_t packed[ST];  // every compute warp has packed its share of the stage's chunk
  EncMeta meta[ST];
  int lnv[2][SC];  // subchunk bit widths, by chunk parity (a fast warp may write the next chunk's)
};

template <class S>
constexpr int enc_smem()
{
  return S::ST * STAGE_BYTES + static_cast<int>((sizeof(EncMisc<S::ST>) + 127) / 128) * 128;
}
template <class S>
constexpr int enc_batch_smem()
{
  return enc_smem<S>() + 8 * (BATCH_MAX_JOBS + 1);  // + the jobs' first chunk ids
}

// barrier among the CW compute warps only (named barrier 1), OR-reducing `pred`
template <int CW>
__device__ __forceinline__ bool cbar_or(bool pred)
{
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"(static_cast<uint32_t>(pred)), "n"(CW * 32)
      : "memory");
  return r != 0;
}

// ORs `v`, placed at bit offset `o` (< 96, warp-uniform) of a 128-bit run, into
// the run's words x0..x3.
__device__ __forceinline__ void place32(uint32_t v, int o, uint32_t& x0, uint32_t& x1, uint32_t& x2, uint32_t& x3)
{
  const int q = o >> 5;
  const int r = o & 31;
  const uint32_t lo = v << r;
  const uint32_t hi = __funnelshift_l(v, 0u, r);  // bits that cross into the next word
  if (q == 0) {
    x0 |= lo;
    x1 |= hi;
  } else if (q == 1) {
    x1 |= lo;
    x2 |= hi;
  } else {
    x2 |= lo;
    x3 |= hi;
  }
}

// Packs one subchunk whose transformed values sit in registers: lane L holds
// values P*L .. P*L+P-1 and writes the bit run [P*L*ln, P*(L+1)*ln) of the
// subchunk's packed bits (LSB-first, 32-bit little-endian words at `pw`).
template <typename T>
__device__ __forceinline__ void pack_subchunk(uint32_t* pw, int ln, const T (&v)[16 / sizeof(T)], int lane)
{
  constexpr int P = 16 / static_cast<int>(sizeof(T));  // values per lane
  constexpr int TB = 8 * static_cast<int>(sizeof(T));
  if (ln == 0) return;
  if (ln == TB) {  // verbatim: the lane's 16 bytes in place
    uint32_t* d = pw + 4 * lane;
    if constexpr (sizeof(T) == 4) {
      if ((reinterpret_cast<uintptr_t>(d) & 15u) == 0u) {
        *reinterpret_cast<uint4*>(d) = make_uint4(v[0], v[1], v[2], v[3]);
      } else {
        d[0] = v[0]; d[1] = v[1]; d[2] = v[2]; d[3] = v[3];
      }
    } else {
      reinterpret_cast<uint2*>(d)[0] = make_uint2(static_cast<uint32_t>(v[0]), static_cast<uint32_t>(v[0] >> 32));
      reinterpret_cast<uint2*>(d)[1] = make_uint2(static_cast<uint32_t>(v[1]), static_cast<uint32_t>(v[1] >> 32));
    }
    return;
  }
  const int R = P * ln;  // bits of the lane's run
  const int rs = lane * R;
  const int w0 = rs >> 5;
  const int s = rs & 31;
  if (R >= 32) {
    // the run as a 128-bit number x3:x2:x1:x0 (the offsets are warp-uniform)
    uint32_t x0, x1 = 0u, x2 = 0u, x3 = 0u;
    if constexpr (sizeof(T) == 4) {
      x0 = v[0];
      place32(v[1], ln, x0, x1, x2, x3);
      place32(v[2], 2 * ln, x0, x1, x2, x3);
      place32(v[3], 3 * ln, x0, x1, x2, x3);
    } else {
      const uint32_t a0 = static_cast<uint32_t>(v[0]), a1 = static_cast<uint32_t>(v[0] >> 32);
      const uint32_t b0 = static_cast<uint32_t>(v[1]), b1 = static_cast<uint32_t>(v[1] >> 32);
      if (ln >= 32) {
        const int r = ln - 32;
        x0 = a0;
        x1 = a1 | (b0 << r);
        x2 = __funnelshift_l(b0, b1, r);
        x3 = __funnelshift_l(b1, 0u, r);
      } else {  // both values fit in 31 bits
        x0 = a0 | (b0 << ln);
        x1 = __funnelshift_l(b0, 0u, ln);
      }
    }
    // shifted into place within the lane's first word
    const uint32_t y0 = x0 << s;
    const uint32_t y1 = __funnelshift_l(x0, x1, s);
    const uint32_t y2 = __funnelshift_l(x1, x2, s);
    const uint32_t y3 = __funnelshift_l(x2, x3, s);
    const uint32_t y4 = __funnelshift_l(x3, 0u, s);
    const int nfull = (s + R) >> 5;  // words 1 .. nfull-1 lie wholly in this run
    const uint32_t tail = nfull == 1 ? y1 : (nfull == 2 ? y2 : (nfull == 3 ? y3 : y4));
    // each word holds bits of at most two adjacent lanes: the next lane completes our tail
    const uint32_t prev = __shfl_up_sync(0xffffffffu, tail, 1);
    uint32_t* const d = pw + w0;
    d[0] = s ? (y0 | prev) : y0;
    if (nfull > 1) d[1] = y1;
    if (nfull > 2) d[2] = y2;
    if (nfull > 3) d[3] = y3;
  } else {
    // short runs: several lanes share a word.  A run of R < 32 bits starts in
    // every word, so the lane whose run starts first in a word stores it
    // plainly (no clearing pass); the other lanes, and the spill of each run
    // into the next word, OR in after that store.  Lane 31's run ends on a
    // word boundary (32 R bits in all), so no spill leaves the packed area.
    uint32_t run = 0;
#pragma unroll
    for (int k = 0; k < P; ++k) run |= static_cast<uint32_t>(v[k]) << (k * ln);
    const uint64_t sh = static_cast<uint64_t>(run) << s;
    const uint32_t lo = static_cast<uint32_t>(sh), hi = static_cast<uint32_t>(sh >> 32);
    const bool first = lane == 0 || (((lane - 1) * R) >> 5) != w0;
    if (first) pw[w0] = lo;
    __syncwarp();
    if (!first && lo) atomicOr(&pw[w0], lo);
    if (hi) atomicOr(&pw[w0 + 1], hi);
  }
}

// The lane's bit run of four 32-bit values of width ln (8 <= ln <= 31) as a
// 128-bit number x3:x2:x1:x0, without branches.
__device__ __forceinline__ void run_words(const uint32_t (&v)[4], int ln, uint32_t& x0, uint32_t& x1, uint32_t& x2,
                                          uint32_t& x3)
{
  // pairs (v0 | v1 << ln) and (v2 | v3 << ln), each below 2^62; then the second
  // pair shifted by 2 ln (16 .. 62) onto the first
  const uint32_t a0 = v[0] | (v[1] << ln), a1 = __funnelshift_l(v[1], 0u, ln);
  const uint32_t b0 = v[2] | (v[3] << ln), b1 = __funnelshift_l(v[3], 0u, ln);
  const int k = 2 * ln;
  const bool q = k >= 32;
  const int r = k & 31;
  const uint32_t t0 = b0 << r, t1 = __funnelshift_l(b0, b1, r), t2 = __funnelshift_l(b1, 0u, r);
  x0 = a0 | (q ? 0u : t0);
  x1 = a1 | (q ? t0 : t1);
  x2 = q ? t1 : t2;
  x3 = q ? t2 : 0u;
}

// Packs a warp's SPW subchunks (offsets wbase, widths lnu).  When every run is
// short, or (32-bit values) every run is long (32 <= P*ln, ln below the value
// width), or (64-bit values) every run is long with values of at most 31 bits,
// the subchunks go through one straight-line sequence each, so their shuffles,
// shifts and stores overlap; other widths take the per-subchunk path.
// (For 64-bit values the branch-free long run costs more than the overlap saves:
// measured -2 % on lossless f64, +3.5-6 % on f32.)
constexpr int PACK_GROUP = 2;  // subchunks whose long runs are built and exchanged together

template <typename T, int SPW>
__device__ __forceinline__ void pack_subchunks(uint32_t* pw, const int (&wbase)[SPW], const int (&lnu)[SPW],
                                               const T (&v)[SPW][16 / sizeof(T)], int lane)
{
  constexpr int P = 16 / static_cast<int>(sizeof(T));
  constexpr int TB = 8 * static_cast<int>(sizeof(T));
  bool all_long = sizeof(T) == 4, all_short = true, all_narrow = sizeof(T) == 8;
#pragma unroll
  for (int u = 0; u < SPW; ++u) {
    all_long &= P * lnu[u] >= 32 && lnu[u] < TB;
    all_short &= P * lnu[u] < 32;
    all_narrow &= P * lnu[u] >= 32 && lnu[u] < 32;  // 64-bit values of 16 .. 31 bits
  }
  if (all_long) {
    if constexpr (sizeof(T) == 4) {
#pragma unroll
      for (int g = 0; g < SPW; g += PACK_GROUP) {
        uint32_t y[SPW][5], tl[SPW], pv[SPW];
        int nf[SPW];
#pragma unroll
        for (int u = g; u < g + PACK_GROUP; ++u) {
          const int R = P * lnu[u];
          const int s = (lane * R) & 31;
          uint32_t x0, x1, x2, x3;
          run_words(v[u], lnu[u], x0, x1, x2, x3);
          y[u][0] = x0 << s;
          y[u][1] = __funnelshift_l(x0, x1, s);
          y[u][2] = __funnelshift_l(x1, x2, s);
          y[u][3] = __funnelshift_l(x2, x3, s);
          y[u][4] = __funnelshift_l(x3, 0u, s);
          nf[u] = (s + R) >> 5;
          tl[u] = nf[u] == 1 ? y[u][1] : (nf[u] == 2 ? y[u][2] : (nf[u] == 3 ? y[u][3] : y[u][4]));
        }
#pragma unroll
        for (int u = g; u < g + PACK_GROUP; ++u) pv[u] = __shfl_up_sync(0xffffffffu, tl[u], 1);
#pragma unroll
        for (int u = g; u < g + PACK_GROUP; ++u) {
          const int rs = lane * P * lnu[u];
          uint32_t* const d = pw + wbase[u] + (rs >> 5);
          d[0] = (rs & 31) ? (y[u][0] | pv[u]) : y[u][0];
          if (nf[u] > 1) d[1] = y[u][1];
          if (nf[u] > 2) d[2] = y[u][2];
          if (nf[u] > 3) d[3] = y[u][3];
        }
      }
    }
  } else if (all_short) {
    // see pack_subchunk: the first run in each word stores it, the rest OR in
    uint32_t lo[SPW], hi[SPW];
    int w[SPW];
    bool first[SPW];
#pragma unroll
    for (int u = 0; u < SPW; ++u) {
      const int ln = lnu[u];
      const int R = P * ln;
      uint32_t run = 0;
#pragma unroll
      for (int k = 0; k < P; ++k) run |= static_cast<uint32_t>(v[u][k]) << (k * ln);
      const uint64_t sh = static_cast<uint64_t>(run) << ((lane * R) & 31);
      lo[u] = static_cast<uint32_t>(sh);
      hi[u] = static_cast<uint32_t>(sh >> 32);
      w[u] = wbase[u] + ((lane * R) >> 5);
      first[u] = ln != 0 && (lane == 0 || (((lane - 1) * R) >> 5) != ((lane * R) >> 5));
      if (first[u]) pw[w[u]] = lo[u];
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < SPW; ++u) {
      if (!first[u] && lo[u]) atomicOr(&pw[w[u]], lo[u]);
      if (hi[u]) atomicOr(&pw[w[u] + 1], hi[u]);
    }
  } else if (all_narrow) {
    if constexpr (sizeof(T) == 8) {
      // 64-bit values that fit in 31 bits (typical of lossy chunks): the lane's two
      // values make a run of 32 .. 62 bits, two words before the shift and at most
      // three after it, built from the low halves only
      uint32_t y0[SPW], y1[SPW], tl[SPW], pv[SPW];
      int nf[SPW];
#pragma unroll
      for (int u = 0; u < SPW; ++u) {
        const int ln = lnu[u];
        const int R = P * ln;
        const int sh = (lane * R) & 31;
        const uint32_t a0 = static_cast<uint32_t>(v[u][0]), b0 = static_cast<uint32_t>(v[u][1]);
        const uint32_t x0 = a0 | (b0 << ln), x1 = __funnelshift_l(b0, 0u, ln);
        y0[u] = x0 << sh;
        y1[u] = __funnelshift_l(x0, x1, sh);
        const uint32_t y2 = __funnelshift_l(x1, 0u, sh);
        nf[u] = (sh + R) >> 5;
        tl[u] = nf[u] == 1 ? y1[u] : y2;
      }
#pragma unroll
      for (int u = 0; u < SPW; ++u) pv[u] = __shfl_up_sync(0xffffffffu, tl[u], 1);
#pragma unroll
      for (int u = 0; u < SPW; ++u) {
        const int rs = lane * P * lnu[u];
        uint32_t* const d = pw + wbase[u] + (rs >> 5);
        d[0] = (rs & 31) ? (y0[u] | pv[u]) : y0[u];
        if (nf[u] > 1) d[1] = y1[u];
      }
    }
  } else {
#pragma unroll
    for (int u = 0; u < SPW; ++u) pack_subchunk<T>(pw + wbase[u], lnu[u], v[u], lane);
  }
}


// The per-chunk work of a compute warp, in three steps shared by both encode
// kernels.  KIND: bit 0 = 64-bit values, bit 1 = lossy.
template <int KIND>
using EncVal = typename std::conditional<(KIND & 1) != 0, uint64_t, uint32_t>::type;

// Phase A: the warp's subchunks cw, cw + CW, ... of the staged chunk into
// registers, transformed or quantized, and their bit widths into lnv (the stage
// always holds a full 16 KB chunk: partial chunks are zero padded).
template <int KIND, class S>
__device__ __forceinline__ void chunk_phase_a(const uint8_t* stg, const QParams& q, int* lnv, int cw, int lane,
                                              EncVal<KIND> (&vals)[S::SPW][16 / sizeof(EncVal<KIND>)])
{
  using T = EncVal<KIND>;
  constexpr bool LOSSY = (KIND & 2) != 0;
  constexpr int P = 16 / static_cast<int>(sizeof(T));
#pragma unroll
  for (int u = 0; u < S::SPW; ++u) {
    const int i = cw + u * S::CW;
    const uint4 w4 = *reinterpret_cast<const uint4*>(stg + i * 512 + lane * 16);
    if constexpr (sizeof(T) == 4) {
      vals[u][0] = w4.x; vals[u][1] = w4.y; vals[u][2] = w4.z; vals[u][3] = w4.w;
    } else {
      vals[u][0] = (static_cast<uint64_t>(w4.y) << 32) | w4.x;
      vals[u][1] = (static_cast<uint64_t>(w4.w) << 32) | w4.z;
    }
    T orv = 0;
#pragma unroll
    for (int p = 0; p < P; ++p) {
      vals[u][p] = encode_value<LOSSY>(vals[u][p], q);
      orv |= vals[u][p];
    }
    const int w = warp_bit_width(orv);
    if (lane == 0) lnv[i] = w;
  }
}

// The chunk's packed words (wtot) and its size in the stream (compressed iff
// 34 + 4 wtot < osize), from every subchunk's width (all lanes, any warp).
struct ChunkSize {
  int ln;    // width of subchunk `lane`
  int wc;    // 32-bit words of subchunk `lane`
  int wtot;  // packed words of the chunk
  int csize;
  bool comp;
};
template <typename T>
__device__ __forceinline__ ChunkSize chunk_size(const int* lnv, int lane, int osize)
{
  using V = VT<T>;
  ChunkSize z;
  z.ln = lnv[lane];
  z.wc = (V::VPS * z.ln) >> 5;
  // totals by warp reductions (independent, no shuffle-scan chain)
  z.wtot = __reduce_add_sync(0xffffffffu, z.wc);
  const int newsize = 34 + 4 * z.wtot;
  z.comp = newsize < osize;
  z.csize = z.comp ? newsize : osize;
  return z;
}

// Packs a compressible chunk from registers to `dst` (16-byte aligned): the 32
// width bytes, the packed words, the int16 trailer.
template <int KIND, class S>
__device__ __forceinline__ void chunk_pack(uint8_t* dst, const ChunkSize& z, int osize, int cw, int lane,
                                           const EncVal<KIND> (&vals)[S::SPW][16 / sizeof(EncVal<KIND>)])
{
  using T = EncVal<KIND>;
  uint32_t* const pw = reinterpret_cast<uint32_t*>(dst + 32);
  int wbase[S::SPW], lnu[S::SPW];  // all offsets and widths first: the reductions overlap
#pragma unroll
  for (int u = 0; u < S::SPW; ++u) {
    const int i = cw + u * S::CW;
    wbase[u] = __reduce_add_sync(0xffffffffu, lane < i ? z.wc : 0);  // words of subchunks before i
    lnu[u] = __shfl_sync(0xffffffffu, z.ln, i);
  }
  pack_subchunks<T, S::SPW>(pw, wbase, lnu, vals, lane);
  if (cw == 0) {
    dst[lane] = static_cast<uint8_t>(z.ln);
    if (lane == 0) *reinterpret_cast<int16_t*>(dst + 32 + 4 * z.wtot) = static_cast<int16_t>(osize);
  }
}

// Transform, size, publish and pack one chunk in place (compute warps of
// k_encode).  The barrier after phase A is the compute warps' only CTA barrier
// per chunk and their point of agreement: every warp arrives there, with `skip`
// (no chunk: the end, or a failed wait) and `fail` (this thread's wait gave up);
// returns 2 if any thread failed, 1 at the end, 0 when the chunk was processed.
template <int KIND, class S>
__device__ __forceinline__ int compute_chunk(uint8_t* stg, EncMeta& me, EncMisc<S::ST>& m, uint64_t* flags, int cw,
                                             int lane, int tid, int par, bool skip, bool fail)
{
  using T = EncVal<KIND>;
  int* const lnv = m.lnv[par];
  T vals[S::SPW][16 / sizeof(T)];
  if (!skip) chunk_phase_a<KIND, S>(stg, me.q, lnv, cw, lane, vals);
  if (cbar_or<S::CW>(fail)) return 2;
  if (skip) return 1;
  const int osize = me.osize;
  const ChunkSize z = chunk_size<T>(lnv, lane, osize);
  if (tid == 0) {
    const int s = static_cast<int>(&me - m.meta);
    me.csize = z.csize;
    me.comp = z.comp;
    st_relaxed_u64(&flags[me.g], (me.c == 0 ? FLAG_INC : FLAG_AGG) | static_cast<uint64_t>(z.csize));
    mbar_arrive(&m.sized[s]);
  }
  if (z.comp) chunk_pack<KIND, S>(stg, z, osize, cw, lane, vals);
  return 0;
}

// Chunk sources: one buffer (the plain entry points) or a table of buffers (the
// batched entry points; every chunk of every buffer is one ticket).
template <bool BATCH>
struct EncSource;

template <>
struct EncSource<false> {
  const EncArgs& a;
  long long chunks;
  __device__ long long total() const { return chunks; }
  // fills the chunk's description; returns its first byte
  __device__ const uint8_t* describe(long long g, EncMeta& me, int kind) const
  {
    me.g = g;
    me.c = g;
    me.seg = 0;
    me.chunks = chunks;
    me.insize = a.insize;
    me.out = a.out;
    me.outsize = a.outsize;
    me.q = a.q;
    me.kind = kind;
    me.osize = static_cast<int>(min(static_cast<long long>(CS), a.insize - g * CS));
    return a.in + g * CS;
  }
};

template <>
struct EncSource<true> {
  const BatchEncArgs& a;
  const long long* cb;  // shared memory: first chunk id of each job, then the total
  __device__ long long total() const { return cb[a.njobs]; }
  __device__ const uint8_t* describe(long long g, EncMeta& me, int) const
  {
    int lo = 0, hi = a.njobs - 1;  // last job whose first chunk id is <= g (empty jobs are skipped)
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cb[mid] <= g) lo = mid;
      else hi = mid - 1;
    }
    const BatchJob& j = a.jobs[lo];
    const long long c = g - cb[lo];
    me.g = g;
    me.c = c;
    me.seg = cb[lo];
    me.chunks = j.chunks;
    me.insize = j.insize;
    me.out = j.out;
    me.outsize = j.outsize;
    me.q = j.q;
    me.kind = j.kind;
    me.osize = static_cast<int>(min(static_cast<long long>(CS), j.insize - c * CS));
    return j.in + c * CS;
  }
};

template <int KIND, bool BATCH, class S>
__global__ void __launch_bounds__(S::NT, S::MINB) k_encode(const typename std::conditional<BATCH, BatchEncArgs, EncArgs>::type a)
{
  constexpr int ENC_STAGES = S::ST;
  constexpr int ENC_AHEAD = S::AHEAD;
  constexpr int ENC_CW = S::CW;
  constexpr int ENC_NT = S::NT;
  extern __shared__ __align__(128) uint8_t smem[];
  uint8_t* const stage0 = smem;
  EncMisc<ENC_STAGES>& m = *reinterpret_cast<EncMisc<ENC_STAGES>*>(smem + ENC_STAGES * STAGE_BYTES);
  long long* const cb = reinterpret_cast<long long*>(smem + enc_smem<S>());

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  // this launch's counter block and flag region: alternating by epoch in the
  // single-buffer form (self-resetting workspace), block 0 and the first region
  // of a workspace cleared before each run in the batched form
  const WsPhase ph = [&]() {
    if constexpr (BATCH) return WsPhase::fixed(a.ws);
    else return WsPhase::of(a.ws, a.flag_cap);
  }();
  uint64_t* const hdr = ph.hdr;
  uint64_t* const flags = ph.flags;

  if constexpr (BATCH) {
    for (int i = tid; i <= a.njobs; i += ENC_NT) cb[i] = a.chunk_base[i];
  }
  if (tid == 0) {
    for (int s = 0; s < ENC_STAGES; ++s) {
      mbar_init(&m.full[s], 1);
      mbar_init(&m.sized[s], 1);
      mbar_init(&m.placed[s], 1);
      mbar_init(&m.packed[s], ENC_CW);  // one arrival per compute warp
    }
    mbar_fence_init();
  }
  // the producer's first ticket, taken while the barriers are set up (the
  // counter was reset by the previous launch's last CTA)
  long long first_ticket = NO_CHUNK;
  if (warp == ENC_CW && lane == 0)
    first_ticket = static_cast<long long>(atomicAdd(reinterpret_cast<unsigned long long*>(&a.ws[WS_TICKET]), 1ull));
  __syncthreads();

  EncSource<BATCH> src = [&]() {
    if constexpr (BATCH) return EncSource<true>{a, cb};
    else return EncSource<false>{a, (a.insize + CS - 1) / CS};
  }();
  const long long total = src.total();

  if (warp == ENC_CW) {
    // ============ producer warp: tickets, TMA copies and the chunks' stores ============
    // Tickets are taken just before their chunk's copy is issued, never earlier:
    // a ticket held long before its chunk is processed makes every later chunk's
    // look-back wait for it.  The stage's previous chunk is stored to the stream by
    // this warp right before the stage is refilled, so the compute warps go from
    // one chunk's pack straight to the next chunk's transform.
    unsigned long long* const tick = reinterpret_cast<unsigned long long*>(&a.ws[WS_TICKET]);
    // stores chunk q (stage q % ENC_STAGES) once it is packed and placed
    auto store_q = [&](int q) -> bool {
      const int sq = q % ENC_STAGES;
      const uint32_t pq = (q / ENC_STAGES) & 1;
      if (!mbar_wait_bounded(&m.packed[sq], pq)) return false;
      if (!mbar_wait_bounded(&m.placed[sq], pq)) return false;
      const EncMeta& me = m.meta[sq];
      const long long excl = me.excl;
      if (excl >= 0) {
        uint8_t* const out = me.out;
        store_shifted<32>(out + 8 + 2 * me.chunks + excl, stage0 + sq * STAGE_BYTES, me.csize, lane);
        if (lane == 0) *reinterpret_cast<uint16_t*>(out + 8 + 2 * me.c) = static_cast<uint16_t>(me.csize);
      }
      // the stage's generic accesses are ordered before the TMA write that refills it
      fence_proxy_async_smem();
      __syncwarp();
      return true;
    };
    unsigned issued = 0;      // stages whose last use was a TMA copy (lane 0's view)
    unsigned issued_par = 0;  // parity of that use
    bool more = true;
    for (int seq = 0;; ++seq) {
      const int s = seq % ENC_STAGES;
      bool ok = true;
      if (seq >= ENC_AHEAD)
        ok = mbar_wait_bounded(&m.sized[(seq - ENC_AHEAD) % ENC_STAGES], ((seq - ENC_AHEAD) / ENC_STAGES) & 1);
      if (ok && seq >= ENC_STAGES) ok = store_q(seq - ENC_STAGES);
      if (__any_sync(0xffffffffu, !ok)) {
        if (lane == 0) set_status(hdr, ST_TIMEOUT, -1);
        break;
      }
      long long t = NO_CHUNK;
      if (lane == 0 && more) t = seq == 0 ? first_ticket : static_cast<long long>(atomicAdd(tick, 1ull));
      t = __shfl_sync(0xffffffffu, t, 0);
      uint8_t* const stg = stage0 + s * STAGE_BYTES;
      EncMeta& me = m.meta[s];
      if (t < total) {
        const uint8_t* in = nullptr;
        if (lane == 0) in = src.describe(t, me, KIND);
        __syncwarp();
        in = reinterpret_cast<const uint8_t*>(__shfl_sync(0xffffffffu, reinterpret_cast<uintptr_t>(in), 0));
        const int osize = me.osize;
        if ((reinterpret_cast<uintptr_t>(in) & 15u) == 0u && osize == CS) {
          if (lane == 0) {
            mbar_arrive_expect_tx(&m.full[s], CS);
            tma_load_1d(stg, in, CS, &m.full[s]);
            issued |= 1u << s;
            issued_par = (issued_par & ~(1u << s)) | (((seq / ENC_STAGES) & 1u) << s);
          }
        } else {
          // last partial chunk or an input that is not 16-byte aligned: 4-byte
          // loads (inputs are at least 4-byte aligned), zero padding up to the full
          // chunk (the padding is encoded too)
          const uint32_t* const gin = reinterpret_cast<const uint32_t*>(in);
          uint32_t* const sv = reinterpret_cast<uint32_t*>(stg);
          constexpr int U = 16;  // independent loads in flight per lane
          for (int k0 = 0; k0 < CS / 4; k0 += 32 * U) {
            uint32_t v[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
              const int k = k0 + u * 32 + lane;
              v[u] = 4 * k < osize ? gin[k] : 0u;
            }
#pragma unroll
            for (int u = 0; u < U; ++u) sv[k0 + u * 32 + lane] = v[u];
          }
          __syncwarp();
          if (lane == 0) {
            issued &= ~(1u << s);
            mbar_arrive(&m.full[s]);  // release: the stores above are visible to its waiters
          }
        }
      } else {
        more = false;
        if (lane == 0) {
          me.g = NO_CHUNK;
          issued &= ~(1u << s);
          mbar_arrive(&m.full[s]);
        }
      }
      if (!more) break;
    }
    // (the chunks still in stages, the last ENC_STAGES - 1, are stored by the
    // compute warps, idle by then: eight warps instead of one at the kernel's end)
    // never leave with a bulk copy still landing in this CTA's shared memory
    if (lane == 0) {
      for (int s = 0; s < ENC_STAGES; ++s)
        if (issued & (1u << s)) mbar_wait_bounded(&m.full[s], (issued_par >> s) & 1u);
    }
  } else if (warp == ENC_CW + 1) {
    // ===================== scanner warp: decoupled look-back =====================
    if constexpr (!BATCH) ph.clear_other_share(lane);
    for (int seq = 0;; ++seq) {
      const int s = seq % ENC_STAGES;
      const uint32_t par = (seq / ENC_STAGES) & 1;
      bool ok = mbar_wait_bounded(&m.full[s], par);
      if (__any_sync(0xffffffffu, !ok)) break;  // the compute warps report it
      EncMeta& me = m.meta[s];
      const long long g = me.g;
      if (g == NO_CHUNK) break;
      // The look-back needs only the predecessors' sizes, so it starts as soon as
      // the chunk has landed and overlaps the compute warps' phase A (measured
      // against starting once the chunk is sized: +1-6 %).
      const long long c = me.c;
      long long excl = 0;
      unsigned err = 0;
      if (c > 0) {
        excl = lookback(flags, g, me.seg, hdr);
        if (excl < 0) err = ST_TIMEOUT;
        else if (excl > c * CS) err = ST_CAPACITY;
        if (err) excl = -1;
      }
      ok = mbar_wait_bounded(&m.sized[s], par);
      if (__any_sync(0xffffffffu, !ok)) {
        if (lane == 0) set_status(hdr, ST_TIMEOUT, g);
        break;
      }
      const int csize = me.csize;
      if (lane == 0) {
        if (c > 0) {
          if (err) set_status(hdr, err, g);
          // an impossible prefix is replaced by the largest legal one so that
          // every later chunk still writes inside the output bound
          st_relaxed_u64(&flags[g], FLAG_INC | static_cast<uint64_t>(excl >= 0 ? excl + csize : (c + 1) * CS));
        }
        me.excl = excl;
        if (c == me.chunks - 1 && excl >= 0) {
          if constexpr (BATCH) {  // the buffer is complete: its header and size
            *reinterpret_cast<long long*>(me.out) = me.insize;
            *me.outsize = 8 + 2 * me.chunks + excl + csize;
          } else {
            hdr[WS_TOTAL] = static_cast<uint64_t>(excl + csize);
          }
        }
        mbar_arrive(&m.placed[s]);
      }
    }
  } else {
    // ===================== compute warps =====================
    // Warps pass each other freely between the barriers of compute_chunk: each
    // waits for its stage itself, and a stage goes back to the producer warp once
    // every compute warp has packed its share of the chunk.
    const int cw = warp;
    bool late = false;  // a wait of this thread gave up
    int seq = 0;
    int r = 0;
    for (;; ++seq) {
      const int s = seq % ENC_STAGES;
      if (!mbar_wait_bounded(&m.full[s], (seq / ENC_STAGES) & 1)) {
        if (lane == 0) set_status(hdr, ST_TIMEOUT, -1);
        late = true;
      }
      EncMeta& me = m.meta[s];
      // warp-uniform: phase A's warp collectives need every lane or none
      const bool wlate = __any_sync(0xffffffffu, late);
      const bool skip = wlate || me.g == NO_CHUNK;
      uint8_t* const stg = stage0 + s * STAGE_BYTES;
      if constexpr (KIND >= 0) {
        r = compute_chunk<KIND, S>(stg, me, m, flags, cw, lane, tid, seq & 1, skip, wlate);
      } else {
        switch (skip ? 0 : me.kind) {
          case 0: r = compute_chunk<0, S>(stg, me, m, flags, cw, lane, tid, seq & 1, skip, wlate); break;
          case 1: r = compute_chunk<1, S>(stg, me, m, flags, cw, lane, tid, seq & 1, skip, wlate); break;
          case 2: r = compute_chunk<2, S>(stg, me, m, flags, cw, lane, tid, seq & 1, skip, wlate); break;
          default: r = compute_chunk<3, S>(stg, me, m, flags, cw, lane, tid, seq & 1, skip, wlate); break;
        }
      }
      if (r != 0) break;  // end of the work (1) or a wait that gave up (2)
      __syncwarp();
      if (lane == 0) mbar_arrive(&m.packed[s]);
    }
    if (r == 1) {
      // The producer stored chunks 0 .. seq - ENC_STAGES as it refilled their
      // stages (seq is the end marker); the rest, packed before the end's
      // barrier, are stored here once placed.
      for (int q = seq >= ENC_STAGES - 1 ? seq - ENC_STAGES + 1 : 0; q < seq; ++q) {
        const int sq = q % ENC_STAGES;
        if (!mbar_wait_bounded(&m.placed[sq], (q / ENC_STAGES) & 1)) {
          if (lane == 0) set_status(hdr, ST_TIMEOUT, -1);
          continue;
        }
        const EncMeta& me = m.meta[sq];
        const long long excl = me.excl;
        if (excl >= 0) {
          store_shifted<ENC_CW * 32>(me.out + 8 + 2 * me.chunks + excl, stage0 + sq * STAGE_BYTES, me.csize, tid);
          if (tid == 0) *reinterpret_cast<uint16_t*>(me.out + 8 + 2 * me.c) = static_cast<uint16_t>(me.csize);
        }
      }
    }
  }

  // ---- epilogue: the last CTA out finishes the outputs -----------------------
  __syncthreads();
  __shared__ int last_cta;
  if (tid == 0) {
    __threadfence();
    const unsigned long long d = atomicAdd(reinterpret_cast<unsigned long long*>(&a.ws[WS_DONE]), 1ull);
    last_cta = d == gridDim.x - 1;
    if (last_cta) __threadfence();
  }
  __syncthreads();
  if (last_cta) {
    const unsigned long long st = ld_relaxed_u64(&hdr[WS_STATUS]);
    if constexpr (BATCH) {
      // buffers without chunks get their header-only stream; an error anywhere
      // turns every size into -status
      for (int i = tid; i < a.njobs; i += ENC_NT) {
        const BatchJob& j = a.jobs[i];
        if (st) {
          *j.outsize = -static_cast<long long>(st);
        } else if (j.chunks == 0) {
          *reinterpret_cast<long long*>(j.out) = 0;
          *j.outsize = 8;
        }
      }
    } else if (tid == 0) {
      const long long chunks = (a.insize + CS - 1) / CS;
      const long long tot = chunks ? static_cast<long long>(ld_relaxed_u64(&hdr[WS_TOTAL])) : 0ll;
      *reinterpret_cast<long long*>(a.out) = a.insize;
      *a.outsize = st ? -static_cast<long long>(st) : 8 + 2 * chunks + tot;
      ph.finish(a.ws, chunks);
    }
  }
}

// ============================================================================
// decode
// ============================================================================
struct DecChunk {
  long long c;
  long long off;
  int cs;
  int sft;
  int ok;
  int pad_;
};

constexpr int DEC_STAGES = 2;

struct DecMisc {
  uint64_t full[DEC_STAGES];   // chunk bytes landed (TMA tx count)
  uint64_t empty[DEC_STAGES];  // every compute warp is done with the stage's chunk
  DecChunk info[DEC_STAGES];
  long long excl;
  long long vb;
  long long red[NT_MAX_WARPS];
  long long pre[NT_MAX_WARPS];
  int bad[NT_MAX_WARPS];
};

// Streams of at most this many chunks place each CTA's range by summing the size
// table before it directly (at most 64 KB read per CTA from L2, no wait on other
// CTAs) instead of the decoupled look-back, whose chain of polls dominates small
// decodes (26 MB: +32 %) and still costs 2-4 % at 18,432 chunks.
constexpr long long DEC_DIRECT_MAX = 32768;

constexpr int DEC_SMEM = DEC_STAGES * STAGE_BYTES + ((sizeof(DecMisc) + 127) / 128) * 128;

__device__ __forceinline__ uint64_t lds_u64_at_byte(const uint8_t* base, int byte_off)
{
  const uint32_t* w = reinterpret_cast<const uint32_t*>(base);
  const int wi = byte_off >> 2;
  const int sh = (byte_off & 3) * 8;
  const uint32_t lo = __funnelshift_r(w[wi], w[wi + 1], sh);
  const uint32_t hi = __funnelshift_r(w[wi + 1], w[wi + 2], sh);
  return (static_cast<uint64_t>(hi) << 32) | lo;
}

// Decodes one staged chunk (payload at byte `sft` of `stg`, `cs` bytes, `osize`
// bytes out) with the calling warp's share of the work and no CTA barrier: every
// warp reads the 32 bit widths, sums and checks them itself (the same result in
// every warp), then unpacks its subchunks cw, cw + NW, ... with consecutive lanes
// on consecutive values, widths and bit offsets in registers.  Returns false for
// a malformed chunk (bit width above the element width, widths not adding up to
// cs, trailer not equal to osize); a raw chunk (cs == osize) is copied.
template <typename T, bool LOSSY, int NW>
__device__ __forceinline__ bool decode_chunk_warp(const uint8_t* stg, int sft, int cs, int osize, T* o,
                                                  const QParams& q, int cw, int lane)
{
  using V = VT<T>;
  const int nv = osize / static_cast<int>(sizeof(T));
  if (cs == osize) {
    for (int e = cw * 32 + lane; e < nv; e += NW * 32) {
      if constexpr (sizeof(T) == 4) o[e] = lds_u32_at_byte(stg, sft + 4 * e);
      else o[e] = lds_u64_at_byte(stg, sft + 8 * e);
    }
    return true;
  }
  const int ln_l = stg[sft + lane];
  const int bitsw = ln_l * V::VPS;
  const int tot = __reduce_add_sync(0xffffffffu, bitsw);
  bool ok = !__any_sync(0xffffffffu, ln_l > V::TB) && (34 + tot / 8 == cs);
  if (ok) {
    const int16_t tr = static_cast<int16_t>(stg[sft + cs - 2] | (stg[sft + cs - 1] << 8));
    ok = tr == osize;
  }
  if (!ok) return false;
  const uint32_t* const w = reinterpret_cast<const uint32_t*>(stg);
  static_assert(SC % NW == 0, "whole subchunks per warp");
  // full chunks (all but a stream's last) are unpacked without the per-value
  // bound test (f32 lossy decode +11 %); 64-bit chunks whose widths are all at
  // most 32 (typical of lossy streams) extract each value from two words
  // instead of three and dequantize it in 32-bit arithmetic (f64 lossy decode
  // +23 %, then +7-13 %).  A zero width needs no test: its mask is 0, and its
  // reads, like every extraction's, end within 12 bytes of a bit inside the
  // chunk's payload (at most 15 + 16383 + 10 bytes into a stage of 16384 + 64).
  auto unpack = [&](auto full, auto narrow) {
#pragma unroll
    for (int u = 0; u < SC / NW; ++u) {  // unrolled: the subchunks' load chains overlap
      const int i = cw + u * NW;
      const int ln = __shfl_sync(0xffffffffu, ln_l, i);
      const int base = 8 * sft + 256 + __reduce_add_sync(0xffffffffu, lane < i ? bitsw : 0);  // first bit of i
      const int k0 = i * V::VPS;
#pragma unroll
      for (int j = lane; j < V::VPS; j += 32) {
        if (decltype(full)::value || k0 + j < nv) {
          if constexpr (sizeof(T) == 8 && LOSSY && decltype(narrow)::value) {
            o[k0 + j] = dequant_fp_narrow(extract_bits32(w, base + j * ln, ln), q);
          } else {
            T e;
            if constexpr (sizeof(T) == 4 || decltype(narrow)::value) e = extract_bits32(w, base + j * ln, ln);
            else e = extract_bits64(w, base + j * ln, ln);
            o[k0 + j] = decode_value<LOSSY>(e, q);
          }
        }
      }
    }
  };
  if (sizeof(T) == 8 && __all_sync(0xffffffffu, ln_l <= 32)) {
    if (osize == CS) unpack(std::true_type{}, std::true_type{});
    else unpack(std::false_type{}, std::true_type{});
  } else {
    if (osize == CS) unpack(std::true_type{}, std::false_type{});
    else unpack(std::false_type{}, std::false_type{});
  }
  return true;
}

template <typename T, bool LOSSY, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_decode(const DecArgs a)
{
  using V = VT<T>;
  constexpr int NW = NT / 32;
  extern __shared__ __align__(128) uint8_t smem[];
  uint8_t* const stage0 = smem;
  DecMisc& m = *reinterpret_cast<DecMisc*>(smem + DEC_STAGES * STAGE_BYTES);

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const WsPhase ph = WsPhase::of(a.ws, a.flag_cap);  // self-resetting workspace
  uint64_t* const hdr = ph.hdr;
  uint64_t* const flags = ph.flags;

  // Speculation: when the caller states the output capacity and the stream's
  // length, the chunk count is usually ceil(capacity / CS), and this CTA's sizes
  // (the prefix before its range, and its range) are read while the header is
  // still on its way, instead of one dependent round trip after it.  Used only if
  // the header agrees; the reads stay inside the stated stream length.
  const long long g_chunks = a.out_cap > 0 ? (a.out_cap + CS - 1) / CS : -1;
  const bool spec = g_chunks > 0 && g_chunks <= DEC_DIRECT_MAX && a.in_len >= 8 + 2 * g_chunks;
  long long s_pre = 0;  // this thread's share of the sizes before the range
  int s_cs = -1;        // this thread's size in the range (ranges of at most NT chunks)
  {
    const uint16_t* const sz = reinterpret_cast<const uint16_t*>(a.in + 8);
    if (spec) {
      const long long kg = (g_chunks + gridDim.x - 1) / gridDim.x;
      const long long c0g = min(static_cast<long long>(blockIdx.x) * kg, g_chunks);
      const long long c1g = min(c0g + kg, g_chunks);
      if (kg <= NT && c0g + tid < c1g) s_cs = sz[c0g + tid];
      const unsigned long long* const s8 = reinterpret_cast<const unsigned long long*>(sz);
      const long long q = c0g >> 2;
      for (long long k = tid; k < q; k += NT) {
        const unsigned long long v = s8[k];
        const unsigned long long p2 = (v & 0x0000ffff0000ffffull) + ((v >> 16) & 0x0000ffff0000ffffull);
        s_pre += static_cast<long long>((p2 & 0xffffffffull) + (p2 >> 32));
      }
      for (long long c = (q << 2) + tid; c < c0g; c += NT) s_pre += sz[c];
    }
  }

  // header checks (every CTA reads the 8-byte header)
  const long long insize = *reinterpret_cast<const long long*>(a.in);
  const long long chunks = insize > 0 ? (insize + CS - 1) / CS : 0;
  bool hdr_ok = insize >= 0 && (insize % static_cast<long long>(sizeof(T))) == 0;
  if (a.in_len >= 0 && 8 + 2 * chunks > a.in_len) hdr_ok = false;
  const bool cap_ok = a.out_cap < 0 || insize <= a.out_cap;
  const long long payload_len = a.in_len >= 0 ? a.in_len - 8 - 2 * chunks : -1;
  const uint16_t* const size_in = reinterpret_cast<const uint16_t*>(a.in + 8);
  const uint8_t* const data_in = a.in + 8 + 2 * chunks;

  if (tid == 0) {
    for (int st = 0; st < DEC_STAGES; ++st) {
      mbar_init(&m.full[st], 1);
      mbar_init(&m.empty[st], NW);  // one arrival per warp
    }
    mbar_fence_init();
    // ranges placed by summing the size table wait on no other CTA, so the
    // block index orders them; the look-back needs ticket order (a CTA waits only
    // on CTAs that started before it)
    m.vb = hdr_ok && cap_ok && chunks <= DEC_DIRECT_MAX
               ? static_cast<long long>(blockIdx.x)
               : static_cast<long long>(atomicAdd(reinterpret_cast<unsigned long long*>(&a.ws[WS_TICKET]), 1ull));
    if (!hdr_ok) set_status(hdr, ST_CORRUPT, -1);
    else if (!cap_ok) set_status(hdr, ST_CAPACITY, -1);
  }
  __syncthreads();

  const bool go = hdr_ok && cap_ok;
  const long long vb = m.vb;
  const long long K = (chunks + gridDim.x - 1) / gridDim.x;
  const long long c0 = go ? min(vb * K, chunks) : 0;
  const long long c1 = go ? min(c0 + K, chunks) : 0;

  // ---- range aggregate + size-table validation ---------------------------------
  {
    const bool direct = go && chunks <= DEC_DIRECT_MAX;
    const bool hit = direct && spec && chunks == g_chunks;  // the speculative reads are this CTA's
    long long sum = 0, pre = 0;
    int bad = 0;
    if (hit && K <= NT) {
      if (c0 + tid < c1) {
        const int cs = s_cs;
        const long long c = c0 + tid;
        const int os = static_cast<int>(min(static_cast<long long>(CS), insize - c * CS));
        bad |= (cs > os) | (cs == 0) | ((cs < os) & (cs < 34));
        sum += cs;
      }
    } else {
      for (long long c = c0 + tid; c < c1; c += NT) {
        const int cs = size_in[c];
        const int os = static_cast<int>(min(static_cast<long long>(CS), insize - c * CS));
        bad |= (cs > os) | (cs == 0) | ((cs < os) & (cs < 34));
        sum += cs;
      }
    }
    if (hit) {
      pre = warp_sum(s_pre);
    } else if (direct) {
      // sizes [0, c0), four per 8-byte load (the table starts 8-byte aligned)
      const unsigned long long* const s8 = reinterpret_cast<const unsigned long long*>(size_in);
      const long long q = c0 >> 2;
      for (long long k = tid; k < q; k += NT) {
        const unsigned long long v = s8[k];
        const unsigned long long p2 = (v & 0x0000ffff0000ffffull) + ((v >> 16) & 0x0000ffff0000ffffull);
        pre += static_cast<long long>((p2 & 0xffffffffull) + (p2 >> 32));
      }
      for (long long c = (q << 2) + tid; c < c0; c += NT) pre += size_in[c];
      pre = warp_sum(pre);
    }
    sum = warp_sum(sum);
    bad = __any_sync(0xffffffffu, bad);
    if (lane == 0) {
      m.red[warp] = sum;
      m.pre[warp] = pre;
      m.bad[warp] = bad;
    }
    __syncthreads();
    if (warp == 0) {
      long long s2 = lane < NW ? m.red[lane] : 0;
      int b2 = lane < NW ? m.bad[lane] : 0;
      s2 = warp_sum(s2);
      b2 = __any_sync(0xffffffffu, b2);
      if (b2 && lane == 0) set_status(hdr, ST_CORRUPT, c0);
      long long excl = 0;
      if (direct) {
        excl = warp_sum(lane < NW ? m.pre[lane] : 0);
      } else {
        if (lane == 0)
          st_relaxed_u64(&flags[vb], (vb == 0 ? FLAG_INC : FLAG_AGG) | (static_cast<uint64_t>(s2) & FLAG_VAL));
      }
      if (!direct && vb > 0) {
        excl = lookback(flags, vb, 0, hdr);
        if (excl < 0) {
          if (lane == 0) set_status(hdr, ST_TIMEOUT, c0);
        }
        if (lane == 0)
          st_relaxed_u64(&flags[vb], FLAG_INC | (static_cast<uint64_t>(excl >= 0 ? excl + s2 : 0) & FLAG_VAL));
      }
      if (lane == 0) m.excl = b2 ? -1 : excl;
    }
    __syncthreads();
  }

  const long long excl = m.excl;
  if (excl >= 0 && c0 < c1) {
    // producer state (warp 0): offsets and sizes of a window of 32 chunks
    long long wbase = -64, woff = 0, run = excl;
    int wcs = 0;
    auto issue = [&](long long c, int stg) {  // warp 0, warp-uniform
      if (c - wbase >= 32) {
        wbase = c;
        const long long cc = c + lane;
        const int cs = cc < c1 ? static_cast<int>(size_in[cc]) : 0;
        long long incl = cs;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const long long t = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += t;
        }
        woff = run + incl - cs;
        wcs = cs;
        run += __shfl_sync(0xffffffffu, incl, 31);
      }
      const int l = static_cast<int>(c - wbase);
      const long long off = __shfl_sync(0xffffffffu, woff, l);
      const int cs = __shfl_sync(0xffffffffu, wcs, l);
      if (lane == 0) {
        const uint8_t* src = data_in + off;
        const int sft = static_cast<int>(reinterpret_cast<uintptr_t>(src) & 15u);
        const uint32_t nb = static_cast<uint32_t>((sft + cs + 15) & ~15);
        const bool ok = cs >= 1 && cs <= CS && (payload_len < 0 || off + cs <= payload_len);
        DecChunk& d = m.info[stg];
        d.c = c;
        d.off = off;
        d.cs = cs;
        d.sft = sft;
        d.ok = ok;
        if (ok) {
          mbar_arrive_expect_tx(&m.full[stg], nb);
          tma_load_1d(stage0 + stg * STAGE_BYTES, src - sft, nb, &m.full[stg]);
        } else {
          mbar_arrive(&m.full[stg]);
        }
      }
    };

    // Warp 0 keeps DEC_STAGES - 1 chunks in flight: at chunk it it issues chunk
    // it + DEC_STAGES - 1 into the stage of chunk it - 1, once every warp has
    // released that stage.  No CTA barrier per chunk: each warp waits for its
    // stages itself and releases them with its own arrival; a wait that gives up
    // ends that warp's loop (the others end by their own bounded waits).
    long long issued = c0;   // next chunk warp 0 issues
    bool feeding = true;     // warp 0 still issues
    auto issue_next = [&]() {  // warp 0, warp-uniform
      const int jt = static_cast<int>(issued - c0);
      const int st = jt % DEC_STAGES;
      if (jt >= DEC_STAGES &&
          __any_sync(0xffffffffu, !mbar_wait_bounded(&m.empty[st], ((jt - DEC_STAGES) / DEC_STAGES) & 1))) {
        if (lane == 0) set_status(hdr, ST_TIMEOUT, issued);
        feeding = false;
        return;
      }
      issue(issued, st);
      ++issued;
    };
    if (warp == 0)
      for (int k = 0; k < DEC_STAGES - 1 && issued < c1; ++k) issue_next();
    int it = 0;
    long long c = c0;
    for (; c < c1; ++c, ++it) {
      const int s = it % DEC_STAGES;
      uint8_t* const stg = stage0 + s * STAGE_BYTES;
      if (warp == 0 && feeding && issued < c1) issue_next();

      if (__any_sync(0xffffffffu, !mbar_wait_bounded(&m.full[s], (it / DEC_STAGES) & 1))) {
        if (lane == 0) set_status(hdr, ST_TIMEOUT, c);
        break;
      }

      const DecChunk d = m.info[s];
      const int osize = static_cast<int>(min(static_cast<long long>(CS), insize - c * CS));
      uint8_t* const outc = a.out + c * CS;
      if (!d.ok) {
        if (tid == 0) set_status(hdr, ST_CORRUPT, c);
      } else if (!decode_chunk_warp<T, LOSSY, NW>(stg, d.sft, d.cs, osize, reinterpret_cast<T*>(outc), a.q,
                                                    warp, lane)) {
        if (tid == 0) set_status(hdr, ST_CORRUPT, c);
      }
      // this warp is done with the stage (generic accesses ordered before the next TMA write)
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&m.empty[s]);
    }
    // never leave with a bulk copy still landing in this CTA's shared memory:
    // warp 0 waits for the chunks it issued but did not consume
    if (warp == 0 && lane == 0) {
      for (long long k = c; k < issued; ++k) {
        const int jt = static_cast<int>(k - c0);
        mbar_wait_bounded(&m.full[jt % DEC_STAGES], (jt / DEC_STAGES) & 1);
      }
    }
  }

  // this CTA's share of the flags the previous launch left in the other region
  // (off the start of the kernel: only the next launch reads them)
  if (warp == NW - 1) ph.clear_other_share(lane);

  // ---- epilogue ------------------------------------------------------------------
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    const unsigned long long dn = atomicAdd(reinterpret_cast<unsigned long long*>(&a.ws[WS_DONE]), 1ull);
    if (dn == gridDim.x - 1) {
      __threadfence();
      const unsigned long long st = ld_relaxed_u64(&hdr[WS_STATUS]);
      *a.outsize = st ? -static_cast<long long>(st) : insize;
      ph.finish(a.ws, gridDim.x);
    }
  }
}

// ============================================================================
// batched decode: a prepass places every chunk, then a persistent kernel with a
// producer warp and 8 compute warps decodes chunks in any order
// ============================================================================
constexpr int DB_STAGES = 4;
constexpr int DB_CW = 8;
constexpr int DB_NT = (DB_CW + 1) * 32;
constexpr int DB_MINB = 3;

struct DecBMeta {
  long long g;      // chunk id across the launch, or NO_CHUNK
  uint8_t* out;     // where the chunk's values go
  QParams q;
  int kind;         // bit 0: 64-bit values, bit 1: lossy
  int osize;
  int cs;
  int sft;          // byte offset of the chunk within the staged copy
  int state;        // 0: nothing to decode, 1: decode
  int pad_;
};

struct DecBMisc {
  uint64_t full[DB_STAGES];
  uint64_t empty[DB_STAGES];
  DecBMeta meta[DB_STAGES];
};

constexpr int DB_SMEM = DB_STAGES * STAGE_BYTES + ((sizeof(DecBMisc) + 127) / 128) * 128 + 8 * (BATCH_MAX_JOBS + 1);

// Prepass, one CTA per buffer: validates the header and size table and writes the
// byte offset of every chunk's payload (an exclusive scan of the sizes).
__global__ void __launch_bounds__(256) k_decode_prepass(const BatchDecArgs a)
{
  __shared__ long long wsum[8];
  __shared__ int wbad[8];
  const int j = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const BatchJob& job = a.jobs[j];
  const uint8_t* const in = job.in;
  const long long len = job.insize;  // stream bytes, -1 when unknown
  const int elem = (job.kind & 1) ? 8 : 4;
  long long insize = (len < 0 || len >= 8) ? *reinterpret_cast<const long long*>(in) : -1;
  bool ok = insize >= 0 && insize % elem == 0 && insize <= job.cap;
  const long long chunks = ok ? (insize + CS - 1) / CS : 0;
  if (ok && len >= 0 && 8 + 2 * chunks > len) ok = false;
  if (!ok) {
    if (tid == 0) set_status(a.ws, insize > job.cap ? ST_CAPACITY : ST_CORRUPT, j);
    return;
  }
  const uint16_t* const size_in = reinterpret_cast<const uint16_t*>(in + 8);
  long long* const offs = a.offsets + a.chunk_base[j];
  long long carry = 0;
  int bad = 0;
  for (long long b = 0; b < chunks; b += 256) {
    const long long c = b + tid;
    int cs = 0;
    if (c < chunks) {
      cs = size_in[c];
      const int os = static_cast<int>(min(static_cast<long long>(CS), insize - c * CS));
      bad |= (cs > os) | (cs == 0) | ((cs < os) & (cs < 34));
    }
    long long incl = cs;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    long long before = carry;
    for (int w = 0; w < warp; ++w) before += wsum[w];
    if (c < chunks) offs[c] = before + incl - cs;
    long long tile = 0;
    for (int w = 0; w < 8; ++w) tile += wsum[w];
    carry += tile;
    __syncthreads();
  }
  bad = __any_sync(0xffffffffu, bad);
  if (lane == 0) wbad[warp] = bad;
  __syncthreads();
  if (tid == 0) {
    int any = 0;
    for (int w = 0; w < 8; ++w) any |= wbad[w];
    if (any || (len >= 0 && 8 + 2 * chunks + carry > len)) {
      set_status(a.ws, ST_CORRUPT, j);
    } else {
      a.actual[j] = chunks;
      a.actual_insize[j] = insize;
      *job.outsize = insize;
    }
  }
}

__global__ void __launch_bounds__(DB_NT, DB_MINB) k_decode_batch(const BatchDecArgs a)
{
  extern __shared__ __align__(128) uint8_t smem[];
  uint8_t* const stage0 = smem;
  DecBMisc& m = *reinterpret_cast<DecBMisc*>(smem + DB_STAGES * STAGE_BYTES);
  long long* const cb = reinterpret_cast<long long*>(smem + DB_STAGES * STAGE_BYTES +
                                                     ((sizeof(DecBMisc) + 127) / 128) * 128);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint64_t* const ws = a.ws;
  for (int i = tid; i <= a.njobs; i += DB_NT) cb[i] = a.chunk_base[i];
  if (tid == 0) {
    for (int s = 0; s < DB_STAGES; ++s) {
      mbar_init(&m.full[s], 1);
      mbar_init(&m.empty[s], DB_CW);  // one arrival per compute warp
    }
    mbar_fence_init();
  }
  __syncthreads();
  const long long total = cb[a.njobs];
  const bool failed_before = ld_relaxed_u64(&ws[WS_STATUS]) != 0ull;  // the prepass found an error

  if (warp == DB_CW) {
    // ===================== producer warp (lane 0 works, the warp follows) =====================
    unsigned long long* const tick = reinterpret_cast<unsigned long long*>(&ws[WS_TICKET]);
    unsigned issued = 0, issued_par = 0;
    for (int seq = 0;; ++seq) {
      const int s = seq % DB_STAGES;
      if (seq >= DB_STAGES) {
        const bool ok = mbar_wait_bounded(&m.empty[s], ((seq - DB_STAGES) / DB_STAGES) & 1);
        if (__any_sync(0xffffffffu, !ok)) {
          if (lane == 0) set_status(ws, ST_TIMEOUT, -1);
          break;
        }
      }
      long long t = NO_CHUNK;
      if (lane == 0 && !failed_before) t = static_cast<long long>(atomicAdd(tick, 1ull));
      t = __shfl_sync(0xffffffffu, t, 0);
      if (lane == 0) {
        DecBMeta& d = m.meta[s];
        bool copy = false;
        if (t < total) {
          int lo = 0, hi = a.njobs - 1;
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (cb[mid] <= t) lo = mid;
            else hi = mid - 1;
          }
          const BatchJob& job = a.jobs[lo];
          const long long c = t - cb[lo];
          const long long chunks = a.actual[lo];
          d.g = t;
          d.state = 0;
          if (c < chunks) {
            const long long insize = a.actual_insize[lo];
            const uint8_t* const data_in = job.in + 8 + 2 * chunks;
            const long long off = a.offsets[t];
            const int cs = reinterpret_cast<const uint16_t*>(job.in + 8)[c];
            const uint8_t* const src = data_in + off;
            const int sft = static_cast<int>(reinterpret_cast<uintptr_t>(src) & 15u);
            d.out = job.out + c * CS;
            d.q = job.q;
            d.kind = job.kind;
            d.osize = static_cast<int>(min(static_cast<long long>(CS), insize - c * CS));
            d.cs = cs;
            d.sft = sft;
            d.state = 1;
            const uint32_t nb = static_cast<uint32_t>((sft + cs + 15) & ~15);
            mbar_arrive_expect_tx(&m.full[s], nb);
            tma_load_1d(stage0 + s * STAGE_BYTES, src - sft, nb, &m.full[s]);
            copy = true;
          }
        } else {
          d.g = NO_CHUNK;
        }
        if (copy) {
          issued |= 1u << s;
          issued_par = (issued_par & ~(1u << s)) | (((seq / DB_STAGES) & 1u) << s);
        } else {
          issued &= ~(1u << s);
          mbar_arrive(&m.full[s]);
        }
      }
      __syncwarp();
      if (t >= total) break;
    }
    if (lane == 0) {
      for (int s = 0; s < DB_STAGES; ++s)
        if (issued & (1u << s)) mbar_wait_bounded(&m.full[s], (issued_par >> s) & 1u);
    }
  } else {
    // ===================== compute warps =====================
    // No CTA barrier: each warp waits for a stage itself, decodes its share of the
    // chunk and frees the stage with its own arrival.  A wait that gives up ends
    // this warp's loop; the others and the producer end by their own bounded waits.
    for (int seq = 0;; ++seq) {
      const int s = seq % DB_STAGES;
      if (__any_sync(0xffffffffu, !mbar_wait_bounded(&m.full[s], (seq / DB_STAGES) & 1))) {
        if (lane == 0) set_status(ws, ST_TIMEOUT, -1);
        break;
      }
      const DecBMeta& d = m.meta[s];
      if (d.g == NO_CHUNK) break;
      if (d.state == 1) {
        const uint8_t* const stg = stage0 + s * STAGE_BYTES;
        bool ok;
        switch (d.kind) {
          case 0: ok = decode_chunk_warp<uint32_t, false, DB_CW>(stg, d.sft, d.cs, d.osize,
                                                                 reinterpret_cast<uint32_t*>(d.out), d.q, warp, lane); break;
          case 1: ok = decode_chunk_warp<uint64_t, false, DB_CW>(stg, d.sft, d.cs, d.osize,
                                                                 reinterpret_cast<uint64_t*>(d.out), d.q, warp, lane); break;
          case 2: ok = decode_chunk_warp<uint32_t, true, DB_CW>(stg, d.sft, d.cs, d.osize,
                                                                reinterpret_cast<uint32_t*>(d.out), d.q, warp, lane); break;
          default: ok = decode_chunk_warp<uint64_t, true, DB_CW>(stg, d.sft, d.cs, d.osize,
                                                                 reinterpret_cast<uint64_t*>(d.out), d.q, warp, lane); break;
        }
        if (!ok && warp == 0 && lane == 0) set_status(ws, ST_CORRUPT, d.g);
      }
      // this warp is done with the stage (generic accesses ordered before the next TMA write)
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&m.empty[s]);
    }
  }

  // ---- epilogue: an error anywhere turns every size into -status ---------------
  __syncthreads();
  __shared__ int last_cta;
  if (tid == 0) {
    __threadfence();
    const unsigned long long dn = atomicAdd(reinterpret_cast<unsigned long long*>(&ws[WS_DONE]), 1ull);
    last_cta = dn == gridDim.x - 1;
    if (last_cta) __threadfence();
  }
  __syncthreads();
  if (last_cta) {
    const unsigned long long st = ld_relaxed_u64(&ws[WS_STATUS]);
    if (st)
      for (int i = tid; i < a.njobs; i += DB_NT) *a.jobs[i].outsize = -static_cast<long long>(st);
  }
}

// ============================================================================
// launchers
// ============================================================================
// Sets the dynamic shared memory limit of `k` once per device.
template <typename K>
static cudaError_t ensure_smem_attr(K k, int bytes, unsigned long long* done_mask)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = 1ull << (dev & 63);
  if (__atomic_load_n(done_mask, __ATOMIC_ACQUIRE) & bit) return cudaSuccess;
  e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) __atomic_fetch_or(done_mask, bit, __ATOMIC_RELEASE);
  return e;
}

// Decode launch shapes: threads per CTA and the CTAs per SM the registers are
// budgeted for (index = the C ABI's shape number).
template <int NT_, int MINB_>
struct DecShape {
  static constexpr int NT = NT_;
  static constexpr int MINB = MINB_;
};
using DecShape0 = DecShape<256, 4>;  // default
using DecShape1 = DecShape<128, 6>;
using DecShape2 = DecShape<512, 2>;
constexpr int DEC_SHAPES = 3;

template <int KIND, class S>
static cudaError_t launch_enc_k(const EncArgs& a, int grid, cudaStream_t st)
{
  auto k = k_encode<KIND, false, S>;
  static unsigned long long attr = 0;
  cudaError_t e = ensure_smem_attr(k, enc_smem<S>(), &attr);
  if (e != cudaSuccess) return e;
  k<<<grid, S::NT, enc_smem<S>(), st>>>(a);
  return cudaGetLastError();
}

template <int KIND, class S>
static int enc_occupancy()
{
  auto k = k_encode<KIND, false, S>;
  // the smem attribute must be set before the occupancy query counts dynamic smem
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, enc_smem<S>());
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, S::NT, enc_smem<S>());
  return n;
}

template <typename T, bool LOSSY, class S>
static cudaError_t launch_dec_k(const DecArgs& a, int grid, cudaStream_t st)
{
  auto k = k_decode<T, LOSSY, S::NT, S::MINB>;
  static unsigned long long attr = 0;
  cudaError_t e = ensure_smem_attr(k, DEC_SMEM, &attr);
  if (e != cudaSuccess) return e;
  k<<<grid, S::NT, DEC_SMEM, st>>>(a);
  return cudaGetLastError();
}

template <typename T, bool LOSSY, class S>
static int dec_occupancy()
{
  auto k = k_decode<T, LOSSY, S::NT, S::MINB>;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, DEC_SMEM);
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, S::NT, DEC_SMEM);
  return n;
}

template <int KIND>
static cudaError_t launch_enc_kind(int shape, const EncArgs& a, int grid, cudaStream_t st)
{
  switch (shape) {
    case 1: return launch_enc_k<KIND, EncShape1>(a, grid, st);
    case 2: return launch_enc_k<KIND, EncShape2>(a, grid, st);
    case 3: return launch_enc_k<KIND, EncShape3>(a, grid, st);
    case 4: return launch_enc_k<KIND, EncShape4>(a, grid, st);
    default: return launch_enc_k<KIND, EncShape0>(a, grid, st);
  }
}

template <int KIND>
static int enc_occupancy_kind(int shape)
{
  switch (shape) {
    case 1: return enc_occupancy<KIND, EncShape1>();
    case 2: return enc_occupancy<KIND, EncShape2>();
    case 3: return enc_occupancy<KIND, EncShape3>();
    case 4: return enc_occupancy<KIND, EncShape4>();
    default: return enc_occupancy<KIND, EncShape0>();
  }
}

template <typename T, bool LOSSY>
static cudaError_t launch_dec_kind(int shape, const DecArgs& a, int grid, cudaStream_t st)
{
  switch (shape) {
    case 1: return launch_dec_k<T, LOSSY, DecShape1>(a, grid, st);
    case 2: return launch_dec_k<T, LOSSY, DecShape2>(a, grid, st);
    default: return launch_dec_k<T, LOSSY, DecShape0>(a, grid, st);
  }
}

template <typename T, bool LOSSY>
static int dec_occupancy_kind(int shape)
{
  switch (shape) {
    case 1: return dec_occupancy<T, LOSSY, DecShape1>();
    case 2: return dec_occupancy<T, LOSSY, DecShape2>();
    default: return dec_occupancy<T, LOSSY, DecShape0>();
  }
}

cudaError_t launch_encode(int width, bool lossy, int shape, const EncArgs& a, int grid, cudaStream_t st)
{
  if (width == 4) return lossy ? launch_enc_kind<2>(shape, a, grid, st) : launch_enc_kind<0>(shape, a, grid, st);
  return lossy ? launch_enc_kind<3>(shape, a, grid, st) : launch_enc_kind<1>(shape, a, grid, st);
}

cudaError_t launch_decode(int width, bool lossy, int shape, const DecArgs& a, int grid, cudaStream_t st)
{
  if (width == 4)
    return lossy ? launch_dec_kind<uint32_t, true>(shape, a, grid, st) : launch_dec_kind<uint32_t, false>(shape, a, grid, st);
  return lossy ? launch_dec_kind<uint64_t, true>(shape, a, grid, st) : launch_dec_kind<uint64_t, false>(shape, a, grid, st);
}

int blocks_per_sm(int width, bool lossy, bool enc, int shape)
{
  if (enc) {
    if (width == 4) return lossy ? enc_occupancy_kind<2>(shape) : enc_occupancy_kind<0>(shape);
    return lossy ? enc_occupancy_kind<3>(shape) : enc_occupancy_kind<1>(shape);
  }
  if (width == 4) return lossy ? dec_occupancy_kind<uint32_t, true>(shape) : dec_occupancy_kind<uint32_t, false>(shape);
  return lossy ? dec_occupancy_kind<uint64_t, true>(shape) : dec_occupancy_kind<uint64_t, false>(shape);
}

ShapeInfo shape_info(bool enc, int shape)
{
  ShapeInfo r{};
  if (enc) {
    switch (shape) {
      case 1: r = {EncShape1::NT, EncShape1::CW, EncShape1::ST, EncShape1::MINB}; break;
      case 2: r = {EncShape2::NT, EncShape2::CW, EncShape2::ST, EncShape2::MINB}; break;
      case 3: r = {EncShape3::NT, EncShape3::CW, EncShape3::ST, EncShape3::MINB}; break;
      case 4: r = {EncShape4::NT, EncShape4::CW, EncShape4::ST, EncShape4::MINB}; break;
      default: r = {EncShape0::NT, EncShape0::CW, EncShape0::ST, EncShape0::MINB}; break;
    }
  } else {
    switch (shape) {
      case 1: r = {DecShape1::NT, DecShape1::NT / 32, DEC_STAGES, DecShape1::MINB}; break;
      case 2: r = {DecShape2::NT, DecShape2::NT / 32, DEC_STAGES, DecShape2::MINB}; break;
      default: r = {DecShape0::NT, DecShape0::NT / 32, DEC_STAGES, DecShape0::MINB}; break;
    }
  }
  return r;
}

int shape_count(bool enc) { return enc ? ENC_SHAPES : DEC_SHAPES; }

cudaError_t launch_encode_batch(const BatchEncArgs& a, int grid, cudaStream_t st)
{
  using S = EncShape0;
  auto k = k_encode<-1, true, S>;
  static unsigned long long attr = 0;
  cudaError_t e = ensure_smem_attr(k, enc_batch_smem<S>(), &attr);
  if (e != cudaSuccess) return e;
  k<<<grid, S::NT, enc_batch_smem<S>(), st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_decode_batch(const BatchDecArgs& a, int grid, cudaStream_t st)
{
  k_decode_prepass<<<a.njobs, 256, 0, st>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  static unsigned long long attr = 0;
  e = ensure_smem_attr(k_decode_batch, DB_SMEM, &attr);
  if (e != cudaSuccess) return e;
  k_decode_batch<<<grid, DB_NT, DB_SMEM, st>>>(a);
  return cudaGetLastError();
}

int decode_batch_blocks_per_sm()
{
  cudaFuncSetAttribute(k_decode_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, DB_SMEM);
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_decode_batch, DB_NT, DB_SMEM);
  return n;
}

int encode_batch_blocks_per_sm()
{
  using S = EncShape0;
  cudaFuncSetAttribute(k_encode<-1, true, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, enc_batch_smem<S>());
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_encode<-1, true, S>, S::NT, enc_batch_smem<S>());
  return n;
}

}  // namespace sleek

// sleek_kernels.cu -- sm_100a encode / decode kernels for one buffer.
//
// Encode (replaces d_encode, include/sleek_common_gpu.h:474-559, 989-1074 of the
// reference): persistent CTAs take 16 KB chunks by atomic ticket, in order.  A
// chunk arrives in shared memory by a 1-D TMA bulk copy issued one chunk ahead;
// warps transform a subchunk each (value arithmetic restated from the reference)
// and take the bit width from a warp max; warp 0 scans the widths, publishes the
// chunk's compressed size and runs a bounded decoupled look-back while the other
// warps pack the chunk in gather form (each thread assembles whole 64-bit words,
// no shared atomics); finally all threads store the chunk at its byte offset with
// 16-byte vector stores.  A chunk whose encoding is not smaller than its input is
// stored raw straight from the staged copy (never re-read from HBM).
//
// Decode (replaces d_decode, :688-768, 1199-1279): CTAs take contiguous chunk
// ranges in ticket order, sum their ranges' compressed sizes, look back over the
// preceding ranges once, then stream their chunks through a two-stage TMA
// pipeline (each copy is the 16-byte aligned superset of the chunk's bytes) and
// unpack with funnel shifts straight into coalesced global stores.  Malformed
// streams set an error status instead of trapping.
#include "sleek_device.cuh"
#include "sleek_launch.h"

namespace sleek {

constexpr int ENC_STAGES = 4;
constexpr int ENC_CW = 8;                    // compute warps
constexpr int ENC_NT = (ENC_CW + 2) * 32;    // + a producer warp and a scanner warp
constexpr int ENC_MINB = 3;
constexpr long long NO_CHUNK = 0x7fffffffffffffffll;

struct EncMeta {
  long long c;     // chunk id, or NO_CHUNK: no more work for this CTA
  long long excl;  // byte offset of the chunk's payload (or -1 after an error)
  int osize;
  int csize;
  int comp;
  int pad_;
};

struct EncMisc {
  uint64_t full[ENC_STAGES];    // chunk bytes landed (TMA tx count)
  uint64_t empty[ENC_STAGES];   // go-ahead for the stage's next copy (its previous chunk is stored)
  uint64_t sized[ENC_STAGES];   // compressed size of the stage's chunk known
  uint64_t placed[ENC_STAGES];  // payload offset of the stage's chunk known
  EncMeta meta[ENC_STAGES];
  int lnv[SC];
};

constexpr int ENC_SMEM = ENC_STAGES * STAGE_BYTES + ((sizeof(EncMisc) + 127) / 128) * 128;

// barrier among the compute warps only (named barrier 1)
__device__ __forceinline__ void cbar()
{
  asm volatile("bar.sync 1, %0;" ::"n"(ENC_CW * 32) : "memory");
}

__device__ __forceinline__ bool cbar_or(bool pred)
{
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"(static_cast<uint32_t>(pred)), "n"(ENC_CW * 32)
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
    // short runs: several lanes share a word; clear the words, then OR in
    const int words = (32 * P * ln) >> 5;
    for (int q = lane; q < words; q += 32) pw[q] = 0u;
    __syncwarp();
    uint32_t run = 0;
#pragma unroll
    for (int k = 0; k < P; ++k) run |= static_cast<uint32_t>(v[k]) << (k * ln);
    const uint64_t sh = static_cast<uint64_t>(run) << s;
    if (static_cast<uint32_t>(sh)) atomicOr(&pw[w0], static_cast<uint32_t>(sh));
    if (static_cast<uint32_t>(sh >> 32)) atomicOr(&pw[w0 + 1], static_cast<uint32_t>(sh >> 32));
  }
}

template <typename T, bool LOSSY, int MINB>
__global__ void __launch_bounds__(ENC_NT, MINB) k_encode(const EncArgs a)
{
  using V = VT<T>;
  constexpr int P = 16 / static_cast<int>(sizeof(T));  // values per lane per subchunk
  constexpr int SPW = SC / ENC_CW;                      // subchunks per compute warp
  extern __shared__ __align__(128) uint8_t smem[];
  uint8_t* const stage0 = smem;
  EncMisc& m = *reinterpret_cast<EncMisc*>(smem + ENC_STAGES * STAGE_BYTES);

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const long long chunks = (a.insize + CS - 1) / CS;
  uint64_t* const ws = a.ws;
  uint64_t* const flags = ws + WS_HDR_WORDS;
  uint8_t* const size_out = a.out + 8;
  uint8_t* const data_out = a.out + 8 + 2 * chunks;
  const bool in_aligned = (reinterpret_cast<uintptr_t>(a.in) & 15u) == 0u;

  if (tid == 0) {
    for (int s = 0; s < ENC_STAGES; ++s) {
      mbar_init(&m.full[s], 1);
      mbar_init(&m.empty[s], 1);
      mbar_init(&m.sized[s], 1);
      mbar_init(&m.placed[s], 1);
    }
    mbar_fence_init();
  }
  __syncthreads();

  if (warp == ENC_CW) {
    // ===================== producer warp: tickets and TMA copies =====================
    // Tickets are taken just before their chunk's copy is issued, never earlier:
    // a ticket held long before its chunk is processed makes every later chunk's
    // look-back wait for it.
    unsigned long long* const tick = reinterpret_cast<unsigned long long*>(&ws[WS_TICKET]);
    unsigned issued = 0;      // stages whose last use was a TMA copy (lane 0's view)
    unsigned issued_par = 0;  // parity of that use
    bool more = true;
    for (int seq = 0;; ++seq) {
      const int s = seq % ENC_STAGES;
      // From seq 2 on, the copy for chunk seq is issued when the compute warps
      // start chunk seq - 1: one chunk of lookahead, and the stage's previous
      // chunk (seq - 4) has been stored by then.
      if (seq >= 2) {
        const bool ok = mbar_wait_bounded(&m.empty[s], ((seq - 2) / ENC_STAGES) & 1);
        if (__any_sync(0xffffffffu, !ok)) {
          if (lane == 0) set_status(ws, ST_TIMEOUT, -1);
          break;
        }
      }
      long long t = NO_CHUNK;
      if (lane == 0 && more) t = static_cast<long long>(atomicAdd(tick, 1ull));
      t = __shfl_sync(0xffffffffu, t, 0);
      uint8_t* const stg = stage0 + s * STAGE_BYTES;
      if (t < chunks) {
        const long long base = t * CS;
        const int osize = static_cast<int>(min(static_cast<long long>(CS), a.insize - base));
        if (in_aligned && osize == CS) {
          if (lane == 0) {
            m.meta[s].c = t;
            mbar_arrive_expect_tx(&m.full[s], CS);
            tma_load_1d(stg, a.in + base, CS, &m.full[s]);
            issued |= 1u << s;
            issued_par = (issued_par & ~(1u << s)) | (((seq / ENC_STAGES) & 1u) << s);
          }
        } else {
          // last partial chunk or an input that is not 16-byte aligned: element
          // loads, zero padding up to the full chunk (the padding is encoded too)
          const int elem = static_cast<int>(sizeof(T));
          const T* const gin = reinterpret_cast<const T*>(a.in + base);
          T* const sv = reinterpret_cast<T*>(stg);
          for (int k = lane; k < CS / elem; k += 32) sv[k] = k * elem < osize ? gin[k] : T(0);
          __syncwarp();
          if (lane == 0) {
            m.meta[s].c = t;
            issued &= ~(1u << s);
            mbar_arrive(&m.full[s]);  // release: the stores above are visible to its waiters
          }
        }
      } else {
        more = false;
        if (lane == 0) {
          m.meta[s].c = NO_CHUNK;
          issued &= ~(1u << s);
          mbar_arrive(&m.full[s]);
        }
      }
      if (!more) break;
    }
    // never leave with a bulk copy still landing in this CTA's shared memory
    if (lane == 0) {
      for (int s = 0; s < ENC_STAGES; ++s)
        if (issued & (1u << s)) mbar_wait_bounded(&m.full[s], (issued_par >> s) & 1u);
    }
  } else if (warp == ENC_CW + 1) {
    // ===================== scanner warp: decoupled look-back =====================
    for (int seq = 0;; ++seq) {
      const int s = seq % ENC_STAGES;
      const uint32_t par = (seq / ENC_STAGES) & 1;
      bool ok = mbar_wait_bounded(&m.full[s], par);
      if (__any_sync(0xffffffffu, !ok)) break;  // the compute warps report it
      const long long c = m.meta[s].c;
      if (c == NO_CHUNK) break;
      ok = mbar_wait_bounded(&m.sized[s], par);
      if (__any_sync(0xffffffffu, !ok)) {
        if (lane == 0) set_status(ws, ST_TIMEOUT, c);
        break;
      }
      const int csize = m.meta[s].csize;
      long long excl = 0;
      if (c > 0) {
        excl = lookback(flags, c, 0, ws);
        unsigned err = 0;
        if (excl < 0) err = ST_TIMEOUT;
        else if (excl > c * CS) err = ST_CAPACITY;
        if (err) excl = -1;
        if (lane == 0) {
          if (err) set_status(ws, err, c);
          // an impossible prefix is replaced by the largest legal one so that
          // every later chunk still writes inside the output bound
          st_relaxed_u64(&flags[c], FLAG_INC | static_cast<uint64_t>(excl >= 0 ? excl + csize : (c + 1) * CS));
        }
      }
      if (lane == 0) {
        m.meta[s].excl = excl;
        if (c == chunks - 1 && excl >= 0) ws[WS_TOTAL] = static_cast<uint64_t>(excl + csize);
        mbar_arrive(&m.placed[s]);
      }
    }
  } else {
    // ===================== compute warps =====================
    const int cw = warp;
    auto store = [&](int sq) {  // all compute threads; placed[] already observed
      const int sp = sq % ENC_STAGES;
      const EncMeta me = m.meta[sp];
      if (me.excl >= 0) {
        store_shifted<ENC_CW * 32>(data_out + me.excl, stage0 + sp * STAGE_BYTES, me.csize);
        if (tid == 0) *reinterpret_cast<uint16_t*>(size_out + 2 * me.c) = static_cast<uint16_t>(me.csize);
      }
    };

    int seq = 0;
    bool failed = false;
    for (;; ++seq) {
      const int s = seq % ENC_STAGES;
      bool ok = mbar_wait_bounded(&m.full[s], (seq / ENC_STAGES) & 1);
      if (seq >= 2) ok = mbar_wait_bounded(&m.placed[(seq - 2) % ENC_STAGES], ((seq - 2) / ENC_STAGES) & 1) && ok;
      if (cbar_or(!ok)) {
        if (tid == 0) set_status(ws, ST_TIMEOUT, -1);
        failed = true;
        break;
      }
      // start of chunk seq: the producer may copy chunk seq + 1 into the stage of
      // seq - 3, whose store every compute warp has finished
      if (seq >= 1 && tid == 0) mbar_arrive(&m.empty[(seq + 1) % ENC_STAGES]);
      const long long c = m.meta[s].c;
      if (c == NO_CHUNK) break;
      uint8_t* const stg = stage0 + s * STAGE_BYTES;

      // ---- phase A: values into registers, transform / quantize, bit widths ----
      // (the stage always holds a full 16 KB chunk: partial chunks are zero padded)
      const long long base = c * CS;
      const int osize = static_cast<int>(min(static_cast<long long>(CS), a.insize - base));
      T vals[SPW][P];
#pragma unroll
      for (int u = 0; u < SPW; ++u) {
        const int i = cw + u * ENC_CW;
        const uint4 q = *reinterpret_cast<const uint4*>(stg + i * 512 + lane * 16);
        if constexpr (sizeof(T) == 4) {
          vals[u][0] = q.x; vals[u][1] = q.y; vals[u][2] = q.z; vals[u][3] = q.w;
        } else {
          vals[u][0] = (static_cast<uint64_t>(q.y) << 32) | q.x;
          vals[u][1] = (static_cast<uint64_t>(q.w) << 32) | q.z;
        }
        T orv = 0;
#pragma unroll
        for (int p = 0; p < P; ++p) {
          vals[u][p] = encode_value<LOSSY>(vals[u][p], a.q);
          orv |= vals[u][p];
        }
        const int w = warp_bit_width(orv);
        if (lane == 0) m.lnv[i] = w;
      }
      cbar();

      // ---- widths scan (every warp, redundantly), size decision ---------------
      const int ln_l = m.lnv[lane];
      const int wc = (V::VPS * ln_l) >> 5;  // 32-bit words of subchunk `lane`
      int incl = wc;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      const int wtot = __shfl_sync(0xffffffffu, incl, 31);
      const int newsize = 34 + 4 * wtot;
      const bool comp = newsize < osize;
      const int csize = comp ? newsize : osize;
      if (tid == 0) {
        m.meta[s].osize = osize;
        m.meta[s].csize = csize;
        m.meta[s].comp = comp;
        st_relaxed_u64(&flags[c], (c == 0 ? FLAG_INC : FLAG_AGG) | static_cast<uint64_t>(csize));
        mbar_arrive(&m.sized[s]);
      }

      // ---- pack this chunk from registers --------------------------------------
      if (comp) {
        uint32_t* const pw = reinterpret_cast<uint32_t*>(stg + 32);
#pragma unroll
        for (int u = 0; u < SPW; ++u) {
          const int i = cw + u * ENC_CW;
          const int wbase = __shfl_sync(0xffffffffu, incl - wc, i);
          const int ln = __shfl_sync(0xffffffffu, ln_l, i);
          pack_subchunk<T>(pw + wbase, ln, vals[u], lane);
        }
        if (cw == 0) {
          stg[lane] = static_cast<uint8_t>(ln_l);
          if (lane == 0) *reinterpret_cast<int16_t*>(stg + 32 + 4 * wtot) = static_cast<int16_t>(osize);
        }
      }

      // ---- store the chunk of seq - 2 (its offset is known) ---------------------
      if (seq >= 2) store(seq - 2);
      fence_proxy_async_smem();  // generic accesses of this iteration before later TMA writes
    }
    if (!failed) {
      // drain: chunks seq - 2 (placed already observed) and seq - 1
      if (seq >= 2) store(seq - 2);
      if (seq >= 1) {
        const bool ok = mbar_wait_bounded(&m.placed[(seq - 1) % ENC_STAGES], ((seq - 1) / ENC_STAGES) & 1);
        if (!cbar_or(!ok)) store(seq - 1);
        else if (tid == 0) set_status(ws, ST_TIMEOUT, -1);
      }
    }
  }

  // ---- epilogue: the last CTA out writes the header and the stream size ------
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    const unsigned long long d = atomicAdd(reinterpret_cast<unsigned long long*>(&ws[WS_DONE]), 1ull);
    if (d == gridDim.x - 1) {
      __threadfence();
      const unsigned long long st = ld_relaxed_u64(&ws[WS_STATUS]);
      const long long total = chunks ? static_cast<long long>(ld_relaxed_u64(&ws[WS_TOTAL])) : 0ll;
      *reinterpret_cast<long long*>(a.out) = a.insize;
      *a.outsize = st ? -static_cast<long long>(st) : 8 + 2 * chunks + total;
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

struct DecMisc {
  uint64_t bar[2];
  DecChunk info[2];
  long long excl;
  long long vb;
  long long red[NT_MAX_WARPS];
  int bad[NT_MAX_WARPS];
  int lnv[SC];
  int bitbase[SC];
  int ok;
  int abort;
};

constexpr int DEC_SMEM = 2 * STAGE_BYTES + ((sizeof(DecMisc) + 127) / 128) * 128;

__device__ __forceinline__ uint64_t lds_u64_at_byte(const uint8_t* base, int byte_off)
{
  const uint32_t* w = reinterpret_cast<const uint32_t*>(base);
  const int wi = byte_off >> 2;
  const int sh = (byte_off & 3) * 8;
  const uint32_t lo = __funnelshift_r(w[wi], w[wi + 1], sh);
  const uint32_t hi = __funnelshift_r(w[wi + 1], w[wi + 2], sh);
  return (static_cast<uint64_t>(hi) << 32) | lo;
}

template <typename T, bool LOSSY, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_decode(const DecArgs a)
{
  using V = VT<T>;
  constexpr int NW = NT / 32;
  extern __shared__ __align__(128) uint8_t smem[];
  uint8_t* const stage0 = smem;
  DecMisc& m = *reinterpret_cast<DecMisc*>(smem + 2 * STAGE_BYTES);

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  uint64_t* const ws = a.ws;
  uint64_t* const flags = ws + WS_HDR_WORDS;

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
    mbar_init(&m.bar[0], 1);
    mbar_init(&m.bar[1], 1);
    mbar_fence_init();
    m.vb = static_cast<long long>(atomicAdd(reinterpret_cast<unsigned long long*>(&ws[WS_TICKET]), 1ull));
    m.abort = 0;
    if (!hdr_ok) set_status(ws, ST_CORRUPT, -1);
    else if (!cap_ok) set_status(ws, ST_CAPACITY, -1);
  }
  __syncthreads();

  const bool go = hdr_ok && cap_ok;
  const long long vb = m.vb;
  const long long K = (chunks + gridDim.x - 1) / gridDim.x;
  const long long c0 = go ? min(vb * K, chunks) : 0;
  const long long c1 = go ? min(c0 + K, chunks) : 0;

  // ---- range aggregate + size-table validation ---------------------------------
  {
    long long sum = 0;
    int bad = 0;
    for (long long c = c0 + tid; c < c1; c += NT) {
      const int cs = size_in[c];
      const int os = static_cast<int>(min(static_cast<long long>(CS), insize - c * CS));
      bad |= (cs > os) | (cs == 0) | ((cs < os) & (cs < 34));
      sum += cs;
    }
    sum = warp_sum(sum);
    bad = __any_sync(0xffffffffu, bad);
    if (lane == 0) {
      m.red[warp] = sum;
      m.bad[warp] = bad;
    }
    __syncthreads();
    if (warp == 0) {
      long long s2 = lane < NW ? m.red[lane] : 0;
      int b2 = lane < NW ? m.bad[lane] : 0;
      s2 = warp_sum(s2);
      b2 = __any_sync(0xffffffffu, b2);
      if (b2 && lane == 0) set_status(ws, ST_CORRUPT, c0);
      if (lane == 0) st_relaxed_u64(&flags[vb], (vb == 0 ? FLAG_INC : FLAG_AGG) | (static_cast<uint64_t>(s2) & FLAG_VAL));
      long long excl = 0;
      if (vb > 0) {
        excl = lookback(flags, vb, 0, ws);
        if (excl < 0) {
          if (lane == 0) set_status(ws, ST_TIMEOUT, c0);
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
          mbar_arrive_expect_tx(&m.bar[stg], nb);
          tma_load_1d(stage0 + stg * STAGE_BYTES, src - sft, nb, &m.bar[stg]);
        } else {
          mbar_arrive(&m.bar[stg]);
        }
      }
    };

    if (warp == 0) issue(c0, 0);
    int it = 0;
    for (long long c = c0; c < c1; ++c, ++it) {
      const int s = it & 1;
      uint8_t* const stg = stage0 + s * STAGE_BYTES;
      if (warp == 0 && c + 1 < c1) issue(c + 1, s ^ 1);

      const bool arrived = mbar_wait_bounded(&m.bar[s], (it >> 1) & 1);
      if (__syncthreads_or(!arrived)) {
        if (tid == 0) set_status(ws, ST_TIMEOUT, c);
        mbar_wait_bounded(&m.bar[s], (it >> 1) & 1);
        if (c + 1 < c1) mbar_wait_bounded(&m.bar[s ^ 1], ((it + 1) >> 1) & 1);
        break;
      }

      const DecChunk d = m.info[s];
      const int osize = static_cast<int>(min(static_cast<long long>(CS), insize - c * CS));
      uint8_t* const outc = a.out + c * CS;
      if (!d.ok) {
        if (tid == 0) set_status(ws, ST_CORRUPT, c);
      } else if (d.cs == osize) {
        // raw chunk: shifted copy from the staged bytes
        T* const o = reinterpret_cast<T*>(outc);
        const int nv = osize / static_cast<int>(sizeof(T));
        for (int e = tid; e < nv; e += NT) {
          if constexpr (sizeof(T) == 4) o[e] = lds_u32_at_byte(stg, d.sft + 4 * e);
          else o[e] = lds_u64_at_byte(stg, d.sft + 8 * e);
        }
      } else {
        if (warp == 0) {
          const int ln = stg[d.sft + lane];
          const int bitsw = ln * V::VPS;
          int incl = bitsw;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
          }
          const int tot = __shfl_sync(0xffffffffu, incl, 31);
          m.lnv[lane] = ln;
          m.bitbase[lane] = 8 * d.sft + 256 + incl - bitsw;
          const bool bad_ln = __any_sync(0xffffffffu, ln > V::TB);
          if (lane == 0) {
            bool ok = !bad_ln && (34 + tot / 8 == d.cs);
            if (ok) {
              const int16_t tr = static_cast<int16_t>(stg[d.sft + d.cs - 2] | (stg[d.sft + d.cs - 1] << 8));
              ok = tr == osize;
            }
            m.ok = ok;
            if (!ok) set_status(ws, ST_CORRUPT, c);
          }
        }
        __syncthreads();
        if (m.ok) {
          const uint32_t* const w = reinterpret_cast<const uint32_t*>(stg);
          T* const o = reinterpret_cast<T*>(outc);
          const int nv = osize / static_cast<int>(sizeof(T));
          for (int k = tid; k < nv; k += NT) {
            const int i = k / V::VPS;
            const int j = k - i * V::VPS;
            const int ln = m.lnv[i];
            T e = 0;
            if (ln) {
              if constexpr (sizeof(T) == 4) e = extract_bits32(w, m.bitbase[i] + j * ln, ln);
              else e = extract_bits64(w, m.bitbase[i] + j * ln, ln);
            }
            o[k] = decode_value<LOSSY>(e, a.q);
          }
        }
      }
      fence_proxy_async_smem();
      __syncthreads();
    }
  }

  // ---- epilogue ------------------------------------------------------------------
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    const unsigned long long dn = atomicAdd(reinterpret_cast<unsigned long long*>(&ws[WS_DONE]), 1ull);
    if (dn == gridDim.x - 1) {
      __threadfence();
      const unsigned long long st = ld_relaxed_u64(&ws[WS_STATUS]);
      *a.outsize = st ? -static_cast<long long>(st) : insize;
    }
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

template <typename T, bool LOSSY>
static cudaError_t launch_encode_t(const EncArgs& a, int grid, cudaStream_t st)
{
  auto k = k_encode<T, LOSSY, ENC_MINB>;
  static unsigned long long attr = 0;
  cudaError_t e = ensure_smem_attr(k, ENC_SMEM, &attr);
  if (e != cudaSuccess) return e;
  k<<<grid, ENC_NT, ENC_SMEM, st>>>(a);
  return cudaGetLastError();
}

template <typename T, bool LOSSY>
static cudaError_t launch_decode_t(const DecArgs& a, int grid, cudaStream_t st)
{
  constexpr int NT = 256, MINB = 4;
  auto k = k_decode<T, LOSSY, NT, MINB>;
  static unsigned long long attr = 0;
  cudaError_t e = ensure_smem_attr(k, DEC_SMEM, &attr);
  if (e != cudaSuccess) return e;
  k<<<grid, NT, DEC_SMEM, st>>>(a);
  return cudaGetLastError();
}

template <typename T, bool LOSSY>
static int occupancy_t(bool enc)
{
  int n = 0;
  if (enc) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_encode<T, LOSSY, ENC_MINB>, ENC_NT, ENC_SMEM);
  else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_decode<T, LOSSY, 256, 4>, 256, DEC_SMEM);
  return n;
}

cudaError_t launch_encode(int width, bool lossy, const EncArgs& a, int grid, cudaStream_t st)
{
  if (width == 4) return lossy ? launch_encode_t<uint32_t, true>(a, grid, st) : launch_encode_t<uint32_t, false>(a, grid, st);
  return lossy ? launch_encode_t<uint64_t, true>(a, grid, st) : launch_encode_t<uint64_t, false>(a, grid, st);
}

cudaError_t launch_decode(int width, bool lossy, const DecArgs& a, int grid, cudaStream_t st)
{
  if (width == 4) return lossy ? launch_decode_t<uint32_t, true>(a, grid, st) : launch_decode_t<uint32_t, false>(a, grid, st);
  return lossy ? launch_decode_t<uint64_t, true>(a, grid, st) : launch_decode_t<uint64_t, false>(a, grid, st);
}

int blocks_per_sm(int width, bool lossy, bool enc)
{
  // the smem attribute must be set before the occupancy query counts dynamic smem
  if (width == 4) {
    if (lossy) {
      cudaFuncSetAttribute(k_encode<uint32_t, true, ENC_MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, ENC_SMEM);
      cudaFuncSetAttribute(k_decode<uint32_t, true, 256, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, DEC_SMEM);
      return occupancy_t<uint32_t, true>(enc);
    }
    cudaFuncSetAttribute(k_encode<uint32_t, false, ENC_MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, ENC_SMEM);
    cudaFuncSetAttribute(k_decode<uint32_t, false, 256, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, DEC_SMEM);
    return occupancy_t<uint32_t, false>(enc);
  }
  if (lossy) {
    cudaFuncSetAttribute(k_encode<uint64_t, true, ENC_MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, ENC_SMEM);
    cudaFuncSetAttribute(k_decode<uint64_t, true, 256, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, DEC_SMEM);
    return occupancy_t<uint64_t, true>(enc);
  }
  cudaFuncSetAttribute(k_encode<uint64_t, false, ENC_MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, ENC_SMEM);
  cudaFuncSetAttribute(k_decode<uint64_t, false, 256, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, DEC_SMEM);
  return occupancy_t<uint64_t, false>(enc);
}

}  // namespace sleek

// radik_common.cuh -- types, flags and device helpers shared by the selection
// engine (radik_engine.cu) and the C-ABI host side (radik_api.cu).
//
// Key space.  Every input value is mapped once to an unsigned "selection key"
// in which smaller means better: the order-preserving image of the float
// (negative: flip all bits, else flip the sign bit -- the same map as RadiK's
// getBinId, radik/RadixSelect/utils.cuh:329-334), complemented for largest-k.
// fp32 keys and every WITHSCALE key (the float difference x - s, RadiK's
// ComputeT<half> = float, utils.cuh:96-101) are 32 bits wide; unscaled
// fp16/bf16 keys are 16 bits wide.  Selection is over the 64-bit composite
// (key << IB | position), IB = bits of the row's largest position, so ties
// at the k-th key resolve to the lowest positions and the result is unique.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace radik {

// ----------------------------------------------------------------------------
// Public constants (mirrored in include/radik_b200.h)
// ----------------------------------------------------------------------------
enum : uint32_t {
  kFlagLargest = 1u,     // top-k largest (else smallest)
  kFlagSorted = 2u,      // sort each row's output
  kFlagAscend = 4u,      // sorted order ascending (else descending)
  kFlagWithScale = 8u,   // RadiK's adaptive scaling: order by x - x[0]
  kFlagWithIdxIn = 16u,  // emit idx_in[row_off + pos] instead of pos
  kFlagIdx64 = 32u,      // idx_in / idx_out are int64 (else int32)
};
enum : int { kF32 = 0, kF16 = 1, kBF16 = 2 };

// ----------------------------------------------------------------------------
// Engine geometry
// ----------------------------------------------------------------------------
constexpr int kThreads = 1024;           // one CTA per SM: 24 consumer, 7 side, 1 producer warp
constexpr int kCtasPerSM = 1;
constexpr int kWarps = kThreads / 32;
constexpr int kCapSB = 6144;             // candidates a finisher resolves in smem (48 KB)
constexpr int kSmemRowCap = 8192;        // rows this short are selected in smem
constexpr int kCtaRowCap = 1 << 15;      // default: rows this short are selected by one CTA
constexpr int kCtaRowCapMin = 1 << 15;   // range of the tunable one-CTA row cap
constexpr int kCtaRowCapMax = 1 << 20;
constexpr int kCapSort = 4096;           // outputs a finisher sorts in smem (32 KB)
constexpr int kMaxD1 = 12;               // widest first digit (16 KB smem hist)
constexpr int kMinD1 = 8;
constexpr int kPrefRatio = 64;           // pre-filter rows with k * 64 <= n
constexpr int kSampleMax = 8192;         // sampled keys per row (32 KB smem)
constexpr int kSampleStream = 16384;     // sampled keys of a streamed side-team sample (no smem)
constexpr int kSampleMin = 1024;
constexpr int kPhaseBSlots = 64;         // rows resolved together in phase B
constexpr int kPhaseBChunk = 65536;      // phase-B chunk length (entries)
constexpr int kSmemBytes = 226 * 1024;   // dynamic smem per CTA
constexpr int kMiscBytes = 4096;         // tail of smem for scalars / scan scratch

// Row kinds (a function of n and k only).
enum : int32_t {
  kKindEmpty = 0,      // k <= 0: nothing to do
  kKindSmem = 1,       // n <= kSmemRowCap: one item, row held in smem
  kKindCta = 2,        // n <= cta_cap (kCtaRowCap by default): one item, one CTA selects the row
  kKindAll = 3,        // k >= n: chunk items copy the whole row
  kKindGridPref = 4,   // large row, small k/n: sample item + filter chunks
  kKindGridRadix = 5,  // large row, large k/n: histogram chunks + filter chunks
};

// Row modes decided after the first level.
enum : int32_t {
  kModeNone = 0,
  kModeFinal = 1,   // matched bin == remaining k: F emits better-or-matched
  kModeSB = 2,      // matched bin fits a finisher's smem: F compacts into it
  kModeCand = 3,    // matched bin compacted into the candidate region
  kModeDefer = 4,   // matched bin too large: levels continue on the input
  kModeAll = 5,     // k >= n: every element is selected
};

// Status bits written by the device (Header::status).
enum : int32_t {
  kStatusTimeout = 1,       // a bounded wait gave up
  kStatusSelect = 2,        // a histogram did not hold k keys (internal)
  kStatusCapacity = 4,      // workspace too small for the planned rows
  kStatusLevels = 16,       // resolution did not converge (internal)
};

// Per-row plan (written by the planning kernel, read by the engine).
struct alignas(16) RowPlan {
  int64_t in_off;    // element offset of the row in val_in / idx_in
  int64_t out_off;   // first output slot of the row
  int64_t cand_off;  // first candidate entry of the row (8 B entries)
  int64_t sort_off;  // first sort-scratch entry (8 B entries), -1 if none
  int32_t n;         // row length
  int32_t k;         // requested k
  int32_t a0;        // first A item of the row
  int32_t b0;        // first B item of the row
  int32_t cand_cap;  // candidate region capacity (entries)
  int32_t slot_use;  // ordinal among histogram rows (hist ring), -1 = none
  int32_t pad0, pad1;
};
static_assert(sizeof(RowPlan) == 64, "RowPlan layout");

// Per-row state, zeroed before every call.
struct alignas(16) RowState {
  int32_t hticket;     // histogram items finished (radix rows)
  int32_t fticket;     // chunk items finished (filter / copy chunks)
  int32_t ready;       // radix rows: first-level decision published
  int32_t mode;        // kMode*
  int32_t krem;        // k still to take from the matched set
  int32_t count;       // size of the matched set
  int32_t out_count;   // output slots reserved so far
  int32_t cand_count;  // candidate entries written
  uint64_t prefix;     // composite prefix of the matched set
  uint64_t tready;     // pre-filter rows: (1 << 32) | threshold key, one release store
  int32_t plen;        // its length in bits
  int32_t src;         // phase B source: 0 = the row, 1 = its candidates
  int32_t src_len;     // entries in the phase-B source
  int32_t final_pass;  // phase B: the next filter is the last
  int32_t sb_count;    // phase B: entries compacted for the finisher
  int32_t pad0;
  uint64_t pb_min;     // phase B: least / greatest composite of the matched set
  uint64_t pb_max;     //   seen by the current histogram pass
  int32_t pad[10];
};
static_assert(sizeof(RowState) == 128, "RowState layout");

// Call header, zeroed before every call.
struct alignas(16) Header {
  uint32_t qhead;       // phase-A claim counter
  uint32_t bar_count;   // grid barrier arrivals
  uint32_t bar_gen;     // grid barrier generation
  int32_t status;       // kStatus* bits
  int32_t nlarge;       // rows handed to phase B
  int32_t na;           // A items planned
  int32_t nb;           // B items planned
  int32_t lag;          // A-ahead-of-B distance in items
  int32_t plan_error;   // planning failed (capacity)
  uint32_t pbhead;      // phase-B claim counter
  int64_t cand_total;   // candidate entries planned
  int64_t sort_total;   // sort-scratch entries planned
  int32_t fin_tail;     // FIN items at the end of the claim order
  int32_t pad0;
  uint64_t t_first;     // %globaltimer (ns) when the engine's first CTA started
  uint64_t t_last;      // ... and when its last CTA ended
  int32_t pad[44];
};
static_assert(sizeof(Header) == 256, "Header layout");

// Row descriptor given to the planning kernel.
struct alignas(8) RowDesc {
  int64_t in_off;
  int64_t out_off;
  int32_t n;
  int32_t k;
};
static_assert(sizeof(RowDesc) == 24, "RowDesc layout");

// Everything the engine kernel needs.  Passed by value (__grid_constant__).
struct EngineParams {
  const void* val_in;
  const void* idx_in;
  void* val_out;
  void* idx_out;
  const RowPlan* plans;     // null in uniform mode
  RowState* rs;
  const int32_t* a_row;     // A item -> row (null in uniform mode)
  const int32_t* b_row;     // B item -> row (null in uniform mode)
  uint32_t* hist_ring;      // S slots of (1 << kMaxD1) counters
  uint32_t* slot_gen;       // S release counters
  Header* hdr;
  int32_t* large_list;      // B entries
  uint64_t* cand;           // candidate entries (valbits << 32 | pos)
  uint64_t* sort_scratch;   // merge-sort scratch
  uint64_t* pb_sb;          // phase-B smem-bound candidates, kPhaseBSlots x kCapSB
  int32_t B;
  int32_t CH;               // chunk length of single-read rows (elements), multiple of 16
  int32_t CHR;              // chunk length of radix rows (elements), multiple of 16
  int32_t D1;               // first digit width of histogram rows
  int32_t cta_cap;          // rows of up to this many keys are selected by one CTA
  int32_t early_copy;       // chunk copies may start before their row's threshold exists
  int32_t l2_ahead;         // ring stages a chunk's L2 prefetch runs ahead of its copies (0: none)
  int32_t S;                // hist ring slots
  int32_t lag;              // uniform mode: A-ahead-of-B distance
  int32_t fin_delay;        // uniform mode: rows a FIN item trails its row
  uint32_t flags;
  uint32_t spin_limit;      // iterations of a bounded wait
  unsigned long long* timeline;  // per-CTA phase stamps (timeline build only; else null)
  // uniform mode: every row has n = u_n, k = u_k, contiguous input,
  // output at r * u_k.
  int32_t uniform;
  int32_t u_n;
  int32_t u_k;
  int32_t u_cand_cap;
  int64_t u_sort_cap;       // sort-scratch entries per row (0 if none)
  int32_t u_tail_rows;      // the last rows, whose pre-filter chunks are u_ch_tail long (0: none)
  int32_t u_ch_tail;
};

// ----------------------------------------------------------------------------
// Host+device helpers
// ----------------------------------------------------------------------------
__host__ __device__ inline int key_bits(int dtype, uint32_t flags) {
  return (dtype == kF32 || (flags & kFlagWithScale)) ? 32 : 16;
}
__host__ __device__ inline int elem_bytes(int dtype) { return dtype == kF32 ? 4 : 2; }
__host__ __device__ inline int index_bits(int64_t n) {
  int b = 1;
  while (b < 32 && ((int64_t)1 << b) < n) ++b;
  return b;
}
__host__ __device__ inline bool is_smem_row(int32_t n) { return n <= kSmemRowCap; }
// cta_cap: rows of up to this many keys are selected by one CTA (tunable).
__host__ __device__ inline int row_kind(int32_t n, int32_t k, int32_t cta_cap) {
  if (k <= 0) return kKindEmpty;
  if (n <= kSmemRowCap) return kKindSmem;
  if (k >= n) return kKindAll;
  if (n <= cta_cap) return kKindCta;
  if ((int64_t)k * kPrefRatio <= (int64_t)n) return kKindGridPref;
  return kKindGridRadix;
}
__host__ __device__ inline int32_t ceil_div32(int64_t a, int64_t b) { return (int32_t)((a + b - 1) / b); }
// Chunk length of a row's streaming items: radix rows re-read their chunks
// and use the short length CHR (the re-read must still be in L2); the
// others read each chunk once and use CH.
__host__ __device__ inline int32_t row_chunk(int kind, int32_t CH, int32_t CHR) {
  return kind == kKindGridRadix ? CHR : CH;
}
// Items of a row.  A items (sample, histogram chunks, single-item rows,
// copy chunks) run first; B items are the row's filter chunks and its finish
// item ("FIN": resolve candidates, sort, map indices), which depends on all
// of the row's chunk items.  A row's FIN item is placed D rows later in the
// B sequence (inside the block of row r + D, or in a tail after the last
// row), so that its chunks are done by the time it is claimed.
__host__ __device__ inline int32_t row_na(int kind, int32_t n, int32_t CH, int32_t CHR) {
  if (kind == kKindAll || kind == kKindGridRadix) return ceil_div32(n, row_chunk(kind, CH, CHR));
  return 1;
}
// B chunk items of a row (its FIN item not counted)
__host__ __device__ inline int32_t row_nbc(int kind, int32_t n, int32_t CH, int32_t CHR) {
  if (kind == kKindGridPref || kind == kKindGridRadix) return ceil_div32(n, row_chunk(kind, CH, CHR));
  return 0;
}
__host__ __device__ inline int32_t row_fin(int kind) {
  return (kind == kKindGridPref || kind == kKindGridRadix || kind == kKindAll) ? 1 : 0;
}
// Chunk items a row's FIN item waits for.
__host__ __device__ inline int32_t row_fin_wait(int kind, int32_t n, int32_t CH, int32_t CHR) {
  return kind == kKindAll ? row_na(kind, n, CH, CHR) : row_nbc(kind, n, CH, CHR);
}

// B items of an equal-length call.  Rows [0, B - R) have nc chunk items,
// the last R rows nct (shorter chunks: the last items of the claim order are
// short, so the CTAs run out of work together), and a row's FIN item (f = 1)
// trails it by D rows.  Order: the chunks of rows [0, D); then, for each row
// r in [D, B), its chunks followed by row r - D's FIN; then the FINs of rows
// [B - D, B).
struct UniformB {
  int32_t B, nc, nct, R, f, D;
  __host__ __device__ int32_t chunks(int64_t r) const { return r >= (int64_t)B - R ? nct : nc; }
  __host__ __device__ int64_t dd() const { return D < B ? D : B; }
  // B index of row r's first chunk (r = B: the first tail FIN)
  __host__ __device__ int64_t first(int64_t r) const {
    const int64_t s = (int64_t)B - R;
    const int64_t head = r < s ? r : s;
    int64_t idx = head * nc + (r - head) * nct;
    if (r > dd()) idx += (int64_t)f * (r - dd());
    return idx;
  }
  __host__ __device__ int64_t count() const { return first(B) + (int64_t)f * dd(); }
  // item j -> row, chunk index (sub) and whether it is a FIN
  __host__ __device__ void decode(int64_t j, int32_t* row, int32_t* sub, int32_t* fin) const {
    const int64_t Dd = dd(), s = (int64_t)B - R;
    const int64_t end = first(B);
    if (j >= end) {
      *row = (int32_t)((int64_t)B - Dd + (j - end));
      *sub = 0;
      *fin = 1;
      return;
    }
    // rows fall in three runs of equal block size: [0, lo), [lo, hi), [hi, B)
    const int64_t lo = Dd < s ? Dd : s, hi = Dd < s ? s : Dd;
    const int64_t starts[3] = {0, lo, hi};
    int k = 2;
    if (j < first(hi)) k = 1;
    if (j < first(lo)) k = 0;
    const int64_t r0 = starts[k];
    const int64_t size = chunks(r0) + (r0 >= Dd ? f : 0);
    const int64_t r = r0 + (j - first(r0)) / size;
    const int64_t o = (j - first(r0)) % size;
    if (o < chunks(r)) {
      *row = (int32_t)r;
      *sub = (int32_t)o;
      *fin = 0;
    } else {
      *row = (int32_t)(r - Dd);
      *sub = 0;
      *fin = 1;
    }
  }
};

// Candidate region capacity of a row: enough for the smem finisher's set or
// one eighth of the row, whichever is larger (never more than n).
__host__ __device__ inline int32_t cand_capacity(int32_t n) {
  int64_t a = n < kCapSB ? n : kCapSB;
  int64_t b = ((int64_t)n + 7) / 8;
  return (int32_t)(a > b ? a : b);
}
__host__ __device__ inline int32_t row_cand_cap(int kind, int32_t n) {
  return (kind == kKindGridPref || kind == kKindGridRadix) ? cand_capacity(n) : 0;
}
__host__ __device__ inline bool row_uses_hist(int kind) { return kind == kKindGridRadix; }
// Pre-filter sample size (a power of two near n / 128, clamped) and the rank
// of the sampled key used as the threshold: about twice the expected rank of
// the k-th key in the sample plus a margin of 8, so that fewer than k keys
// pass only with negligible probability for i.i.d. rows.
__host__ __device__ inline int32_t sample_size(int32_t n) {
  int32_t s = kSampleMin;
  while (s < kSampleMax && (int64_t)s * 2 * 128 <= n) s *= 2;
  return s;
}
__host__ __device__ inline int32_t sample_rank(int32_t n, int32_t k, int32_t S) {
  const int64_t r = (2 * (int64_t)k * S + n - 1) / n + 8;
  return (int32_t)(r < S ? r : S);
}

}  // namespace radik

// topk_oracle.cpp -- CPU restatement of RadiK's batched radix top-k selection.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
// library in radik_b200/ and the OpenMP CPU baseline that bench.py reports
// beside the GPU numbers.  Only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg may load it.  The product path never calls it.
//
// What it restates (file:line are paths inside the leefige/radik project):
//   * radik/RadixSelect/topk_radixselect.h:59-323  topKRadixSelectL: per row,
//     select the K largest (LARGEST=1) or smallest keys of val_in, write them
//     to val_out/idx_out at row*K, optionally sorted (ASCEND picks the order),
//     with the "idle fill" idx=-1 / val=0 for the K-n slots of a short row
//     (topk_radixselect.h:312-320).
//   * radik/RadixSelect/utils.cuh:329-334  getBinId: the order-preserving
//     unsigned key of a float (negative: flip all bits, else flip the sign).
//   * radik/RadixSelect/utils.cuh:255-324  sampleScaler/scaling: WITHSCALE
//     subtracts the row's first element (0 if it is NaN/Inf) in float before
//     any comparison; the emitted values stay the original ones
//     (radixselect_l.cuh:410-436 stage the unscaled value).
//   * radik/RadixSelect/utils.cuh:96-101  ComputeT<half> = float, so a scaled
//     half row is ordered by the float difference.
//   * radik/RadixSelect/radixselect_l.cuh:498-506  WITHIDXIN: the emitted index
//     is idx_in[row_offset + position] instead of the position.
//
// Where RadiK leaves a choice open this restatement fixes it, and the CUDA
// library follows the same rule:
//   * Ties at the k-th key are broken by the lowest position in the row.
//     RadiK takes them in arrival order (radixselect_l.cuh:417-421).
//   * Keys are compared as the order-preserving unsigned integer, so -0.0 ranks
//     below +0.0 and a NaN ranks by its bit pattern (a positive NaN above
//     +inf).  RadiK compares floats in its filter and skips NaN only in its
//     first histogram (radixselect_l.cuh:189-194).
//   * Sorted output orders by value in the requested direction and then by
//     ascending position.  Unsorted output is written here in ascending
//     position order; the GPU library's unsorted order is unspecified, so the
//     tests compare unsorted rows as sets.
//
// The selection itself is std::nth_element on a 64-bit composite
// (selection key << 32 | position), which is exactly "the k smallest
// composites": unique, deterministic, independent of thread count.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

namespace {

enum : uint32_t {
  kLargest = 1u,
  kSorted = 2u,
  kAscend = 4u,
  kWithScale = 8u,
  kWithIdxIn = 16u,
  kIdx64 = 32u,
};
enum : int { kF32 = 0, kF16 = 1, kBF16 = 2 };

inline uint32_t f32_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}
inline float bits_f32(uint32_t u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

// Exact widening of a binary16 / bfloat16 bit pattern to float.
inline float half_to_float(uint16_t h) {
  _Float16 x;
  std::memcpy(&x, &h, 2);
  return static_cast<float>(x);
}
inline float bf16_to_float(uint16_t h) { return bits_f32(static_cast<uint32_t>(h) << 16); }

// Order-preserving key of a 32-bit float pattern (utils.cuh:329-334).
inline uint32_t ukey32(uint32_t u) { return u ^ ((u >> 31) ? 0xFFFFFFFFu : 0x80000000u); }
// Same for a 16-bit float pattern.
inline uint32_t ukey16(uint32_t u) { return (u ^ ((u >> 15) ? 0xFFFFu : 0x8000u)) & 0xFFFFu; }

struct RowCtx {
  int dtype;
  uint32_t flags;
  const uint8_t* vals;  // row start
  float scaler;
  int key_bits;
};

inline uint32_t raw_bits(const RowCtx& c, int64_t i) {
  if (c.dtype == kF32) {
    uint32_t u;
    std::memcpy(&u, c.vals + 4 * i, 4);
    return u;
  }
  uint16_t h;
  std::memcpy(&h, c.vals + 2 * i, 2);
  return h;
}

inline float as_float(const RowCtx& c, uint32_t bits) {
  if (c.dtype == kF32) return bits_f32(bits);
  if (c.dtype == kF16) return half_to_float(static_cast<uint16_t>(bits));
  return bf16_to_float(static_cast<uint16_t>(bits));
}

// Unsigned key in value order (smaller key = smaller value), before the
// largest/smallest flip.  WITHSCALE orders by the float difference x - s.
inline uint32_t value_key(const RowCtx& c, uint32_t bits) {
  if (c.flags & kWithScale) {
    volatile float d = as_float(c, bits) - c.scaler;  // one IEEE single subtraction
    return ukey32(f32_bits(d));
  }
  return c.dtype == kF32 ? ukey32(bits) : ukey16(bits);
}

// Selection key: smaller is better.
inline uint32_t select_key(const RowCtx& c, uint32_t bits) {
  uint32_t k = value_key(c, bits);
  if (c.flags & kLargest) k = (c.key_bits == 32) ? ~k : (~k & 0xFFFFu);
  return k;
}

// Key used to sort the output: unscaled value order in the requested direction
// (RadiK's bitonic sort compares the emitted, unscaled values,
// bitonic_sort.cuh:39-75).
inline uint32_t sort_key(const RowCtx& c, uint32_t bits) {
  uint32_t k = c.dtype == kF32 ? ukey32(bits) : ukey16(bits);
  if (!(c.flags & kAscend)) k = ~k;
  return k;
}

float row_scaler(int dtype, uint32_t flags, const uint8_t* row, int64_t n) {
  if (!(flags & kWithScale) || n <= 0) return 0.0f;
  RowCtx c{dtype, flags, row, 0.0f, 32};
  float s = as_float(c, raw_bits(c, 0));
  if (std::isnan(s) || std::isinf(s)) s = 0.0f;
  return s;
}

// Top-kk composites of [lo, hi) appended to out (unordered).
void partial_select(const RowCtx& c, int64_t lo, int64_t hi, int64_t kk, std::vector<uint64_t>& out) {
  std::vector<uint64_t> comp(static_cast<size_t>(hi - lo));
  for (int64_t i = lo; i < hi; ++i)
    comp[i - lo] = (static_cast<uint64_t>(select_key(c, raw_bits(c, i))) << 32) | static_cast<uint64_t>(i);
  int64_t take = std::min<int64_t>(kk, hi - lo);
  if (take < hi - lo && take > 0) std::nth_element(comp.begin(), comp.begin() + (take - 1), comp.end());
  out.insert(out.end(), comp.begin(), comp.begin() + take);
}

void write_row(const RowCtx& c, uint32_t flags, const std::vector<uint64_t>& sel, int64_t k,
               const void* idx_in, int64_t in_off, void* val_out, void* idx_out, int64_t out_off) {
  const int es = c.dtype == kF32 ? 4 : 2;
  const int64_t kk = static_cast<int64_t>(sel.size());
  for (int64_t j = 0; j < k; ++j) {
    uint32_t vb = 0;
    int64_t idx = -1;
    if (j < kk) {
      const int64_t pos = static_cast<int64_t>(sel[j] & 0xFFFFFFFFull);
      vb = raw_bits(c, pos);
      if (flags & kWithIdxIn) {
        idx = (flags & kIdx64) ? static_cast<const int64_t*>(idx_in)[in_off + pos]
                               : static_cast<const int32_t*>(idx_in)[in_off + pos];
      } else {
        idx = pos;
      }
    }
    uint8_t* vo = static_cast<uint8_t*>(val_out) + (out_off + j) * es;
    if (es == 4) std::memcpy(vo, &vb, 4);
    else {
      uint16_t h = static_cast<uint16_t>(vb);
      std::memcpy(vo, &h, 2);
    }
    if (flags & kIdx64) static_cast<int64_t*>(idx_out)[out_off + j] = idx;
    else static_cast<int32_t*>(idx_out)[out_off + j] = static_cast<int32_t>(idx);
  }
}

// Orders the selected composites for output: sorted by (sort key, position)
// when kSorted, else by position.
void order_selection(const RowCtx& c, uint32_t flags, std::vector<uint64_t>& sel) {
  if (flags & kSorted) {
    for (auto& e : sel) {
      const uint64_t pos = e & 0xFFFFFFFFull;
      e = (static_cast<uint64_t>(sort_key(c, raw_bits(c, static_cast<int64_t>(pos)))) << 32) | pos;
    }
    std::sort(sel.begin(), sel.end());
  } else {
    for (auto& e : sel) e &= 0xFFFFFFFFull;
    std::sort(sel.begin(), sel.end());
  }
}

}  // namespace

extern "C" {

// Number of key bits the selection works in: 32 for fp32 or any scaled row
// (ComputeT = float), 16 for unscaled fp16/bf16.
int oracle_key_bits(int dtype, uint32_t flags) {
  return (dtype == kF32 || (flags & kWithScale)) ? 32 : 16;
}

// Batched exact top-k.
//   row_off[B+1]: element offsets of the rows in val_in (and idx_in).
//   row_k[B]:     k of each row.  out_off[B]: first output slot of each row.
//   nthreads <= 0 uses omp_get_max_threads().
// Returns 0, or -1 on bad arguments.
int oracle_topk(int dtype, uint32_t flags, const void* val_in, const void* idx_in,
                const int64_t* row_off, const int32_t* row_k, const int64_t* out_off, int B,
                void* val_out, void* idx_out, int nthreads) {
  if (dtype < kF32 || dtype > kBF16 || B < 0 || !row_off || !row_k || !out_off) return -1;
  if ((flags & kWithIdxIn) && !idx_in) return -1;
  const int es = dtype == kF32 ? 4 : 2;
  const int kb = oracle_key_bits(dtype, flags);
  const int T = nthreads > 0 ? nthreads : omp_get_max_threads();

  auto run_row = [&](int r, int inner_threads) {
    const int64_t n = row_off[r + 1] - row_off[r];
    const int64_t k = row_k[r];
    if (k <= 0) return;
    const uint8_t* row = static_cast<const uint8_t*>(val_in) + row_off[r] * es;
    RowCtx c{dtype, flags, row, row_scaler(dtype, flags, row, n), kb};
    const int64_t kk = std::min(n, k);
    std::vector<uint64_t> sel;
    if (inner_threads <= 1 || n < (int64_t)inner_threads * 65536) {
      partial_select(c, 0, n, kk, sel);
    } else {
      // Per-thread chunks, then a merge of the per-chunk winners.
      std::vector<std::vector<uint64_t>> part(inner_threads);
#pragma omp parallel for num_threads(inner_threads) schedule(static)
      for (int t = 0; t < inner_threads; ++t) {
        const int64_t lo = n * t / inner_threads, hi = n * (t + 1) / inner_threads;
        partial_select(c, lo, hi, kk, part[t]);
      }
      std::vector<uint64_t> all;
      for (auto& p : part) all.insert(all.end(), p.begin(), p.end());
      if (kk < (int64_t)all.size() && kk > 0) std::nth_element(all.begin(), all.begin() + (kk - 1), all.end());
      all.resize(kk);
      sel.swap(all);
    }
    order_selection(c, flags, sel);
    write_row(c, flags, sel, k, idx_in, row_off[r], val_out, idx_out, out_off[r]);
  };

  if (B >= T || B == 0) {
#pragma omp parallel for num_threads(T) schedule(dynamic, 1)
    for (int r = 0; r < B; ++r) run_row(r, 1);
  } else {
    for (int r = 0; r < B; ++r) run_row(r, T);
  }
  return 0;
}

// The selection key of one value (exposed so tests can check key order).
uint32_t oracle_select_key(int dtype, uint32_t flags, uint32_t bits, float scaler) {
  RowCtx c{dtype, flags, nullptr, scaler, oracle_key_bits(dtype, flags)};
  return select_key(c, bits);
}

int oracle_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"

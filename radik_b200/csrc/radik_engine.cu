// radik_engine.cu -- the B200 radix top-k selection engine.
//
// One persistent launch (one 1024-thread CTA per SM) selects every row of a
// batch.  It replaces RadiK's chain of ~10 launches and 2 host syncs per call
// (radik/RadixSelect/topk_radixselect.h:117-307):
//
//   countBinEx + selectBin   (radixselect_l.cuh:173-267, :45-126)
//       -> H items: histogram of the first digit of a chunk, fused into the
//          first read of the keys; the CTA finishing a row's last H item
//          scans the row histogram and publishes the selected bin (no
//          separate selectBin launch, no host sync).
//   selectCandidateEx + filter (radixselect_l.cuh:269-408, :438-832)
//       -> F items: one re-read of the chunk (served from L2: F items trail
//          the H items by a fixed lag of chunks) that writes keys of better
//          bins straight to the output and compacts the selected bin's keys
//          into a candidate region.  RadiK's third full read (filter) is gone.
//   countBin/selectCandidate passes 2-3 (radixselect_l.cuh:14-43, :128-168)
//       -> the row's finisher (the CTA finishing its last F item) resolves
//          the candidates in shared memory with 8-bit digits over the
//          composite (key, position), so ties go to the lowest positions.
//   bitonicSort_* / thrust::sort_by_key (bitonic_sort.cuh:195-553,
//       topk_radixselect.h:285-307)
//       -> the finisher sorts the row's outputs in shared memory.
//
// Work items are claimed from one global counter.  Their order is
// H[0..L), then H and F alternating, then the trailing F: every F item of a
// row comes after all H items of that row (L >= chunks per row), so a CTA
// that waits for a row's selection only waits for items already claimed by
// running CTAs, and the smallest unfinished item can always progress.
// Every wait is bounded (spin_limit); a wait that gives up sets a status bit
// and the kernel still exits.

#include "radik_common.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace radik {
namespace dev {

constexpr unsigned kFull = 0xFFFFFFFFu;

// ----------------------------------------------------------------------------
// PTX helpers
// ----------------------------------------------------------------------------
__device__ __forceinline__ int32_t ld_acquire(const int32_t* p) {
  int32_t v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int32_t* p, int32_t v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// Streaming 16-byte load of read-only input.
__device__ __forceinline__ uint4 ld_stream16(const void* p) {
  uint4 r;
  asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
               : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
               : "l"(p));
  return r;
}
__device__ __forceinline__ uint32_t ld_cg_u32(const uint32_t* p) { return __ldcg(p); }
__device__ __forceinline__ uint64_t ld_cg_u64(const uint64_t* p) {
  return (uint64_t)__ldcg(reinterpret_cast<const unsigned long long*>(p));
}

__device__ __forceinline__ uint64_t shr64(uint64_t x, int s) { return s >= 64 ? 0ull : (x >> s); }

// ----------------------------------------------------------------------------
// Keys
// ----------------------------------------------------------------------------
template <int VT, bool SCALE>
struct KT {
  static constexpr int ES = VT == kF32 ? 4 : 2;            // element bytes
  static constexpr int VEC = 16 / ES;                       // elements per 16 B
  static constexpr int KB = (VT == kF32 || SCALE) ? 32 : 16;
  static constexpr uint32_t KMASK = KB == 32 ? 0xFFFFFFFFu : 0xFFFFu;
};

template <int VT>
__device__ __forceinline__ float to_float(uint32_t bits) {
  if constexpr (VT == kF32) return __uint_as_float(bits);
  else if constexpr (VT == kF16) return __half2float(__ushort_as_half((unsigned short)bits));
  else return __uint_as_float(bits << 16);
}

__device__ __forceinline__ uint32_t ukey32(uint32_t u) {
  return u ^ ((uint32_t)((int32_t)u >> 31) | 0x80000000u);
}
__device__ __forceinline__ uint32_t ukey16(uint32_t u) {
  return (u ^ ((u & 0x8000u) ? 0xFFFFu : 0x8000u)) & 0xFFFFu;
}
__device__ __forceinline__ uint32_t unkey32(uint32_t k) { return (k & 0x80000000u) ? (k ^ 0x80000000u) : ~k; }
__device__ __forceinline__ uint32_t unkey16(uint32_t k) {
  return ((k & 0x8000u) ? (k ^ 0x8000u) : (~k)) & 0xFFFFu;
}

// Selection key (smaller = better).  flip is 0 (smallest) or KMASK (largest).
template <int VT, bool SCALE>
__device__ __forceinline__ uint32_t sel_key(uint32_t bits, uint32_t flip, float scaler) {
  if constexpr (SCALE) {
    const float d = __fsub_rn(to_float<VT>(bits), scaler);
    return ukey32(__float_as_uint(d)) ^ flip;
  } else if constexpr (VT == kF32) {
    return ukey32(bits) ^ flip;
  } else {
    return ukey16(bits) ^ flip;
  }
}

// Output-order key (unscaled value order, direction by ASCEND) and inverse.
template <int VT>
__device__ __forceinline__ uint32_t out_key(uint32_t bits, bool ascend) {
  if constexpr (VT == kF32) return ascend ? ukey32(bits) : ~ukey32(bits);
  else return ascend ? ukey16(bits) : (~ukey16(bits) & 0xFFFFu);
}
template <int VT>
__device__ __forceinline__ uint32_t out_key_inv(uint32_t k, bool ascend) {
  if constexpr (VT == kF32) return unkey32(ascend ? k : ~k);
  else return unkey16(ascend ? k : (~k & 0xFFFFu));
}

// ----------------------------------------------------------------------------
// Shared-memory scratch at the tail of the dynamic allocation
// ----------------------------------------------------------------------------
struct Misc {
  uint32_t hist256[256];
  uint32_t scan[64];
  int32_t next_q;
  int32_t bcast;
  int32_t bcast2;
  uint32_t sel_bin, sel_cum, sel_cnt, sel_found;
  uint32_t counter;
  // row-state snapshot taken by thread 0 after an acquire
  int32_t st_mode, st_krem, st_count, st_plen;
  uint64_t st_prefix;
  int32_t st_candn;
  int32_t pad[7];
};
static_assert(sizeof(Misc) <= kMiscBytes, "Misc too large");

__device__ __forceinline__ Misc* misc_of(uint8_t* smem) {
  return reinterpret_cast<Misc*>(smem + (kSmemBytes - kMiscBytes));
}

// ----------------------------------------------------------------------------
// Block primitives
// ----------------------------------------------------------------------------
// Exclusive scan of one value per thread; *total gets the block sum.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* scan, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) scan[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = scan[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, w, o);
      if (lane >= o) w += y;
    }
    scan[lane] = w;
  }
  __syncthreads();
  const uint32_t base = warp ? scan[warp - 1] : 0u;
  if (total) *total = scan[kWarps - 1];
  __syncthreads();
  return base + x - v;
}

// Finds the bin b of h[0..NB) with cum(<b) < krem <= cum(<=b).
// Result in m->sel_*; m->sel_found = 0 if the bins hold fewer than krem.
template <bool GLOBAL>
__device__ void block_select(const uint32_t* h, int NB, uint32_t krem, Misc* m) {
  if (threadIdx.x == 0) m->sel_found = 0;
  const int per = (NB + kThreads - 1) / kThreads;
  const int lo = threadIdx.x * per;
  const int hi = min(NB, lo + per);
  uint32_t s = 0;
  if ((per & 3) == 0) {
    for (int i = lo; i < hi; i += 4) {
      uint4 v;
      if constexpr (GLOBAL) v = __ldcg(reinterpret_cast<const uint4*>(h + i));
      else v = *reinterpret_cast<const uint4*>(h + i);
      s += v.x + v.y + v.z + v.w;
    }
  } else {
    for (int i = lo; i < hi; ++i) s += GLOBAL ? ld_cg_u32(h + i) : h[i];
  }
  const uint32_t ex = block_excl_scan(s, m->scan, nullptr);
  if (lo < hi && ex < krem && krem <= ex + s) {
    uint32_t run = ex;
    for (int i = lo; i < hi; ++i) {
      const uint32_t c = GLOBAL ? ld_cg_u32(h + i) : h[i];
      if (run + c >= krem) {
        m->sel_bin = (uint32_t)i;
        m->sel_cum = run;
        m->sel_cnt = c;
        m->sel_found = 1;
        break;
      }
      run += c;
    }
  }
  __syncthreads();
}

// Shared-memory histogram increment.  All 32 lanes must call it together.
// The bin of the first valid lane is aggregated with one atomic, which turns
// a heavily repeated key (constant-heavy rows) into one update per warp.
__device__ __forceinline__ void hist_add(uint32_t* hist, uint32_t bin, bool valid) {
  const unsigned vm = __ballot_sync(kFull, valid);
  if (vm == 0) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(vm) - 1;
  const uint32_t lb = __shfl_sync(kFull, bin, leader);
  const bool same = valid && bin == lb;
  const unsigned sm = __ballot_sync(kFull, same);
  if (valid && !same) atomicAdd(&hist[bin], 1u);
  if (lane == leader) atomicAdd(&hist[lb], (uint32_t)__popc(sm));
}

// Bitonic sort of n (power of two, >= 2) uint64 keys in shared memory.
__device__ void block_bitonic_sort(uint64_t* s, int n) {
  for (int size = 2; size <= n; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < (n >> 1); i += kThreads) {
        const int lo = 2 * i - (i & (stride - 1));
        const int hi = lo + stride;
        const bool up = (lo & size) == 0;
        const uint64_t a = s[lo], b = s[hi];
        if ((a > b) == up) {
          s[lo] = b;
          s[hi] = a;
        }
      }
      __syncthreads();
    }
  }
}

// ----------------------------------------------------------------------------
// Row context
// ----------------------------------------------------------------------------
enum : int { kKindEmpty = 0, kKindSmem = 1, kKindAll = 2, kKindMulti = 3 };

__host__ __device__ __forceinline__ int row_kind(int32_t n, int32_t k) {
  if (k <= 0) return kKindEmpty;
  if (is_smem_row(n)) return kKindSmem;
  if (k >= n) return kKindAll;
  return kKindMulti;
}

struct RowCtx {
  int64_t in_off, out_off, cand_off, sort_off;
  int32_t n, k, chunk0, nch, cand_cap, slot_use;
  int32_t kind, IB;
  uint32_t flip;
  float scaler;
};

template <int VT, bool SCALE>
__device__ __forceinline__ RowCtx load_row(const EngineParams& p, int r) {
  RowCtx c;
  if (p.uniform) {
    c.n = p.u_n;
    c.k = p.u_k;
    c.in_off = (int64_t)r * p.u_n;
    c.out_off = (int64_t)r * p.u_k;
    c.chunk0 = r * p.u_nch;
    c.nch = p.u_nch;
    c.cand_cap = p.u_cand_cap;
    c.cand_off = (int64_t)r * p.u_cand_cap;
    c.sort_off = p.u_sort_cap ? (int64_t)r * p.u_sort_cap : -1;
    c.kind = row_kind(c.n, c.k);
    c.slot_use = c.kind == kKindMulti ? r : -1;
  } else {
    const RowPlan& pl = p.plans[r];
    c.in_off = pl.in_off;
    c.out_off = pl.out_off;
    c.cand_off = pl.cand_off;
    c.sort_off = pl.sort_off;
    c.n = pl.n;
    c.k = pl.k;
    c.chunk0 = pl.chunk0;
    c.nch = pl.nch;
    c.cand_cap = pl.cand_cap;
    c.slot_use = pl.slot_use;
    c.kind = row_kind(c.n, c.k);
  }
  c.IB = index_bits(c.n);
  c.flip = (p.flags & kFlagLargest) ? KT<VT, SCALE>::KMASK : 0u;
  c.scaler = 0.f;
  if constexpr (SCALE) {
    if (c.n > 0) {
      float s;
      if constexpr (VT == kF32) s = __ldg(static_cast<const float*>(p.val_in) + c.in_off);
      else s = to_float<VT>((uint32_t)__ldg(static_cast<const unsigned short*>(p.val_in) + c.in_off));
      if (isnan(s) || isinf(s)) s = 0.f;
      c.scaler = s;
    }
  }
  return c;
}

__device__ __forceinline__ int chunk_to_row(const EngineParams& p, int c) {
  return p.uniform ? c / p.u_nch : p.chunk_row[c];
}

// ----------------------------------------------------------------------------
// Element iteration over positions [a, b) of a row, 16-byte vector loads
// in the aligned middle.  f(bits, pos, valid) is called by every thread the
// same number of times (warp-uniform), so f may use warp collectives.
// ----------------------------------------------------------------------------
template <int VT, bool SCALE, int U, typename F>
__device__ __forceinline__ void for_range(const void* base, int64_t in_off, int64_t a, int64_t b, F&& f) {
  using K = KT<VT, SCALE>;
  constexpr int ES = K::ES, VEC = K::VEC;
  if (b <= a) return;
  const char* row = static_cast<const char*>(base) + in_off * ES;
  const uintptr_t addr_a = reinterpret_cast<uintptr_t>(row + a * ES);
  int64_t head = (int64_t)(((16u - (unsigned)(addr_a & 15u)) & 15u) / ES);
  if (head > b - a) head = b - a;
  const int64_t va = a + head;
  const int64_t nvec = (b - va) / VEC;
  const int64_t vb = va + nvec * VEC;
  const int64_t tail = b - vb;
  // head and tail: fewer than VEC elements each
  {
    const int t = threadIdx.x;
    const bool vh = t < head;
    const bool vt = t < tail;
    uint32_t bh = 0, bt = 0;
    if (vh) bh = ES == 4 ? reinterpret_cast<const uint32_t*>(row)[a + t]
                         : (uint32_t)reinterpret_cast<const unsigned short*>(row)[a + t];
    if (vt) bt = ES == 4 ? reinterpret_cast<const uint32_t*>(row)[vb + t]
                         : (uint32_t)reinterpret_cast<const unsigned short*>(row)[vb + t];
    if (head > 0) f(bh, a + t, vh);
    if (tail > 0) f(bt, vb + t, vt);
  }
  const uint4* vp = reinterpret_cast<const uint4*>(row + va * ES);
  const int64_t iters = (nvec + (int64_t)kThreads * U - 1) / ((int64_t)kThreads * U);
  int64_t v0 = threadIdx.x;
  for (int64_t it = 0; it < iters; ++it, v0 += (int64_t)kThreads * U) {
    uint4 x[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t v = v0 + (int64_t)u * kThreads;
      if (v < nvec) x[u] = ld_stream16(vp + v);
      else x[u] = make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t v = v0 + (int64_t)u * kThreads;
      const bool ok = v < nvec;
      const int64_t p0 = va + v * VEC;
      const uint32_t w[4] = {x[u].x, x[u].y, x[u].z, x[u].w};
      if constexpr (ES == 4) {
#pragma unroll
        for (int e = 0; e < 4; ++e) f(w[e], p0 + e, ok);
      } else {
#pragma unroll
        for (int e = 0; e < 8; ++e) f((w[e >> 1] >> ((e & 1) * 16)) & 0xFFFFu, p0 + e, ok);
      }
    }
  }
}

// ----------------------------------------------------------------------------
// Output / candidate sinks with warp-aggregated reservations
// ----------------------------------------------------------------------------
template <int VT>
__device__ __forceinline__ void write_out(const EngineParams& p, int64_t slot, uint32_t bits, int64_t pos) {
  if constexpr (VT == kF32) static_cast<uint32_t*>(p.val_out)[slot] = bits;
  else static_cast<unsigned short*>(p.val_out)[slot] = (unsigned short)bits;
  if (p.flags & kFlagIdx64) static_cast<int64_t*>(p.idx_out)[slot] = pos;
  else static_cast<int32_t*>(p.idx_out)[slot] = (int32_t)pos;
}

// Warp-level reservation: every lane passes its count; returns the lane's
// first slot (base + exclusive prefix).  ctr may be global or shared.
__device__ __forceinline__ uint32_t warp_reserve(uint32_t cnt, uint32_t* ctr) {
  const int lane = threadIdx.x & 31;
  uint32_t x = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  const uint32_t tot = __shfl_sync(kFull, x, 31);
  uint32_t base = 0;
  if (tot) {
    if (lane == 31) base = atomicAdd(ctr, tot);
    base = __shfl_sync(kFull, base, 31);
  }
  return base + x - cnt;
}

// ----------------------------------------------------------------------------
// Shared-memory resolution of a candidate set
// ----------------------------------------------------------------------------
// Entries get(i) -> (bits, pos), all matching (prefix, plen).  Refines the
// prefix with 8-bit digits over the composite (key << IB | pos) until the
// matched set size equals krem.  On return the selected entries are those
// whose composite prefix is <= prefix.
template <int VT, bool SCALE, typename G>
__device__ void smem_resolve(G get, int cnt, const RowCtx& rc, uint64_t& prefix, int& plen, int& krem,
                             int count, Misc* m, int32_t* status) {
  using K = KT<VT, SCALE>;
  const int W = K::KB + rc.IB;
  while (count != krem) {
    if (plen >= W || count < krem) {
      if (threadIdx.x == 0) atomicOr(status, kStatusLevels);
      break;
    }
    const int D = min(8, W - plen);
    for (int i = threadIdx.x; i < 256; i += kThreads) m->hist256[i] = 0;
    __syncthreads();
    const int sh = W - plen;
    const int sd = W - plen - D;
    const uint32_t dm = (1u << D) - 1u;
    for (int i = threadIdx.x; i < cnt; i += kThreads) {
      uint32_t bits;
      int64_t pos;
      get(i, bits, pos);
      const uint64_t c = ((uint64_t)sel_key<VT, SCALE>(bits, rc.flip, rc.scaler) << rc.IB) | (uint64_t)pos;
      if (shr64(c, sh) == prefix) atomicAdd(&m->hist256[(uint32_t)shr64(c, sd) & dm], 1u);
    }
    __syncthreads();
    block_select<false>(m->hist256, 1 << D, (uint32_t)krem, m);
    if (!m->sel_found) {
      if (threadIdx.x == 0) atomicOr(status, kStatusSelect);
      break;
    }
    prefix = (prefix << D) | m->sel_bin;
    plen += D;
    krem -= (int)m->sel_cum;
    count = (int)m->sel_cnt;
    __syncthreads();
  }
}

// Emits the entries selected by (prefix, plen) to the row's output, in entry
// order, reserving the slots with one atomic on the row's out_count.
template <int VT, bool SCALE, typename G>
__device__ void smem_emit(const EngineParams& p, G get, int cnt, const RowCtx& rc, uint64_t prefix, int plen,
                          RowState* rs, Misc* m) {
  using K = KT<VT, SCALE>;
  const int W = K::KB + rc.IB;
  const int sh = W - plen;
  const int per = (cnt + kThreads - 1) / kThreads;
  const int lo = min(cnt, (int)threadIdx.x * per);
  const int hi = min(cnt, lo + per);
  uint32_t mine = 0;
  for (int i = lo; i < hi; ++i) {
    uint32_t bits;
    int64_t pos;
    get(i, bits, pos);
    const uint64_t c = ((uint64_t)sel_key<VT, SCALE>(bits, rc.flip, rc.scaler) << rc.IB) | (uint64_t)pos;
    mine += shr64(c, sh) <= prefix;
  }
  uint32_t total;
  const uint32_t ex = block_excl_scan(mine, m->scan, &total);
  if (threadIdx.x == 0) m->counter = total ? atomicAdd(reinterpret_cast<uint32_t*>(&rs->out_count), total) : 0u;
  __syncthreads();
  int64_t slot = (int64_t)m->counter + ex;
  for (int i = lo; i < hi; ++i) {
    uint32_t bits;
    int64_t pos;
    get(i, bits, pos);
    const uint64_t c = ((uint64_t)sel_key<VT, SCALE>(bits, rc.flip, rc.scaler) << rc.IB) | (uint64_t)pos;
    if (shr64(c, sh) <= prefix) {
      if (slot < rc.k) write_out<VT>(p, rc.out_off + slot, bits, pos);
      ++slot;
    }
  }
  __syncthreads();
}

// ----------------------------------------------------------------------------
// Row post-processing: sort, index mapping, idle fill
// ----------------------------------------------------------------------------
template <int VT, bool SCALE>
__device__ void post_process(const EngineParams& p, const RowCtx& rc, uint8_t* smem, Misc* m) {
  const int64_t kk = min((int64_t)rc.n, (int64_t)rc.k);
  const bool idx64 = (p.flags & kFlagIdx64) != 0;
  const bool withidx = (p.flags & kFlagWithIdxIn) != 0;
  __threadfence();
  __syncthreads();
  auto load_pos = [&](int64_t i) -> int64_t {
    return idx64 ? (int64_t)__ldcg(reinterpret_cast<const long long*>(p.idx_out) + rc.out_off + i)
                 : (int64_t)__ldcg(static_cast<const int32_t*>(p.idx_out) + rc.out_off + i);
  };
  auto load_bits = [&](int64_t i) -> uint32_t {
    if constexpr (VT == kF32) return __ldcg(static_cast<const uint32_t*>(p.val_out) + rc.out_off + i);
    else return (uint32_t)__ldcg(static_cast<const unsigned short*>(p.val_out) + rc.out_off + i);
  };
  auto map_idx = [&](int64_t pos) -> int64_t {
    if (!withidx) return pos;
    return idx64 ? (int64_t)__ldg(static_cast<const long long*>(p.idx_in) + rc.in_off + pos)
                 : (int64_t)__ldg(static_cast<const int32_t*>(p.idx_in) + rc.in_off + pos);
  };
  if ((p.flags & kFlagSorted) && kk > 1) {
    const bool ascend = (p.flags & kFlagAscend) != 0;
    if (kk <= kCapSort) {
      uint64_t* s = reinterpret_cast<uint64_t*>(smem);
      int np = 2;
      while (np < kk) np <<= 1;
      for (int i = threadIdx.x; i < np; i += kThreads) {
        uint64_t v = ~0ull;
        if (i < kk) v = ((uint64_t)out_key<VT>(load_bits(i), ascend) << 32) | (uint64_t)(uint32_t)load_pos(i);
        s[i] = v;
      }
      __syncthreads();
      block_bitonic_sort(s, np);
      for (int i = threadIdx.x; i < kk; i += kThreads) {
        const uint64_t v = s[i];
        const int64_t pos = (int64_t)(uint32_t)v;
        write_out<VT>(p, rc.out_off + i, out_key_inv<VT>((uint32_t)(v >> 32), ascend), map_idx(pos));
      }
    } else if (rc.sort_off >= 0) {
      // Merge sort through global scratch: runs of kCapSort sorted in smem,
      // then pairwise merges (each thread merges a contiguous output range
      // found by a merge-path search).
      uint64_t* a = p.sort_scratch + rc.sort_off;
      uint64_t* b = a + kk;
      uint64_t* s = reinterpret_cast<uint64_t*>(smem);
      for (int64_t r0 = 0; r0 < kk; r0 += kCapSort) {
        const int len = (int)min((int64_t)kCapSort, kk - r0);
        for (int i = threadIdx.x; i < kCapSort; i += kThreads) {
          uint64_t v = ~0ull;
          if (i < len)
            v = ((uint64_t)out_key<VT>(load_bits(r0 + i), ascend) << 32) | (uint64_t)(uint32_t)load_pos(r0 + i);
          s[i] = v;
        }
        __syncthreads();
        block_bitonic_sort(s, kCapSort);
        for (int i = threadIdx.x; i < len; i += kThreads) a[r0 + i] = s[i];
        __syncthreads();
      }
      __threadfence_block();
      __syncthreads();
      for (int64_t run = kCapSort; run < kk; run <<= 1) {
        for (int64_t m0 = 0; m0 < kk; m0 += 2 * run) {
          const int64_t l0 = m0, l1 = min(kk, m0 + run), r1 = min(kk, m0 + 2 * run);
          const int64_t tot = r1 - l0;
          const int64_t per = (tot + kThreads - 1) / kThreads;
          const int64_t d0 = min(tot, (int64_t)threadIdx.x * per), d1 = min(tot, d0 + per);
          auto split = [&](int64_t d) -> int64_t {  // elements taken from the left run
            int64_t lo = max((int64_t)0, d - (r1 - l1)), hi = min(d, l1 - l0);
            while (lo < hi) {
              const int64_t mid = (lo + hi) >> 1;
              if (__ldcg(reinterpret_cast<const unsigned long long*>(a + l0 + mid)) <=
                  __ldcg(reinterpret_cast<const unsigned long long*>(a + l1 + (d - mid - 1))))
                lo = mid + 1;
              else
                hi = mid;
            }
            return lo;
          };
          if (d0 < d1) {
            int64_t i = l0 + split(d0), j = l1 + (d0 - (i - l0));
            for (int64_t d = d0; d < d1; ++d) {
              const uint64_t x = i < l1 ? (uint64_t)__ldcg(reinterpret_cast<const unsigned long long*>(a + i)) : ~0ull;
              const uint64_t y = j < r1 ? (uint64_t)__ldcg(reinterpret_cast<const unsigned long long*>(a + j)) : ~0ull;
              const bool takel = (j >= r1) || (i < l1 && x <= y);
              b[l0 + d] = takel ? x : y;
              if (takel) ++i;
              else ++j;
            }
          }
        }
        __threadfence_block();
        __syncthreads();
        uint64_t* t = a;
        a = b;
        b = t;
      }
      for (int64_t i = threadIdx.x; i < kk; i += kThreads) {
        const uint64_t v = (uint64_t)__ldcg(reinterpret_cast<const unsigned long long*>(a + i));
        write_out<VT>(p, rc.out_off + i, out_key_inv<VT>((uint32_t)(v >> 32), ascend), map_idx((int64_t)(uint32_t)v));
      }
    }
  } else if (withidx) {
    for (int64_t i = threadIdx.x; i < kk; i += kThreads) {
      const int64_t pos = load_pos(i);
      const int64_t mapped = map_idx(pos);
      if (idx64) static_cast<int64_t*>(p.idx_out)[rc.out_off + i] = mapped;
      else static_cast<int32_t*>(p.idx_out)[rc.out_off + i] = (int32_t)mapped;
    }
  }
  for (int64_t i = kk + threadIdx.x; i < rc.k; i += kThreads) write_out<VT>(p, rc.out_off + i, 0u, -1);
  __syncthreads();
}

// ----------------------------------------------------------------------------
// Items
// ----------------------------------------------------------------------------
template <int VT, bool SCALE>
struct Engine {
  using K = KT<VT, SCALE>;
  static constexpr int U = 4;

  const EngineParams& p;
  uint8_t* smem;
  Misc* m;

  __device__ Engine(const EngineParams& p_, uint8_t* s) : p(p_), smem(s), m(misc_of(s)) {}

  __device__ bool spin_until_ge(const uint32_t* addr, uint32_t target) {
    for (uint32_t it = 0; it < p.spin_limit; ++it) {
      if (ld_acquire(addr) >= target) return true;
      __nanosleep(64);
    }
    atomicOr(&p.hdr->status, kStatusTimeout);
    return false;
  }

  // Whole row selected in shared memory (n <= kSmemRowCap).
  __device__ void smem_row_full(int r, const RowCtx& rc) {
    uint32_t* vals = reinterpret_cast<uint32_t*>(smem);
    for_range<VT, SCALE, U>(p.val_in, rc.in_off, 0, rc.n, [&](uint32_t bits, int64_t pos, bool ok) {
      if (ok) vals[pos] = bits;
    });
    __syncthreads();
    const int kk = min(rc.n, rc.k);
    uint64_t prefix = 0;
    int plen = 0, krem = kk;
    auto get = [&](int i, uint32_t& bits, int64_t& pos) {
      bits = vals[i];
      pos = i;
    };
    smem_resolve<VT, SCALE>(get, rc.n, rc, prefix, plen, krem, rc.n, m, &p.hdr->status);
    smem_emit<VT, SCALE>(p, get, rc.n, rc, prefix, plen, p.rs + r, m);
    // the sort area must not overlap the values while they are read: the
    // emission above has finished (it ends with a barrier)
    post_process<VT, SCALE>(p, rc, smem + 65536, m);
  }

  // H item: histogram of the first digit over chunk j of row r.
  __device__ void h_item(int r, const RowCtx& rc, int j) {
    if (rc.kind == kKindSmem) {
      smem_row_full(r, rc);
      return;
    }
    if (rc.kind != kKindMulti) return;
    const int D1 = p.D1;
    const int NB = 1 << D1;
    const int s = rc.slot_use % p.S;
    const uint32_t use = (uint32_t)(rc.slot_use / p.S);
    uint32_t* hist = reinterpret_cast<uint32_t*>(smem);
    uint32_t* ghist = p.hist_ring + (size_t)s * NB;
    if (threadIdx.x == 0) m->bcast = use == 0 ? 1 : (int)spin_until_ge(p.slot_gen + s, use);
    for (int i = threadIdx.x * 4; i < NB; i += kThreads * 4) *reinterpret_cast<uint4*>(hist + i) = make_uint4(0, 0, 0, 0);
    __syncthreads();
    const bool slot_ok = m->bcast != 0;
    const int shift = K::KB - D1;
    const int64_t a = (int64_t)j * p.CH, b = min((int64_t)rc.n, a + p.CH);
    for_range<VT, SCALE, U>(p.val_in, rc.in_off, a, b, [&](uint32_t bits, int64_t, bool ok) {
      const uint32_t key = sel_key<VT, SCALE>(bits, rc.flip, rc.scaler);
      hist_add(hist, key >> shift, ok);
    });
    __syncthreads();
    if (slot_ok) {
      for (int i = threadIdx.x * 4; i < NB; i += kThreads * 4) {
        const uint4 v = *reinterpret_cast<const uint4*>(hist + i);
        if (v.x) atomicAdd(ghist + i + 0, v.x);
        if (v.y) atomicAdd(ghist + i + 1, v.y);
        if (v.z) atomicAdd(ghist + i + 2, v.z);
        if (v.w) atomicAdd(ghist + i + 3, v.w);
      }
    }
    __threadfence();
    __syncthreads();
    RowState* rs = p.rs + r;
    if (threadIdx.x == 0) m->bcast2 = atomicAdd(&rs->hticket, 1) == rc.nch - 1;
    __syncthreads();
    if (!m->bcast2) return;
    // Last H item of the row: select the first digit's bin.
    __threadfence();
    block_select<true>(ghist, NB, (uint32_t)rc.k, m);
    const bool found = m->sel_found != 0;
    const uint32_t bin = m->sel_bin, cum = m->sel_cum, cnt = m->sel_cnt;
    for (int i = threadIdx.x * 4; i < NB; i += kThreads * 4) *reinterpret_cast<uint4*>(ghist + i) = make_uint4(0, 0, 0, 0);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      int mode;
      const int krem = rc.k - (int)cum;
      if (!found || !slot_ok) {
        mode = kModeNone;
        if (!found) atomicOr(&p.hdr->status, kStatusSelect);
      } else if ((int)cnt == krem) {
        mode = kModeFinal;
      } else if ((int)cnt <= kCapSB) {
        mode = kModeSB;
      } else if ((int)cnt <= rc.cand_cap) {
        mode = kModeCand;
      } else {
        mode = kModeDefer;
      }
      rs->mode = mode;
      rs->krem = krem;
      rs->count = (int)cnt;
      rs->prefix = bin;
      rs->plen = D1;
      __threadfence();
      st_release(p.slot_gen + s, use + 1);
      st_release(&rs->ready, 1);
    }
  }

  // Classify-and-emit pass over positions [a, b) of a row for a level-1
  // prefix: digit < prefix -> output; digit == prefix -> output (FINAL) or
  // candidate (SB/CAND); ALL mode -> output.
  __device__ void f_range(const RowCtx& rc, RowState* rs, int64_t a, int64_t b, int mode, uint32_t prefix,
                          int shift) {
    uint32_t* out_ctr = reinterpret_cast<uint32_t*>(&rs->out_count);
    uint32_t* cand_ctr = reinterpret_cast<uint32_t*>(&rs->cand_count);
    uint64_t* cand = p.cand + rc.cand_off;
    const bool all = mode == kModeAll;
    const bool final_mode = mode == kModeFinal;
    for_range<VT, SCALE, U>(p.val_in, rc.in_off, a, b, [&](uint32_t bits, int64_t pos, bool ok) {
      bool to_out = false, to_cand = false;
      if (ok) {
        if (all) {
          to_out = true;
        } else {
          const uint32_t d = sel_key<VT, SCALE>(bits, rc.flip, rc.scaler) >> shift;
          to_out = d < prefix || (final_mode && d == prefix);
          to_cand = !final_mode && d == prefix;
        }
      }
      const unsigned any = __ballot_sync(kFull, to_out || to_cand);
      if (!any) return;
      const uint32_t so = warp_reserve(to_out ? 1u : 0u, out_ctr);
      if (to_out && so < (uint32_t)rc.k) write_out<VT>(p, rc.out_off + so, bits, pos);
      const uint32_t sc = warp_reserve(to_cand ? 1u : 0u, cand_ctr);
      if (to_cand) {
        if (sc < (uint32_t)rc.cand_cap) cand[sc] = ((uint64_t)bits << 32) | (uint64_t)(uint32_t)pos;
        else atomicOr(&p.hdr->status, kStatusOverflow);
      }
    });
  }

  // F item: filter chunk j of row r.  Returns true if this CTA finished the
  // row's last F item (it then owes the row's finisher work).
  __device__ bool f_item(int r, const RowCtx& rc, int j) {
    if (rc.kind != kKindMulti && rc.kind != kKindAll) return false;
    RowState* rs = p.rs + r;
    const int64_t a = (int64_t)j * p.CH, b = min((int64_t)rc.n, a + p.CH);
    if (rc.kind == kKindAll) {
      f_range(rc, rs, a, b, kModeAll, 0u, 0);
    } else {
      if (threadIdx.x == 0) {
        int mode = kModeNone;
        if (spin_until_ge(reinterpret_cast<const uint32_t*>(&rs->ready), 1u)) mode = __ldcg(&rs->mode);
        m->st_mode = mode;
        m->st_prefix = __ldcg(reinterpret_cast<const unsigned long long*>(&rs->prefix));
      }
      __syncthreads();
      const int mode = m->st_mode;
      const uint32_t prefix = (uint32_t)m->st_prefix;
      if (mode == kModeFinal || mode == kModeSB || mode == kModeCand)
        f_range(rc, rs, a, b, mode, prefix, K::KB - p.D1);
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) m->bcast2 = atomicAdd(&rs->fticket, 1) == rc.nch - 1;
    __syncthreads();
    return m->bcast2 != 0;
  }

  // ---- single-CTA continuation for a row whose matched set is too large
  // for shared memory.  Source: the candidate region (CAND) or the row
  // itself (DEFER).  Levels of 12-bit digits over the composite until the
  // matched set fits in shared memory (or equals krem), then one filter pass.
  template <typename Fn>
  __device__ void for_source(const RowCtx& rc, bool from_cand, int ncand, Fn&& fn) {
    if (from_cand) {
      const uint64_t* cand = p.cand + rc.cand_off;
      const int iters = (ncand + kThreads - 1) / kThreads;
      for (int it = 0; it < iters; ++it) {
        const int i = it * kThreads + threadIdx.x;
        const bool ok = i < ncand;
        uint64_t e = 0;
        if (ok) e = ld_cg_u64(cand + i);
        fn((uint32_t)(e >> 32), (int64_t)(uint32_t)e, ok);
      }
    } else {
      for_range<VT, SCALE, U>(p.val_in, rc.in_off, 0, rc.n, fn);
    }
  }

  __device__ void large_row(int r, const RowCtx& rc, bool from_cand) {
    RowState* rs = p.rs + r;
    if (threadIdx.x == 0) {
      m->st_krem = __ldcg(&rs->krem);
      m->st_count = __ldcg(&rs->count);
      m->st_plen = __ldcg(&rs->plen);
      m->st_prefix = __ldcg(reinterpret_cast<const unsigned long long*>(&rs->prefix));
      m->st_candn = __ldcg(&rs->cand_count);
    }
    __syncthreads();
    uint64_t prefix = m->st_prefix;
    int plen = m->st_plen, krem = m->st_krem, count = m->st_count;
    const int ncand = min(m->st_candn, rc.cand_cap);
    const int W = K::KB + rc.IB;
    uint32_t* hist = reinterpret_cast<uint32_t*>(smem);
    uint32_t* out_ctr = reinterpret_cast<uint32_t*>(&rs->out_count);
    __syncthreads();
    for (int guard = 0; guard < 16; ++guard) {
      if (count == krem || count <= kCapSB) break;
      const int D = min(12, W - plen);
      if (D <= 0) break;
      const int NB = 1 << D;
      for (int i = threadIdx.x; i < NB; i += kThreads) hist[i] = 0;
      __syncthreads();
      const int sh = W - plen, sd = W - plen - D;
      const uint32_t dm = (uint32_t)NB - 1u;
      for_source(rc, from_cand, ncand, [&](uint32_t bits, int64_t pos, bool ok) {
        bool hit = false;
        uint32_t dig = 0;
        if (ok) {
          const uint64_t c = ((uint64_t)sel_key<VT, SCALE>(bits, rc.flip, rc.scaler) << rc.IB) | (uint64_t)pos;
          hit = shr64(c, sh) == prefix;
          dig = (uint32_t)shr64(c, sd) & dm;
        }
        hist_add(hist, dig, hit);
      });
      __syncthreads();
      block_select<false>(hist, NB, (uint32_t)krem, m);
      if (!m->sel_found) {
        if (threadIdx.x == 0) atomicOr(&p.hdr->status, kStatusSelect);
        return;
      }
      prefix = (prefix << D) | m->sel_bin;
      plen += D;
      krem -= (int)m->sel_cum;
      count = (int)m->sel_cnt;
      __syncthreads();
    }
    if (count != krem && count > kCapSB) {
      if (threadIdx.x == 0) atomicOr(&p.hdr->status, kStatusLevels);
      return;
    }
    // Final filter pass over the source.
    const bool final_mode = count == krem;
    uint64_t* ent = reinterpret_cast<uint64_t*>(smem);
    if (threadIdx.x == 0) m->counter = 0;
    __syncthreads();
    const int sh = W - plen;
    for_source(rc, from_cand, ncand, [&](uint32_t bits, int64_t pos, bool ok) {
      bool to_out = false, to_ent = false;
      if (ok) {
        const uint64_t c = ((uint64_t)sel_key<VT, SCALE>(bits, rc.flip, rc.scaler) << rc.IB) | (uint64_t)pos;
        const uint64_t t = shr64(c, sh);
        to_out = t < prefix || (final_mode && t == prefix);
        to_ent = !final_mode && t == prefix;
      }
      const unsigned any = __ballot_sync(kFull, to_out || to_ent);
      if (!any) return;
      const uint32_t so = warp_reserve(to_out ? 1u : 0u, out_ctr);
      if (to_out && so < (uint32_t)rc.k) write_out<VT>(p, rc.out_off + so, bits, pos);
      const uint32_t se = warp_reserve(to_ent ? 1u : 0u, &m->counter);
      if (to_ent && se < (uint32_t)kCapSB) ent[se] = ((uint64_t)bits << 32) | (uint64_t)(uint32_t)pos;
    });
    __syncthreads();
    if (!final_mode) {
      const int ne = min((int)m->counter, kCapSB);
      auto get = [&](int i, uint32_t& bits, int64_t& pos) {
        const uint64_t e = ent[i];
        bits = (uint32_t)(e >> 32);
        pos = (int64_t)(uint32_t)e;
      };
      smem_resolve<VT, SCALE>(get, ne, rc, prefix, plen, krem, ne, m, &p.hdr->status);
      smem_emit<VT, SCALE>(p, get, ne, rc, prefix, plen, rs, m);
    }
  }

  // Finisher work of a multi-chunk row (all of its F items are done).
  __device__ void finish_row(int r) {
    const RowCtx rc = load_row<VT, SCALE>(p, r);
    RowState* rs = p.rs + r;
    __threadfence();
    if (threadIdx.x == 0) {
      m->st_mode = rc.kind == kKindAll ? kModeAll : __ldcg(&rs->mode);
      m->st_krem = __ldcg(&rs->krem);
      m->st_count = __ldcg(&rs->count);
      m->st_plen = __ldcg(&rs->plen);
      m->st_prefix = __ldcg(reinterpret_cast<const unsigned long long*>(&rs->prefix));
      m->st_candn = __ldcg(&rs->cand_count);
    }
    __syncthreads();
    const int mode = m->st_mode;
    if (mode == kModeSB) {
      const int ne = min(m->st_candn, kCapSB);
      uint64_t* ent = reinterpret_cast<uint64_t*>(smem);
      const uint64_t* cand = p.cand + rc.cand_off;
      for (int i = threadIdx.x; i < ne; i += kThreads) ent[i] = ld_cg_u64(cand + i);
      uint64_t prefix = m->st_prefix;
      int plen = m->st_plen, krem = m->st_krem;
      __syncthreads();
      auto get = [&](int i, uint32_t& bits, int64_t& pos) {
        const uint64_t e = ent[i];
        bits = (uint32_t)(e >> 32);
        pos = (int64_t)(uint32_t)e;
      };
      smem_resolve<VT, SCALE>(get, ne, rc, prefix, plen, krem, ne, m, &p.hdr->status);
      smem_emit<VT, SCALE>(p, get, ne, rc, prefix, plen, rs, m);
    } else if (mode == kModeCand) {
      large_row(r, rc, true);
    } else if (mode == kModeDefer) {
      large_row(r, rc, false);
    }
    if (mode != kModeNone) post_process<VT, SCALE>(p, rc, smem, m);
  }
};

// Maps a claim index to an item: true = H item, chunk id in c.
__device__ __forceinline__ bool decode_item(int q, int NC, int L, int& c) {
  if (q < L) {
    c = q;
    return true;
  }
  const int alt_end = 2 * NC - L;
  if (q < alt_end) {
    const int t = q - L;
    if ((t & 1) == 0) {
      c = L + (t >> 1);
      return true;
    }
    c = t >> 1;
    return false;
  }
  c = q - NC;
  return false;
}

template <int VT, bool SCALE>
__global__ void __launch_bounds__(kThreads, 1) engine_kernel(const __grid_constant__ EngineParams p) {
  extern __shared__ __align__(16) uint8_t smem[];
  Engine<VT, SCALE> e(p, smem);
  Misc* m = e.m;
  const int NC = p.uniform ? p.B * p.u_nch : __ldcg(&p.hdr->nc);
  if (!p.uniform && __ldcg(&p.hdr->plan_error)) return;
  const int lag = p.uniform ? p.lag : __ldcg(&p.hdr->lag);
  const int L = min(max(lag, 1), NC);
  const int NQ = 2 * NC;
  if (threadIdx.x == 0) m->next_q = (int)atomicAdd(&p.hdr->qhead, 1u);
  __syncthreads();
  int q = m->next_q;
  int pending = -1;
  while (true) {
    if (q >= NQ) {
      if (pending >= 0) e.finish_row(pending);
      break;
    }
    __syncthreads();
    const bool prefetch = pending < 0;
    uint32_t nq = 0;
    if (threadIdx.x == 0 && prefetch) nq = atomicAdd(&p.hdr->qhead, 1u);
    int c;
    const bool isH = decode_item(q, NC, L, c);
    const int r = chunk_to_row(p, c);
    const RowCtx rc = load_row<VT, SCALE>(p, r);
    const int j = c - rc.chunk0;
    int fin = -1;
    if (isH) e.h_item(r, rc, j);
    else if (e.f_item(r, rc, j)) fin = r;
    if (pending >= 0) {
      e.finish_row(pending);
      pending = -1;
    }
    pending = fin;
    __syncthreads();
    if (threadIdx.x == 0) m->next_q = prefetch ? (int)nq : (int)atomicAdd(&p.hdr->qhead, 1u);
    __syncthreads();
    q = m->next_q;
  }
}

// ----------------------------------------------------------------------------
// Planning kernel (non-uniform batches): one CTA scans the row descriptors.
// ----------------------------------------------------------------------------
__device__ int64_t block_excl_scan64(int64_t v, int64_t* scan, int64_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) scan[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int64_t w = scan[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(kFull, w, o);
      if (lane >= o) w += y;
    }
    scan[lane] = w;
  }
  __syncthreads();
  const int64_t base = warp ? scan[warp - 1] : 0;
  if (total) *total = scan[kWarps - 1];
  __syncthreads();
  return base + x - v;
}

__global__ void __launch_bounds__(kThreads, 1)
    plan_kernel(const RowDesc* desc, int B, int CH, uint32_t flags, RowPlan* plans, int32_t* chunk_row,
                Header* hdr, int64_t nc_cap, int64_t cand_cap_total, int64_t sort_cap_total, int grid) {
  __shared__ int64_t scan[32];
  __shared__ int64_t run[4];
  __shared__ int32_t maxnch;
  if (threadIdx.x < 4) run[threadIdx.x] = 0;
  if (threadIdx.x == 0) maxnch = 1;
  __syncthreads();
  const bool sorted = (flags & kFlagSorted) != 0;
  for (int base = 0; base < B; base += kThreads) {
    const int r = base + threadIdx.x;
    int64_t nch = 0, cand = 0, sortn = 0, multi = 0;
    RowDesc d{0, 0, 0, 0};
    int kind = kKindEmpty;
    if (r < B) {
      d = desc[r];
      kind = row_kind(d.n, d.k);
      nch = (kind == kKindMulti || kind == kKindAll) ? ((int64_t)d.n + CH - 1) / CH : 1;
      multi = kind == kKindMulti;
      cand = multi ? cand_capacity(d.n) : 0;
      const int64_t kk = min((int64_t)d.n, (int64_t)d.k);
      sortn = (sorted && kk > kCapSort) ? 2 * kk : 0;
      atomicMax(&maxnch, (int32_t)nch);
    }
    int64_t t0, t1, t2, t3;
    const int64_t e0 = block_excl_scan64(nch, scan, &t0);
    const int64_t e1 = block_excl_scan64(cand, scan, &t1);
    const int64_t e2 = block_excl_scan64(sortn, scan, &t2);
    const int64_t e3 = block_excl_scan64(multi, scan, &t3);
    if (r < B) {
      RowPlan pl;
      pl.in_off = d.in_off;
      pl.out_off = d.out_off;
      pl.cand_off = run[1] + e1;
      pl.sort_off = sortn ? run[2] + e2 : -1;
      pl.n = d.n;
      pl.k = d.k;
      pl.chunk0 = (int32_t)(run[0] + e0);
      pl.nch = (int32_t)nch;
      pl.cand_cap = (int32_t)cand;
      pl.slot_use = multi ? (int32_t)(run[3] + e3) : -1;
      pl.pad0 = pl.pad1 = 0;
      plans[r] = pl;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      run[0] += t0;
      run[1] += t1;
      run[2] += t2;
      run[3] += t3;
    }
    __syncthreads();
  }
  const bool ok = run[0] <= nc_cap && run[1] <= cand_cap_total && run[2] <= sort_cap_total && run[0] < (1ll << 30);
  if (threadIdx.x == 0) {
    hdr->nc = (int32_t)run[0];
    hdr->cand_total = run[1];
    hdr->sort_total = run[2];
    hdr->lag = max(maxnch, 2 * grid);
    hdr->plan_error = ok ? 0 : 1;
    if (!ok) atomicOr(&hdr->status, kStatusCapacity);
  }
  if (!ok) return;
  __syncthreads();
  // one warp per row fills the row's chunk -> row map
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int r = warp; r < B; r += kWarps) {
    const int32_t c0 = plans[r].chunk0, nch = plans[r].nch;
    for (int c = lane; c < nch; c += 32) chunk_row[c0 + c] = r;
  }
}

}  // namespace dev

// ----------------------------------------------------------------------------
// Host-side launchers (called from radik_api.cu)
// ----------------------------------------------------------------------------
template <int VT, bool SCALE>
static cudaError_t launch_typed(const EngineParams& p, int grid, cudaStream_t stream) {
  auto kern = dev::engine_kernel<VT, SCALE>;
  // The smem opt-in is per device; remember which devices have it.
  static bool attr_set[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64 || !attr_set[dev]) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) attr_set[dev] = true;
  }
  kern<<<grid, kThreads, kSmemBytes, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_engine(int dtype, const EngineParams& p, int grid, cudaStream_t stream) {
  const bool scale = (p.flags & kFlagWithScale) != 0;
  switch (dtype) {
    case kF32: return scale ? launch_typed<kF32, true>(p, grid, stream) : launch_typed<kF32, false>(p, grid, stream);
    case kF16: return scale ? launch_typed<kF16, true>(p, grid, stream) : launch_typed<kF16, false>(p, grid, stream);
    case kBF16: return scale ? launch_typed<kBF16, true>(p, grid, stream) : launch_typed<kBF16, false>(p, grid, stream);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_plan(const RowDesc* desc, int B, int CH, uint32_t flags, RowPlan* plans, int32_t* chunk_row,
                        Header* hdr, int64_t nc_cap, int64_t cand_cap_total, int64_t sort_cap_total, int grid,
                        cudaStream_t stream) {
  dev::plan_kernel<<<1, kThreads, 0, stream>>>(desc, B, CH, flags, plans, chunk_row, hdr, nc_cap, cand_cap_total,
                                               sort_cap_total, grid);
  return cudaGetLastError();
}

}  // namespace radik

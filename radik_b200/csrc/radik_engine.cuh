// radik_engine.cu -- the B200 radix top-k selection engine.
//
// One cooperative persistent launch (one 1024-thread CTA per SM) selects every
// row of a batch.  It replaces RadiK's chain of ~10 launches and 2 host syncs
// per call (radik/RadixSelect/topk_radixselect.h:117-307).
//
// Phase A: a work queue of items claimed from one global counter.
//   * smem rows (n <= 16K): one item loads the row into shared memory and
//     selects it there (8-bit radix digits over the composite key).
//   * CTA rows (n <= 256K): one item; one CTA samples the row, filters it
//     against the sampled threshold into shared memory and resolves it, or
//     runs radix levels over the row (second reads come from L2).
//   * large rows with k * 64 <= n ("pre-filter" rows): a sample item picks a
//     threshold key T (the r-th smallest of a strided sample, r about twice
//     the expected rank of the k-th key plus a margin); then one read of the
//     row (filter items, one per chunk) compacts the keys <= T into the row's
//     candidate region.  This fuses RadiK's first histogram and candidate
//     passes (countBinEx + selectCandidateEx, radixselect_l.cuh:173-408)
//     and its final filter (:438-832) into a single read of the keys.
//   * other large rows ("radix" rows): histogram items compute the first
//     digit (14 bits) of each chunk in shared memory (countBinEx); the CTA
//     finishing a row's last histogram item selects the bin (selectBin,
//     radixselect_l.cuh:45-126) in the same kernel; filter items then re-read
//     the chunks (from L2: they trail the histogram items by a lag) and emit
//     keys of better bins and compact the selected bin.
//   The CTA finishing a row's last item resolves the row's candidates in
//   shared memory (RadiK's passes 2-3 and filter) and sorts the outputs
//   (bitonicSort_*, bitonic_sort.cuh:195-553).
// Phase B (after a grid barrier; empty for i.i.d. data): rows whose
//   threshold missed, whose candidates exceed shared memory, or whose
//   selected bin is huge (skewed / adversarial rows) run multi-CTA radix
//   levels of 12-bit digits over their candidates or the row, with grid
//   barriers between histogram, bin selection, filter and finish.
//
// Ties at the k-th key go to the lowest positions: selection is over the
// composite (key << IB | position).  Every wait is bounded (spin_limit); a wait
// that gives up sets a status bit and the kernel still exits.
//
// Queue order: A items (sample / histogram / single-item rows / copy chunks)
// and B items (filter chunks) interleave after the first L A items; every B
// item of a row comes after all A items of that row (L is planned so), so a
// CTA that waits for a row's threshold or bin only waits for items already
// claimed by running CTAs, and the smallest unfinished item always progresses.

#pragma once

#include "radik_common.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <mutex>

namespace radik {
namespace dev {

constexpr unsigned kFull = 0xFFFFFFFFu;

// Timeline build (-DRADIK_TIMELINE): thread 0 of a team writes %globaltimer
// (ns) into slot s of its CTA's row of p.timeline at the engine's phase
// boundaries (kTl* below), for radik_b200.timeline.  In the normal build the
// stamps compile to nothing.
constexpr int kTlSlots = 32;
enum TlSlot : int {
  kTlStart = 0, kTlFirstSample = 1, kTlConsDone = 2, kTlSideDone = 3, kTlFinEnd = 4, kTlPhaseB = 5, kTlEnd = 6,
  kTlFinStart = 7, kTlSampleIn = 8, kTlSampleIssue = 9, kTlSampleKeys = 10, kTlItemStart = 14, kTlChunkEnd = 15,
  kTlFinBegin = 16, kTlFinLoaded = 17,
  kTlFinResolved = 18, kTlFinEmitted = 19, kTlFinPost = 20, kTlFinCands = 31,
  // per-CTA sums (SM clock cycles, or counts) of where the teams wait
  kTlNChunks = 11, kTlNSide = 12, kTlNFin = 13,
  kTlAccSideQ = 21,     // producer: blocked pushing to a full side queue
  kTlAccConsQ = 22,     // producer: blocked pushing to a full consumer queue
  kTlAccRing = 23,      // producer: waiting for a drained ring stage
  kTlAccThr = 24,       // producer: waiting for a chunk's threshold
  kTlAccFull = 25,      // consumer team: waiting for a stage's data
  kTlAccPre = 26,       // consumer team: waiting for a threshold before a chunk
  kTlAccConsIdle = 27,  // consumer team: waiting for an item
  kTlAccFinWait = 28,   // a finish waiting for its row's chunks
  kTlAccSideIdle = 29,  // side team: waiting for an item
  kTlAccClaim = 30      // producer: claim round trips not hidden behind copies
};
#ifdef RADIK_TIMELINE
__device__ __forceinline__ void tl_write(unsigned long long* tl, int slot, unsigned long long v) {
  if (tl) tl[(size_t)blockIdx.x * kTlSlots + slot] = v;
}
__device__ __forceinline__ unsigned long long tl_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void tl_add(unsigned long long* tl, int slot, unsigned long long v) {
  if (tl) tl[(size_t)blockIdx.x * kTlSlots + slot] += v;
}
#define RADIK_TL(p, slot) tl_write((p).timeline, (slot), tl_now())
#define RADIK_TL_VALUE(p, slot, v) tl_write((p).timeline, (slot), (unsigned long long)(v))
// RADIK_TL_T0(t) starts a wait; RADIK_TL_ACC(p, slot, t) adds its cycles.
#define RADIK_TL_T0(t) const long long t = clock64()
#define RADIK_TL_ACC(p, slot, t) tl_add((p).timeline, (slot), (unsigned long long)(clock64() - (t)))
#define RADIK_TL_COUNT(p, slot) tl_add((p).timeline, (slot), 1ull)
#else
#define RADIK_TL(p, slot) ((void)0)
#define RADIK_TL_VALUE(p, slot, v) ((void)0)
#define RADIK_TL_T0(t) ((void)0)
#define RADIK_TL_ACC(p, slot, t) ((void)0)
#define RADIK_TL_COUNT(p, slot) ((void)0)
#endif

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
__device__ __forceinline__ uint64_t ld_acquire_u64(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ void st_release_u64(uint64_t* p, uint64_t v) {
  asm volatile("st.release.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
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

// mbarrier + bulk asynchronous copy (TMA, no multicast) into this CTA's smem.
__device__ __forceinline__ uint32_t smem_u32(const void* ptr) {
  return (uint32_t)__cvta_generic_to_shared(ptr);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile(
      "{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}" ::"r"(smem_u32(bar)),
      "r"(bytes)
      : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Orders this thread's earlier generic-proxy smem accesses before later
// async-proxy (bulk copy) writes to the same smem.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// 16-byte asynchronous copy global -> smem (no registers held while in flight).
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// Bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned) from
// global to this CTA's smem; completion is counted on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Prefetch of [src, src + bytes) into L2 (both 16-byte multiples; this GPU's
// memory only).
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

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
// Shared memory of a CTA (kSmemBytes):
//   ring           kStages x kStageBytes, filled by the producer's bulk copies
//   consumer area  per-warp staging buffers / first-digit histogram
//   side area      sampled keys, candidate entries, sort and resolve scratch
//   control        per-team scratch (Misc), ring and queue mbarriers
constexpr int kStages = 4;
constexpr int kStageVecs = 24 * 32 * 3;                 // three 16-byte vectors per consumer thread
constexpr int kStageBytes = kStageVecs * 16;            // 36 KB
constexpr int kRingBytes = kStages * kStageBytes;       // 144 KB
// Stages a dtype's engine cycles through.  Every stage costs a handoff (each
// consumer warp arrives, the producer waits for all 24 before refilling), so
// the ring is a few large stages: 256 x 2^20, k = 256, fp32 / fp16 took
// 206.5 / 163.5 us with six 24 KB stages, 200.5 / 158.4 us with four 36 KB
// ones, 206.3 / 172.9 us with three 48 KB ones and 264 / 184 us with twelve
// 12 KB ones.
template <int VT>
__host__ __device__ constexpr int ring_stages() { return kStages; }
constexpr int kConsAreaOff = kRingBytes;
constexpr int kConsAreaBytes = 24 * 1024;
constexpr int kSideAreaOff = kConsAreaOff + kConsAreaBytes;
constexpr int kSideAreaBytes = 50 * 1024;
constexpr int kCtrlOff = kSideAreaOff + kSideAreaBytes;  // 218 KB
constexpr int kSinkCand = 96;                           // filter items: candidate entries per warp
constexpr int kSinkOut = 32;                            // filter / copy items: output entries per warp
constexpr int kSinkPf = 128;                            // pre-filter items: candidate entries per warp
// offsets inside an area
constexpr int kHistOff = 0;                             // first-digit histogram (<= 16 KB)
constexpr int kResolveHistOff = kCapSB * 8;             // 256-bin histogram behind a finisher's entries
constexpr int kSmemRowHistOff = kSmemRowCap * 4;        // behind an smem row's values
constexpr int kSampleHistOff = kSampleMax * 4;          // behind the sampled keys
constexpr int kSampleRawOff = kSampleHistOff + 1024;    // 16-bit sampled values before conversion
static_assert(24 * kSinkPf * 8 <= kConsAreaBytes, "pre-filter staging");
static_assert(24 * (kSinkCand + kSinkOut) * 8 <= kConsAreaBytes, "filter staging");
static_assert(32 * (kSinkCand + kSinkOut) * 8 <= kSideAreaBytes, "phase-B staging");
static_assert((4 << kMaxD1) <= kConsAreaBytes, "histogram");
static_assert(kResolveHistOff + 1024 <= kSideAreaBytes && 16384 <= kSideAreaBytes, "finisher area");
static_assert(kSmemRowHistOff + 1024 <= kSideAreaBytes && kCapSort * 8 <= kSideAreaBytes, "smem-row area");
static_assert(32 * 128 * 8 <= kSideAreaBytes, "phase-B staging");
static_assert(kSampleHistOff + 1024 <= kSideAreaBytes, "sample area");
static_assert(kSampleRawOff + kSampleMax * 2 <= kSideAreaBytes, "16-bit sample staging");

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
  int32_t rel_row;     // row whose chunk counter the next item releases (-1: none)
  int32_t t_row;       // row of the cached pre-filter threshold (-1: none)
  uint32_t t_val;      // the cached threshold
  int32_t pad[4];
  uint64_t red_lo, red_hi;
  uint64_t red_hi_w[32];
  int32_t pbtab[200];  // phase-B row table (row ids, chunk counts, prefix)
};
static_assert(sizeof(Misc) <= 3072, "Misc too large");

// A claimed work item, handed from the producer to a team.
struct alignas(16) ItemDesc {
  int32_t q;     // claim index, -1 = end of the queue
  int32_t row;
  int32_t isA;   // an A item (else a B item)
  int32_t fin;   // a FIN item
  int32_t sub;   // chunk index within the row
  int32_t nst;   // bulk-copy stages of a streaming item
  uint32_t g0;   // its first global ring stage
  uint32_t thr;  // pre-filter threshold, if the producer found it published
  int32_t thr_ok;
  int32_t pad[3];
  int64_t a, b;  // positions [a, b) of the chunk
  int64_t va;    // first 16-byte aligned position
  int64_t nvec;  // aligned 16-byte vectors from va
};
constexpr int kQ = 4;  // queue slots per team
constexpr int kCapTail = 16384;  // candidates a tail finish on the consumer team resolves in the ring
static_assert(kCapTail * 8 + 1024 <= kRingBytes && 32768 * 4 + 1024 <= kRingBytes, "ring as scratch");
constexpr int kSideCandMax = 1 << 17;  // candidate sets the side team resolves itself (else phase B)
// Batches of fewer rows leave the grid idle at their end, so there every set
// too large for smem goes to phase B, which resolves it with all CTAs --
// except sets of up to kTailResolveMax in a finish on the consumer team,
// which resolves them from L2 itself in less time than phase B's barriers.
constexpr int kSideResolveMinRows = 32;
constexpr int kTailResolveMax = 1 << 15;

struct Ctrl {
  uint64_t full[kStages];   // ring slot filled
  uint64_t empty[kStages];  // ring slot drained by every consumer warp
  uint64_t cq_full[kQ], cq_empty[kQ], sq_full[kQ], sq_empty[kQ];
  ItemDesc cq[kQ], sq[kQ];
  uint32_t side_done;       // side items finished (written by the side team)
  uint32_t cons_done;       // consumer items finished (written by the consumer team)
};
static_assert(kCtrlOff + 2 * 3072 + sizeof(Ctrl) <= kSmemBytes, "control area");

__device__ __forceinline__ Misc* cons_misc(uint8_t* smem) { return reinterpret_cast<Misc*>(smem + kCtrlOff); }
__device__ __forceinline__ Misc* side_misc(uint8_t* smem) { return reinterpret_cast<Misc*>(smem + kCtrlOff + 3072); }
__device__ __forceinline__ Ctrl* ctrl_of(uint8_t* smem) { return reinterpret_cast<Ctrl*>(smem + kCtrlOff + 6144); }

// ----------------------------------------------------------------------------
// Thread teams.  The CTA is split by warp role: warps 0-23 stream chunks
// (consumers), warps 24-30 do latency-bound work (samples, finishes, short
// rows), warp 31 claims items and issues the bulk copies (producer).  Each
// team synchronises on its own named barrier; the whole CTA on barrier 0.
// ----------------------------------------------------------------------------
template <int BASE, int SIZE, int BAR>
struct TeamT {
  static constexpr int kBase = BASE;
  static constexpr int kSize = SIZE;
  static constexpr int kWarps = SIZE / 32;
  __device__ __forceinline__ static int tid() { return (int)threadIdx.x - BASE; }
  __device__ __forceinline__ static int wid() { return ((int)threadIdx.x - BASE) >> 5; }
  __device__ __forceinline__ static void sync() {
    if constexpr (BAR == 0) __syncthreads();
    else asm volatile("bar.sync %0, %1;" ::"n"(BAR), "n"(SIZE) : "memory");
  }
};
constexpr int kConsWarps = 24;
constexpr int kSideWarps = 7;
constexpr int kProducerWarp = 31;
using ConsTeam = TeamT<0, kConsWarps * 32, 1>;
using SideTeam = TeamT<kConsWarps * 32, kSideWarps * 32, 2>;
using FullTeam = TeamT<0, kThreads, 0>;
static_assert(kConsWarps + kSideWarps + 1 == kWarps, "warp roles");

// ----------------------------------------------------------------------------
// Block primitives
// ----------------------------------------------------------------------------
// Exclusive scan of one value per thread; *total gets the block sum.
template <class Tm>
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* scan, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = Tm::wid();
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) scan[warp] = x;
  Tm::sync();
  if (warp == 0) {
    uint32_t w = lane < Tm::kWarps ? scan[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, w, o);
      if (lane >= o) w += y;
    }
    scan[lane] = w;
  }
  Tm::sync();
  const uint32_t base = warp ? scan[warp - 1] : 0u;
  if (total) *total = scan[Tm::kWarps - 1];
  Tm::sync();
  return base + x - v;
}

// Finds the bin b of h[0..NB) with cum(<b) < krem <= cum(<=b).
// Result in m->sel_*; m->sel_found = 0 if the bins hold fewer than krem.
template <class Tm, bool GLOBAL>
__device__ void block_select(const uint32_t* h, int NB, uint32_t krem, Misc* m) {
  if (Tm::tid() == 0) m->sel_found = 0;
  const int per = (NB + Tm::kSize - 1) / Tm::kSize;
  const int lo = Tm::tid() * per;
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
  const uint32_t ex = block_excl_scan<Tm>(s, m->scan, nullptr);
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
  Tm::sync();
}

// Shared-memory histogram increment, aggregated: the bin of the first valid
// lane is added once with the count of lanes that share it, which turns a
// heavily repeated key (constant-heavy rows) into one update per warp.  One
// predicated atomic per lane.  All 32 lanes must call it together; returns
// how many lanes shared the leader's bin.
__device__ __forceinline__ int hist_add_agg(uint32_t* hist, uint32_t bin, bool valid) {
  const unsigned vm = __ballot_sync(kFull, valid);
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(vm) - 1;
  const uint32_t lb = __shfl_sync(kFull, bin, leader & 31);
  const bool same = valid && bin == lb;
  const unsigned sm = __ballot_sync(kFull, same);
  const uint32_t add = same ? (lane == leader ? (uint32_t)__popc(sm) : 0u) : (valid ? 1u : 0u);
  if (add) atomicAdd(&hist[bin], add);
  return __popc(sm);
}

// Histogram update for the e-th element of a 16-byte vector.  Element 0 goes
// through the aggregated path and decides, per warp, whether the rest of the
// vector does too (only when lanes repeat a bin); otherwise one plain atomic.
__device__ __forceinline__ void hist_add(uint32_t* hist, uint32_t bin, bool valid, int e, bool& agg) {
  if (e == 0) {
    agg = hist_add_agg(hist, bin, valid) >= 3;
  } else if (agg) {
    hist_add_agg(hist, bin, valid);
  } else if (valid) {
    atomicAdd(&hist[bin], 1u);
  }
}

// Bitonic sort of n (power of two, >= 2) uint64 keys in shared memory.
template <class Tm>
__device__ inline void block_bitonic_sort(uint64_t* s, int n) {
  for (int size = 2; size <= n; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = Tm::tid(); i < (n >> 1); i += Tm::kSize) {
        const int lo = 2 * i - (i & (stride - 1));
        const int hi = lo + stride;
        const bool up = (lo & size) == 0;
        const uint64_t a = s[lo], b = s[hi];
        if ((a > b) == up) {
          s[lo] = b;
          s[hi] = a;
        }
      }
      Tm::sync();
    }
  }
}

// ----------------------------------------------------------------------------
// Row context
// ----------------------------------------------------------------------------
struct RowCtx {
  int64_t in_off, out_off, cand_off, sort_off;
  int32_t n, k, a0, b0, na, nbc, fin_wait, cand_cap, slot_use;
  int32_t kind, IB, ch;
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
    c.kind = row_kind(c.n, c.k, p.cta_cap);
    c.na = row_na(c.kind, c.n, p.CH, p.CHR);
    c.nbc = row_nbc(c.kind, c.n, p.CH, p.CHR);
    c.a0 = r * c.na;
    c.b0 = 0;  // uniform batches decode B items arithmetically
    c.cand_cap = p.u_cand_cap;
    c.cand_off = (int64_t)r * p.u_cand_cap;
    c.sort_off = p.u_sort_cap ? (int64_t)r * p.u_sort_cap : -1;
    c.slot_use = row_uses_hist(c.kind) ? r : -1;
  } else {
    const RowPlan& pl = p.plans[r];
    c.in_off = pl.in_off;
    c.out_off = pl.out_off;
    c.cand_off = pl.cand_off;
    c.sort_off = pl.sort_off;
    c.n = pl.n;
    c.k = pl.k;
    c.kind = row_kind(c.n, c.k, p.cta_cap);
    c.na = row_na(c.kind, c.n, p.CH, p.CHR);
    c.nbc = row_nbc(c.kind, c.n, p.CH, p.CHR);
    c.a0 = pl.a0;
    c.b0 = pl.b0;
    c.cand_cap = pl.cand_cap;
    c.slot_use = pl.slot_use;
  }
  c.IB = index_bits(c.n);
  c.ch = row_chunk(c.kind, p.CH, p.CHR);
  if (p.uniform && p.u_tail_rows > 0 && c.kind == kKindGridPref && r >= p.B - p.u_tail_rows) {
    c.ch = p.u_ch_tail;  // the short chunks at the end of the claim order
    c.nbc = row_nbc(c.kind, c.n, c.ch, p.CHR);
  }
  c.fin_wait = c.kind == kKindAll ? c.na : c.nbc;
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

// ----------------------------------------------------------------------------
// Iteration over positions [a, b) of a row.  The unaligned head and tail go
// through fe(bits, pos, ok) one element per thread; the aligned middle
// through fv(x, pos0, ok) one 16-byte vector per thread, U vectors in flight.
// Both callbacks are called by every thread the same number of times (warp
// collectives are allowed inside).
// ----------------------------------------------------------------------------
template <class Tm, int ES, int U, typename FE, typename FV>
__device__ __forceinline__ void for_range_v(const void* base, int64_t in_off, int64_t a, int64_t b, FE&& fe,
                                            FV&& fv) {
  constexpr int VEC = 16 / ES;
  if (b <= a) return;
  const char* row = static_cast<const char*>(base) + in_off * ES;
  const uintptr_t addr_a = reinterpret_cast<uintptr_t>(row + a * ES);
  int64_t head = (int64_t)(((16u - (unsigned)(addr_a & 15u)) & 15u) / ES);
  if (head > b - a) head = b - a;
  const int64_t va = a + head;
  const int64_t nvec = (b - va) / VEC;
  const int64_t vb = va + nvec * VEC;
  const int64_t tail = b - vb;
  if (head > 0 || tail > 0) {
    const int t = Tm::tid();
    const bool vh = t < head;
    const bool vt = t < tail;
    uint32_t bh = 0, bt = 0;
    if (vh) bh = ES == 4 ? reinterpret_cast<const uint32_t*>(row)[a + t]
                         : (uint32_t)reinterpret_cast<const unsigned short*>(row)[a + t];
    if (vt) bt = ES == 4 ? reinterpret_cast<const uint32_t*>(row)[vb + t]
                         : (uint32_t)reinterpret_cast<const unsigned short*>(row)[vb + t];
    if (head > 0) fe(bh, a + t, vh);
    if (tail > 0) fe(bt, vb + t, vt);
  }
  const uint4* vp = reinterpret_cast<const uint4*>(row + va * ES);
  const int64_t step = (int64_t)Tm::kSize * U;
  const int64_t iters = (nvec + step - 1) / step;
  int64_t v0 = Tm::tid();
  for (int64_t it = 0; it < iters; ++it, v0 += step) {
    uint4 x[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t v = v0 + (int64_t)u * Tm::kSize;
      x[u] = v < nvec ? ld_stream16(vp + v) : make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t v = v0 + (int64_t)u * Tm::kSize;
      fv(x[u], va + v * VEC, v < nvec);
    }
  }
}

// Element e of a 16-byte vector as a raw bit pattern.
template <int ES>
__device__ __forceinline__ uint32_t vec_elem(const uint4& x, int e) {
  if constexpr (ES == 4) {
    return e == 0 ? x.x : e == 1 ? x.y : e == 2 ? x.z : x.w;
  } else {
    const uint32_t w = (e >> 1) == 0 ? x.x : (e >> 1) == 1 ? x.y : (e >> 1) == 2 ? x.z : x.w;
    return (e & 1) ? (w >> 16) : (w & 0xFFFFu);
  }
}

// ----------------------------------------------------------------------------
// Output writes and warp-staged sinks
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

__device__ __forceinline__ uint64_t make_entry(uint32_t bits, int64_t pos) {
  return ((uint64_t)bits << 32) | (uint64_t)(uint32_t)pos;
}

// A warp's private staging buffer in shared memory.  Hits are appended with
// a ballot (no atomics); a full buffer is flushed with one global atomic.
struct WarpBuf {
  uint64_t* buf;
  uint32_t n;  // warp-uniform
};

template <typename Flush>
__device__ __forceinline__ void sink_push(WarpBuf& s, int cap, bool want, uint64_t e, Flush&& flush) {
  const unsigned b = __ballot_sync(kFull, want);
  if (b == 0) return;
  const unsigned lane = threadIdx.x & 31u;
  if (want) s.buf[s.n + __popc(b & ((1u << lane) - 1u))] = e;
  s.n += (uint32_t)__popc(b);
  if (s.n > (uint32_t)(cap - 32)) {
    __syncwarp();
    flush(s);
    s.n = 0;
    __syncwarp();
  }
}

// Flushes a warp buffer to the row's output slots.
template <int VT>
__device__ __forceinline__ void flush_out(const EngineParams& p, const WarpBuf& s, uint32_t* ctr, int64_t out_off,
                                          int32_t k) {
  const unsigned lane = threadIdx.x & 31u;
  uint32_t base = 0;
  if (lane == 0) base = atomicAdd(ctr, s.n);
  base = __shfl_sync(kFull, base, 0);
  for (uint32_t i = lane; i < s.n; i += 32) {
    const uint64_t e = s.buf[i];
    if (base + i < (uint32_t)k) write_out<VT>(p, out_off + base + i, (uint32_t)(e >> 32), (int64_t)(uint32_t)e);
  }
}

// Flushes a warp buffer to a candidate region of capacity cap.  Entries past
// the capacity are dropped but still counted, so the reader sees the true
// count and takes its fallback (a pre-filter row whose threshold let more
// than cand_cap keys through is resolved over the row itself in phase B).
__device__ __forceinline__ void flush_cand(const WarpBuf& s, uint32_t* ctr, uint64_t* dst, int32_t cap) {
  const unsigned lane = threadIdx.x & 31u;
  uint32_t base = 0;
  if (lane == 0) base = atomicAdd(ctr, s.n);
  base = __shfl_sync(kFull, base, 0);
  for (uint32_t i = lane; i < s.n; i += 32)
    if (base + i < (uint32_t)cap) dst[base + i] = s.buf[i];
}

// ----------------------------------------------------------------------------
// Shared-memory selection
// ----------------------------------------------------------------------------
// Warp-wide min / max of 64-bit values with the 32-bit redux unit: the high
// words first, then the low words of the lanes holding that high word.
__device__ __forceinline__ uint64_t warp_min64(uint64_t v) {
  const uint32_t h = __reduce_min_sync(kFull, (uint32_t)(v >> 32));
  const uint32_t l = __reduce_min_sync(kFull, (uint32_t)(v >> 32) == h ? (uint32_t)v : 0xFFFFFFFFu);
  return ((uint64_t)h << 32) | l;
}
__device__ __forceinline__ uint64_t warp_max64(uint64_t v) {
  const uint32_t h = __reduce_max_sync(kFull, (uint32_t)(v >> 32));
  const uint32_t l = __reduce_max_sync(kFull, (uint32_t)(v >> 32) == h ? (uint32_t)v : 0u);
  return ((uint64_t)h << 32) | l;
}

// Block-wide min of lo and max of hi over all threads (pass ~0 / 0 to abstain).
template <class Tm>
__device__ __forceinline__ void block_minmax(uint64_t lo, uint64_t hi, uint64_t* mn, uint64_t* mx, Misc* m) {
  lo = warp_min64(lo);
  hi = warp_max64(hi);
  uint64_t* red = reinterpret_cast<uint64_t*>(m->scan);  // 64 x u32 = 32 x u64
  const int warp = Tm::wid(), lane = threadIdx.x & 31;
  Tm::sync();
  if (lane == 0) {
    red[warp] = lo;
    m->red_hi_w[warp] = hi;
  }
  Tm::sync();
  if (warp == 0) {
    uint64_t a = lane < Tm::kWarps ? red[lane] : ~0ull, b = lane < Tm::kWarps ? m->red_hi_w[lane] : 0ull;
    a = warp_min64(a);
    b = warp_max64(b);
    if (lane == 0) {
      m->red_lo = a;
      m->red_hi = b;
    }
  }
  Tm::sync();
  *mn = m->red_lo;
  *mx = m->red_hi;
  Tm::sync();
}

// Threshold key of a sample: the r-th smallest (1-based) of cnt KB-bit keys
// in shared memory, or an upper bound of it.  The bits every key shares are
// skipped (min/max reduction); then at most two 12-bit digits refine it.
// When bits remain after that, the upper edge of the r-th key's bin is
// returned (at least r keys are <= it).  hist: 4096 counters of smem.
// Finds the bin b of h[0..256) with cum(<b) < krem <= cum(<=b) using one
// warp.  Lane l holds bins 8l .. 8l + 7 (two 16-byte loads; h is 16-byte
// aligned), the lanes scan their sums, and the lane whose range reaches krem
// walks its eight bins.  Few live registers: inside the finishes, where the
// kernel's register budget is tight, a wider form spilled and took ~8 us.
// Result in m->sel_*; m->sel_found = 0 if the bins hold fewer than krem (or
// krem is 0).  Ends with a team barrier.
template <class Tm>
__device__ void select256(const uint32_t* hist, uint32_t krem, Misc* m) {
  if (Tm::wid() == 0) {
    const int lane = threadIdx.x & 31;
    const uint4 a = reinterpret_cast<const uint4*>(hist)[lane * 2];
    const uint4 b = reinterpret_cast<const uint4*>(hist)[lane * 2 + 1];
    const uint32_t sum = a.x + a.y + a.z + a.w + b.x + b.y + b.z + b.w;
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += y;
    }
    const unsigned hit = __ballot_sync(kFull, krem > 0 && incl >= krem);
    if (hit == 0) {
      if (lane == 0) m->sel_found = 0;
    } else if (lane == __ffs(hit) - 1) {
      uint32_t cum = incl - sum, cnt = 0;
      int bin = -1;
      const uint32_t v[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        if (bin < 0) {
          if (cum + v[t] >= krem) {
            bin = t;
            cnt = v[t];
          } else {
            cum += v[t];
          }
        }
      }
      m->sel_bin = (uint32_t)(lane * 8 + bin);
      m->sel_cum = cum;
      m->sel_cnt = cnt;
      m->sel_found = 1;
    }
  }
  Tm::sync();
}

// Threshold of a pre-filter row from its sampled keys: an upper bound of the
// r-th smallest of the cnt keys (each thread passes the min / max of the keys
// it stored).  Past the bits all keys share, 8-bit digit levels narrow the
// bin holding the r-th key until it holds at most 8 keys; the bin's upper end
// is returned, so at least r sampled keys are <= the result.  256-bin levels
// keep the clearing and the bin search to a few instructions per thread.
template <class Tm, int KB>
__device__ uint32_t block_sample_threshold(const uint32_t* keys, int cnt, int r, uint64_t lo, uint64_t hi,
                                           uint32_t* hist, Misc* m, int32_t* status) {
  // Small ranks (r <= a quarter of the team) select among the per-thread
  // minimums instead of all cnt keys: the r-th smallest minimum has r
  // distinct sampled keys at or below it, so it bounds the r-th smallest key
  // from above, and for r << team size it sits at nearly the same quantile
  // (the minimum of m keys is below x with probability about m times that of
  // one key).  Each level then counts one value a thread instead of cnt /
  // team: the shared-memory atomics were most of a level's time.
  const bool by_mins = r * 4 <= Tm::kSize;
  uint64_t mn, mx;
  block_minmax<Tm>(lo, by_mins ? (lo == ~0ull ? 0ull : lo) : hi, &mn, &mx, m);
  if (mn >= mx) return (uint32_t)mn;
  int plen = __clzll((long long)(mn ^ mx)) - (64 - KB);  // shared leading bits
  uint32_t prefix = plen > 0 ? (uint32_t)(mn >> (KB - plen)) : 0u;
  uint32_t krem = (uint32_t)r;
  while (plen < KB) {
    const int D = min(8, KB - plen);
    const int NB = 1 << D;
    for (int i = Tm::tid(); i < 256; i += Tm::kSize) hist[i] = 0;
    Tm::sync();
    const int sd = KB - plen - D;
    if (by_mins) {
      const uint32_t v = (uint32_t)lo;
      if (lo != ~0ull && (plen == 0 || (v >> (KB - plen)) == prefix)) atomicAdd(&hist[(v >> sd) & (uint32_t)(NB - 1)], 1u);
    } else {
      for (int b = 0; b < cnt; b += 4 * Tm::kSize) {  // four keys a thread in flight
        uint32_t k[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int i = b + u * Tm::kSize + Tm::tid();
          k[u] = i < cnt ? keys[i] : 0u;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int i = b + u * Tm::kSize + Tm::tid();
          if (i < cnt && (plen == 0 || (k[u] >> (KB - plen)) == prefix))
            atomicAdd(&hist[(k[u] >> sd) & (uint32_t)(NB - 1)], 1u);
        }
      }
    }
    Tm::sync();
    select256<Tm>(hist, krem, m);
    if (!m->sel_found) {
      if (Tm::tid() == 0) atomicOr(status, kStatusSelect);
      return (uint32_t)(((uint64_t)1 << KB) - 1);
    }
    prefix = (prefix << D) | m->sel_bin;
    plen += D;
    krem -= m->sel_cum;
    const uint32_t cnt_bin = m->sel_cnt;
    Tm::sync();
    if (cnt_bin <= 8) break;
  }
  if (plen >= KB) return prefix;
  return (uint32_t)(((uint64_t)prefix << (KB - plen)) | (((uint64_t)1 << (KB - plen)) - 1));
}

// Copies cnt 64-bit entries from global memory (L2) into smem.  Each thread
// issues eight loads before its first store: a plain copy loop would wait a
// full memory round trip per element, because the compiler cannot move a
// load above a store it cannot prove disjoint.
template <class Tm>
__device__ __forceinline__ void load_entries(uint64_t* dst, const uint64_t* src, int cnt) {
  constexpr int U = 8;
  for (int b = 0; b < cnt; b += Tm::kSize * U) {
    uint64_t v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = b + u * Tm::kSize + Tm::tid();
      v[u] = i < cnt ? ld_cg_u64(src + i) : 0ull;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = b + u * Tm::kSize + Tm::tid();
      if (i < cnt) dst[i] = v[u];
    }
  }
}

// Entries get(i) -> (bits, pos), all matching (prefix, plen).  Refines the
// prefix over the composite (key << IB | pos) until the matched set size
// equals krem: first past the bits all entries share (min/max reduction),
// then with 12-bit digits (hist: 4096 counters of smem).  On return the
// selected entries are those whose composite prefix is <= prefix.
template <class Tm, int VT, bool SCALE, typename G>
__device__ void smem_resolve(G get, int cnt, const RowCtx& rc, uint64_t& prefix, int& plen, int& krem, int count,
                             uint32_t* hist, Misc* m, int32_t* status) {
  using K = KT<VT, SCALE>;
  const int W = K::KB + rc.IB;
  if (count != krem && cnt > 0) {
    uint64_t lo = ~0ull, hi = 0;
    for (int i = Tm::tid(); i < cnt; i += Tm::kSize) {
      uint32_t bits;
      int64_t pos;
      get(i, bits, pos);
      const uint64_t c = ((uint64_t)sel_key<VT, SCALE>(bits, rc.flip, rc.scaler) << rc.IB) | (uint64_t)pos;
      if (shr64(c, W - plen) == prefix) {
        lo = min(lo, c);
        hi = max(hi, c);
      }
    }
    uint64_t mn, mx;
    block_minmax<Tm>(lo, hi, &mn, &mx, m);
    if (mn != ~0ull) {
      const int common = (mn == mx) ? W : (__clzll((long long)(mn ^ mx)) - (64 - W));
      if (common > plen) {
        plen = common;
        prefix = shr64(mn, W - plen);
      }
    }
  }
  while (count != krem) {
    if (plen >= W || count < krem) {
      if (Tm::tid() == 0) atomicOr(status, kStatusLevels);
      break;
    }
    // 8-bit digits: the sets here are small (smem), so a level's fixed cost
    // (clearing the bins, finding the bin) matters more than its pass count
    const int D = min(8, W - plen);
    const int NB = 1 << D;
    for (int i = Tm::tid(); i < 256; i += Tm::kSize) hist[i] = 0;
    Tm::sync();
    const int sh = W - plen;
    const int sd = W - plen - D;
    const uint32_t dm = (uint32_t)NB - 1u;
    for (int i = Tm::tid(); i < cnt; i += Tm::kSize) {
      uint32_t bits;
      int64_t pos;
      get(i, bits, pos);
      const uint64_t c = ((uint64_t)sel_key<VT, SCALE>(bits, rc.flip, rc.scaler) << rc.IB) | (uint64_t)pos;
      if (shr64(c, sh) == prefix) atomicAdd(&hist[(uint32_t)shr64(c, sd) & dm], 1u);
    }
    Tm::sync();
    select256<Tm>(hist, (uint32_t)krem, m);
    if (!m->sel_found) {
      if (Tm::tid() == 0) atomicOr(status, kStatusSelect);
      break;
    }
    prefix = (prefix << D) | m->sel_bin;
    plen += D;
    krem -= (int)m->sel_cum;
    count = (int)m->sel_cnt;
    Tm::sync();
  }
}

// Emits the entries selected by (prefix, plen) to the row's output, in entry
// order, reserving the slots with one atomic on the row's out_count -- or,
// when the team is the row's only writer (sole), from slot 0 without it: the
// atomic's round trip sits on the finish's critical path.  Warp w owns a
// contiguous run of entries and walks it 32 at a time (conflict-free smem
// reads; a ballot ranks the selected lanes, so the writes coalesce).
template <class Tm, int VT, bool SCALE, typename G>
__device__ void smem_emit(const EngineParams& p, G get, int cnt, const RowCtx& rc, uint64_t prefix, int plen,
                          RowState* rs, Misc* m, bool sole = false) {
  using K = KT<VT, SCALE>;
  const int W = K::KB + rc.IB;
  const int sh = W - plen;
  const int lane = threadIdx.x & 31;
  const int span = (cnt + Tm::kWarps * 32 - 1) / (Tm::kWarps * 32) * 32;
  const int lo = min(cnt, Tm::wid() * span);
  const int hi = min(cnt, lo + span);
  auto selected = [&](int i, uint32_t& bits, int64_t& pos) -> bool {
    if (i >= hi) return false;
    get(i, bits, pos);
    const uint64_t c = ((uint64_t)sel_key<VT, SCALE>(bits, rc.flip, rc.scaler) << rc.IB) | (uint64_t)pos;
    return shr64(c, sh) <= prefix;
  };
  uint32_t mine = 0;
  for (int b = lo; b < hi; b += 32) {
    uint32_t bits;
    int64_t pos;
    mine += (uint32_t)__popc(__ballot_sync(kFull, selected(b + lane, bits, pos)));
  }
  uint32_t total;
  const uint32_t ex = block_excl_scan<Tm>(lane == 0 ? mine : 0u, m->scan, &total);
  uint32_t base = __shfl_sync(kFull, ex, 0);
  if (!sole) {
    if (Tm::tid() == 0) m->counter = total ? atomicAdd(reinterpret_cast<uint32_t*>(&rs->out_count), total) : 0u;
    Tm::sync();
    base += m->counter;
  }
  for (int b = lo; b < hi; b += 32) {
    uint32_t bits = 0;
    int64_t pos = 0;
    const bool s = selected(b + lane, bits, pos);
    const unsigned bal = __ballot_sync(kFull, s);
    const int64_t slot = (int64_t)base + __popc(bal & ((1u << lane) - 1u));
    if (s && slot < rc.k) write_out<VT>(p, rc.out_off + slot, bits, pos);
    base += (uint32_t)__popc(bal);
  }
  Tm::sync();
}

// ----------------------------------------------------------------------------
// Row post-processing: sort, index mapping, idle fill
// ----------------------------------------------------------------------------
template <class Tm, int VT, bool SCALE>
__device__ void post_process(const EngineParams& p, const RowCtx& rc, uint8_t* smem, Misc* m) {
  const int64_t kk = min((int64_t)rc.n, (int64_t)rc.k);
  const bool idx64 = (p.flags & kFlagIdx64) != 0;
  const bool withidx = (p.flags & kFlagWithIdxIn) != 0;
  const bool sorting = (p.flags & kFlagSorted) && kk > 1;
  if (!sorting && !withidx && kk == rc.k) return;  // unsorted, positions, no idle slots: nothing to do
  __threadfence();
  Tm::sync();
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
      for (int i = Tm::tid(); i < np; i += Tm::kSize) {
        uint64_t v = ~0ull;
        if (i < kk) v = ((uint64_t)out_key<VT>(load_bits(i), ascend) << 32) | (uint64_t)(uint32_t)load_pos(i);
        s[i] = v;
      }
      Tm::sync();
      block_bitonic_sort<Tm>(s, np);
      for (int i = Tm::tid(); i < kk; i += Tm::kSize) {
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
        for (int i = Tm::tid(); i < kCapSort; i += Tm::kSize) {
          uint64_t v = ~0ull;
          if (i < len)
            v = ((uint64_t)out_key<VT>(load_bits(r0 + i), ascend) << 32) | (uint64_t)(uint32_t)load_pos(r0 + i);
          s[i] = v;
        }
        Tm::sync();
        block_bitonic_sort<Tm>(s, kCapSort);
        for (int i = Tm::tid(); i < len; i += Tm::kSize) a[r0 + i] = s[i];
        Tm::sync();
      }
      for (int64_t run = kCapSort; run < kk; run <<= 1) {
        for (int64_t m0 = 0; m0 < kk; m0 += 2 * run) {
          const int64_t l0 = m0, l1 = min(kk, m0 + run), r1 = min(kk, m0 + 2 * run);
          const int64_t tot = r1 - l0;
          const int64_t per = (tot + Tm::kSize - 1) / Tm::kSize;
          const int64_t d0 = min(tot, (int64_t)Tm::tid() * per), d1 = min(tot, d0 + per);
          auto split = [&](int64_t d) -> int64_t {  // elements taken from the left run
            int64_t lo = max((int64_t)0, d - (r1 - l1)), hi = min(d, l1 - l0);
            while (lo < hi) {
              const int64_t mid = (lo + hi) >> 1;
              if (ld_cg_u64(a + l0 + mid) <= ld_cg_u64(a + l1 + (d - mid - 1))) lo = mid + 1;
              else hi = mid;
            }
            return lo;
          };
          if (d0 < d1) {
            int64_t i = l0 + split(d0), j = l1 + (d0 - (i - l0));
            for (int64_t d = d0; d < d1; ++d) {
              const uint64_t x = i < l1 ? ld_cg_u64(a + i) : ~0ull;
              const uint64_t y = j < r1 ? ld_cg_u64(a + j) : ~0ull;
              const bool takel = (j >= r1) || (i < l1 && x <= y);
              b[l0 + d] = takel ? x : y;
              if (takel) ++i;
              else ++j;
            }
          }
        }
        Tm::sync();
        uint64_t* t = a;
        a = b;
        b = t;
      }
      for (int64_t i = Tm::tid(); i < kk; i += Tm::kSize) {
        const uint64_t v = ld_cg_u64(a + i);
        write_out<VT>(p, rc.out_off + i, out_key_inv<VT>((uint32_t)(v >> 32), ascend), map_idx((int64_t)(uint32_t)v));
      }
    }
  } else if (withidx) {
    for (int64_t i = Tm::tid(); i < kk; i += Tm::kSize) {
      const int64_t pos = load_pos(i);
      const int64_t mapped = map_idx(pos);
      if (idx64) static_cast<int64_t*>(p.idx_out)[rc.out_off + i] = mapped;
      else static_cast<int32_t*>(p.idx_out)[rc.out_off + i] = (int32_t)mapped;
    }
  }
  for (int64_t i = kk + Tm::tid(); i < rc.k; i += Tm::kSize) write_out<VT>(p, rc.out_off + i, 0u, -1);
  Tm::sync();
}

// ----------------------------------------------------------------------------
// Grid barrier (cooperative launch: all CTAs are resident).  Bounded.
// ----------------------------------------------------------------------------
template <class Tm>
__device__ inline void grid_barrier(Header* h, uint32_t spin_limit) {
  // bar_count only grows during a call (the header is cleared per call):
  // every CTA takes the barriers in the same order, so barrier b completes at
  // (b + 1) * gridDim.x arrivals -- one atomic per CTA, then a poll.  The
  // arrival is a release at GPU scope (it orders the CTA's writes, gathered
  // by the team barrier before it) and the poll an acquire; a sequentially
  // consistent fence on each side cost about 8 us per barrier on B200.
  Tm::sync();
  if (Tm::tid() == 0) {
    uint32_t old;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], 1;" : "=r"(old) : "l"(&h->bar_count) : "memory");
    const uint32_t target = (old / gridDim.x + 1u) * gridDim.x;
    uint32_t it = 0;
    // the last arrival has seen every other one through its own atomic
    while (old + 1u != target && ld_acquire(&h->bar_count) < target) {
      if (++it > spin_limit) {
        atomicOr(&h->status, kStatusTimeout);
        break;
      }
      __nanosleep(32);
    }
  }
  Tm::sync();
}

// ----------------------------------------------------------------------------
// Items
// ----------------------------------------------------------------------------
template <int VT, bool SCALE>
struct Engine {
  using K = KT<VT, SCALE>;
  static constexpr int ES = K::ES;
  static constexpr int VEC = K::VEC;
  static constexpr int U = 4;

  const EngineParams& p;
  uint8_t* base;  // the CTA's shared memory
  uint8_t* smem;  // this team's area (consumer or side)
  Misc* m;        // this team's scratch
  Ctrl* ctl;
  int pending_rel = -1;  // consumer team: row whose chunk counter is still to be released

  __device__ Engine(const EngineParams& p_, uint8_t* b, uint8_t* area, Misc* m_)
      : p(p_), base(b), smem(area), m(m_), ctl(ctrl_of(b)) {}

  template <class Tm>
  __device__ uint64_t* cand_sink() const {
    return reinterpret_cast<uint64_t*>(smem) + Tm::wid() * kSinkCand;
  }
  template <class Tm>
  __device__ uint64_t* out_sink() const {
    return reinterpret_cast<uint64_t*>(smem + Tm::kWarps * kSinkCand * 8) + Tm::wid() * kSinkOut;
  }

  // Releases the previous chunk item's completion on its row's counter: one
  // consumer thread fences (the item's writes by all consumer warps precede
  // it through the item's closing barrier) and increments.  Called after
  // the next item's threshold wait, so its stall overlaps the ring's data.
  __device__ void do_release() {
    if (pending_rel >= 0) {
      if (ConsTeam::tid() == ConsTeam::kSize - 32) {
        // one release reduction: orders every consumer's candidate writes
        // (seen through the team barrier) before the count the FIN acquires
        asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(&p.rs[pending_rel].fticket) : "memory");
      }
      pending_rel = -1;
    }
  }

  // Consumes a streaming item's chunk: pre() (e.g. a threshold wait), the
  // unaligned head and tail (< 16 bytes each) through fe(bits, pos, ok), and
  // the aligned middle from the ring, kStageVecs / 768 16-byte vectors per consumer
  // thread per stage, through fv(x, pos0, ok).  Each consumer warp arrives
  // on a stage's "empty" barrier once done with it; the producer refills the
  // slot when all have.  All callbacks are called warp-uniformly.
  template <typename PRE, typename FE, typename FV>
  __device__ void consume_chunk(const RowCtx& rc, const ItemDesc& d, PRE&& pre, FE&& fe, FV&& fv) {
    const char* row = static_cast<const char*>(p.val_in) + rc.in_off * ES;
    RADIK_TL_T0(tp);
    pre();
    if (ConsTeam::tid() == 0) {
      RADIK_TL_ACC(p, kTlAccPre, tp);
      RADIK_TL_COUNT(p, kTlNChunks);
      RADIK_TL(p, kTlItemStart);
    }
    do_release();
    const int64_t head = d.va - d.a;
    const int64_t vb = d.va + d.nvec * VEC;
    const int64_t tail = d.b - vb;
    if (head > 0 || tail > 0) {
      const int t = ConsTeam::tid();
      const bool vh = t < head, vt = t < tail;
      uint32_t bh = 0, bt = 0;
      if (vh) bh = ES == 4 ? reinterpret_cast<const uint32_t*>(row)[d.a + t]
                           : (uint32_t)reinterpret_cast<const unsigned short*>(row)[d.a + t];
      if (vt) bt = ES == 4 ? reinterpret_cast<const uint32_t*>(row)[vb + t]
                           : (uint32_t)reinterpret_cast<const unsigned short*>(row)[vb + t];
      if (head > 0) fe(bh, d.a + t, vh);
      if (tail > 0) fe(bt, vb + t, vt);
    }
    // Stage loop.  Full stages (all but a ragged last one) take no bounds
    // checks; the slot and its phase parity advance without divisions.
    constexpr int kPer = kStageVecs / ConsTeam::kSize;
    const uint4* ring = reinterpret_cast<const uint4*>(base) + ConsTeam::tid();
    constexpr uint32_t NS = ring_stages<VT>();
    uint32_t slot = d.g0 % NS, parity = (d.g0 / NS) & 1u;
    const int nfull = (int)(d.nvec / kStageVecs);
    int64_t pos = d.va + (int64_t)ConsTeam::tid() * VEC;  // first element of this thread's vector in the stage
    for (int i = 0; i < d.nst; ++i) {
      uint32_t it = 0;
      RADIK_TL_T0(tw);
      while (!mbar_try_wait(&ctl->full[slot], parity)) {
        if (++it > p.spin_limit) {
          if (ConsTeam::tid() == 0) atomicOr(&p.hdr->status, kStatusTimeout);
          break;
        }
      }
      if (ConsTeam::tid() == 0) RADIK_TL_ACC(p, kTlAccFull, tw);
      const uint4* st = ring + slot * kStageVecs;
      // The warp's vectors of the stage are read into registers, then the
      // slot is released before they are processed: a warp that meets hits
      // (the compaction is the slow path) no longer holds the refill of the
      // slot for every other warp.
      uint4 v[kPer];
      if (i < nfull) {
#pragma unroll
        for (int j = 0; j < kPer; ++j) v[j] = st[j * ConsTeam::kSize];
        __syncwarp();
        if ((threadIdx.x & 31) == 0) mbar_arrive(&ctl->empty[slot]);
#pragma unroll
        for (int j = 0; j < kPer; ++j) fv(v[j], pos + (int64_t)j * ConsTeam::kSize * VEC, true);
      } else {
        const int cnt = (int)(d.nvec - (int64_t)i * kStageVecs);
#pragma unroll
        for (int j = 0; j < kPer; ++j)
          v[j] = j * ConsTeam::kSize + ConsTeam::tid() < cnt ? st[j * ConsTeam::kSize] : make_uint4(0, 0, 0, 0);
        __syncwarp();
        if ((threadIdx.x & 31) == 0) mbar_arrive(&ctl->empty[slot]);
#pragma unroll
        for (int j = 0; j < kPer; ++j)
          fv(v[j], pos + (int64_t)j * ConsTeam::kSize * VEC, j * ConsTeam::kSize + ConsTeam::tid() < cnt);
      }
      pos += (int64_t)kStageVecs * VEC;
      if (++slot == NS) {
        slot = 0;
        parity ^= 1u;
      }
    }
  }

  // Bounded wait by one thread until *addr >= target.
  __device__ bool spin_until_ge(const uint32_t* addr, uint32_t target) {
    for (uint32_t it = 0; it < p.spin_limit; ++it) {
      if (ld_acquire(addr) >= target) return true;
      __nanosleep(64);
    }
    atomicOr(&p.hdr->status, kStatusTimeout);
    return false;
  }

  __device__ uint32_t key_of(uint32_t bits, const RowCtx& rc) const {
    return sel_key<VT, SCALE>(bits, rc.flip, rc.scaler);
  }

  __device__ uint32_t load_bits(const RowCtx& rc, int64_t pos) const {
    if constexpr (ES == 4) return __ldg(static_cast<const uint32_t*>(p.val_in) + rc.in_off + pos);
    else return (uint32_t)__ldg(static_cast<const unsigned short*>(p.val_in) + rc.in_off + pos);
  }

  // ---- threshold from a strided sample of the row (one team of a CTA).
  // The sample is S keys in S / (128 / ES) whole 128-byte lines spread evenly
  // over the row's aligned lines (pre-filter rows hold more than 2^18 keys,
  // far more lines than the sample needs).  All lines are fetched at once by
  // 16-byte asynchronous copies into smem, so the sample costs about one
  // memory round trip and holds no registers while in flight.
  // With big = true (a whole CTA at the kernel's start, before anything
  // streams) the ring is the scratch, and long rows take a larger sample (up
  // to n / 64 keys and kSampleBig: 128 KB of fp32 keys, or 64 KB of 16-bit
  // ones plus their staging): the threshold then sits closer to the k-th
  // key, leaving fewer candidates for the row's finish.
  template <class Tm>
  __device__ uint32_t sample_threshold(const RowCtx& rc, bool big = false) {
    uint8_t* scratch = big ? base : smem;
    uint32_t* keys = reinterpret_cast<uint32_t*>(scratch);
    int S = sample_size(rc.n);
    if (big) {
      constexpr int kSampleBig = ES == 4 ? 32768 : 16384;
      while (S < kSampleBig && (int64_t)S * 2 * 64 <= rc.n) S *= 2;
    }
    constexpr int SL = 128 / ES;  // keys per line
    const uintptr_t a = reinterpret_cast<uintptr_t>(p.val_in) + (uintptr_t)rc.in_off * ES;
    const int64_t first = (int64_t)((a + 127) / 128);
    const int64_t nfull = (int64_t)((a + (uintptr_t)rc.n * ES) / 128) - first;  // whole lines in the row
    if (!big) {
      // A larger sample streamed through registers.  When the threshold comes
      // from per-thread minimums (small ranks), no sampled key is stored, so
      // the sample is not bound by the team's area: up to n / 64 keys
      // (kSampleStream).  For 2^20-key rows at k = 256 the threshold then
      // passes about 1000 keys instead of 2500: fewer vectors take the
      // consumers' exact test and the finish resolves fewer candidates.
      int S2 = S;
      while (S2 < kSampleStream && (int64_t)S2 * 2 * 64 <= rc.n) S2 *= 2;
      const int r2 = sample_rank(rc.n, rc.k, S2);
      if (S2 > S && r2 * 4 <= Tm::kSize) {
        const int nv = S2 / SL * 8;  // 16-byte pieces of whole lines
        const uint64_t step2 = ((uint64_t)(nfull - 1) << 32) / (uint64_t)(S2 / SL - 1);
        uint32_t lo32 = 0xFFFFFFFFu, hi32 = 0;
        constexpr int UL = 4;  // loads a thread keeps in flight
        for (int b = Tm::tid(); b < nv; b += UL * Tm::kSize) {
          uint4 v[UL];
#pragma unroll
          for (int u = 0; u < UL; ++u) {
            const int j = b + u * Tm::kSize;
            const int64_t line = first + (int64_t)(((uint64_t)(j >> 3) * step2) >> 32);
            v[u] = j < nv ? ld_stream16(reinterpret_cast<const void*>((uintptr_t)line * 128 + (uintptr_t)(j & 7) * 16))
                          : make_uint4(0, 0, 0, 0);
          }
#pragma unroll
          for (int u = 0; u < UL; ++u) {
            if (b + u * Tm::kSize < nv) {
#pragma unroll
              for (int e = 0; e < VEC; ++e) {
                const uint32_t k = key_of(vec_elem<ES>(v[u], e), rc);
                lo32 = min(lo32, k);
                hi32 = max(hi32, k);
              }
            }
          }
        }
        const uint64_t lo = lo32 == 0xFFFFFFFFu && hi32 == 0 ? ~0ull : (uint64_t)lo32, hi = hi32;
        uint32_t* hist = reinterpret_cast<uint32_t*>(smem + kSampleHistOff);
        const uint32_t t = block_sample_threshold<Tm, K::KB>(nullptr, S2, r2, lo, hi, hist, m, &p.hdr->status);
        Tm::sync();
        return t;
      }
    }
    const int nlines = S / SL;
    // fp32 values are converted to keys in place; 16-bit values are staged apart
    uint8_t* raw = ES == 4 ? scratch : big ? scratch + S * 4 + 1024 : smem + kSampleRawOff;
    // line i sits at first + floor(i * (nfull - 1) / (nlines - 1)), stepped in
    // 32.32 fixed point (one division per thread instead of one per line)
    const uint64_t step = nlines > 1 ? ((uint64_t)(nfull - 1) << 32) / (uint64_t)(nlines - 1) : 0;
    if (Tm::kSize == FullTeam::kSize && Tm::tid() == 0) RADIK_TL(p, kTlSampleIssue);
    for (int j = Tm::tid(); j < 8 * nlines; j += Tm::kSize) {
      const int i = j >> 3;
      const int64_t line = first + (int64_t)(((uint64_t)i * step) >> 32);
      cp_async16(raw + (size_t)j * 16, reinterpret_cast<const void*>((uintptr_t)line * 128 + (uintptr_t)(j & 7) * 16));
    }
    cp_async_wait_all();
    Tm::sync();
    if (Tm::kSize == FullTeam::kSize && Tm::tid() == 0) RADIK_TL(p, kTlSampleIn);
    uint32_t lo32 = 0xFFFFFFFFu, hi32 = 0;
    for (int b = 0; b < S; b += 4 * Tm::kSize) {  // four keys a thread in flight
      uint32_t bits[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int i = b + u * Tm::kSize + Tm::tid();
        bits[u] = i >= S ? 0u
                         : ES == 4 ? reinterpret_cast<const uint32_t*>(raw)[i]
                                   : (uint32_t)reinterpret_cast<const unsigned short*>(raw)[i];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int i = b + u * Tm::kSize + Tm::tid();
        if (i < S) {
          const uint32_t k = key_of(bits[u], rc);
          keys[i] = k;
          lo32 = min(lo32, k);
          hi32 = max(hi32, k);
        }
      }
    }
    const uint64_t lo = lo32 == 0xFFFFFFFFu && hi32 == 0 ? ~0ull : (uint64_t)lo32, hi = hi32;
    Tm::sync();
    if (Tm::kSize == FullTeam::kSize && Tm::tid() == 0) RADIK_TL(p, kTlSampleKeys);
    uint32_t* hist = reinterpret_cast<uint32_t*>(big ? scratch + S * 4 : smem + kSampleHistOff);  // behind the keys
    const uint32_t t = block_sample_threshold<Tm, K::KB>(keys, S, sample_rank(rc.n, rc.k, S), lo, hi, hist, m,
                                                         &p.hdr->status);
    Tm::sync();
    return t;
  }

  // ---- whole row in shared memory (n <= kSmemRowCap)
  template <class Tm = SideTeam>
  __device__ void smem_row(int r, const RowCtx& rc) {
    uint32_t* vals = reinterpret_cast<uint32_t*>(smem);
    for_range_v<Tm, ES, U>(
        p.val_in, rc.in_off, 0, rc.n, [&](uint32_t bits, int64_t pos, bool ok) { if (ok) vals[pos] = bits; },
        [&](const uint4& x, int64_t pos0, bool ok) {
          if (ok) {
#pragma unroll
            for (int e = 0; e < VEC; ++e) vals[pos0 + e] = vec_elem<ES>(x, e);
          }
        });
    Tm::sync();
    const int kk = min(rc.n, rc.k);
    uint64_t prefix = 0;
    int plen = 0, krem = kk;
    auto get = [&](int i, uint32_t& bits, int64_t& pos) {
      bits = vals[i];
      pos = i;
    };
    smem_resolve<Tm, VT, SCALE>(get, rc.n, rc, prefix, plen, krem, rc.n, reinterpret_cast<uint32_t*>(smem + kSmemRowHistOff), m,
                            &p.hdr->status);
    smem_emit<Tm, VT, SCALE>(p, get, rc.n, rc, prefix, plen, p.rs + r, m, true);
    // The outputs are written, so the row's values are dead: the sort takes
    // the area from its base (up to kCapSort entries, 32 KB).  Behind the
    // values it would run 14 KB past the side area into the control block.
    post_process<Tm, VT, SCALE>(p, rc, smem, m);
  }

  // ---- one CTA, the whole row from global memory (n <= p.cta_cap)
  // Pass over the row classifying by a composite prefix; to_out hits go to
  // the output, to_ent hits into the smem entry array (cap kCapSB).
  template <class Tm = SideTeam>
  __device__ void cta_filter(const RowCtx& rc, RowState* rs, uint64_t prefix, int plen, bool final_mode,
                             uint64_t* ent) {
    const int W = K::KB + rc.IB;
    const int sh = W - plen;
    uint32_t* out_ctr = reinterpret_cast<uint32_t*>(&rs->out_count);
    auto one = [&](uint32_t bits, int64_t pos, bool ok) {
      bool to_out = false, to_ent = false;
      if (ok) {
        const uint64_t c = ((uint64_t)key_of(bits, rc) << rc.IB) | (uint64_t)pos;
        const uint64_t t = shr64(c, sh);
        to_out = t < prefix || (final_mode && t == prefix);
        to_ent = !final_mode && t == prefix;
      }
      if (!__any_sync(kFull, to_out || to_ent)) return;
      const uint32_t so = warp_reserve(to_out ? 1u : 0u, out_ctr);
      if (to_out && so < (uint32_t)rc.k) write_out<VT>(p, rc.out_off + so, bits, pos);
      const uint32_t se = warp_reserve(to_ent ? 1u : 0u, &m->counter);
      if (to_ent && se < (uint32_t)kCapSB) ent[se] = make_entry(bits, pos);
    };
    for_range_v<Tm, ES, U>(p.val_in, rc.in_off, 0, rc.n, one, [&](const uint4& x, int64_t pos0, bool ok) {
#pragma unroll
      for (int e = 0; e < VEC; ++e) one(vec_elem<ES>(x, e), pos0 + e, ok);
    });
  }

  template <class Tm = SideTeam>
  __device__ void cta_row(int r, const RowCtx& rc) {
    RowState* rs = p.rs + r;
    uint64_t* ent = reinterpret_cast<uint64_t*>(smem);
    auto get = [&](int i, uint32_t& bits, int64_t& pos) {
      const uint64_t e = ent[i];
      bits = (uint32_t)(e >> 32);
      pos = (int64_t)(uint32_t)e;
    };
    if ((int64_t)rc.k * kPrefRatio <= rc.n) {
      // pre-filter inside the CTA
      const uint32_t T = sample_threshold<Tm>(rc);
      if (Tm::tid() == 0) m->counter = 0;
      Tm::sync();
      auto one = [&](uint32_t bits, int64_t pos, bool ok) {
        const bool hit = ok && key_of(bits, rc) <= T;
        if (!__any_sync(kFull, hit)) return;
        const uint32_t se = warp_reserve(hit ? 1u : 0u, &m->counter);
        if (hit && se < (uint32_t)kCapSB) ent[se] = make_entry(bits, pos);
      };
      for_range_v<Tm, ES, U>(p.val_in, rc.in_off, 0, rc.n, one, [&](const uint4& x, int64_t pos0, bool ok) {
#pragma unroll
        for (int e = 0; e < VEC; ++e) one(vec_elem<ES>(x, e), pos0 + e, ok);
      });
      Tm::sync();
      const int c = (int)m->counter;
      Tm::sync();
      if (c >= rc.k && c <= kCapSB) {
        uint64_t prefix = 0;
        int plen = 0, krem = rc.k;
        smem_resolve<Tm, VT, SCALE>(get, c, rc, prefix, plen, krem, c, reinterpret_cast<uint32_t*>(smem + kResolveHistOff), m,
                                &p.hdr->status);
        smem_emit<Tm, VT, SCALE>(p, get, c, rc, prefix, plen, rs, m, true);
        post_process<Tm, VT, SCALE>(p, rc, smem, m);
        return;
      }
      // threshold missed: radix levels below
    }
    uint64_t prefix = 0;
    int plen = 0, krem = rc.k, count = rc.n;
    const int W = K::KB + rc.IB;
    uint32_t* hist = reinterpret_cast<uint32_t*>(smem);
    for (int guard = 0; guard < 16 && count != krem && count > kCapSB; ++guard) {
      const int D = min(12, W - plen);
      const int NB = 1 << D;
      for (int i = Tm::tid(); i < NB; i += Tm::kSize) hist[i] = 0;
      Tm::sync();
      const int sh = W - plen, sd = W - plen - D;
      const uint32_t dm = (uint32_t)NB - 1u;
      auto one = [&](uint32_t bits, int64_t pos, bool ok) {
        const uint64_t c = ((uint64_t)key_of(bits, rc) << rc.IB) | (uint64_t)pos;
        hist_add_agg(hist, (uint32_t)shr64(c, sd) & dm, ok && shr64(c, sh) == prefix);
      };
      for_range_v<Tm, ES, U>(p.val_in, rc.in_off, 0, rc.n, one, [&](const uint4& x, int64_t pos0, bool ok) {
#pragma unroll
        for (int e = 0; e < VEC; ++e) one(vec_elem<ES>(x, e), pos0 + e, ok);
      });
      Tm::sync();
      block_select<Tm, false>(hist, NB, (uint32_t)krem, m);
      if (!m->sel_found) {
        if (Tm::tid() == 0) atomicOr(&p.hdr->status, kStatusSelect);
        return;
      }
      prefix = (prefix << D) | m->sel_bin;
      plen += D;
      krem -= (int)m->sel_cum;
      count = (int)m->sel_cnt;
      Tm::sync();
    }
    const bool final_mode = count == krem;
    if (Tm::tid() == 0) m->counter = 0;
    Tm::sync();
    cta_filter<Tm>(rc, rs, prefix, plen, final_mode, ent);
    Tm::sync();
    if (!final_mode) {
      const int ne = min((int)m->counter, kCapSB);
      Tm::sync();
      smem_resolve<Tm, VT, SCALE>(get, ne, rc, prefix, plen, krem, ne, reinterpret_cast<uint32_t*>(smem + kResolveHistOff), m,
                              &p.hdr->status);
      smem_emit<Tm, VT, SCALE>(p, get, ne, rc, prefix, plen, rs, m);
    }
    post_process<Tm, VT, SCALE>(p, rc, smem, m);
  }

  // ---- copy chunk ia of a k >= n row (every element is selected)
  __device__ void all_item(int r, const RowCtx& rc, const ItemDesc& d) {
    RowState* rs = p.rs + r;
    const int warp = ConsTeam::wid();
    WarpBuf ob{out_sink<ConsTeam>(), 0};
    uint32_t* ctr = reinterpret_cast<uint32_t*>(&rs->out_count);
    auto fl = [&](const WarpBuf& s) { flush_out<VT>(p, s, ctr, rc.out_off, rc.k); };
    consume_chunk(
        rc, d, [] {},
        [&](uint32_t bits, int64_t pos, bool ok) { sink_push(ob, kSinkOut, ok, make_entry(bits, pos), fl); },
        [&](const uint4& x, int64_t pos0, bool ok) {
#pragma unroll
          for (int e = 0; e < VEC; ++e) sink_push(ob, kSinkOut, ok, make_entry(vec_elem<ES>(x, e), pos0 + e), fl);
        });
    if (ob.n) fl(ob);
    defer_release(r);
  }

  // A chunk item's completion is counted on the row's fticket by one
  // thread after the item's closing barrier, without waiting for the result
  // (the release's latency overlaps the next item).
  __device__ void defer_release(int r) {
    if (ConsTeam::tid() == 0) m->rel_row = r;
  }

  // ---- FIN item: wait for the row's chunk items, then finish the row
  template <class Tm>
  __device__ void fin_item_t(int r, const RowCtx& rc) {
    if (Tm::tid() == 0) {
      const int32_t* t = &p.rs[r].fticket;
      uint32_t it = 0;
      RADIK_TL_T0(tw);
      RADIK_TL_COUNT(p, kTlNFin);
      while (ld_acquire(t) < rc.fin_wait) {
        if (++it > p.spin_limit) {
          atomicOr(&p.hdr->status, kStatusTimeout);
          break;
        }
        __nanosleep(128);
      }
      RADIK_TL_ACC(p, kTlAccFinWait, tw);
    }
    Tm::sync();
    if (Tm::tid() == 0) RADIK_TL(p, kTlFinStart);
    finish_row<Tm>(r);
    if (Tm::tid() == 0) RADIK_TL(p, kTlFinEnd);
  }  __device__ void fin_item(int r, const RowCtx& rc) { fin_item_t<SideTeam>(r, rc); }


  // ---- sample item of a pre-filter row: publish the threshold
  template <class Tm>
  __device__ void sample_item_t(int r, const RowCtx& rc, bool big = false) {
    const uint32_t T = sample_threshold<Tm>(rc, big);
    if (Tm::tid() == 0) st_release_u64(&p.rs[r].tready, (1ull << 32) | T);
  }
  __device__ void sample_item(int r, const RowCtx& rc) { sample_item_t<SideTeam>(r, rc); }

  // ---- filter item of a pre-filter row: keys <= T into the candidates.
  // Hot loop: a float (or half2) compare against the threshold's value with
  // the unordered predicate, so NaN always passes; it keeps a superset of
  // the keys <= T.  Only vectors with a passing element take the exact
  // integer-key test and the warp-scan compaction into the warp's buffer.
  template <bool LARGEST>
  __device__ void pf_item_t(int r, const RowCtx& rc, const ItemDesc& d) {
    RowState* rs = p.rs + r;
    uint32_t T = 0;
    auto pre = [&]() {
      if (d.thr_ok) {  // read by the producer when it routed the item
        T = d.thr;
        return;
      }
      // The wait below may depend on this team's held-back chunk release
      // (a finish waiting for that count can sit ahead of the threshold's
      // sample on a side team), so the release goes first.
      do_release();
      if (ConsTeam::tid() == 0 && m->t_row != r) {
        uint64_t v = ld_acquire_u64(&rs->tready);
        for (uint32_t it = 0; !(v >> 32); ++it) {
          if (it > p.spin_limit) {
            atomicOr(&p.hdr->status, kStatusTimeout);  // only keys <= 0 pass then
            break;
          }
          __nanosleep(64);
          v = ld_acquire_u64(&rs->tready);
        }
        m->t_val = (uint32_t)v;
        m->t_row = r;
      }
      ConsTeam::sync();
      T = m->t_val;
    };
    const int warp = ConsTeam::wid();
    const unsigned lane = threadIdx.x & 31u;
    constexpr int kCap = kSinkPf;
    WarpBuf cb{reinterpret_cast<uint64_t*>(smem) + warp * kCap, 0};
    uint32_t* ctr = reinterpret_cast<uint32_t*>(&rs->cand_count);
    uint64_t* dst = p.cand + rc.cand_off;
    const uint32_t flip = rc.flip;
    const float sc = rc.scaler;
    // lane's hit mask over up to VEC elements -> warp buffer
    auto push = [&](uint32_t hm, uint32_t e0bits_unused, auto elem_bits, int64_t pos0) {
      (void)e0bits_unused;
      const uint32_t h = (uint32_t)__popc(hm);
      // Usual case: a single lane holds all of the warp's hits.
      const unsigned lanes = __ballot_sync(kFull, hm != 0u);
      if (__popc(lanes) == 1) {
        const int src = __ffs(lanes) - 1;
        const uint32_t tot = __shfl_sync(kFull, h, src);
        if (cb.n + tot > (uint32_t)kCap) {
          __syncwarp();
          flush_cand(cb, ctr, dst, rc.cand_cap);
          cb.n = 0;
          __syncwarp();
        }
        if ((int)lane == src) {
          uint32_t w = cb.n;
          for (uint32_t mm = hm; mm; mm &= mm - 1) {
            const int e = __ffs(mm) - 1;
            cb.buf[w++] = make_entry(elem_bits(e), pos0 + e);
          }
        }
        cb.n += tot;
        return;
      }
      uint32_t x = h;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= (unsigned)o) x += y;
      }
      const uint32_t tot = __shfl_sync(kFull, x, 31);
      if (cb.n + tot > (uint32_t)kCap) {
        __syncwarp();
        flush_cand(cb, ctr, dst, rc.cand_cap);
        cb.n = 0;
        __syncwarp();
      }
      uint32_t w = cb.n + x - h;
      for (uint32_t mm = hm; mm; mm &= mm - 1) {
        const int e = __ffs(mm) - 1;
        cb.buf[w++] = make_entry(elem_bits(e), pos0 + e);
      }
      cb.n += tot;
    };
    consume_chunk(
        rc, d, pre,
        [&](uint32_t bits, int64_t pos, bool ok) {
          const bool hit = ok && sel_key<VT, SCALE>(bits, flip, sc) <= T;
          if (__any_sync(kFull, hit)) push(hit ? 1u : 0u, 0u, [&](int) { return bits; }, pos);
        },
        [&](const uint4& x, int64_t pos0, bool ok) {
          // threshold as a value (computed here so it is live only in the loop)
          const uint32_t ukT = LARGEST ? (~T & K::KMASK) : T;
          bool any;
          if constexpr (SCALE) {
            const float tv = __uint_as_float(unkey32(ukT));
            any = false;
#pragma unroll
            for (int e = 0; e < VEC; ++e) {
              const float d = __fsub_rn(to_float<VT>(vec_elem<ES>(x, e)), sc);
              any |= LARGEST ? !(d < tv) : !(d > tv);
            }
          } else if constexpr (VT == kF32) {
            const float tv = __uint_as_float(unkey32(ukT));
            const float f0 = __uint_as_float(x.x), f1 = __uint_as_float(x.y);
            const float f2 = __uint_as_float(x.z), f3 = __uint_as_float(x.w);
            if (LARGEST) any = !(f0 < tv) | !(f1 < tv) | !(f2 < tv) | !(f3 < tv);
            else any = !(f0 > tv) | !(f1 > tv) | !(f2 > tv) | !(f3 > tv);
          } else {
            const uint32_t tb = unkey16(ukT);
            const uint32_t t2 = tb | (tb << 16);
            uint32_t mk;
            if constexpr (VT == kF16) {
              const __half2 th = *reinterpret_cast<const __half2*>(&t2);
              const __half2 h0 = *reinterpret_cast<const __half2*>(&x.x), h1 = *reinterpret_cast<const __half2*>(&x.y);
              const __half2 h2 = *reinterpret_cast<const __half2*>(&x.z), h3 = *reinterpret_cast<const __half2*>(&x.w);
              // the vector's extreme (NaN-propagating), then one unordered compare:
              // 256 x 2^20 fp16, k = 256: 157.9 -> 154.7 us against four compares
              const __half2 e = LARGEST ? __hmax2_nan(__hmax2_nan(h0, h1), __hmax2_nan(h2, h3))
                                        : __hmin2_nan(__hmin2_nan(h0, h1), __hmin2_nan(h2, h3));
              mk = LARGEST ? __hgeu2_mask(e, th) : __hleu2_mask(e, th);
            } else {
              const __nv_bfloat162 th = *reinterpret_cast<const __nv_bfloat162*>(&t2);
              const __nv_bfloat162 h0 = *reinterpret_cast<const __nv_bfloat162*>(&x.x);
              const __nv_bfloat162 h1 = *reinterpret_cast<const __nv_bfloat162*>(&x.y);
              const __nv_bfloat162 h2 = *reinterpret_cast<const __nv_bfloat162*>(&x.z);
              const __nv_bfloat162 h3 = *reinterpret_cast<const __nv_bfloat162*>(&x.w);
              const __nv_bfloat162 e = LARGEST ? __hmax2_nan(__hmax2_nan(h0, h1), __hmax2_nan(h2, h3))
                                               : __hmin2_nan(__hmin2_nan(h0, h1), __hmin2_nan(h2, h3));
              mk = LARGEST ? __hgeu2_mask(e, th) : __hleu2_mask(e, th);
            }
            any = mk != 0;
          }
          any = any && ok;
          if (__any_sync(kFull, any)) {
            uint32_t hm = 0;
            if (any) {
#pragma unroll
              for (int e = 0; e < VEC; ++e)
                if (sel_key<VT, SCALE>(vec_elem<ES>(x, e), flip, sc) <= T) hm |= 1u << e;
            }
            push(hm, 0u, [&](int e) { return vec_elem<ES>(x, e); }, pos0);
          }
        });
    if (ConsTeam::tid() == 0) RADIK_TL(p, kTlChunkEnd);
    if (cb.n) flush_cand(cb, ctr, dst, rc.cand_cap);
    defer_release(r);
  }

  __device__ void pf_item(int r, const RowCtx& rc, const ItemDesc& d) {
    if (p.flags & kFlagLargest) pf_item_t<true>(r, rc, d);
    else pf_item_t<false>(r, rc, d);
  }

  // ---- histogram item of a radix row: first digit of chunk ia
  __device__ void h_item(int r, const RowCtx& rc, const ItemDesc& d) {
    const int D1 = p.D1;
    const int NB = 1 << D1;
    const int s = rc.slot_use % p.S;
    const uint32_t use = (uint32_t)(rc.slot_use / p.S);
    uint32_t* hist = reinterpret_cast<uint32_t*>(smem + kHistOff);  // consumer area
    uint32_t* ghist = p.hist_ring + (size_t)s * ((size_t)1 << kMaxD1);
    do_release();  // before a wait that a finish holding back the slot may need it for
    if (ConsTeam::tid() == 0) m->bcast = use == 0 ? 1 : (int)spin_until_ge(p.slot_gen + s, use);
    for (int i = ConsTeam::tid() * 4; i < NB; i += ConsTeam::kSize * 4) *reinterpret_cast<uint4*>(hist + i) = make_uint4(0, 0, 0, 0);
    ConsTeam::sync();
    const bool slot_ok = m->bcast != 0;
    const int shift = K::KB - D1;
    const uint32_t flip = rc.flip;
    const float sc = rc.scaler;
    bool agg = false;
    consume_chunk(
        rc, d, [] {},
        [&](uint32_t bits, int64_t, bool ok) { hist_add_agg(hist, sel_key<VT, SCALE>(bits, flip, sc) >> shift, ok); },
        [&](const uint4& x, int64_t, bool ok) {
#pragma unroll
          for (int e = 0; e < VEC; ++e) hist_add(hist, sel_key<VT, SCALE>(vec_elem<ES>(x, e), flip, sc) >> shift, ok, e, agg);
        });
    ConsTeam::sync();
    if (slot_ok) {
      for (int i = ConsTeam::tid() * 4; i < NB; i += ConsTeam::kSize * 4) {
        const uint4 v = *reinterpret_cast<const uint4*>(hist + i);
        if (v.x) atomicAdd(ghist + i + 0, v.x);
        if (v.y) atomicAdd(ghist + i + 1, v.y);
        if (v.z) atomicAdd(ghist + i + 2, v.z);
        if (v.w) atomicAdd(ghist + i + 3, v.w);
      }
    }
    // The team's histogram atomics precede the count (team barrier, then one
    // fence on each side of it by the counting thread).
    ConsTeam::sync();
    RowState* rs = p.rs + r;
    if (ConsTeam::tid() == 0) {
      __threadfence();
      m->bcast2 = atomicAdd(&rs->hticket, 1) == rc.na - 1;
      __threadfence();
    }
    ConsTeam::sync();
    if (!m->bcast2) return;
    // Last histogram item of the row: select the first digit's bin.
    block_select<ConsTeam, true>(ghist, NB, (uint32_t)rc.k, m);
    const bool found = m->sel_found != 0;
    const uint32_t bin = m->sel_bin, cum = m->sel_cum, cnt = m->sel_cnt;
    for (int i = ConsTeam::tid() * 4; i < NB; i += ConsTeam::kSize * 4) *reinterpret_cast<uint4*>(ghist + i) = make_uint4(0, 0, 0, 0);
    ConsTeam::sync();
    if (ConsTeam::tid() == 0) {
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

  // ---- filter item of a radix row
  __device__ void f_item(int r, const RowCtx& rc, const ItemDesc& d) {
    RowState* rs = p.rs + r;
    do_release();  // the bin wait below must not hold back another row's finish
    if (ConsTeam::tid() == 0) {
      int mode = kModeNone;
      if (spin_until_ge(reinterpret_cast<const uint32_t*>(&rs->ready), 1u)) mode = __ldcg(&rs->mode);
      m->st_mode = mode;
      m->st_prefix = ld_cg_u64(&rs->prefix);
    }
    ConsTeam::sync();
    const int mode = m->st_mode;
    if (mode == kModeFinal || mode == kModeSB || mode == kModeCand) {
      const uint32_t prefix = (uint32_t)m->st_prefix;
      const int shift = K::KB - p.D1;
      const bool final_mode = mode == kModeFinal;
      const int warp = ConsTeam::wid();
      WarpBuf cb{cand_sink<ConsTeam>(), 0};
      WarpBuf ob{out_sink<ConsTeam>(), 0};
      uint32_t* cctr = reinterpret_cast<uint32_t*>(&rs->cand_count);
      uint32_t* octr = reinterpret_cast<uint32_t*>(&rs->out_count);
      uint64_t* dst = p.cand + rc.cand_off;
      auto flc = [&](const WarpBuf& s) { flush_cand(s, cctr, dst, rc.cand_cap); };
      auto flo = [&](const WarpBuf& s) { flush_out<VT>(p, s, octr, rc.out_off, rc.k); };
      const uint32_t flip = rc.flip;
      const float sc = rc.scaler;
      auto one = [&](uint32_t bits, int64_t pos, bool ok) {
        const uint32_t d = sel_key<VT, SCALE>(bits, flip, sc) >> shift;
        const bool to_out = ok && (d < prefix || (final_mode && d == prefix));
        const bool to_cand = ok && !final_mode && d == prefix;
        sink_push(ob, kSinkOut, to_out, make_entry(bits, pos), flo);
        sink_push(cb, kSinkCand, to_cand, make_entry(bits, pos), flc);
      };
      consume_chunk(rc, d, [] {}, one, [&](const uint4& x, int64_t pos0, bool ok) {
        bool any = false;
#pragma unroll
        for (int e = 0; e < VEC; ++e) any |= ok && (sel_key<VT, SCALE>(vec_elem<ES>(x, e), flip, sc) >> shift) <= prefix;
        if (__any_sync(kFull, any)) {
#pragma unroll
          for (int e = 0; e < VEC; ++e) one(vec_elem<ES>(x, e), pos0 + e, ok);
        }
      });
      if (ob.n) flo(ob);
      if (cb.n) flc(cb);
    } else {
      // nothing to filter (the row continues in phase B, or timed out): the
      // producer has issued this chunk's copies all the same, so drain them
      consume_chunk(rc, d, [] {}, [](uint32_t, int64_t, bool) {}, [](const uint4&, int64_t, bool) {});
    }
    defer_release(r);
  }

  // Hands a row to phase B.
  template <class Tm>
  __device__ void to_phase_b(int r, int src, int src_len, uint64_t prefix, int plen, int krem, int count) {
    if (Tm::tid() == 0) {
      RowState* rs = p.rs + r;
      rs->src = src;
      rs->src_len = src_len;
      rs->prefix = prefix;
      rs->plen = plen;
      rs->krem = krem;
      rs->count = count;
      rs->final_pass = 0;
      rs->sb_count = 0;
      rs->pb_min = ~0ull;
      rs->pb_max = 0;
      __threadfence();
      const int slot = atomicAdd(&p.hdr->nlarge, 1);
      p.large_list[slot] = r;
    }
  }

  // Resolves a row whose matched set -- the entries of its candidate region
  // [0, src_n) that match (prefix, plen), count of them -- is too large for
  // smem: 12-bit histogram levels over the region (read from L2) until the
  // matched set fits in smem or equals krem, then one pass that emits the
  // better entries and gathers the matched ones into smem to resolve there.
  template <class Tm>
  __device__ void side_cand_resolve(int r, const RowCtx& rc, int src_n, uint64_t prefix, int plen, int krem,
                                    int count) {
    RowState* rs = p.rs + r;
    const uint64_t* cand = p.cand + rc.cand_off;
    uint32_t* hist = reinterpret_cast<uint32_t*>(smem);  // 12-bit levels; ent[] reuses it after the last
    uint64_t* ent = reinterpret_cast<uint64_t*>(smem);
    const int W = K::KB + rc.IB;
    // entries in groups of eight per thread, loaded before they are used
    constexpr int U = 8;
    const int iters = (src_n + Tm::kSize * U - 1) / (Tm::kSize * U);
    auto for_entries = [&](auto&& fn) {
      for (int it = 0; it < iters; ++it) {
        uint64_t e[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int i = (it * U + u) * Tm::kSize + Tm::tid();
          e[u] = i < src_n ? ld_cg_u64(cand + i) : 0ull;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int i = (it * U + u) * Tm::kSize + Tm::tid();
          const uint32_t bits = (uint32_t)(e[u] >> 32);
          const int64_t pos = (int64_t)(uint32_t)e[u];
          const uint64_t c = ((uint64_t)key_of(bits, rc) << rc.IB) | (uint64_t)pos;
          fn(bits, pos, c, i < src_n);
        }
      }
    };
    for (int guard = 0; guard < 8 && count != krem && count > kCapSB && plen < W; ++guard) {
      const int D = min(12, W - plen);
      const int NB = 1 << D;
      for (int i = Tm::tid(); i < NB; i += Tm::kSize) hist[i] = 0;
      Tm::sync();
      const int sh = W - plen, sd = W - plen - D;
      const uint32_t dm = (uint32_t)NB - 1u;
      for_entries([&](uint32_t, int64_t, uint64_t c, bool ok) {
        hist_add_agg(hist, (uint32_t)shr64(c, sd) & dm, ok && shr64(c, sh) == prefix);
      });
      Tm::sync();
      block_select<Tm, false>(hist, NB, (uint32_t)krem, m);
      if (!m->sel_found) {
        if (Tm::tid() == 0) atomicOr(&p.hdr->status, kStatusSelect);
        return;
      }
      prefix = (prefix << D) | m->sel_bin;
      plen += D;
      krem -= (int)m->sel_cum;
      count = (int)m->sel_cnt;
      Tm::sync();
    }
    if (count != krem && count > kCapSB) {
      if (Tm::tid() == 0) atomicOr(&p.hdr->status, kStatusLevels);
      return;
    }
    const bool final_mode = count == krem;
    const int sh = W - plen;
    uint32_t* out_ctr = reinterpret_cast<uint32_t*>(&rs->out_count);
    if (Tm::tid() == 0) m->counter = 0;
    Tm::sync();
    for_entries([&](uint32_t bits, int64_t pos, uint64_t c, bool ok) {
      const uint64_t t = shr64(c, sh);
      const bool to_out = ok && (t < prefix || (final_mode && t == prefix));
      const bool to_ent = ok && !final_mode && t == prefix;
      if (!__any_sync(kFull, to_out || to_ent)) return;
      const uint32_t so = warp_reserve(to_out ? 1u : 0u, out_ctr);
      if (to_out && so < (uint32_t)rc.k) write_out<VT>(p, rc.out_off + so, bits, pos);
      const uint32_t se = warp_reserve(to_ent ? 1u : 0u, &m->counter);
      if (to_ent && se < (uint32_t)kCapSB) ent[se] = make_entry(bits, pos);
    });
    Tm::sync();
    if (!final_mode) {
      const int ne = min((int)m->counter, kCapSB);
      auto get = [&](int i, uint32_t& bits, int64_t& pos) {
        const uint64_t e = ent[i];
        bits = (uint32_t)(e >> 32);
        pos = (int64_t)(uint32_t)e;
      };
      smem_resolve<Tm, VT, SCALE>(get, ne, rc, prefix, plen, krem, ne,
                                        reinterpret_cast<uint32_t*>(smem + kResolveHistOff), m, &p.hdr->status);
      smem_emit<Tm, VT, SCALE>(p, get, ne, rc, prefix, plen, rs, m);
    }
    post_process<Tm, VT, SCALE>(p, rc, smem, m);
  }

  // Finisher work of a large row (all of its items are done).
  template <class Tm>
  __device__ void finish_row(int r) {
    const RowCtx rc = load_row<VT, SCALE>(p, r);
    RowState* rs = p.rs + r;
    // thread 0 of the team acquired the row's chunk counter (fin_item_t) and
    // the team barrier there passed that on: the row's state is visible
    if (Tm::tid() == 0) {
      m->st_mode = rc.kind == kKindAll ? kModeAll : __ldcg(&rs->mode);
      m->st_krem = __ldcg(&rs->krem);
      m->st_count = __ldcg(&rs->count);
      m->st_plen = __ldcg(&rs->plen);
      m->st_prefix = ld_cg_u64(&rs->prefix);
      m->st_candn = __ldcg(&rs->cand_count);
    }
    Tm::sync();
    uint64_t* ent = reinterpret_cast<uint64_t*>(smem);
    auto get = [&](int i, uint32_t& bits, int64_t& pos) {
      const uint64_t e = ent[i];
      bits = (uint32_t)(e >> 32);
      pos = (int64_t)(uint32_t)e;
    };
    const uint64_t* cand = p.cand + rc.cand_off;
    // the consumer team finishes in the idle ring (kCapTail entries)
    constexpr int kCap = Tm::kSize == ConsTeam::kSize ? kCapTail : kCapSB;
    if (rc.kind == kKindGridPref) {
      // c counts every key that passed the threshold, including those its
      // region (rc.cand_cap entries) had no room for: every branch that
      // reads the region first checks that all c entries are in it
      const int c = m->st_candn;
      if (Tm::tid() == 0) {
        RADIK_TL(p, kTlFinBegin);
        RADIK_TL_VALUE(p, kTlFinCands, c);
      }
      if (c >= rc.k && c <= kCap && c <= rc.cand_cap) {
        load_entries<Tm>(ent, cand, c);
        Tm::sync();
        if (Tm::tid() == 0) RADIK_TL(p, kTlFinLoaded);
        uint64_t prefix = 0;
        int plen = 0, krem = rc.k;
        smem_resolve<Tm, VT, SCALE>(get, c, rc, prefix, plen, krem, c, reinterpret_cast<uint32_t*>(smem + kCap * 8), m,
                                &p.hdr->status);
        if (Tm::tid() == 0) RADIK_TL(p, kTlFinResolved);
        // a pre-filter row's outputs are written by its finish alone
        smem_emit<Tm, VT, SCALE>(p, get, c, rc, prefix, plen, rs, m, true);
        if (Tm::tid() == 0) RADIK_TL(p, kTlFinEmitted);
        post_process<Tm, VT, SCALE>(p, rc, smem, m);
        if (Tm::tid() == 0) RADIK_TL(p, kTlFinPost);
      } else if (c >= rc.k && c <= min(rc.cand_cap, kSideCandMax) &&
                 (p.B >= kSideResolveMinRows || (Tm::kSize == ConsTeam::kSize && c <= kTailResolveMax))) {
        side_cand_resolve<Tm>(r, rc, c, 0, 0, rc.k, c);
      } else if (c >= rc.k && c <= rc.cand_cap) {
        to_phase_b<Tm>(r, 1, c, 0, 0, rc.k, c);
      } else {
        to_phase_b<Tm>(r, 0, rc.n, 0, 0, rc.k, rc.n);
      }
      return;
    }
    const int mode = m->st_mode;
    if (mode == kModeSB) {
      const int ne = min(m->st_candn, kCapSB);
      load_entries<Tm>(ent, cand, ne);
      uint64_t prefix = m->st_prefix;
      int plen = m->st_plen, krem = m->st_krem;
      Tm::sync();
      smem_resolve<Tm, VT, SCALE>(get, ne, rc, prefix, plen, krem, ne, reinterpret_cast<uint32_t*>(smem + kResolveHistOff), m,
                              &p.hdr->status);
      smem_emit<Tm, VT, SCALE>(p, get, ne, rc, prefix, plen, rs, m);
      post_process<Tm, VT, SCALE>(p, rc, smem, m);
    } else if (mode == kModeCand) {
      const int src_n = min(m->st_candn, rc.cand_cap);
      if (src_n <= kSideCandMax && p.B >= kSideResolveMinRows)
        side_cand_resolve<Tm>(r, rc, src_n, m->st_prefix, m->st_plen, m->st_krem, m->st_count);
      else to_phase_b<Tm>(r, 1, src_n, m->st_prefix, m->st_plen, m->st_krem, m->st_count);
    } else if (mode == kModeDefer) {
      to_phase_b<Tm>(r, 0, rc.n, m->st_prefix, m->st_plen, m->st_krem, m->st_count);
    } else if (mode == kModeFinal || mode == kModeAll) {
      post_process<Tm, VT, SCALE>(p, rc, smem, m);
    }
  }

  // ---- phase B: multi-CTA radix levels over the listed rows ----
  struct PBTable {
    int32_t row[kPhaseBSlots];
    int32_t nch[kPhaseBSlots];
    int32_t c0[kPhaseBSlots + 1];
    int32_t chunk;  // entries per work unit this pass
  };

  // Runs f(bits, pos, ok) over entries [a, b) of a phase-B source.
  template <typename Fn>
  __device__ void pb_source(const RowCtx& rc, int src, int64_t a, int64_t b, Fn&& fn) {
    if (src == 1) {
      // candidate entries from L2, eight loads a thread in flight
      constexpr int UE = 8;
      const uint64_t* cand = p.cand + rc.cand_off;
      for (int64_t base = a; base < b; base += (int64_t)UE * FullTeam::kSize) {
        uint64_t e[UE];
#pragma unroll
        for (int u = 0; u < UE; ++u) {
          const int64_t i = base + (int64_t)u * FullTeam::kSize + FullTeam::tid();
          e[u] = i < b ? ld_cg_u64(cand + i) : 0ull;
        }
#pragma unroll
        for (int u = 0; u < UE; ++u) {
          const int64_t i = base + (int64_t)u * FullTeam::kSize + FullTeam::tid();
          fn((uint32_t)(e[u] >> 32), (int64_t)(uint32_t)e[u], i < b);
        }
      }
    } else {
      for_range_v<FullTeam, ES, U>(p.val_in, rc.in_off, a, b, fn, [&](const uint4& x, int64_t pos0, bool ok) {
#pragma unroll
        for (int e = 0; e < VEC; ++e) fn(vec_elem<ES>(x, e), pos0 + e, ok);
      });
    }
  }

  // Builds the table of the first nG listed rows whose flag matches `want`
  // (0: rows that still need a histogram level, 1: rows due for the final
  // filter).  Returns the number of chunks.
  __device__ int pb_table(PBTable* t, int nG, int want) {
    if (FullTeam::tid() == 0) {
      // work units sized so the pass spreads over the whole grid (at least
      // 2048 entries, at most kPhaseBChunk)
      int64_t sum = 0;
      for (int i = 0; i < nG; ++i) {
        const RowState* rs = p.rs + p.large_list[i];
        if (__ldcg(&rs->final_pass) == want) sum += __ldcg(&rs->src_len);
      }
      int64_t ch = (sum + gridDim.x - 1) / gridDim.x;
      ch = (ch + 2047) / 2048 * 2048;
      const int chunk = ch < 2048 ? 2048 : ch > kPhaseBChunk ? kPhaseBChunk : (int)ch;
      int c = 0;
      for (int i = 0; i < nG; ++i) {
        const int r = p.large_list[i];
        const RowState* rs = p.rs + r;
        const int fp = __ldcg(&rs->final_pass);
        const int len = __ldcg(&rs->src_len);
        t->row[i] = r;
        t->c0[i] = c;
        t->nch[i] = (fp == want) ? (len + chunk - 1) / chunk : 0;
        c += t->nch[i];
      }
      t->c0[nG] = c;
      t->chunk = chunk;
    }
    FullTeam::sync();
    return t->c0[nG];
  }

  __device__ void phase_b() {
    PBTable* t = reinterpret_cast<PBTable*>(m->pbtab);
    for (int round = 0; round < 64; ++round) {
      grid_barrier<FullTeam>(p.hdr, p.spin_limit);
      const int nL = __ldcg(&p.hdr->nlarge);
      if (nL <= 0) return;
      const int nG = min(nL, kPhaseBSlots);
      // Round 0: every histogram slot is cleared (the call clears the ring only
      // for radix rows; later each selection clears the slot it read), and
      // rows already small enough skip the histogram.  Rows reaching the
      // window later start from to_phase_b's state.
      for (int i = blockIdx.x; round == 0 && i < kPhaseBSlots; i += gridDim.x) {
        uint32_t* gh = p.hist_ring + (size_t)i * ((size_t)1 << kMaxD1);
        for (int j = FullTeam::tid(); j < 4096; j += FullTeam::kSize) gh[j] = 0;
        if (FullTeam::tid() == 0 && i < nG) {
          RowState* rs = p.rs + p.large_list[i];
          const int cnt = __ldcg(&rs->count), kr = __ldcg(&rs->krem);
          rs->final_pass = (cnt == kr || cnt <= kCapSB) ? 1 : 0;
          rs->pb_min = ~0ull;
          rs->pb_max = 0;
        }
      }
      if (round == 0) grid_barrier<FullTeam>(p.hdr, p.spin_limit);
      // ---- histogram of the next 12-bit digit
      int total = pb_table(t, nG, 0);
      uint32_t* hist = reinterpret_cast<uint32_t*>(smem);
      for (int w = blockIdx.x; w < total; w += gridDim.x) {
        int i = 0;
        while (t->c0[i + 1] <= w) ++i;
        const int r = t->row[i];
        const RowCtx rc = load_row<VT, SCALE>(p, r);
        const RowState* rs = p.rs + r;
        const uint64_t prefix = ld_cg_u64(&rs->prefix);
        const int plen = __ldcg(&rs->plen);
        const int src = __ldcg(&rs->src);
        const int len = __ldcg(&rs->src_len);
        const int W = K::KB + rc.IB;
        const int D = min(12, W - plen);
        const int NB = 1 << D;
        for (int j = FullTeam::tid(); j < NB; j += FullTeam::kSize) hist[j] = 0;
        FullTeam::sync();
        const int sh = W - plen, sd = W - plen - D;
        const uint32_t dm = (uint32_t)NB - 1u;
        const int64_t a = (int64_t)(w - t->c0[i]) * t->chunk, b = min((int64_t)len, a + t->chunk);
        uint64_t lo = ~0ull, hi = 0;
        pb_source(rc, src, a, b, [&](uint32_t bits, int64_t pos, bool ok) {
          const uint64_t c = ((uint64_t)key_of(bits, rc) << rc.IB) | (uint64_t)pos;
          const bool match = ok && shr64(c, sh) == prefix;
          hist_add_agg(hist, (uint32_t)shr64(c, sd) & dm, match);
          if (match) {
            lo = min(lo, c);
            hi = max(hi, c);
          }
        });
        // the matched set's extremes: a level that does not split the set
        // lets the selection jump to their common prefix instead
        uint64_t mn, mx;
        block_minmax<FullTeam>(lo, hi, &mn, &mx, m);
        RowState* rsw = p.rs + r;
        if (FullTeam::tid() == 0 && mn != ~0ull) {
          atomicMin(reinterpret_cast<unsigned long long*>(&rsw->pb_min), (unsigned long long)mn);
          atomicMax(reinterpret_cast<unsigned long long*>(&rsw->pb_max), (unsigned long long)mx);
        }
        uint32_t* gh = p.hist_ring + (size_t)i * ((size_t)1 << kMaxD1);
        for (int j = FullTeam::tid(); j < NB; j += FullTeam::kSize)
          if (hist[j]) atomicAdd(gh + j, hist[j]);
        FullTeam::sync();
      }
      grid_barrier<FullTeam>(p.hdr, p.spin_limit);
      // ---- bin selection, one CTA per row
      for (int i = blockIdx.x; i < nG; i += gridDim.x) {
        const int r = p.large_list[i];
        RowState* rs = p.rs + r;
        if (__ldcg(&rs->final_pass)) continue;
        const RowCtx rc = load_row<VT, SCALE>(p, r);
        const int plen = __ldcg(&rs->plen);
        const int W = K::KB + rc.IB;
        const int D = min(12, W - plen);
        const int NB = 1 << D;
        uint32_t* gh = p.hist_ring + (size_t)i * ((size_t)1 << kMaxD1);
        const int krem = __ldcg(&rs->krem);
        block_select<FullTeam, true>(gh, NB, (uint32_t)krem, m);
        const bool found = m->sel_found != 0;
        const uint32_t bin = m->sel_bin, cum = m->sel_cum, cnt = m->sel_cnt;
        for (int j = FullTeam::tid(); j < NB; j += FullTeam::kSize) gh[j] = 0;
        FullTeam::sync();
        if (FullTeam::tid() == 0) {
          if (!found) {
            atomicOr(&p.hdr->status, kStatusSelect);
            rs->count = krem;  // give up on this row: finish what is there
            rs->final_pass = 1;
          } else {
            const uint64_t mn = ld_cg_u64(&rs->pb_min), mx = ld_cg_u64(&rs->pb_max);
            rs->pb_min = ~0ull;  // for the next round's histogram pass
            rs->pb_max = 0;
            const int common = mn == mx ? W : __clzll((long long)(mn ^ mx)) - (64 - W);
            if (mn != ~0ull && common > plen + D) {
              // every matched entry fell in one bin: take all the bits they share
              rs->prefix = shr64(mn, W - common);
              rs->plen = common;
            } else {
              rs->prefix = (ld_cg_u64(&rs->prefix) << D) | bin;
              rs->plen = plen + D;
            }
            rs->krem = krem - (int)cum;
            rs->count = (int)cnt;
            rs->final_pass = ((int)cnt == krem - (int)cum || (int)cnt <= kCapSB) ? 1 : 0;
          }
        }
        FullTeam::sync();
      }
      grid_barrier<FullTeam>(p.hdr, p.spin_limit);
      // ---- final filter for the rows that are due
      total = pb_table(t, nG, 1);
      const int warp = FullTeam::wid();
      for (int w = blockIdx.x; w < total; w += gridDim.x) {
        int i = 0;
        while (t->c0[i + 1] <= w) ++i;
        const int r = t->row[i];
        const RowCtx rc = load_row<VT, SCALE>(p, r);
        RowState* rs = p.rs + r;
        const uint64_t prefix = ld_cg_u64(&rs->prefix);
        const int plen = __ldcg(&rs->plen);
        const int src = __ldcg(&rs->src);
        const int len = __ldcg(&rs->src_len);
        const bool final_mode = __ldcg(&rs->count) == __ldcg(&rs->krem);
        const int W = K::KB + rc.IB;
        const int sh = W - plen;
        WarpBuf cb{cand_sink<FullTeam>(), 0};
        WarpBuf ob{out_sink<FullTeam>(), 0};
        uint32_t* cctr = reinterpret_cast<uint32_t*>(&rs->sb_count);
        uint32_t* octr = reinterpret_cast<uint32_t*>(&rs->out_count);
        uint64_t* dst = p.pb_sb + (size_t)i * kCapSB;
        auto flc = [&](const WarpBuf& s) { flush_cand(s, cctr, dst, kCapSB); };
        auto flo = [&](const WarpBuf& s) { flush_out<VT>(p, s, octr, rc.out_off, rc.k); };
        const int64_t a = (int64_t)(w - t->c0[i]) * t->chunk, b = min((int64_t)len, a + t->chunk);
        pb_source(rc, src, a, b, [&](uint32_t bits, int64_t pos, bool ok) {
          const uint64_t c = ((uint64_t)key_of(bits, rc) << rc.IB) | (uint64_t)pos;
          const uint64_t tt = shr64(c, sh);
          sink_push(ob, kSinkOut, ok && (tt < prefix || (final_mode && tt == prefix)), make_entry(bits, pos), flo);
          sink_push(cb, kSinkCand, ok && !final_mode && tt == prefix, make_entry(bits, pos), flc);
        });
        if (ob.n) flo(ob);
        if (cb.n) flc(cb);
        FullTeam::sync();
      }
      grid_barrier<FullTeam>(p.hdr, p.spin_limit);
      // ---- finish the rows that were filtered
      uint64_t* ent = reinterpret_cast<uint64_t*>(smem);
      for (int i = blockIdx.x; i < nG; i += gridDim.x) {
        const int r = p.large_list[i];
        RowState* rs = p.rs + r;
        if (!__ldcg(&rs->final_pass)) continue;
        const RowCtx rc = load_row<VT, SCALE>(p, r);
        const int count = __ldcg(&rs->count), krem0 = __ldcg(&rs->krem);
        if (count != krem0) {
          const int ne = min(__ldcg(&rs->sb_count), kCapSB);
          const uint64_t* sb = p.pb_sb + (size_t)i * kCapSB;
          load_entries<FullTeam>(ent, sb, ne);
          uint64_t prefix = ld_cg_u64(&rs->prefix);
          int plen = __ldcg(&rs->plen), krem = krem0;
          FullTeam::sync();
          auto get = [&](int j, uint32_t& bits, int64_t& pos) {
            const uint64_t e = ent[j];
            bits = (uint32_t)(e >> 32);
            pos = (int64_t)(uint32_t)e;
          };
          smem_resolve<FullTeam, VT, SCALE>(get, ne, rc, prefix, plen, krem, ne, reinterpret_cast<uint32_t*>(smem + kResolveHistOff), m,
                              &p.hdr->status);
          smem_emit<FullTeam, VT, SCALE>(p, get, ne, rc, prefix, plen, rs, m);
        }
        post_process<FullTeam, VT, SCALE>(p, rc, smem, m);
        if (FullTeam::tid() == 0) rs->final_pass = 2;  // done
      }
      grid_barrier<FullTeam>(p.hdr, p.spin_limit);
      // ---- drop the finished rows from the list (CTA 0)
      if (blockIdx.x == 0 && FullTeam::tid() == 0) {
        int w = 0;
        for (int i = 0; i < nL; ++i) {
          const int r = p.large_list[i];
          if (i < nG && __ldcg(&p.rs[r].final_pass) == 2) continue;
          p.large_list[w++] = r;
        }
        p.hdr->nlarge = w;
        __threadfence();
      }
    }
    if (FullTeam::tid() == 0 && blockIdx.x == 0) atomicOr(&p.hdr->status, kStatusLevels);
  }
};

// Maps a claim index to an item.  Returns true for an A item; idx is the
// item's index in its sequence.
__device__ __forceinline__ bool decode_item(int q, int NA, int NB, int L, int& idx) {
  const int L1 = min(L, NA);
  if (q < L1) {
    idx = q;
    return true;
  }
  const int q1 = q - L1;
  const int P = min(NA - L1, NB);
  if (q1 < 2 * P) {
    const int mth = q1 >> 1;
    if ((q1 & 1) == 0) {
      idx = L1 + mth;
      return true;
    }
    idx = mth;
    return false;
  }
  const int rest = q1 - 2 * P;
  if (NA - L1 > P) {
    idx = L1 + P + rest;
    return true;
  }
  idx = P + rest;
  return false;
}

// Item geometry of a claim: which row, A or B item, chunk, FIN.
// The B-item layout of an equal-length call (see UniformB).
__device__ __forceinline__ UniformB uniform_b(const EngineParams& p, int unc, int ufin) {
  const int R = p.u_tail_rows;
  const int nct = R > 0 ? (int)ceil_div32(p.u_n, p.u_ch_tail) : unc;
  return UniformB{p.B, unc, nct, R, ufin, p.fin_delay};
}

struct ItemRef {
  int32_t row, sub, isA, fin;
};

__device__ __forceinline__ ItemRef resolve_item(const EngineParams& p, int q, int NA, int NB, int lag, int una, int unc,
                                                int ufin) {
  ItemRef it{0, 0, 0, 0};
  int idx;
  it.isA = decode_item(q, NA, NB, lag, idx);
  if (it.isA) {
    it.row = p.uniform ? idx / una : p.a_row[idx];
    it.sub = idx;  // made row-relative once the row's a0 is known
  } else if (p.uniform) {
    uniform_b(p, unc, ufin).decode(idx, &it.row, &it.sub, &it.fin);
  } else {
    const int32_t v = p.b_row[idx];
    it.row = v & 0x7FFFFFFF;
    it.fin = (v >> 31) & 1;
    it.sub = idx;  // made row-relative once the row's b0 is known
  }
  return it;
}

__device__ __forceinline__ bool is_streaming(int kind, int isA, int fin) {
  return isA ? (kind == kKindAll || kind == kKindGridRadix)
             : (!fin && (kind == kKindGridPref || kind == kKindGridRadix));
}

// Claims the next work item.  Items 0 .. gridDim.x - 1 are the CTAs' first
// items, taken by block index without a claim; the counter hands out the rest.
__device__ __forceinline__ int claim_item(const EngineParams& p) {
  return (int)(gridDim.x + atomicAdd(&p.hdr->qhead, 1u));
}

// Producer (one thread): claims items in order, routes streaming items to
// the consumer queue and the rest to the side queue, and issues the bulk
// copies of each streaming chunk into the ring as slots drain.
template <int VT, bool SCALE>
__device__ void producer_loop(const EngineParams& p, Ctrl* ctl, int NA, int NB, int lag, int una, int unc, int ufin,
                              int fin_tail, int first_q) {
  constexpr int ES = KT<VT, SCALE>::ES, VEC = KT<VT, SCALE>::VEC;
  const int NQ = NA + NB;
  uint32_t g = 0, ci = 0, si = 0;
  auto push = [&](uint64_t* full, uint64_t* empty, ItemDesc* slots, uint32_t& i, const ItemDesc& d) {
    const uint32_t slot = i % kQ;
    if (i >= (uint32_t)kQ) {
      const uint32_t parity = ((i / kQ) - 1u) & 1u;
      uint32_t it = 0;
      RADIK_TL_T0(tw);
      while (!mbar_try_wait(&empty[slot], parity)) {
        if (++it > p.spin_limit) {
          atomicOr(&p.hdr->status, kStatusTimeout);
          break;
        }
      }
      RADIK_TL_ACC(p, full == ctl->sq_full ? kTlAccSideQ : kTlAccConsQ, tw);
    }
    slots[slot] = d;
    mbar_arrive(&full[slot]);
    ++i;
  };
  // In the tail of FIN items a claim is made only once this CTA's side team
  // has finished what it holds, so the last finishes spread over the CTAs.
  auto throttle = [&](int last_q) {
    if (fin_tail > 0 && last_q + 1 >= NQ - fin_tail) {
      uint32_t it = 0;
      while (*reinterpret_cast<volatile uint32_t*>(&ctl->side_done) < si ||
             *reinterpret_cast<volatile uint32_t*>(&ctl->cons_done) < ci) {
        if (++it > p.spin_limit) {
          atomicOr(&p.hdr->status, kStatusTimeout);
          break;
        }
        __nanosleep(256);
      }
    }
  };
  int q = first_q >= 0 ? first_q : claim_item(p);
  // Threshold word of the next chunk item's row, loaded while the current
  // item's copies are issued (pf_row: its row, -1 = none).  The word holds
  // the threshold itself, so a relaxed load suffices; a word read before the
  // threshold existed is read again below.
  int pf_row = -1;
  uint64_t pf_tr = 0;
  while (true) {
    ItemDesc d{};
    if (q >= NQ) {
      d.q = -1;
      push(ctl->cq_full, ctl->cq_empty, ctl->cq, ci, d);
      push(ctl->sq_full, ctl->sq_empty, ctl->sq, si, d);
      break;
    }
    const ItemRef ir = resolve_item(p, q, NA, NB, lag, una, unc, ufin);
    const RowCtx rc = load_row<VT, SCALE>(p, ir.row);
    d.q = q;
    d.row = ir.row;
    d.isA = ir.isA;
    d.fin = ir.fin;
    d.sub = ir.isA ? ir.sub - rc.a0 : (p.uniform ? ir.sub : ir.sub - rc.b0);
    if (!is_streaming(rc.kind, ir.isA, ir.fin)) {
      // Finishes in the tail of the claim order go to the consumer team (three
      // times the side team's threads): nothing streams after them.
      if (ir.fin && fin_tail > 0 && q >= NQ - fin_tail) push(ctl->cq_full, ctl->cq_empty, ctl->cq, ci, d);
      else push(ctl->sq_full, ctl->sq_empty, ctl->sq, si, d);
      if (q + 1 >= NQ) {  // the last item: every later claim falls past the end
        q = NQ;
        continue;
      }
      throttle(q);
      q = claim_item(p);
      continue;
    }
    if (!ir.isA && rc.kind == kKindGridPref) {
      // The chunk is useless before its row's threshold exists, so in a large
      // call its copies wait for it: at the start this keeps the ring fills of
      // all CTAs from queueing ahead of the sample reads that produce the
      // thresholds.  The sample item precedes the chunk in the claim order, so
      // the wait ends.  A small call (early_copy) streams its few megabytes
      // while the thresholds are computed; its consumers wait for them.
      uint64_t v = ir.row == pf_row ? pf_tr : 0ull;
      RADIK_TL_T0(tw);
      if (!(v >> 32)) v = ld_acquire_u64(&p.rs[ir.row].tready);
      for (uint32_t it = 0; !(v >> 32) && !p.early_copy && it < p.spin_limit; ++it) {
        __nanosleep(128);
        v = ld_acquire_u64(&p.rs[ir.row].tready);
      }
      RADIK_TL_ACC(p, kTlAccThr, tw);
      d.thr = (uint32_t)v;
      d.thr_ok = (int32_t)(v >> 32);
    }
    // chunk geometry: the aligned middle goes through the ring
    const int64_t a = (int64_t)d.sub * rc.ch, b = min((int64_t)rc.n, a + rc.ch);
    const char* row = static_cast<const char*>(p.val_in) + rc.in_off * ES;
    int64_t head = 0, nvec = 0;
    if (b > a) {
      const uintptr_t addr_a = reinterpret_cast<uintptr_t>(row + a * ES);
      head = (int64_t)(((16u - (unsigned)(addr_a & 15u)) & 15u) / ES);
      if (head > b - a) head = b - a;
      nvec = (b - a - head) / VEC;
    }
    d.a = a;
    d.b = b;
    d.va = a + head;
    d.nvec = nvec;
    d.nst = (int32_t)((nvec + kStageVecs - 1) / kStageVecs);
    d.g0 = g;
    push(ctl->cq_full, ctl->cq_empty, ctl->cq, ci, d);
    // Claim the next item now, so the claim's latency overlaps this chunk's
    // copies -- except next to the FIN tail, where the claim may wait for the
    // side team, which may need this chunk: there it follows the copies.
    // The last grid of items is claimed only when this item's copies are all
    // issued: a claim made early holds an item that an idle CTA could start.
    const bool near_tail = fin_tail > 0 && q + 1 >= NQ - fin_tail;
    const bool late_claim = near_tail || q + 1 >= NQ - fin_tail - (int)gridDim.x;
    const bool last = q + 1 >= NQ;
    int nq = last ? NQ : late_claim ? -1 : claim_item(p);
    const uint4* src = reinterpret_cast<const uint4*>(row + d.va * ES);
    uint4* ring = reinterpret_cast<uint4*>(reinterpret_cast<uint8_t*>(ctl) - (kCtrlOff + 6144));
    // L2 prefetch p.l2_ahead stages ahead of the copies: the ring's copies
    // then wait for L2 rather than DRAM, and more of the row is in flight
    // than the ring holds.
    const int ahead = p.l2_ahead;
    auto stage_bytes = [&](int i) { return (uint32_t)min((int64_t)kStageVecs, nvec - (int64_t)i * kStageVecs) * 16u; };
    for (int i = 0; i < min(ahead, d.nst); ++i) bulk_prefetch_l2(src + (int64_t)i * kStageVecs, stage_bytes(i));
    for (int i = 0; i < d.nst; ++i, ++g) {
      constexpr uint32_t NS = ring_stages<VT>();
      const uint32_t slot = g % NS;
      if (g >= NS) {
        const uint32_t parity = ((g / NS) - 1u) & 1u;
        uint32_t it = 0;
        RADIK_TL_T0(tw);
        while (!mbar_try_wait(&ctl->empty[slot], parity)) {
          if (++it > p.spin_limit) {
            atomicOr(&p.hdr->status, kStatusTimeout);
            break;
          }
        }
        RADIK_TL_ACC(p, kTlAccRing, tw);
      }
      const int64_t v0 = (int64_t)i * kStageVecs;
      const uint32_t bytes = stage_bytes(i);
      mbar_expect_tx(&ctl->full[slot], bytes);
      bulk_g2s(ring + (size_t)slot * kStageVecs, src + v0, bytes, &ctl->full[slot]);
      if (ahead > 0 && i + ahead < d.nst) bulk_prefetch_l2(src + (int64_t)(i + ahead) * kStageVecs, stage_bytes(i + ahead));
      if (i == d.nst / 2) {  // the claim has long returned: reading it does not stall the copies
        pf_row = -1;
        if (nq >= 0 && nq < NQ) {
          const ItemRef nir = resolve_item(p, nq, NA, NB, lag, una, unc, ufin);
          if (!nir.isA && !nir.fin) {
            pf_row = nir.row;
            pf_tr = ld_relaxed_u64(&p.rs[nir.row].tready);
          }
        }
      }
    }
    if (late_claim && !last) {
      throttle(q);
      RADIK_TL_T0(tw);
      nq = claim_item(p);
      RADIK_TL_ACC(p, kTlAccClaim, tw);
    }
    q = nq;
  }
}

// Pops the team's next item (every thread of the team calls it).
template <class Tm>
__device__ __forceinline__ ItemDesc pop_item(uint64_t* full, uint64_t* empty, const ItemDesc* slots, uint32_t i,
                                             const EngineParams& p) {
  const uint32_t slot = i % kQ;
  const uint32_t parity = (i / kQ) & 1u;
  uint32_t it = 0;
  while (!mbar_try_wait(&full[slot], parity)) {
    if (++it > p.spin_limit) {
      if (Tm::tid() == 0) atomicOr(&p.hdr->status, kStatusTimeout);
      break;
    }
  }
  const ItemDesc d = slots[slot];
  Tm::sync();
  if (Tm::tid() == 0) mbar_arrive(&empty[slot]);
  return d;
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <int VT, bool SCALE>
__global__ void __launch_bounds__(kThreads, kCtasPerSM) engine_kernel(const __grid_constant__ EngineParams p) {
  extern __shared__ __align__(128) uint8_t smem[];
  Ctrl* ctl = ctrl_of(smem);
  if (threadIdx.x == 0) {
    RADIK_TL(p, kTlStart);
    // the call's device span (radik_get_call_span): the first CTA to start
    // sets the start, every CTA raises the end as it leaves
    atomicCAS(reinterpret_cast<unsigned long long*>(&p.hdr->t_first), 0ull, globaltimer_ns());
  }
  if (!p.uniform && __ldcg(&p.hdr->plan_error)) return;
  if (threadIdx.x == 0) {
    for (int i = 0; i < ring_stages<VT>(); ++i) {
      mbar_init(&ctl->full[i], 1);
      mbar_init(&ctl->empty[i], ConsTeam::kWarps);
    }
    for (int i = 0; i < kQ; ++i) {
      mbar_init(&ctl->cq_full[i], 1);
      mbar_init(&ctl->cq_empty[i], 1);
      mbar_init(&ctl->sq_full[i], 1);
      mbar_init(&ctl->sq_empty[i], 1);
    }
    mbar_fence_init();
    ctl->side_done = 0;
    ctl->cons_done = 0;
    for (Misc* mm : {cons_misc(smem), side_misc(smem)}) {
      mm->rel_row = -1;
      mm->t_row = -1;
    }
  }
  __syncthreads();
  int NA, NB, lag, fin_tail;
  int una = 1, unc = 0, ufin = 0;
  if (p.uniform) {
    const int kind = row_kind(p.u_n, p.u_k, p.cta_cap);
    una = row_na(kind, p.u_n, p.CH, p.CHR);
    unc = row_nbc(kind, p.u_n, p.CH, p.CHR);
    ufin = row_fin(kind);
    NA = p.B * una;
    NB = (int)uniform_b(p, unc, ufin).count();
    lag = p.lag;
    fin_tail = ufin ? min(p.fin_delay, p.B) : 0;
  } else {
    NA = __ldcg(&p.hdr->na);
    NB = __ldcg(&p.hdr->nb);
    lag = __ldcg(&p.hdr->lag);
    fin_tail = __ldcg(&p.hdr->fin_tail);
  }
  // The CTA's first item is its block index.  A pre-filter sample taken here
  // is computed by the whole CTA before the teams start: nothing streams
  // until the first thresholds exist, so these samples are on every CTA's
  // critical path.
  int first_q = (int)blockIdx.x;
  if (first_q < NA + NB) {
    const ItemRef ir = resolve_item(p, first_q, NA, NB, lag, una, unc, ufin);
    const RowCtx rc = load_row<VT, SCALE>(p, ir.row);
    if (ir.isA && rc.kind == kKindGridPref) {
      Engine<VT, SCALE> e(p, smem, smem + kSideAreaOff, side_misc(smem));
      e.template sample_item_t<FullTeam>(ir.row, rc, true);
      if (threadIdx.x == 0) RADIK_TL(p, kTlFirstSample);
      first_q = -1;
    }
  }
  const int warp = threadIdx.x >> 5;
  if (warp == kProducerWarp) {
    if ((threadIdx.x & 31) == 0) producer_loop<VT, SCALE>(p, ctl, NA, NB, lag, una, unc, ufin, fin_tail, first_q);
  } else if (warp < kConsWarps) {
    // consumer team: streaming items
    Engine<VT, SCALE> e(p, smem, smem + kConsAreaOff, cons_misc(smem));
    Misc* m = e.m;
    const bool releaser = ConsTeam::tid() == ConsTeam::kSize - 32;
    for (uint32_t i = 0;; ++i) {
      // The previous item's chunk counter is released during the next item
      // when one is already queued (its fence then overlaps that item's
      // data); with nothing queued it is released before waiting, so no
      // release is ever held by an idle team.
      if (releaser) {
        e.pending_rel = m->rel_row;
        if (e.pending_rel >= 0 && !mbar_try_wait(&ctl->cq_full[i % kQ], (i / kQ) & 1u)) e.do_release();
      }
      RADIK_TL_T0(tw);
      const ItemDesc d = pop_item<ConsTeam>(ctl->cq_full, ctl->cq_empty, ctl->cq, i, p);
      if (ConsTeam::tid() == 0) {
        RADIK_TL_ACC(p, kTlAccConsIdle, tw);
        m->rel_row = -1;
      }
      if (d.q < 0) break;
      const RowCtx rc = load_row<VT, SCALE>(p, d.row);
      if (d.fin) {
        // A finish from the tail of the claim order: this team has streamed
        // all of its chunks and no copies follow, so the ring is its scratch.
        // Its own last chunk may belong to this row: release it first.
        e.do_release();
        ConsTeam::sync();
        Engine<VT, SCALE> ef(p, smem, smem, m);
        ef.template fin_item_t<ConsTeam>(d.row, rc);
      } else if (d.isA) {
        if (rc.kind == kKindAll) e.all_item(d.row, rc, d);
        else e.h_item(d.row, rc, d);
      } else if (rc.kind == kKindGridPref) {
        e.pf_item(d.row, rc, d);
      } else {
        e.f_item(d.row, rc, d);
      }
      ConsTeam::sync();
      if (ConsTeam::tid() == 0) *reinterpret_cast<volatile uint32_t*>(&ctl->cons_done) = i + 1;
    }
    if (ConsTeam::tid() == 0) RADIK_TL(p, kTlConsDone);
    e.do_release();
  } else {
    // side team: samples, single-item rows, FIN items
    Engine<VT, SCALE> e(p, smem, smem + kSideAreaOff, side_misc(smem));
    for (uint32_t i = 0;; ++i) {
      RADIK_TL_T0(tw);
      const ItemDesc d = pop_item<SideTeam>(ctl->sq_full, ctl->sq_empty, ctl->sq, i, p);
      if (SideTeam::tid() == 0) {
        RADIK_TL_ACC(p, kTlAccSideIdle, tw);
        RADIK_TL_COUNT(p, kTlNSide);
      }
      if (d.q < 0) break;
      const RowCtx rc = load_row<VT, SCALE>(p, d.row);
      if (d.isA) {
        switch (rc.kind) {
          case kKindSmem: e.smem_row(d.row, rc); break;
          case kKindCta: e.cta_row(d.row, rc); break;
          case kKindGridPref: e.sample_item(d.row, rc); break;
          default: break;
        }
      } else if (d.fin) {
        e.fin_item(d.row, rc);
      }
      SideTeam::sync();
      if (SideTeam::tid() == 0) *reinterpret_cast<volatile uint32_t*>(&ctl->side_done) = i + 1;
    }
    if (SideTeam::tid() == 0) RADIK_TL(p, kTlSideDone);
  }
  __syncthreads();
  if (threadIdx.x == 0) RADIK_TL(p, kTlPhaseB);
  // phase B: the whole CTA, scratch in the side area
  Engine<VT, SCALE> e(p, smem, smem + kSideAreaOff, side_misc(smem));
  e.phase_b();
  if (threadIdx.x == 0) {
    RADIK_TL(p, kTlEnd);
    atomicMax(reinterpret_cast<unsigned long long*>(&p.hdr->t_last), globaltimer_ns());
  }
}

// ----------------------------------------------------------------------------
// Short-row kernel: calls whose rows are each selected by one team (smem
// rows, n <= 8192, or one-CTA rows, n <= cta_cap), of equal length or, with
// the planning kernel run first, of lengths known on the host.  No row needs the
// grid, so nothing streams through a ring and no CTA waits for another: four
// 256-thread teams per CTA each claim whole rows from the call's counter and
// select them with the side team's code, each in a side-sized area of its own.
// In the engine these rows run on the 7-warp side team alone.
// ----------------------------------------------------------------------------
constexpr int kRowTeams = 4;
constexpr int kRowTeamThreads = kThreads / kRowTeams;
constexpr int kRowMiscOff = kRowTeams * kSideAreaBytes;
constexpr int kShortSmemBytes = kRowMiscOff + kRowTeams * 3072;
static_assert(kShortSmemBytes <= 227 * 1024, "short-row kernel smem");

template <int VT, bool SCALE, int T>
__device__ __forceinline__ void row_team_loop(const EngineParams& p, uint8_t* smem) {
  using Tm = TeamT<T * kRowTeamThreads, kRowTeamThreads, 3 + T>;
  Misc* m = reinterpret_cast<Misc*>(smem + kRowMiscOff + T * 3072);
  Engine<VT, SCALE> e(p, smem, smem + T * kSideAreaBytes, m);
  for (;;) {
    if (Tm::tid() == 0) m->bcast = (int)atomicAdd(&p.hdr->qhead, 1u);
    Tm::sync();
    const int r = m->bcast;
    Tm::sync();
    if (r >= p.B) break;
    const RowCtx rc = load_row<VT, SCALE>(p, r);
    if (rc.kind == kKindSmem) e.template smem_row<Tm>(r, rc);
    else if (rc.kind == kKindCta) e.template cta_row<Tm>(r, rc);
    Tm::sync();
  }
}

template <int VT, bool SCALE>
__global__ void __launch_bounds__(kThreads, 1) short_rows_kernel(const __grid_constant__ EngineParams p) {
  extern __shared__ __align__(128) uint8_t smem[];
  if (!p.uniform && __ldcg(&p.hdr->plan_error)) return;
  if (threadIdx.x == 0)
    atomicCAS(reinterpret_cast<unsigned long long*>(&p.hdr->t_first), 0ull, globaltimer_ns());
  switch (threadIdx.x / kRowTeamThreads) {
    case 0: row_team_loop<VT, SCALE, 0>(p, smem); break;
    case 1: row_team_loop<VT, SCALE, 1>(p, smem); break;
    case 2: row_team_loop<VT, SCALE, 2>(p, smem); break;
    default: row_team_loop<VT, SCALE, 3>(p, smem); break;
  }
  __syncthreads();
  if (threadIdx.x == 0) atomicMax(reinterpret_cast<unsigned long long*>(&p.hdr->t_last), globaltimer_ns());
}

}  // namespace dev

template <int VT, bool SCALE>
inline cudaError_t launch_short_typed(const EngineParams& p, int grid, cudaStream_t stream) {
  auto kern = dev::short_rows_kernel<VT, SCALE>;
  static std::mutex attr_mu;
  static bool attr_set[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  {
    std::lock_guard<std::mutex> lock(attr_mu);
    if (dev < 0 || dev >= 64 || !attr_set[dev]) {
      e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, dev::kShortSmemBytes);
      if (e != cudaSuccess) return e;
      if (dev >= 0 && dev < 64) attr_set[dev] = true;
    }
  }
  kern<<<grid, kThreads, dev::kShortSmemBytes, stream>>>(p);
  return cudaGetLastError();
}

// coop = false launches the same grid without the cooperative attribute: for
// a grid below the device's, whose caller keeps the grids of concurrent
// launches within the SM count, so every CTA finds a free SM.
template <int VT, bool SCALE>
inline cudaError_t launch_typed(const EngineParams& p, int grid, cudaStream_t stream, bool coop = true) {
  auto kern = dev::engine_kernel<VT, SCALE>;
  // The smem opt-in is per device; remember which devices have it.  Callers
  // on several host threads (a serving worker beside the application) may
  // launch at once, so the table is guarded.
  static std::mutex attr_mu;
  static bool attr_set[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  {
    std::lock_guard<std::mutex> lock(attr_mu);
    if (dev < 0 || dev >= 64 || !attr_set[dev]) {
      e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
      if (e != cudaSuccess) return e;
      if (dev >= 0 && dev < 64) attr_set[dev] = true;
    }
  }
  // Cooperative launch: phase B synchronises the grid, so every CTA must be
  // resident (one per SM).
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = kSmemBytes;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = coop ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, p);
}

// Occupancy of one engine instantiation (CTAs per SM with its smem opt-in).
template <int VT, bool SCALE>
inline cudaError_t engine_occupancy(int* per_sm) {
  const void* fn = (const void*)dev::engine_kernel<VT, SCALE>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, fn, kThreads, kSmemBytes);
}

// Per value type entry points (one translation unit each).
cudaError_t launch_engine_f32(const EngineParams& p, int grid, cudaStream_t stream, bool coop);
cudaError_t launch_short_f32(const EngineParams& p, int grid, cudaStream_t stream);
cudaError_t launch_short_f16(const EngineParams& p, int grid, cudaStream_t stream);
cudaError_t launch_short_bf16(const EngineParams& p, int grid, cudaStream_t stream);
cudaError_t launch_engine_f16(const EngineParams& p, int grid, cudaStream_t stream, bool coop);
cudaError_t launch_engine_bf16(const EngineParams& p, int grid, cudaStream_t stream, bool coop);
cudaError_t occupancy_f32(uint32_t flags, int* per_sm);
cudaError_t occupancy_f16(uint32_t flags, int* per_sm);
cudaError_t occupancy_bf16(uint32_t flags, int* per_sm);

}  // namespace radik

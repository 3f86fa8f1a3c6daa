// radik_split.cu -- one row split over several GPUs (C ABI radik_shard_*).
//
// RadiK selects each row on one GPU (radik/RadixSelect/topk_radixselect.h).
// A row too long for one GPU, or one its caller spreads over its ranks, is
// held as contiguous shards: rank r's shard holds global positions
// [pos_base, pos_base + n).  Selection runs radix levels over the composite
// (selection key << ib | global position), ib the index bits of the whole
// row, so every rank orders keys exactly as a single GPU would and ties go
// to the lowest global positions.  Per level every rank histograms the next
// digit of the composites that match the current prefix
// (radik_shard_histogram); the caller sums the 4096 counters over its ranks
// (one all-reduce of 16 KB) and every rank picks the same bin; finally each
// rank compacts the keys whose composite prefix is below the final prefix
// (certainly selected) and those equal to it (the tie set, resolved after a
// gather) with radik_shard_collect.  Neither kernel waits on another rank:
// the exchanges are the caller's collectives between the launches.

#include "radik_engine.cuh"
#include "radik_b200.h"

#include <algorithm>

namespace radik {
namespace dev {

constexpr int kShardThreads = 512;
constexpr int kShardBins = 1 << kMaxD1;

template <int VT, bool SCALE>
__device__ __forceinline__ uint64_t shard_composite(const void* val_in, int64_t i, int64_t pos_base, int ib,
                                                    uint32_t flip, float scaler, uint32_t* bits_out) {
  uint32_t bits;
  if constexpr (VT == kF32) bits = __ldg(static_cast<const uint32_t*>(val_in) + i);
  else bits = (uint32_t)__ldg(static_cast<const unsigned short*>(val_in) + i);
  *bits_out = bits;
  return ((uint64_t)sel_key<VT, SCALE>(bits, flip, scaler) << ib) | (uint64_t)(pos_base + i);
}

// Histogram of digit [w - plen - d, w - plen) of the composites whose top
// plen bits equal prefix; hist (kShardBins counters) was cleared by the host.
template <int VT, bool SCALE>
__global__ void __launch_bounds__(kShardThreads) shard_hist_kernel(const void* val_in, int64_t n, int64_t pos_base,
                                                                   int ib, int w, uint64_t prefix, int plen, int d,
                                                                   uint32_t flip, float scaler, uint32_t* hist) {
  __shared__ uint32_t sh[kShardBins];
  const int nb = 1 << d;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const int s_hi = w - plen, s_lo = w - plen - d;
  const uint32_t dm = (uint32_t)nb - 1u;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  // every lane of a warp runs the same number of iterations (warp collectives)
  const int64_t span = (n + stride - 1) / stride * stride;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < span; i += stride) {
    bool match = false;
    uint32_t bin = 0;
    if (i < n) {
      uint32_t bits;
      const uint64_t c = shard_composite<VT, SCALE>(val_in, i, pos_base, ib, flip, scaler, &bits);
      match = shr64(c, s_hi) == prefix;
      bin = (uint32_t)shr64(c, s_lo) & dm;
    }
    hist_add_agg(sh, bin, match);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nb; i += blockDim.x)
    if (sh[i]) atomicAdd(hist + i, sh[i]);
}

// Compacts entries (value bits << 32 | global position) of the composites
// whose top plen bits are below prefix into better[] and equal to it into
// tied[]; counts[0] / counts[1] receive how many there were (entries past a
// capacity are counted but not stored).
template <int VT, bool SCALE>
__global__ void __launch_bounds__(kShardThreads) shard_collect_kernel(const void* val_in, int64_t n,
                                                                      int64_t pos_base, int ib, int w, uint64_t prefix,
                                                                      int plen, uint32_t flip, float scaler,
                                                                      uint64_t* better, int cap_better,
                                                                      uint64_t* tied, int cap_tied, uint32_t* counts) {
  const int s_hi = w - plen;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t span = (n + stride - 1) / stride * stride;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < span; i += stride) {
    bool to_b = false, to_t = false;
    uint32_t bits = 0;
    if (i < n) {
      const uint64_t c = shard_composite<VT, SCALE>(val_in, i, pos_base, ib, flip, scaler, &bits);
      const uint64_t t = shr64(c, s_hi);
      to_b = t < prefix;
      to_t = t == prefix;
    }
    if (!__any_sync(kFull, to_b || to_t)) continue;
    const uint64_t e = ((uint64_t)bits << 32) | (uint64_t)(uint32_t)(pos_base + i);
    const uint32_t sb = warp_reserve(to_b ? 1u : 0u, counts);
    if (to_b && sb < (uint32_t)cap_better) better[sb] = e;
    const uint32_t st = warp_reserve(to_t ? 1u : 0u, counts + 1);
    if (to_t && st < (uint32_t)cap_tied) tied[st] = e;
  }
}

}  // namespace dev

namespace {

int shard_grid(int64_t n) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (n + 4LL * dev::kShardThreads - 1) / (4LL * dev::kShardThreads);
  return (int)std::max<int64_t>(1, std::min<int64_t>(want, 4LL * sms));
}

bool shard_args_ok(int dtype, uint32_t flags, const void* val_in, int64_t n, int64_t pos_base, int ib) {
  if (dtype != kF32 && dtype != kF16 && dtype != kBF16) return false;
  if (flags & ~(uint32_t)(kFlagLargest | kFlagWithScale)) return false;
  if (n < 0 || pos_base < 0 || ib < 1 || ib > 32 || (n > 0 && !val_in)) return false;
  if (pos_base + n > ((int64_t)1 << ib)) return false;  // positions must fit in ib bits
  return true;
}

}  // namespace
}  // namespace radik

using namespace radik;

extern "C" {

int radik_shard_histogram(int dtype, uint32_t flags, const void* val_in, int64_t n, int64_t pos_base, int ib,
                          uint64_t prefix, int plen, int digit_bits, float scaler, uint32_t* hist, void* stream_) {
  if (!shard_args_ok(dtype, flags, val_in, n, pos_base, ib) || !hist) return RADIK_EINVAL;
  const int w = key_bits(dtype, flags) + ib;
  if (plen < 0 || digit_bits < 1 || digit_bits > kMaxD1 || plen + digit_bits > w) return RADIK_EINVAL;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  cudaError_t e = cudaMemsetAsync(hist, 0, sizeof(uint32_t) * dev::kShardBins, stream);
  if (e != cudaSuccess) return RADIK_ECUDA;
  if (n == 0) return RADIK_OK;
  const uint32_t flip = (flags & kFlagLargest) ? (key_bits(dtype, flags) == 32 ? 0xFFFFFFFFu : 0xFFFFu) : 0u;
  const int grid = shard_grid(n);
  const bool scale = (flags & kFlagWithScale) != 0;
#define RADIK_SHARD_HIST(VT, SC)                                                                              \
  dev::shard_hist_kernel<VT, SC><<<grid, dev::kShardThreads, 0, stream>>>(val_in, n, pos_base, ib, w, prefix, \
                                                                          plen, digit_bits, flip, scaler, hist)
  if (dtype == kF32) {
    if (scale) RADIK_SHARD_HIST(kF32, true);
    else RADIK_SHARD_HIST(kF32, false);
  } else if (dtype == kF16) {
    if (scale) RADIK_SHARD_HIST(kF16, true);
    else RADIK_SHARD_HIST(kF16, false);
  } else {
    if (scale) RADIK_SHARD_HIST(kBF16, true);
    else RADIK_SHARD_HIST(kBF16, false);
  }
#undef RADIK_SHARD_HIST
  return cudaGetLastError() == cudaSuccess ? RADIK_OK : RADIK_ECUDA;
}

int radik_shard_collect(int dtype, uint32_t flags, const void* val_in, int64_t n, int64_t pos_base, int ib,
                        uint64_t prefix, int plen, float scaler, uint64_t* better, int cap_better, uint64_t* tied,
                        int cap_tied, uint32_t* counts, void* stream_) {
  if (!shard_args_ok(dtype, flags, val_in, n, pos_base, ib) || !counts || cap_better < 0 || cap_tied < 0 ||
      (cap_better > 0 && !better) || (cap_tied > 0 && !tied))
    return RADIK_EINVAL;
  const int w = key_bits(dtype, flags) + ib;
  if (plen < 0 || plen > w) return RADIK_EINVAL;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  cudaError_t e = cudaMemsetAsync(counts, 0, 2 * sizeof(uint32_t), stream);
  if (e != cudaSuccess) return RADIK_ECUDA;
  if (n == 0) return RADIK_OK;
  const uint32_t flip = (flags & kFlagLargest) ? (key_bits(dtype, flags) == 32 ? 0xFFFFFFFFu : 0xFFFFu) : 0u;
  const int grid = shard_grid(n);
  const bool scale = (flags & kFlagWithScale) != 0;
#define RADIK_SHARD_COLLECT(VT, SC)                                                                       \
  dev::shard_collect_kernel<VT, SC><<<grid, dev::kShardThreads, 0, stream>>>(                             \
      val_in, n, pos_base, ib, w, prefix, plen, flip, scaler, better, cap_better, tied, cap_tied, counts)
  if (dtype == kF32) {
    if (scale) RADIK_SHARD_COLLECT(kF32, true);
    else RADIK_SHARD_COLLECT(kF32, false);
  } else if (dtype == kF16) {
    if (scale) RADIK_SHARD_COLLECT(kF16, true);
    else RADIK_SHARD_COLLECT(kF16, false);
  } else {
    if (scale) RADIK_SHARD_COLLECT(kBF16, true);
    else RADIK_SHARD_COLLECT(kBF16, false);
  }
#undef RADIK_SHARD_COLLECT
  return cudaGetLastError() == cudaSuccess ? RADIK_OK : RADIK_ECUDA;
}

}  // extern "C"

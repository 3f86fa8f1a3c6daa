// radik_plan.cu -- planning kernel of the uneven batched form and the
// dtype dispatch of the engine launch.
#include "radik_engine.cuh"

namespace radik {
namespace dev {

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
    int64_t w = lane < kWarps ? scan[lane] : 0;
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

// Plans a batch: per row its kind, A items (a0) and B block (b0), candidate
// and sort-scratch regions, histogram-ring ordinal; the A and B item -> row
// maps (a B entry with the top bit set is the row's FIN item, placed at the
// end of the block of row r + D, or in a tail after the last block); and
// the claim-order lag that keeps every B item after its row's A items.
__global__ void __launch_bounds__(kThreads, 1)
    plan_kernel(const RowDesc* desc, int B, int CH, int CHR, int cta_cap, int D, uint32_t flags, RowPlan* plans,
                int32_t* a_row, int32_t* b_row, Header* hdr, int64_t na_cap, int64_t nb_cap, int64_t cand_cap_total,
                int64_t sort_cap_total, int grid) {
  __shared__ int64_t scan[32];
  __shared__ int64_t run[5];
  __shared__ long long maxlag;
  __shared__ int has_radix;
  if (threadIdx.x < 5) run[threadIdx.x] = 0;
  if (threadIdx.x == 0) {
    maxlag = 0;
    has_radix = 0;
  }
  __syncthreads();
  const bool sorted = (flags & kFlagSorted) != 0;
  auto kind_of = [&](int r) {
    const RowDesc d = desc[r];
    return row_kind(d.n < 0 ? 0 : d.n, d.k, cta_cap);
  };
  for (int base = 0; base < B; base += kThreads) {
    const int r = base + threadIdx.x;
    int64_t na = 0, blk = 0, cand = 0, sortn = 0, hist = 0;
    RowDesc d{0, 0, 0, 0};
    int kind = kKindEmpty;
    if (r < B) {
      d = desc[r];
      if (d.n < 0) d.n = 0;
      kind = row_kind(d.n, d.k, cta_cap);
      na = row_na(kind, d.n, CH, CHR);
      blk = row_nbc(kind, d.n, CH, CHR) + ((r >= D) ? row_fin(kind_of(r - D)) : 0);
      cand = row_cand_cap(kind, d.n);
      hist = row_uses_hist(kind);
      if (kind == kKindGridRadix) has_radix = 1;
      const int64_t kk = min((int64_t)d.n, (int64_t)d.k);
      sortn = (sorted && kk > kCapSort) ? 2 * kk : 0;
    }
    int64_t t0, t1, t2, t3, t4;
    const int64_t e0 = block_excl_scan64(na, scan, &t0);
    const int64_t e1 = block_excl_scan64(blk, scan, &t1);
    const int64_t e2 = block_excl_scan64(cand, scan, &t2);
    const int64_t e3 = block_excl_scan64(sortn, scan, &t3);
    const int64_t e4 = block_excl_scan64(hist, scan, &t4);
    if (r < B) {
      RowPlan pl;
      pl.in_off = d.in_off;
      pl.out_off = d.out_off;
      pl.cand_off = run[2] + e2;
      pl.sort_off = sortn ? run[3] + e3 : -1;
      pl.n = d.n;
      pl.k = d.k;
      pl.a0 = (int32_t)(run[0] + e0);
      pl.b0 = (int32_t)(run[1] + e1);
      pl.cand_cap = (int32_t)cand;
      pl.slot_use = hist ? (int32_t)(run[4] + e4) : -1;
      pl.pad0 = pl.pad1 = 0;
      plans[r] = pl;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      run[0] += t0;
      run[1] += t1;
      run[2] += t2;
      run[3] += t3;
      run[4] += t4;
    }
    __syncthreads();
  }
  // FIN items of the last min(D, B) rows form the tail of the B sequence
  const int Dd = D < B ? D : B;
  int64_t tail = 0;
  for (int r = B - Dd; r < B; ++r) tail += row_fin(kind_of(r)) ? 1 : 0;  // same value in every thread
  const int64_t nb_total = run[1] + tail;
  const bool ok = run[0] <= na_cap && nb_total <= nb_cap && run[2] <= cand_cap_total && run[3] <= sort_cap_total &&
                  run[0] + nb_total < (1ll << 30);
  if (threadIdx.x == 0) {
    hdr->na = (int32_t)run[0];
    hdr->nb = (int32_t)nb_total;
    hdr->fin_tail = (int32_t)tail;
    hdr->cand_total = run[2];
    hdr->sort_total = run[3];
    hdr->plan_error = ok ? 0 : 1;
    if (!ok) atomicOr(&hdr->status, kStatusCapacity);
  }
  if (!ok) return;
  __syncthreads();
  // item -> row maps, one warp per row; FIN positions and the lag
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t tail_base = run[1];
  for (int r = warp; r < B; r += kWarps) {
    const RowPlan& pl = plans[r];
    const int kind = row_kind(pl.n, pl.k, cta_cap);
    const int32_t na = row_na(kind, pl.n, CH, CHR), nbc = row_nbc(kind, pl.n, CH, CHR);
    for (int c = lane; c < na; c += 32) a_row[pl.a0 + c] = r;
    for (int c = lane; c < nbc; c += 32) b_row[pl.b0 + c] = r;
    if (lane == 0) {
      int64_t first_b = nbc > 0 ? pl.b0 : -1;
      if (row_fin(kind)) {
        int64_t pos;
        if (r + D < B) {
          const RowPlan& q = plans[r + D];
          pos = q.b0 + row_nbc(row_kind(q.n, q.k, cta_cap), q.n, CH, CHR);
        } else {
          int64_t t = 0;  // FIN items of rows B-Dd .. r-1
          for (int x = B - Dd; x < r; ++x) t += row_fin(kind_of(x)) ? 1 : 0;
          pos = tail_base + t;
        }
        b_row[pos] = (int32_t)((uint32_t)r | 0x80000000u);
        if (first_b < 0) first_b = pos;
      }
      if (first_b >= 0) atomicMax(&maxlag, (long long)(pl.a0 + na - first_b));
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // see lag_floor() on the host side
    const long long floor_ = has_radix ? 2LL * grid : (long long)max(2, grid / 4);
    hdr->lag = (int32_t)max(floor_, maxlag + 1);
  }
}

}  // namespace dev

cudaError_t launch_short_rows(int dtype, const EngineParams& p, int grid, cudaStream_t stream) {
  switch (dtype) {
    case kF32: return launch_short_f32(p, grid, stream);
    case kF16: return launch_short_f16(p, grid, stream);
    case kBF16: return launch_short_bf16(p, grid, stream);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_engine(int dtype, const EngineParams& p, int grid, cudaStream_t stream, bool coop) {
  switch (dtype) {
    case kF32: return launch_engine_f32(p, grid, stream, coop);
    case kF16: return launch_engine_f16(p, grid, stream, coop);
    case kBF16: return launch_engine_bf16(p, grid, stream, coop);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_plan(const RowDesc* desc, int B, int CH, int CHR, int cta_cap, int D, uint32_t flags,
                        RowPlan* plans, int32_t* a_row, int32_t* b_row, Header* hdr, int64_t na_cap, int64_t nb_cap,
                        int64_t cand_cap_total, int64_t sort_cap_total, int grid, cudaStream_t stream) {
  dev::plan_kernel<<<1, kThreads, 0, stream>>>(desc, B, CH, CHR, cta_cap, D, flags, plans, a_row, b_row, hdr, na_cap,
                                               nb_cap, cand_cap_total, sort_cap_total, grid);
  return cudaGetLastError();
}

// Largest grid the engine can be launched with cooperatively: one CTA per SM
// when one fits.
cudaError_t engine_max_grid(int dtype, uint32_t flags, int* grid) {
  int dev = 0, sms = 0, per = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  switch (dtype) {
    case kF32: e = occupancy_f32(flags, &per); break;
    case kF16: e = occupancy_f16(flags, &per); break;
    default: e = occupancy_bf16(flags, &per); break;
  }
  if (e != cudaSuccess) return e;
  *grid = sms * (per < kCtasPerSM ? per : kCtasPerSM);
  return cudaSuccess;
}

}  // namespace radik

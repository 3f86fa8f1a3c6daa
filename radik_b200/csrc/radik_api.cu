// radik_api.cu -- host side of the C ABI declared in include/radik_b200.h.
//
// Each call: validate, lay out the caller's workspace, clear the per-call
// state with one cudaMemsetAsync, and launch the selection engine (plus the
// one-CTA planning kernel when the rows are not uniform).  No host
// synchronisation, unlike RadiK's two cudaStreamSynchronize per call
// (radik/RadixSelect/topk_radixselect.h:157,195).

#include "radik_common.cuh"
#include "radik_b200.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace radik {

cudaError_t launch_engine(int dtype, const EngineParams& p, int grid, cudaStream_t stream);
cudaError_t launch_plan(const RowDesc* desc, int B, int CH, int CHR, int D, uint32_t flags, RowPlan* plans, int32_t* a_row,
                        int32_t* b_row, Header* hdr, int64_t na_cap, int64_t nb_cap, int64_t cand_cap_total,
                        int64_t sort_cap_total, int grid, cudaStream_t stream);
cudaError_t engine_max_grid(int dtype, uint32_t flags, int* grid);

namespace {

constexpr uint32_t kKnownFlags = kFlagLargest | kFlagSorted | kFlagAscend | kFlagWithScale | kFlagWithIdxIn | kFlagIdx64;
constexpr int kSlots = 64;             // level-1 histogram ring slots
constexpr int kMinCH = 4096;           // chunk length bounds (elements)
constexpr int kMaxCH = 1 << 18;
constexpr uint32_t kSpinLimit = 1u << 23;

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  return fail(RADIK_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Cooperative grid of the engine on the current device (one CTA per SM).
int engine_grid(int dtype, uint32_t flags, int* grid) {
  static std::mutex mu;
  static int cache[64][2] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  const int key = (flags & kFlagWithScale) ? 1 : 0;
  std::lock_guard<std::mutex> lock(mu);
  if (dev >= 0 && dev < 64 && cache[dev][key] > 0) {
    *grid = cache[dev][key];
    return RADIK_OK;
  }
  int g = 0;
  e = engine_max_grid(dtype, flags, &g);
  if (e != cudaSuccess) return cuda_fail(e, "engine occupancy");
  if (g <= 0) return fail(RADIK_ECUDA, "radik: the engine does not fit on this device");
  if (dev >= 0 && dev < 64) cache[dev][key] = g;
  *grid = g;
  return RADIK_OK;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

struct Layout {
  size_t hdr, rs, slot_gen, hist, zero_end;
  size_t plans, a_row, b_row, large, descs, pb_sb, cand, sort, total;
};

Layout make_layout(int64_t B, int64_t na_cap, int64_t nb_cap, int64_t cand_cap, int64_t sort_cap) {
  Layout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += align256(bytes);
    return o;
  };
  L.hdr = take(sizeof(Header));
  L.rs = take((size_t)B * sizeof(RowState));
  L.slot_gen = take((size_t)kSlots * 4);
  L.hist = take((size_t)kSlots * ((size_t)1 << kMaxD1) * 4);
  L.zero_end = off;
  L.plans = take((size_t)B * sizeof(RowPlan));
  L.a_row = take((size_t)na_cap * 4);
  L.b_row = take((size_t)nb_cap * 4);
  L.large = take((size_t)B * 4);
  L.descs = take((size_t)B * sizeof(RowDesc));
  L.pb_sb = take((size_t)kPhaseBSlots * kCapSB * 8);
  L.cand = take((size_t)cand_cap * 8);
  L.sort = take((size_t)sort_cap * 8);
  L.total = off;
  return L;
}

struct Bounds {
  int64_t na, nb, cand, sort;
};

int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

Bounds bounds_uniform(int64_t B, int64_t n_max, int64_t K, uint32_t flags) {
  Bounds b{};
  const int64_t nch = std::max<int64_t>(1, ceil_div(n_max, kMinCH));
  b.na = B * nch;
  b.nb = B * (nch + 1);
  b.cand = n_max > kCtaRowCap ? B * (int64_t)cand_capacity((int32_t)n_max) : 0;
  const int64_t kk = std::min(n_max, K);
  b.sort = ((flags & kFlagSorted) && kk > kCapSort) ? B * 2 * kk : 0;
  return b;
}

Bounds bounds_rows(int64_t B, int64_t total_n, int64_t n_max, int64_t k_max, uint32_t flags) {
  Bounds b{};
  b.na = total_n / kMinCH + B;
  b.nb = total_n / kMinCH + 2 * B;
  b.cand = std::min(total_n, B * (int64_t)kCapSB) + total_n / 8 + B;
  const int64_t kk = std::min(n_max, k_max);
  b.sort = ((flags & kFlagSorted) && kk > kCapSort) ? 2 * std::min(total_n, B * k_max) : 0;
  return b;
}

int env_int(const char* name, int dflt) {
  const char* v = std::getenv(name);
  if (!v || !*v) return dflt;
  return std::atoi(v);
}

// Tunables: chunk lengths and first-digit width.  Single-read rows use
// chunks of 4K..256K elements, aiming at about eight chunks per CTA so the
// work queue balances (the last chunks bound the tail) while each chunk
// streams long enough to amortise its item overhead; radik_autotune can
// replace that choice per shape bucket.  Radix rows use 32K-element chunks:
// their filter items re-read chunks that the histogram items read two grids
// earlier, and that window (2 x 148 x 128 KB) must stay in L2.  The 12-bit
// first digit (4096 bins, 16 KB of smem) leaves about n/4096 keys of an
// i.i.d. row in the selected bin.  RADIK_CH / RADIK_CHR / RADIK_D1 override
// everything (tuning sweeps).
struct Config {
  int CH, CHR, D1;
};

// Autotuned chunk lengths, per shape bucket (radik_autotune).
std::mutex g_tune_mu;
std::map<uint64_t, int> g_tuned_ch;

int ilog2(int64_t v) {
  int l = 0;
  while (v > 1) {
    v >>= 1;
    ++l;
  }
  return l;
}

// Shape bucket of a call: dtype, form (uniform / rows), sorted, and the log2
// of the row count, the longest row and k.
uint64_t shape_bucket(int dtype, uint32_t flags, bool rows_form, int64_t B, int64_t n_max, int64_t K) {
  return (uint64_t)dtype | ((uint64_t)rows_form << 2) | ((uint64_t)((flags & kFlagSorted) != 0) << 3) |
         ((uint64_t)ilog2(std::max<int64_t>(B, 1)) << 4) | ((uint64_t)ilog2(std::max<int64_t>(n_max, 1)) << 12) |
         ((uint64_t)ilog2(std::max<int64_t>(K, 1)) << 20);
}

int tuned_ch(uint64_t bucket) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  const auto it = g_tuned_ch.find(bucket);
  return it == g_tuned_ch.end() ? 0 : it->second;
}

Config choose_config(int64_t stream_elems, int grid, uint64_t bucket) {
  Config c{};
  const int64_t target = std::max<int64_t>(1, stream_elems / ((int64_t)grid * 8));
  int ch = kMinCH;
  while (ch < kMaxCH && ch * 2 <= target) ch *= 2;
  // Few large rows (2^24 keys or more in all): per-item overhead outweighs
  // balance, so no chunk is shorter than 128K keys (single 2^24-key rows:
  // 154 -> 111 us from 8K to 128K chunks).
  if (stream_elems >= ((int64_t)1 << 24)) ch = std::max(ch, 1 << 17);
  const int tc = tuned_ch(bucket);
  c.CH = tc ? tc : ch;
  c.CHR = 32768;
  c.D1 = kMaxD1;
  const int ech = env_int("RADIK_CH", 0);
  if (ech >= kMinCH && ech <= (1 << 24) && (ech % 16) == 0) c.CH = ech;
  const int echr = env_int("RADIK_CHR", 0);
  if (echr >= kMinCH && echr <= (1 << 24) && (echr % 16) == 0) c.CHR = echr;
  const int ed1 = env_int("RADIK_D1", 0);
  if (ed1 >= kMinD1 && ed1 <= kMaxD1) c.D1 = ed1;
  return c;
}

int check_common(int dtype, uint32_t flags, const void* val_in, const void* idx_in, void* val_out, void* idx_out,
                 void* ws) {
  if (dtype != kF32 && dtype != kF16 && dtype != kBF16) return fail(RADIK_EINVAL, "radik: unknown dtype");
  if (flags & ~kKnownFlags) return fail(RADIK_EINVAL, "radik: unknown flag bits");
  if (!val_in || !val_out || !idx_out) return fail(RADIK_EINVAL, "radik: null input/output pointer");
  if ((flags & kFlagWithIdxIn) && !idx_in) return fail(RADIK_EINVAL, "radik: RADIK_WITHIDXIN needs idx_in");
  if (!ws) return fail(RADIK_EWORKSPACE, "radik: workspace should not be null");
  if ((reinterpret_cast<uintptr_t>(ws) & 255u) != 0) return fail(RADIK_EWORKSPACE, "radik: workspace must be 256-byte aligned");
  const uintptr_t es = (uintptr_t)elem_bytes(dtype);
  if ((reinterpret_cast<uintptr_t>(val_in) % es) || (reinterpret_cast<uintptr_t>(val_out) % es))
    return fail(RADIK_EINVAL, "radik: value pointers must be aligned to the element size");
  return RADIK_OK;
}

EngineParams base_params(const void* val_in, const void* idx_in, void* val_out, void* idx_out, uint8_t* ws,
                         const Layout& L, int B, const Config& c, uint32_t flags) {
  EngineParams p{};
  p.val_in = val_in;
  p.idx_in = idx_in;
  p.val_out = val_out;
  p.idx_out = idx_out;
  p.rs = reinterpret_cast<RowState*>(ws + L.rs);
  p.hist_ring = reinterpret_cast<uint32_t*>(ws + L.hist);
  p.slot_gen = reinterpret_cast<uint32_t*>(ws + L.slot_gen);
  p.hdr = reinterpret_cast<Header*>(ws + L.hdr);
  p.large_list = reinterpret_cast<int32_t*>(ws + L.large);
  p.cand = reinterpret_cast<uint64_t*>(ws + L.cand);
  p.sort_scratch = reinterpret_cast<uint64_t*>(ws + L.sort);
  p.pb_sb = reinterpret_cast<uint64_t*>(ws + L.pb_sb);
  p.B = B;
  p.CH = c.CH;
  p.CHR = c.CHR;
  p.D1 = c.D1;
  p.S = kSlots;
  p.flags = flags;
  p.spin_limit = kSpinLimit;
  return p;
}

// Bytes cleared before a call: the header, row states and ring release
// counters always; the histogram ring only when radix rows may use it in
// phase A (phase B clears the slots it uses).
size_t zero_bytes(const Layout& L, bool with_hist) { return with_hist ? L.zero_end : L.hist; }

// How far A items run ahead of B items beyond what correctness needs.
// Radix rows re-read their chunks in B items, so their A items run two grids
// ahead and the re-reads hit L2.  Pre-filter rows read their chunks once and
// only need their sample item done, so a short lead suffices for fp32; 16-bit
// rows stream twice the keys per byte, so their start weighs more: there a
// full grid of samples leads and every CTA opens with a whole-CTA sample
// (fp16 256 x 2^20, k = 256: +2.4 %; neutral for fp32).
int64_t lag_floor(bool has_radix, int grid, int dtype) {
  if (has_radix) return 2 * (int64_t)grid;
  return dtype == kF32 ? std::max(2, grid / 4) : (int64_t)grid;
}

// Rows a FIN item trails its row in the B sequence: about one and a half
// grids of chunk items for uniform rows (their chunks are done by then); a
// fixed 64 rows for planned batches.
constexpr int kFinDelayRows = 64;
int fin_delay_uniform(int nc, int grid) { return std::max(1, (3 * grid + 2 * std::max(nc, 1) - 1) / (2 * std::max(nc, 1))); }

// Workspace of radik_topk_static(): static device memory of this module, one
// copy per device the module is loaded on.
static __device__ __align__(256) unsigned char g_static_scratch[RADIK_STATIC_SCRATCH_BYTES];

}  // namespace
}  // namespace radik

using namespace radik;

extern "C" {

int radik_version(void) { return 100; }

const char* radik_last_error(void) { return g_last_error.c_str(); }

const char* radik_strerror(int status) {
  switch (status) {
    case RADIK_OK: return "success";
    case RADIK_EINVAL: return "invalid argument";
    case RADIK_EWORKSPACE: return "workspace null or too small";
    case RADIK_ECUDA: return "CUDA runtime error";
    case RADIK_ETIMEOUT: return "a bounded device wait timed out";
    case RADIK_EINTERNAL: return "internal selection error";
    case RADIK_ENOTSUP: return "unsupported combination";
    default: return "unknown status";
  }
}

int radik_get_workspace_size(int dtype, uint32_t flags, int K, int n_max, int task_num, size_t* bytes) {
  if (!bytes) return fail(RADIK_EINVAL, "radik: bytes is null");
  if (dtype != kF32 && dtype != kF16 && dtype != kBF16) return fail(RADIK_EINVAL, "radik: unknown dtype");
  if (K < 0 || n_max < 0 || task_num < 0) return fail(RADIK_EINVAL, "radik: negative size");
  const Bounds b = bounds_uniform(std::max(task_num, 1), n_max, K, flags);
  *bytes = make_layout(std::max(task_num, 1), b.na, b.nb, b.cand, b.sort).total;
  return RADIK_OK;
}

int radik_get_workspace_size_rows(int dtype, uint32_t flags, int task_num, int64_t total_n, int n_max, int k_max,
                                  size_t* bytes) {
  if (!bytes) return fail(RADIK_EINVAL, "radik: bytes is null");
  if (dtype != kF32 && dtype != kF16 && dtype != kBF16) return fail(RADIK_EINVAL, "radik: unknown dtype");
  if (task_num < 0 || total_n < 0 || n_max < 0 || k_max < 0) return fail(RADIK_EINVAL, "radik: negative size");
  const Bounds b = bounds_rows(std::max(task_num, 1), total_n, n_max, k_max, flags);
  *bytes = make_layout(std::max(task_num, 1), b.na, b.nb, b.cand, b.sort).total;
  return RADIK_OK;
}

int radik_topk(int dtype, uint32_t flags, const void* val_in, const void* idx_in, void* val_out, void* idx_out,
               void* workspace, size_t workspace_bytes, const int* task_len, int task_num, int K, void* stream_) {
  int rc = check_common(dtype, flags, val_in, idx_in, val_out, idx_out, workspace);
  if (rc) return rc;
  if (task_num < 0 || K < 0) return fail(RADIK_EINVAL, "radik: negative task_num or K");
  if (task_num == 0 || K == 0) return RADIK_OK;
  if (!task_len) return fail(RADIK_EINVAL, "radik: task_len is null");
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  const int B = task_num;
  bool uniform = true;
  int64_t multi_elems = 0;
  for (int i = 0; i < B; ++i) {
    const int n = task_len[i];
    if (n < 0) return fail(RADIK_EINVAL, "radik: negative task length");
    uniform = uniform && n == task_len[0];
    const int kind = row_kind(n, K);
    if (kind == kKindAll || kind == kKindGridPref || kind == kKindGridRadix) multi_elems += n;
  }
  if ((int64_t)B * K > ((int64_t)1 << 40)) return fail(RADIK_EINVAL, "radik: output too large");
  int grid = 0;
  rc = engine_grid(dtype, flags, &grid);
  if (rc) return rc;
  int n_max_call = 0;
  for (int i = 0; i < B; ++i) n_max_call = std::max(n_max_call, task_len[i]);
  const Config cfg = choose_config(multi_elems, grid, shape_bucket(dtype, flags, false, B, n_max_call, K));
  // exact needs of this call
  int64_t na = 0, nb = 0, cand = 0, sortn = 0;
  bool has_radix = false;
  for (int i = 0; i < B; ++i) {
    const int n = task_len[i];
    const int kind = row_kind(n, K);
    has_radix = has_radix || kind == kKindGridRadix;
    na += row_na(kind, n, cfg.CH, cfg.CHR);
    nb += row_nbc(kind, n, cfg.CH, cfg.CHR) + row_fin(kind);
    cand += row_cand_cap(kind, n);
    const int64_t kk = std::min<int64_t>(n, K);
    if ((flags & kFlagSorted) && kk > kCapSort) sortn += 2 * kk;
  }
  if (na + nb >= ((int64_t)1 << 30)) return fail(RADIK_EINVAL, "radik: too many work items");
  const Layout L = make_layout(B, na, nb, cand, sortn);
  if (workspace_bytes < L.total) return fail(RADIK_EWORKSPACE, "radik: workspace too small");
  uint8_t* ws = static_cast<uint8_t*>(workspace);
  cudaError_t e = cudaMemsetAsync(ws, 0, zero_bytes(L, has_radix), stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
  EngineParams p = base_params(val_in, idx_in, val_out, idx_out, ws, L, B, cfg, flags);
  if (uniform) {
    const int n = task_len[0];
    const int kind = row_kind(n, K);
    p.uniform = 1;
    p.u_n = n;
    p.u_k = K;
    p.u_cand_cap = row_cand_cap(kind, n);
    const int64_t kk = std::min<int64_t>(n, K);
    p.u_sort_cap = ((flags & kFlagSorted) && kk > kCapSort) ? 2 * kk : 0;
    // B sequence layout (see uniform_b_item) and the lag it needs
    const int64_t una = row_na(kind, n, cfg.CH, cfg.CHR), nc = row_nbc(kind, n, cfg.CH, cfg.CHR);
    const int64_t f = row_fin(kind);
    const int D = fin_delay_uniform((int)nc, grid);
    const int64_t Dd = std::min<int64_t>(D, B);
    auto b0 = [&](int64_t q) { return q < Dd ? q * nc : Dd * nc + (q - Dd) * (nc + f); };
    int64_t maxlag = 0;
    for (int64_t r = 0; r < B && (nc > 0 || f); ++r) {
      int64_t first_b;
      if (nc > 0) first_b = b0(r);
      else first_b = (r + Dd < B) ? b0(r + Dd) + nc : (int64_t)B * nc + f * (B - Dd) + (r - (B - Dd));
      maxlag = std::max(maxlag, (r + 1) * una - first_b);
    }
    p.fin_delay = D;
    p.lag = (int32_t)std::max<int64_t>(maxlag + 1, lag_floor(has_radix, grid, dtype));
  } else {
    std::vector<RowDesc> d(B);
    int64_t off = 0;
    for (int i = 0; i < B; ++i) {
      d[i].in_off = off;
      d[i].out_off = (int64_t)i * K;
      d[i].n = task_len[i];
      d[i].k = K;
      off += task_len[i];
    }
    RowDesc* dd = reinterpret_cast<RowDesc*>(ws + L.descs);
    e = cudaMemcpyAsync(dd, d.data(), sizeof(RowDesc) * B, cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync");
    p.plans = reinterpret_cast<RowPlan*>(ws + L.plans);
    p.a_row = reinterpret_cast<int32_t*>(ws + L.a_row);
    p.b_row = reinterpret_cast<int32_t*>(ws + L.b_row);
    e = launch_plan(dd, B, cfg.CH, cfg.CHR, kFinDelayRows, flags, reinterpret_cast<RowPlan*>(ws + L.plans), reinterpret_cast<int32_t*>(ws + L.a_row),
                    reinterpret_cast<int32_t*>(ws + L.b_row), p.hdr, na, nb, cand, sortn, grid, stream);
    if (e != cudaSuccess) return cuda_fail(e, "plan launch");
  }
  e = launch_engine(dtype, p, grid, stream);
  if (e != cudaSuccess) return cuda_fail(e, "engine launch");
  return RADIK_OK;
}

int radik_topk_rows(int dtype, uint32_t flags, const void* val_in, const void* idx_in, void* val_out,
                    void* idx_out, void* workspace, size_t workspace_bytes, const radik_row_desc* rows,
                    int task_num, int64_t total_n, int n_max, int k_max, void* stream_) {
  int rc = check_common(dtype, flags, val_in, idx_in, val_out, idx_out, workspace);
  if (rc) return rc;
  if (task_num < 0 || total_n < 0 || n_max < 0 || k_max < 0) return fail(RADIK_EINVAL, "radik: negative size");
  if (task_num == 0) return RADIK_OK;
  if (!rows) return fail(RADIK_EINVAL, "radik: rows is null");
  static_assert(sizeof(radik_row_desc) == sizeof(RowDesc), "descriptor layout");
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  const int B = task_num;
  const Bounds b = bounds_rows(B, total_n, n_max, k_max, flags);
  if (b.na + b.nb >= ((int64_t)1 << 30)) return fail(RADIK_EINVAL, "radik: too many work items");
  const Layout L = make_layout(B, b.na, b.nb, b.cand, b.sort);
  if (workspace_bytes < L.total) return fail(RADIK_EWORKSPACE, "radik: workspace too small");
  int grid = 0;
  rc = engine_grid(dtype, flags, &grid);
  if (rc) return rc;
  const Config cfg = choose_config(total_n, grid, shape_bucket(dtype, flags, true, B, n_max, k_max));
  uint8_t* ws = static_cast<uint8_t*>(workspace);
  cudaError_t e = cudaMemsetAsync(ws, 0, zero_bytes(L, true), stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
  EngineParams p = base_params(val_in, idx_in, val_out, idx_out, ws, L, B, cfg, flags);
  p.plans = reinterpret_cast<RowPlan*>(ws + L.plans);
  p.a_row = reinterpret_cast<int32_t*>(ws + L.a_row);
  p.b_row = reinterpret_cast<int32_t*>(ws + L.b_row);
  // The item budget assumed kMinCH-long chunks; with the chosen CH the true
  // count is smaller, so the bound still holds.
  e = launch_plan(reinterpret_cast<const RowDesc*>(rows), B, cfg.CH, cfg.CHR, kFinDelayRows, flags, reinterpret_cast<RowPlan*>(ws + L.plans),
                  reinterpret_cast<int32_t*>(ws + L.a_row), reinterpret_cast<int32_t*>(ws + L.b_row), p.hdr, b.na, b.nb,
                  b.cand, b.sort, grid, stream);
  if (e != cudaSuccess) return cuda_fail(e, "plan launch");
  e = launch_engine(dtype, p, grid, stream);
  if (e != cudaSuccess) return cuda_fail(e, "engine launch");
  return RADIK_OK;
}

int radik_get_status(void* workspace, void* stream_, int* device_bits) {
  if (!workspace) return fail(RADIK_EWORKSPACE, "radik: workspace should not be null");
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  cudaError_t e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
  int32_t bits = 0;
  e = cudaMemcpy(&bits, static_cast<uint8_t*>(workspace) + offsetof(Header, status), sizeof(bits),
                 cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy status");
  if (device_bits) *device_bits = bits;
  if (bits & kStatusCapacity) return fail(RADIK_EWORKSPACE, "radik: rows exceed the workspace bounds");
  if (bits & kStatusTimeout) return fail(RADIK_ETIMEOUT, "radik: a device wait timed out");
  if (bits) return fail(RADIK_EINTERNAL, "radik: internal selection error");
  return RADIK_OK;
}

int radik_autotune(int dtype, uint32_t flags, const void* val_in, const void* idx_in, void* val_out, void* idx_out,
                   void* workspace, size_t workspace_bytes, const int* task_len, int task_num, int K, void* stream_,
                   int* chunk) {
  if (task_num <= 0 || K <= 0 || !task_len) return fail(RADIK_EINVAL, "radik_autotune: empty call");
  int n_max = 0;
  int64_t total = 0;
  for (int i = 0; i < task_num; ++i) {
    if (task_len[i] < 0) return fail(RADIK_EINVAL, "radik: negative task length");
    n_max = std::max(n_max, task_len[i]);
    total += task_len[i];
  }
  int grid = 0;
  int rc = engine_grid(dtype, flags, &grid);
  if (rc) return rc;
  const uint64_t bucket = shape_bucket(dtype, flags, false, task_num, n_max, K);
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  cudaEvent_t a = nullptr, b = nullptr;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return fail(RADIK_ECUDA, "cudaEventCreate");
  // candidates: powers of two from a quarter to four times the default's pick
  const Config dflt = choose_config(total, grid, ~0ull);
  int best = 0;
  float best_ms = 1e30f;
  for (int ch = std::max(kMinCH, dflt.CH / 4); ch <= std::min(kMaxCH, dflt.CH * 4); ch *= 2) {
    {
      std::lock_guard<std::mutex> lock(g_tune_mu);
      g_tuned_ch[bucket] = ch;
    }
    float ms_sum = 0.f;
    for (int rep = 0; rep < 4 && rc == RADIK_OK; ++rep) {
      cudaEventRecord(a, stream);
      rc = radik_topk(dtype, flags, val_in, idx_in, val_out, idx_out, workspace, workspace_bytes, task_len, task_num,
                      K, stream_);
      cudaEventRecord(b, stream);
      if (rc == RADIK_OK && cudaEventSynchronize(b) != cudaSuccess) rc = fail(RADIK_ECUDA, "cudaEventSynchronize");
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      if (rep > 0) ms_sum += ms;  // the first run warms up
    }
    if (rc != RADIK_OK) break;
    if (ms_sum < best_ms) {
      best_ms = ms_sum;
      best = ch;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    if (best) g_tuned_ch[bucket] = best;
    else g_tuned_ch.erase(bucket);
  }
  if (rc != RADIK_OK) return rc;
  if (chunk) *chunk = best;
  return radik_get_status(workspace, stream_, nullptr);
}

void radik_autotune_reset(void) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tuned_ch.clear();
}

int radik_topk_static(int dtype, uint32_t flags, const void* val_in, const void* idx_in, void* val_out,
                      void* idx_out, const int* task_len, int task_num, int K, void* stream, void** scratch) {
  if (scratch) *scratch = nullptr;
  void* ws = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&ws, g_static_scratch);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(static scratch)");
  if (scratch) *scratch = ws;
  const int rc = radik_topk(dtype, flags, val_in, idx_in, val_out, idx_out, ws, RADIK_STATIC_SCRATCH_BYTES, task_len,
                            task_num, K, stream);
  // ws is non-null and aligned, so RADIK_EWORKSPACE can only mean too small
  if (rc == RADIK_EWORKSPACE) {
    int n_max = 0;
    for (int i = 0; i < task_num; ++i) n_max = std::max(n_max, task_len[i]);
    size_t need = 0;
    radik_get_workspace_size(dtype, flags, K, n_max, task_num, &need);
    return fail(RADIK_EWORKSPACE, "radik_topk_static: " + std::to_string(task_num) + " rows of up to " +
                                      std::to_string(n_max) + " values with K = " + std::to_string(K) +
                                      " need up to " + std::to_string(need) + " bytes of scratch, more than the " +
                                      std::to_string(RADIK_STATIC_SCRATCH_BYTES) +
                                      "-byte static array; call radik_topk with a caller-owned workspace");
  }
  return rc;
}

}  // extern "C"

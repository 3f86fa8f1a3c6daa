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
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace radik {

cudaError_t launch_engine(int dtype, const EngineParams& p, int grid, cudaStream_t stream, bool coop = true);
cudaError_t launch_short_rows(int dtype, const EngineParams& p, int grid, cudaStream_t stream);
cudaError_t launch_plan(const RowDesc* desc, int B, int CH, int CHR, int cta_cap, int D, uint32_t flags,
                        RowPlan* plans, int32_t* a_row, int32_t* b_row, Header* hdr, int64_t na_cap, int64_t nb_cap,
                        int64_t cand_cap_total, int64_t sort_cap_total, int grid, cudaStream_t stream);
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

// Cooperative grid of the engine on the current device (one CTA per SM),
// cached per device and per engine instantiation (value type x WITHSCALE).
int engine_grid(int dtype, uint32_t flags, int* grid) {
  static std::mutex mu;
  static int cache[64][6] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  const int key = dtype * 2 + ((flags & kFlagWithScale) ? 1 : 0);
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
  // rows above the one-CTA cap keep cand_capacity(n) candidates each; the
  // cap is tunable down to kCtaRowCapMin
  b.cand = n_max > kCtaRowCapMin ? B * (int64_t)cand_capacity((int32_t)n_max) : 0;
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

// Tunables.  Single-read rows use chunks of 4K..256K elements, aiming at
// about eight chunks per CTA so the work queue balances (the last chunks
// bound the tail) while each chunk streams long enough to amortise its item
// overhead.  Radix rows use 32K-element chunks: their filter items re-read
// chunks that the histogram items read two grids earlier, and that window
// (2 x 148 x 128 KB) must stay in L2.  The 12-bit first digit (4096 bins,
// 16 KB of smem) leaves about n/4096 keys of an i.i.d. row in the selected
// bin.  Rows of up to 2^15 keys are selected by one CTA.  The autotuner
// (radik_autotune*) can replace each choice per shape bucket; RADIK_CH /
// RADIK_CHR / RADIK_D1 / RADIK_CTA_CAP override everything (tuning sweeps).
struct Config {
  int CH, CHR, D1, cta_cap;
  int early_copy;  // chunk copies may start before their row's threshold exists
  int l2_ahead;    // ring stages a chunk's L2 prefetch runs ahead of its copies
  int tail_div;    // the last rows' pre-filter chunks are CH / tail_div long (1: no split)
};

// A tuned shape bucket: a field of 0 keeps the built-in choice.
struct Tuned {
  int ch = 0;      // chunk length of single-read rows
  int d1 = 0;      // first-digit width of histogram rows
  int cta_cap = 0; // rows of up to this many keys go to one CTA
};

std::mutex g_tune_mu;
std::map<uint64_t, Tuned> g_tuned;

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

void load_tune_file_once();

Tuned tuned_for(uint64_t bucket) {
  load_tune_file_once();
  std::lock_guard<std::mutex> lock(g_tune_mu);
  const auto it = g_tuned.find(bucket);
  return it == g_tuned.end() ? Tuned{} : it->second;
}

// Rows of up to this many keys are selected by one CTA (on its side team,
// which streams them with plain loads); longer rows spread over the grid as
// pre-filter rows.  Measured on a B200 with caps of 2^15 / 2^18:
// 1024 x 2^17 keys, k = 256: 238 / 822 us; 512 x 2^18: 174 / 670 us;
// 256 x 100000, k = 1000: 97 / 265 us; 2048 x 2^16, k = 32: 279 / 761 us;
// 4096 uneven rows of n log-uniform in [2^10, 2^22]: 1.66 / 2.51 ms.
int cta_cap_of(const Tuned& t) {
  const int ecap = env_int("RADIK_CTA_CAP", 0);
  if (ecap >= kCtaRowCapMin && ecap <= kCtaRowCapMax) return ecap;
  if (t.cta_cap) return t.cta_cap;
  return kCtaRowCap;
}

// stream_elems: keys of the call's streamed rows; es: bytes per key; uniform_n:
// the common row length of an equal-length call (0 otherwise) and B its rows.
Config choose_config(int64_t stream_elems, int grid, const Tuned& t, int es, int uniform_n, int B = 0) {
  Config c{};
  const int64_t target = std::max<int64_t>(1, stream_elems / ((int64_t)grid * 8));
  int ch = kMinCH;
  while (ch < kMaxCH && ch * 2 <= target) ch *= 2;
  // Few large rows (2^24 keys or more in all): per-item overhead outweighs
  // balance, so no chunk is shorter than 128K keys (single 2^24-key rows:
  // 154 -> 111 us from 8K to 128K chunks).
  if (stream_elems >= ((int64_t)1 << 24)) ch = std::max(ch, 1 << 17);
  // A chunk item costs about 2 us of turnover whatever its length, so 16-bit
  // keys take chunks of the same bytes, not the same keys (fp16 256 x 2^20:
  // 175.7 -> 165.3 us from 128K to 256K keys).
  if (es == 2 && ch >= (1 << 17)) ch = std::min(kMaxCH, ch * 2);
  // Small equal-length calls: one chunk per CTA at most, so no CTA claims a
  // second item (single 2^20-key rows took 256 chunks of 4K keys over 148
  // CTAs before).  Each row splits into as many chunks as the grid has CTAs
  // per row, rounded down; a few rows leave their sampling CTAs out.
  const int spread = std::max(1, grid - (B > 0 && B * 2 < grid ? B : 0));
  const int64_t per_cta = (stream_elems + spread - 1) / spread;
  if (uniform_n > 0 && per_cta <= kMaxCH) {
    const int64_t cpr = std::max<int64_t>(1, uniform_n / std::max<int64_t>(1, per_cta));
    int64_t len = (uniform_n + cpr - 1) / cpr;
    len = (len + 31) / 32 * 32;
    ch = (int)std::min<int64_t>(kMaxCH, std::max<int64_t>(kMinCH, len));
  }
  c.CH = t.ch ? t.ch : ch;
  c.CHR = 32768;
  c.D1 = t.d1 ? t.d1 : kMaxD1;
  c.cta_cap = cta_cap_of(t);
  const int ech = env_int("RADIK_CH", 0);
  if (ech >= kMinCH && ech <= (1 << 24) && (ech % 16) == 0) c.CH = ech;
  const int echr = env_int("RADIK_CHR", 0);
  if (echr >= kMinCH && echr <= (1 << 24) && (echr % 16) == 0) c.CHR = echr;
  const int ed1 = env_int("RADIK_D1", 0);
  if (ed1 >= kMinD1 && ed1 <= kMaxD1) c.D1 = ed1;
  // Calls that stream at most 64 MiB copy their chunks while the thresholds
  // are computed: their ring fills cannot delay the sample reads by much.
  c.early_copy = stream_elems * es <= ((int64_t)64 << 20) ? 1 : 0;
  const int eec = env_int("RADIK_EARLY", -1);
  if (eec == 0 || eec == 1) c.early_copy = eec;
  // An L2 prefetch two stages ahead of the ring's copies: 256 x 2^20 fp32
  // k = 256 / 1024 / 32: 202 / 230 / 196 us without, 196 / 226 / 191 us with
  // it; farther ahead is slower (16 stages: 212 us), and 16-bit rows gain
  // nothing (156 us at 0, 1 or 2 stages).
  c.l2_ahead = es == 4 ? 2 : 0;
  c.tail_div = 1;
  const int etd = env_int("RADIK_TAIL_DIV", 0);
  if (etd >= 1 && etd <= 8) c.tail_div = etd;
  const int ela = env_int("RADIK_L2_AHEAD", -1);
  if (ela >= 0 && ela <= 64) c.l2_ahead = ela;
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

// Device buffer of the timeline build's per-CTA phase stamps (null: none).
std::atomic<unsigned long long*> g_timeline{nullptr};

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
  p.cta_cap = c.cta_cap;
  p.early_copy = c.early_copy;
  p.l2_ahead = c.l2_ahead;
  p.S = kSlots;
  p.flags = flags;
  p.spin_limit = kSpinLimit;
  p.timeline = g_timeline.load();
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

// A radik_topk call after validation: the engine configuration, the exact
// item and scratch counts of its rows, and the workspace layout they need.
struct CallPlan {
  int B = 0, grid = 0;
  bool uniform = true, has_radix = false;
  bool short_only = true;  // every row is a smem or one-CTA row (one team's work)
  Config cfg{};
  int64_t na = 0, nb = 0, cand = 0, sortn = 0;
  Layout L{};
};

int plan_call(int dtype, uint32_t flags, const int* task_len, int task_num, int K, CallPlan* cp) {
  if (!task_len) return fail(RADIK_EINVAL, "radik: task_len is null");
  const int B = task_num;
  bool uniform = true;
  int n_max = 0;
  for (int i = 0; i < B; ++i) {
    const int n = task_len[i];
    if (n < 0) return fail(RADIK_EINVAL, "radik: negative task length");
    uniform = uniform && n == task_len[0];
    n_max = std::max(n_max, n);
  }
  if ((int64_t)B * K > ((int64_t)1 << 40)) return fail(RADIK_EINVAL, "radik: output too large");
  const Tuned t = tuned_for(shape_bucket(dtype, flags, false, B, n_max, K));
  int grid = 0;
  int rc = engine_grid(dtype, flags, &grid);
  if (rc) return rc;
  const int cta_cap = cta_cap_of(t);
  int64_t multi_elems = 0;
  for (int i = 0; i < B; ++i) {
    const int kind = row_kind(task_len[i], K, cta_cap);
    if (kind == kKindAll || kind == kKindGridPref || kind == kKindGridRadix) multi_elems += task_len[i];
  }
  const Config cfg = choose_config(multi_elems, grid, t, (int)elem_bytes(dtype), uniform ? n_max : 0, B);
  int64_t na = 0, nb = 0, cand = 0, sortn = 0;
  bool has_radix = false, short_only = true;
  for (int i = 0; i < B; ++i) {
    const int n = task_len[i];
    const int kind = row_kind(n, K, cta_cap);
    has_radix = has_radix || kind == kKindGridRadix;
    short_only = short_only && (kind == kKindSmem || kind == kKindCta);
    na += row_na(kind, n, cfg.CH, cfg.CHR);
    nb += row_nbc(kind, n, cfg.CH, cfg.CHR) + row_fin(kind);
    cand += row_cand_cap(kind, n);
    const int64_t kk = std::min<int64_t>(n, K);
    if ((flags & kFlagSorted) && kk > kCapSort) sortn += 2 * kk;
  }
  if (na + nb >= ((int64_t)1 << 30)) return fail(RADIK_EINVAL, "radik: too many work items");
  cp->B = B;
  cp->grid = grid;
  cp->uniform = uniform;
  cp->has_radix = has_radix;
  cp->short_only = short_only;
  cp->cfg = cfg;
  cp->na = na;
  cp->nb = nb;
  cp->cand = cand;
  cp->sortn = sortn;
  cp->L = make_layout(B, na, nb, cand, sortn);
  return RADIK_OK;
}

// Clears the call's state and launches it (planning kernel for uneven
// lengths, then the engine).  The workspace holds at least cp.L.total bytes.
int launch_call(int dtype, uint32_t flags, const void* val_in, const void* idx_in, void* val_out, void* idx_out,
                uint8_t* ws, const int* task_len, int K, const CallPlan& cp, cudaStream_t stream) {
  const int B = cp.B, grid = cp.grid;
  const Config& cfg = cp.cfg;
  const Layout& L = cp.L;
  if (!cp.uniform) {
    // Uneven lengths travel to the device as descriptors copied from host
    // memory that lives only for this call: a stream capture would record a
    // copy from freed memory, so it is refused (radik_topk_rows takes device
    // descriptors and can be captured).
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t ce = cudaStreamIsCapturing(stream, &cs);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamIsCapturing");
    if (cs != cudaStreamCaptureStatusNone)
      return fail(RADIK_ENOTSUP, "radik: rows of unequal length cannot be captured in a CUDA graph (their "
                                 "descriptors are copied from host memory); use radik_topk_rows");
  }
  cudaError_t e = cudaMemsetAsync(ws, 0, zero_bytes(L, cp.has_radix), stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
  EngineParams p = base_params(val_in, idx_in, val_out, idx_out, ws, L, B, cfg, flags);
  if (cp.uniform) {
    const int n = task_len[0];
    const int kind = row_kind(n, K, cfg.cta_cap);
    p.uniform = 1;
    p.u_n = n;
    p.u_k = K;
    p.u_cand_cap = row_cand_cap(kind, n);
    const int64_t kk = std::min<int64_t>(n, K);
    p.u_sort_cap = ((flags & kFlagSorted) && kk > kCapSort) ? 2 * kk : 0;
    if (kind == kKindSmem || kind == kKindCta) {
      // every row is one team's work: the short-row kernel, four teams a CTA
      // (4096 x 32768 keys, k = 64: 0.92 ms on the engine's side teams)
      const int g = (int)std::max<int64_t>(1, std::min<int64_t>(grid, (B + 3) / 4));
      e = launch_short_rows(dtype, p, g, stream);
      if (e != cudaSuccess) return cuda_fail(e, "short-row launch");
      return RADIK_OK;
    }
    // B sequence layout (see UniformB) and the lag it needs
    const int64_t una = row_na(kind, n, cfg.CH, cfg.CHR), nc = row_nbc(kind, n, cfg.CH, cfg.CHR);
    const int64_t f = row_fin(kind);
    const int D = fin_delay_uniform((int)nc, grid);
    const int64_t Dd = std::min<int64_t>(D, B);
    // Pre-filter rows in a call of several chunk waves: the last rows take
    // chunks of half the length, so the last items of the claim order are
    // short and the CTAs run out of work together.
    int tail_rows = 0, ch_tail = cfg.CH;
    if (kind == kKindGridPref && cfg.tail_div > 1 && (int64_t)B * nc >= 4LL * grid) {
      ch_tail = std::max(kMinCH, (cfg.CH / cfg.tail_div + 31) / 32 * 32);
      const int nct = ceil_div32(n, ch_tail);
      tail_rows = (int)std::min<int64_t>(B - Dd, (3LL * grid + 2LL * nct - 1) / (2LL * nct));
      if (tail_rows < 1 || nct <= nc) tail_rows = 0;
    }
    p.u_tail_rows = tail_rows;
    p.u_ch_tail = ch_tail;
    const UniformB ub{B, (int32_t)nc, tail_rows ? ceil_div32(n, ch_tail) : (int32_t)nc, tail_rows, (int32_t)f, D};
    int64_t maxlag = 0;
    for (int64_t r = 0; r < B && (nc > 0 || f); ++r) {
      int64_t first_b;
      if (nc > 0) first_b = ub.first(r);
      else first_b = (r + Dd < B) ? ub.first(r + Dd) + nc : ub.first(B) + (r - (B - Dd));
      maxlag = std::max(maxlag, (r + 1) * una - first_b);
    }
    p.fin_delay = D;
    p.lag = (int32_t)std::max<int64_t>(maxlag + 1, lag_floor(cp.has_radix, grid, dtype));
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
    // pageable source: the copy is staged before this call returns
    e = cudaMemcpyAsync(dd, d.data(), sizeof(RowDesc) * B, cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync");
    p.plans = reinterpret_cast<RowPlan*>(ws + L.plans);
    p.a_row = reinterpret_cast<int32_t*>(ws + L.a_row);
    p.b_row = reinterpret_cast<int32_t*>(ws + L.b_row);
    e = launch_plan(dd, B, cfg.CH, cfg.CHR, cfg.cta_cap, kFinDelayRows, flags, reinterpret_cast<RowPlan*>(ws + L.plans),
                    reinterpret_cast<int32_t*>(ws + L.a_row), reinterpret_cast<int32_t*>(ws + L.b_row), p.hdr, cp.na,
                    cp.nb, cp.cand, cp.sortn, grid, stream);
    if (e != cudaSuccess) return cuda_fail(e, "plan launch");
    if (cp.short_only) {
      // rows of unequal length, each one team's work: the short-row kernel
      // reads them from the plans
      const int g = (int)std::max<int64_t>(1, std::min<int64_t>(grid, (B + 3) / 4));
      e = launch_short_rows(dtype, p, g, stream);
      if (e != cudaSuccess) return cuda_fail(e, "short-row launch");
      return RADIK_OK;
    }
  }
  e = launch_engine(dtype, p, grid, stream);
  if (e != cudaSuccess) return cuda_fail(e, "engine launch");
  return RADIK_OK;
}

// Workspace of radik_topk_static(): static device memory of this module, one
// copy per device the module is loaded on.
static __device__ __align__(256) unsigned char g_static_scratch[RADIK_STATIC_SCRATCH_BYTES];

// Times one call of fn (4 runs, the first discarded) with CUDA events on
// the stream; returns RADIK_OK and the summed milliseconds of three runs.
template <typename Fn>
int time_call(cudaStream_t stream, cudaEvent_t a, cudaEvent_t b, Fn&& fn, float* ms_sum) {
  *ms_sum = 0.f;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(a, stream);
    const int rc = fn();
    cudaEventRecord(b, stream);
    if (rc != RADIK_OK) return rc;
    if (cudaEventSynchronize(b) != cudaSuccess) return fail(RADIK_ECUDA, "cudaEventSynchronize");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    if (rep > 0) *ms_sum += ms;
  }
  return RADIK_OK;
}

// Coordinate descent over a bucket's knobs: each candidate value of a knob
// is timed with the others at their best so far; the fastest is kept.  The
// bucket's entry is live while it is timed (the calls read it), and holds
// the winner afterwards.  Knobs whose candidates cannot change the call are
// skipped (no histogram row, no row in the CTA-cap range).
template <typename Call>
int tune_bucket(uint64_t bucket, cudaStream_t stream, bool has_radix, bool cap_matters, int ch_default, Call&& call,
                radik_tune_choice* out) {
  cudaEvent_t a = nullptr, b = nullptr;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return fail(RADIK_ECUDA, "cudaEventCreate");
  auto set = [&](const Tuned& t) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tuned[bucket] = t;
  };
  Tuned best{};
  float best_ms = 1e30f;
  int rc = RADIK_OK;
  auto trial = [&](const Tuned& t) {
    if (rc != RADIK_OK) return;
    set(t);
    float ms = 0.f;
    rc = time_call(stream, a, b, call, &ms);
    if (rc == RADIK_OK && ms < best_ms) {
      best_ms = ms;
      best = t;
    }
  };
  trial(best);  // the built-in choice
  // 1. chunk length of single-read rows: a quarter to four times the pick
  {
    const Tuned base = best;
    for (int ch = std::max(kMinCH, ch_default / 4); ch <= std::min(kMaxCH, ch_default * 4); ch *= 2) {
      Tuned t = base;
      t.ch = (ch + 31) / 32 * 32;  // whole 128-byte lines of 32-bit keys
      trial(t);
    }
  }
  // 2. first-digit width of histogram rows
  if (has_radix) {
    const Tuned base = best;
    for (int d1 : {8, 11}) {
      Tuned t = base;
      t.d1 = d1;
      trial(t);
    }
  }
  // 3. the one-CTA row cap
  if (cap_matters) {
    const Tuned base = best;
    for (int cap = kCtaRowCapMin; cap <= kCtaRowCapMax; cap *= 2) {
      if (cap == kCtaRowCap) continue;
      Tuned t = base;
      t.cta_cap = cap;
      trial(t);
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    if (rc == RADIK_OK) g_tuned[bucket] = best;
    else g_tuned.erase(bucket);
  }
  if (rc != RADIK_OK) return rc;
  if (out) {
    out->chunk = best.ch;
    out->d1 = best.d1;
    out->cta_cap = best.cta_cap;
    out->ms = best_ms / 3.f;
  }
  return RADIK_OK;
}

// The tuning table as text: one bucket per line, "key ch d1 cta_cap".
std::once_flag g_tune_file_once;

int load_tune_table(const char* path, bool replace) {
  FILE* f = std::fopen(path, "r");
  if (!f) return fail(RADIK_EINVAL, std::string("radik: cannot read tuning table ") + path);
  std::map<uint64_t, Tuned> m;
  char line[256];
  int bad = 0;
  while (std::fgets(line, sizeof line, f)) {
    if (line[0] == '#' || line[0] == '\n') continue;
    unsigned long long key = 0;
    Tuned t;
    if (std::sscanf(line, "%llx %d %d %d", &key, &t.ch, &t.d1, &t.cta_cap) != 4) {
      ++bad;
      continue;
    }
    const bool ok = (t.ch == 0 || (t.ch >= kMinCH && t.ch <= kMaxCH && t.ch % 16 == 0)) &&
                    (t.d1 == 0 || (t.d1 >= kMinD1 && t.d1 <= kMaxD1)) &&
                    (t.cta_cap == 0 || (t.cta_cap >= kCtaRowCapMin && t.cta_cap <= kCtaRowCapMax));
    if (!ok) {
      ++bad;
      continue;
    }
    m[(uint64_t)key] = t;
  }
  std::fclose(f);
  if (bad) return fail(RADIK_EINVAL, std::string("radik: malformed lines in tuning table ") + path);
  std::lock_guard<std::mutex> lock(g_tune_mu);
  if (replace) g_tuned.clear();
  for (const auto& kv : m) g_tuned[kv.first] = kv.second;
  return RADIK_OK;
}

// RADIK_TUNE_FILE names a table that the first call in the process loads.
void load_tune_file_once() {
  std::call_once(g_tune_file_once, [] {
    const char* path = std::getenv("RADIK_TUNE_FILE");
    if (path && *path) load_tune_table(path, false);
  });
}

}  // namespace
}  // namespace radik

using namespace radik;

extern "C" {

int radik_version(void) { return 100; }

int radik_timeline_attach(void* stamps) {
#ifdef RADIK_TIMELINE
  g_timeline.store(static_cast<unsigned long long*>(stamps));
  return RADIK_OK;
#else
  (void)stamps;
  return fail(RADIK_ENOTSUP, "radik_timeline_attach: this library was built without RADIK_TIMELINE");
#endif
}

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
  CallPlan cp;
  rc = plan_call(dtype, flags, task_len, task_num, K, &cp);
  if (rc) return rc;
  if (workspace_bytes < cp.L.total) return fail(RADIK_EWORKSPACE, "radik: workspace too small");
  return launch_call(dtype, flags, val_in, idx_in, val_out, idx_out, static_cast<uint8_t*>(workspace), task_len, K,
                     cp, static_cast<cudaStream_t>(stream_));
}

int radik_topk_rows(int dtype, uint32_t flags, const void* val_in, const void* idx_in, void* val_out,
                    void* idx_out, void* workspace, size_t workspace_bytes, const radik_row_desc* rows,
                    int task_num, int64_t total_n, int n_max, int k_max, void* stream_) {
  return radik_topk_rows_ctas(dtype, flags, val_in, idx_in, val_out, idx_out, workspace, workspace_bytes, rows,
                              task_num, total_n, n_max, k_max, 0, stream_);
}

int radik_topk_rows_ctas(int dtype, uint32_t flags, const void* val_in, const void* idx_in, void* val_out,
                         void* idx_out, void* workspace, size_t workspace_bytes, const radik_row_desc* rows,
                         int task_num, int64_t total_n, int n_max, int k_max, int max_ctas, void* stream_) {
  if (max_ctas < 0) return fail(RADIK_EINVAL, "radik: negative max_ctas");
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
  // A smaller grid leaves SMs free for other work.  Its launch is not
  // cooperative, so that launches on other streams can run beside it; its
  // CTAs are all resident as long as the grids of the calls in flight add up
  // to at most the SM count (the contract of this entry point).
  const bool coop = !(max_ctas > 0 && max_ctas < grid);
  if (max_ctas > 0) grid = std::min(grid, max_ctas);
  const Config cfg = choose_config(total_n, grid, tuned_for(shape_bucket(dtype, flags, true, B, n_max, k_max)),
                                   (int)elem_bytes(dtype), 0, B);
  uint8_t* ws = static_cast<uint8_t*>(workspace);
  cudaError_t e = cudaMemsetAsync(ws, 0, zero_bytes(L, true), stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
  EngineParams p = base_params(val_in, idx_in, val_out, idx_out, ws, L, B, cfg, flags);
  p.plans = reinterpret_cast<RowPlan*>(ws + L.plans);
  p.a_row = reinterpret_cast<int32_t*>(ws + L.a_row);
  p.b_row = reinterpret_cast<int32_t*>(ws + L.b_row);
  // The item budget assumed kMinCH-long chunks; with the chosen CH the true
  // count is smaller, so the bound still holds.
  e = launch_plan(reinterpret_cast<const RowDesc*>(rows), B, cfg.CH, cfg.CHR, cfg.cta_cap, kFinDelayRows, flags, reinterpret_cast<RowPlan*>(ws + L.plans),
                  reinterpret_cast<int32_t*>(ws + L.a_row), reinterpret_cast<int32_t*>(ws + L.b_row), p.hdr, b.na, b.nb,
                  b.cand, b.sort, grid, stream);
  if (e != cudaSuccess) return cuda_fail(e, "plan launch");
  e = launch_engine(dtype, p, grid, stream, coop);
  if (e != cudaSuccess) return cuda_fail(e, "engine launch");
  return RADIK_OK;
}

int radik_get_call_span(void* workspace, void* stream_, uint64_t* start_ns, uint64_t* end_ns) {
  if (!workspace) return fail(RADIK_EWORKSPACE, "radik: workspace should not be null");
  cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream_));
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
  uint64_t t[2] = {0, 0};
  e = cudaMemcpy(t, static_cast<uint8_t*>(workspace) + offsetof(Header, t_first), sizeof(t), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy span");
  if (start_ns) *start_ns = t[0];
  if (end_ns) *end_ns = t[1];
  return RADIK_OK;
}

int radik_engine_ctas(int* ctas) {
  if (!ctas) return fail(RADIK_EINVAL, "radik: ctas is null");
  return engine_grid(kF32, 0, ctas);
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

int radik_autotune_ex(int dtype, uint32_t flags, const void* val_in, const void* idx_in, void* val_out,
                      void* idx_out, void* workspace, size_t workspace_bytes, const int* task_len, int task_num,
                      int K, void* stream_, radik_tune_choice* out) {
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
  bool has_radix = false, cap_matters = false;
  for (int i = 0; i < task_num; ++i) {
    const int n = task_len[i];
    has_radix = has_radix || row_kind(n, K, kCtaRowCapMax) == kKindGridRadix ||
                row_kind(n, K, kCtaRowCapMin) == kKindGridRadix;
    cap_matters = cap_matters || (n > kCtaRowCapMin && n <= kCtaRowCapMax && K < n);
  }
  bool uniform = true;
  for (int i = 0; i < task_num; ++i) uniform = uniform && task_len[i] == task_len[0];
  const Config dflt = choose_config(total, grid, Tuned{}, (int)elem_bytes(dtype), uniform ? n_max : 0, task_num);
  rc = tune_bucket(bucket, static_cast<cudaStream_t>(stream_), has_radix, cap_matters, dflt.CH,
                   [&] {
                     return radik_topk(dtype, flags, val_in, idx_in, val_out, idx_out, workspace, workspace_bytes,
                                       task_len, task_num, K, stream_);
                   },
                   out);
  if (rc != RADIK_OK) return rc;
  return radik_get_status(workspace, stream_, nullptr);
}

int radik_autotune(int dtype, uint32_t flags, const void* val_in, const void* idx_in, void* val_out, void* idx_out,
                   void* workspace, size_t workspace_bytes, const int* task_len, int task_num, int K, void* stream_,
                   int* chunk) {
  radik_tune_choice c{};
  const int rc = radik_autotune_ex(dtype, flags, val_in, idx_in, val_out, idx_out, workspace, workspace_bytes,
                                   task_len, task_num, K, stream_, &c);
  if (rc == RADIK_OK && chunk) *chunk = c.chunk;
  return rc;
}

int radik_autotune_rows(int dtype, uint32_t flags, const void* val_in, const void* idx_in, void* val_out,
                        void* idx_out, void* workspace, size_t workspace_bytes, const radik_row_desc* rows,
                        int task_num, int64_t total_n, int n_max, int k_max, void* stream_, radik_tune_choice* out) {
  if (task_num <= 0 || !rows) return fail(RADIK_EINVAL, "radik_autotune_rows: empty call");
  int grid = 0;
  int rc = engine_grid(dtype, flags, &grid);
  if (rc) return rc;
  const uint64_t bucket = shape_bucket(dtype, flags, true, task_num, n_max, k_max);
  // the rows live on the device: every knob is tried
  const Config dflt = choose_config(total_n, grid, Tuned{}, (int)elem_bytes(dtype), 0, task_num);
  rc = tune_bucket(bucket, static_cast<cudaStream_t>(stream_), true, n_max > kCtaRowCapMin, dflt.CH,
                   [&] {
                     return radik_topk_rows(dtype, flags, val_in, idx_in, val_out, idx_out, workspace, workspace_bytes,
                                            rows, task_num, total_n, n_max, k_max, stream_);
                   },
                   out);
  if (rc != RADIK_OK) return rc;
  return radik_get_status(workspace, stream_, nullptr);
}

void radik_autotune_reset(void) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tuned.clear();
}

int radik_autotune_save(const char* path) {
  if (!path) return fail(RADIK_EINVAL, "radik_autotune_save: path is null");
  std::map<uint64_t, Tuned> m;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    m = g_tuned;
  }
  FILE* f = std::fopen(path, "w");
  if (!f) return fail(RADIK_EINVAL, std::string("radik: cannot write tuning table ") + path);
  std::fprintf(f, "# radik_b200 tuning table: bucket chunk d1 cta_cap (0: built-in)\n");
  std::fprintf(f, "# bucket = dtype | rows_form << 2 | sorted << 3 | log2(rows) << 4 | log2(n_max) << 12 | "
                  "log2(k) << 20\n");
  for (const auto& kv : m)
    std::fprintf(f, "%llx %d %d %d\n", (unsigned long long)kv.first, kv.second.ch, kv.second.d1,
                 kv.second.cta_cap);
  const bool ok = std::fclose(f) == 0;
  return ok ? RADIK_OK : fail(RADIK_EINVAL, std::string("radik: cannot write tuning table ") + path);
}

int radik_autotune_load(const char* path) {
  if (!path) return fail(RADIK_EINVAL, "radik_autotune_load: path is null");
  load_tune_file_once();
  return load_tune_table(path, true);
}

int radik_topk_static(int dtype, uint32_t flags, const void* val_in, const void* idx_in, void* val_out,
                      void* idx_out, const int* task_len, int task_num, int K, void* stream, void** scratch) {
  if (scratch) *scratch = nullptr;
  // validated with a stand-in workspace: the array's address is looked up
  // only once the call is known to fit
  int rc = check_common(dtype, flags, val_in, idx_in, val_out, idx_out, reinterpret_cast<void*>(uintptr_t(256)));
  if (rc) return rc;
  if (task_num < 0 || K < 0) return fail(RADIK_EINVAL, "radik: negative task_num or K");
  CallPlan cp;
  if (task_num > 0 && K > 0) {
    rc = plan_call(dtype, flags, task_len, task_num, K, &cp);
    if (rc) return rc;
    if (cp.L.total > RADIK_STATIC_SCRATCH_BYTES) {
      int n_max = 0;
      for (int i = 0; i < task_num; ++i) n_max = std::max(n_max, task_len[i]);
      return fail(RADIK_EWORKSPACE, "radik_topk_static: " + std::to_string(task_num) + " rows of up to " +
                                        std::to_string(n_max) + " values with K = " + std::to_string(K) + " need " +
                                        std::to_string(cp.L.total) + " bytes of scratch, more than the " +
                                        std::to_string(RADIK_STATIC_SCRATCH_BYTES) +
                                        "-byte static array; call radik_topk with a caller-owned workspace");
    }
  }
  void* ws = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&ws, g_static_scratch);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(static scratch)");
  if (scratch) *scratch = ws;
  if (task_num == 0 || K == 0) return RADIK_OK;
  return launch_call(dtype, flags, val_in, idx_in, val_out, idx_out, static_cast<uint8_t*>(ws), task_len, K, cp,
                     static_cast<cudaStream_t>(stream));
}

}  // extern "C"

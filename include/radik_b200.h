/* radik_b200.h -- C ABI of the B200 radix top-k selection library.
 *
 * Drop-in boundary for RadiK's batched radix top-k (leefige/radik,
 * radik/RadixSelect/topk_radixselect.h).  Plain pointers and sizes only; no
 * C++ types cross it and no exception escapes it.  Every entry point returns a
 * radik_status code (0 = success).  Launches are asynchronous on the given
 * stream; device-side failures are reported by radik_get_status().
 *
 * Values: fp32, fp16 or bf16 (radik_dtype).  Indices: int32 by default,
 * int64 with RADIK_IDX64 (applies to idx_in and idx_out together, as RadiK's
 * single IdxType template parameter does).
 */
#ifndef RADIK_B200_H_
#define RADIK_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Value types (RadiK: ValType = float / half; bf16 is declared by RadiK,
 * radik/RadixSelect/utils.cuh:11-14, but cannot build there). */
enum radik_dtype { RADIK_F32 = 0, RADIK_F16 = 1, RADIK_BF16 = 2 };

/* Flags: RadiK's template parameters and needSorting as run-time bits
 * (topk_radixselect.h:59-70). */
#define RADIK_LARGEST 1u    /* LARGEST: top-k largest (else smallest)           */
#define RADIK_SORTED 2u     /* needSorting: sort each row's k outputs           */
#define RADIK_ASCEND 4u     /* ASCEND: sorted order ascending (else descending) */
#define RADIK_WITHSCALE 8u  /* WITHSCALE: order by x - x[row start]             */
#define RADIK_WITHIDXIN 16u /* WITHIDXIN: emit idx_in[row_off + pos]            */
#define RADIK_IDX64 32u     /* idx_in / idx_out are int64 (else int32)          */

enum radik_status {
  RADIK_OK = 0,
  RADIK_EINVAL = 1,      /* bad argument (RadiK throws std::runtime_error)      */
  RADIK_EWORKSPACE = 2,  /* workspace null or too small (topk_radixselect.h:77) */
  RADIK_ECUDA = 3,       /* a CUDA runtime call failed (error_check.hpp:14-58)  */
  RADIK_ETIMEOUT = 4,    /* a bounded device wait gave up                       */
  RADIK_EINTERNAL = 5,   /* the device reported an inconsistent selection       */
  RADIK_ENOTSUP = 6      /* combination not supported                           */
};

/* Row descriptor of the uneven batched form: row r reads n values at
 * val_in[in_off ..) (and idx_in[in_off ..) with RADIK_WITHIDXIN) and writes k
 * results at val_out/idx_out[out_off ..). */
typedef struct radik_row_desc {
  int64_t in_off;
  int64_t out_off;
  int32_t n;
  int32_t k;
} radik_row_desc;

/* Replaces getRadixSelectLWorkSpaceSize<ValType>(K, n, taskNum, &bytes)
 * (radik/RadixSelect/topk_radixselect.h:22-33): bytes of device workspace for
 * radik_topk() on task_num rows of at most n_max values.  flags must carry
 * RADIK_SORTED if the calls will sort (a merge-sort scratch is reserved for
 * k > 4096, the outputs a finisher sorts in shared memory). */
int radik_get_workspace_size(int dtype, uint32_t flags, int K, int n_max, int task_num, size_t* bytes);

/* Replaces topKRadixSelectL<IdxType, LARGEST, ASCEND, WITHSCALE, WITHIDXIN,
 * ValType>(valIn, idxIn, valOut, idxOut, workSpace, taskLen, taskNum, K,
 * stream, needSorting) (radik/RadixSelect/topk_radixselect.h:59-70).
 *   val_in       device, the task_num rows back to back (no padding)
 *   idx_in       device, same layout, only read with RADIK_WITHIDXIN
 *   val_out/idx_out  device, task_num x K, row r at r * K
 *   task_len     HOST array of task_num row lengths (as in RadiK)
 * Rows shorter than K fill slots [n, K) with index -1 and value 0 (RadiK does
 * this on its sorted path, topk_radixselect.h:312-320).  Ties at the k-th
 * value go to the lowest positions.  Unsorted output order is unspecified. */
int radik_topk(int dtype, uint32_t flags, const void* val_in, const void* idx_in, void* val_out, void* idx_out,
               void* workspace, size_t workspace_bytes, const int* task_len, int task_num, int K,
               void* stream);

/* Workspace for radik_topk_rows(): task_num rows, total_n values in all,
 * the longest n_max, the largest k k_max.  The same four bounds must be
 * passed to radik_topk_rows(), which lays the workspace out from them. */
int radik_get_workspace_size_rows(int dtype, uint32_t flags, int task_num, int64_t total_n, int n_max, int k_max,
                                  size_t* bytes);

/* Uneven batched one-launch form: per-row n and k from a DEVICE array of
 * descriptors.  No host synchronisation and no host-side planning, so the
 * call can be captured in a CUDA graph.  Semantics per row as radik_topk.
 * total_n / n_max / k_max are upper bounds of the rows' sum of n, largest n
 * and largest k (the values given to radik_get_workspace_size_rows); a
 * descriptor set that exceeds them is rejected on the device
 * (radik_get_status -> RADIK_EWORKSPACE).  RadiK's batch has one K for all
 * rows (topk_radixselect.h:107-110); this form stands beside the plain one. */
int radik_topk_rows(int dtype, uint32_t flags, const void* val_in, const void* idx_in, void* val_out,
                    void* idx_out, void* workspace, size_t workspace_bytes, const radik_row_desc* rows,
                    int task_num, int64_t total_n, int n_max, int k_max, void* stream);

/* radik_topk_rows on at most max_ctas SMs (0: the whole device; the engine
 * runs one CTA per SM).  Below the whole device the launch is not cooperative,
 * so calls on other streams run side by side with it.  The engine's CTAs wait
 * for one another, so the caller keeps the max_ctas of the calls in flight at
 * once within radik_engine_ctas(): a CTA that finds no free SM delays its
 * call, and one that never finds one makes the call's waits give up
 * (RADIK_ETIMEOUT from radik_get_status).  The serving loop sizes its batches
 * this way.  No RadiK counterpart: RadiK sizes its grid from the shape alone
 * (topk_radixselect.h:117-130). */
int radik_topk_rows_ctas(int dtype, uint32_t flags, const void* val_in, const void* idx_in, void* val_out,
                         void* idx_out, void* workspace, size_t workspace_bytes, const radik_row_desc* rows,
                         int task_num, int64_t total_n, int n_max, int k_max, int max_ctas, void* stream);

/* Engine CTAs a call on the current device can use at most (one per SM):
 * the limit that radik_topk_rows_ctas calls share. */
int radik_engine_ctas(int* ctas);

/* Synchronises the stream and reads when the last call made with this
 * workspace ran on the device: the GPU global timer (ns) at which its
 * selection kernel's first CTA started and its last CTA ended (0 if the
 * kernel did not run).  Spans of calls on different streams share one time
 * base, so they show whether the calls ran at the same time. */
int radik_get_call_span(void* workspace, void* stream, uint64_t* start_ns, uint64_t* end_ns);

/* Synchronises the stream and returns the status of the last call made with
 * this workspace (RADIK_OK, RADIK_ETIMEOUT, RADIK_EINTERNAL, RADIK_EWORKSPACE).
 * device_bits (nullable) receives the raw device status word. */
int radik_get_status(void* workspace, void* stream, int* device_bits);

/* ---- Autotuner (no RadiK counterpart; RadiK fixes its grid and filter
 * cache per shape in code, topk_radixselect.h:117-130, 233-258).
 * A tuned shape bucket -- dtype, form (radik_topk / radik_topk_rows),
 * sortedness and log2 of the row count, longest row and K -- holds:
 *   chunk    chunk length (keys) of single-read rows: how a row's work is
 *            split over the CTAs
 *   d1       first-digit width of histogram rows (8, 11 or 12 bits)
 *   cta_cap  rows of up to this many keys (2^15 .. 2^20) are selected by one
 *            CTA instead of being spread over the grid
 * A field of 0 keeps the built-in choice.  ms is the tuned call's time in
 * milliseconds. */
typedef struct radik_tune_choice {
  int chunk, d1, cta_cap;
  float ms;
} radik_tune_choice;

/* Times radik_topk on the caller's buffers by coordinate descent over the
 * knobs above (4 runs a candidate, CUDA events, the first discarded) and
 * keeps the fastest for the call's bucket, for every later call in this
 * process.  Knobs that cannot change the call are skipped.  Synchronises the
 * stream: do not call it inside a stream capture.  The outputs hold a valid
 * result afterwards.  RADIK_CH / RADIK_D1 / RADIK_CTA_CAP still override. */
int radik_autotune_ex(int dtype, uint32_t flags, const void* val_in, const void* idx_in, void* val_out,
                      void* idx_out, void* workspace, size_t workspace_bytes, const int* task_len, int task_num,
                      int K, void* stream, radik_tune_choice* out);
/* radik_autotune_ex reporting only the chunk length (nullable). */
int radik_autotune(int dtype, uint32_t flags, const void* val_in, const void* idx_in, void* val_out, void* idx_out,
                   void* workspace, size_t workspace_bytes, const int* task_len, int task_num, int K, void* stream,
                   int* chunk);
/* The same for radik_topk_rows (device descriptors; the engine's knobs). */
int radik_autotune_rows(int dtype, uint32_t flags, const void* val_in, const void* idx_in, void* val_out,
                        void* idx_out, void* workspace, size_t workspace_bytes, const radik_row_desc* rows,
                        int task_num, int64_t total_n, int n_max, int k_max, void* stream, radik_tune_choice* out);
/* Forgets every tuned bucket. */
void radik_autotune_reset(void);
/* Writes the tuned buckets to a text file / replaces them with a file's.
 * A process whose environment names a file in RADIK_TUNE_FILE loads it at
 * its first call. */
int radik_autotune_save(const char* path);
int radik_autotune_load(const char* path);

/* Size of the fixed device scratch behind radik_topk_static(). */
#define RADIK_STATIC_SCRATCH_BYTES ((size_t)32 << 20)

/* No counterpart in RadiK.  radik_topk() for callers that may not allocate
 * device memory at the call site: a custom allocator's own eviction or
 * defragmentation pass that ranks blocks (calling cudaMalloc there re-enters
 * the allocator), a hook that runs while the allocator reports out-of-memory,
 * or a latency-bound loop where cudaFree's implicit device synchronisation is
 * not acceptable.  The workspace is a RADIK_STATIC_SCRATCH_BYTES array of
 * static device memory in this library, one per device, allocated when the
 * library's device code is loaded on that device; this function allocates
 * nothing and calls no allocating routine.
 *   - Arguments and results as radik_topk() without workspace/workspace_bytes.
 *   - The first call on a device looks the array up (cudaGetSymbolAddress),
 *     which may load the library's device code; make that first call before
 *     any stream capture on the device.
 *   - A call whose workspace need exceeds the array fails with
 *     RADIK_EWORKSPACE before touching the device; radik_last_error() states
 *     the need.  Use radik_topk() with a caller-owned workspace for it.
 *   - Nothing has to start at zero: each call clears the state it needs at
 *     the front of the array (one memset on the stream) before its kernels.
 *   - One array per device: two calls that can be in flight at the same time
 *     on one device (different streams, or host threads without ordering)
 *     race on it and corrupt each other's results.  Calls ordered on one
 *     stream are safe.
 *   - scratch (nullable) receives the array's device address, so that
 *     radik_get_status(*scratch, stream, ...) reads the call's device status. */
int radik_topk_static(int dtype, uint32_t flags, const void* val_in, const void* idx_in, void* val_out,
                      void* idx_out, const int* task_len, int task_num, int K, void* stream, void** scratch);

/* ---- One row split over several GPUs (no RadiK counterpart: RadiK selects
 * each row on one GPU).  Rank r holds a contiguous shard of the row: global
 * positions [pos_base, pos_base + n) of a row whose positions fit in ib bits
 * (ib = bits of the row length).  Selection is radix levels over the
 * composite (selection key << ib | global position), the order a single GPU
 * uses, so ties go to the lowest global positions.  The caller runs the
 * levels: every rank histograms the next digit of its shard, the histograms
 * are summed over the ranks (an all-reduce of 4096 counters), every rank
 * picks the same bin; when the matched set is small, every rank collects its
 * certainly-selected and tied keys and the caller gathers them.
 * radik_b200.sharding.topk_split_row drives both over torch.distributed.
 * flags: RADIK_LARGEST, RADIK_WITHSCALE (scaler = the row's first value, 0 if
 * it is NaN or infinite).  Both are asynchronous on the stream. */
/* hist (device, 4096 counters, cleared here) receives the counts of digit
 * [w - plen - digit_bits, w - plen) of this shard's composites whose top plen
 * bits equal prefix, w = key bits (32 for fp32 or scaled rows, else 16) + ib. */
int radik_shard_histogram(int dtype, uint32_t flags, const void* val_in, int64_t n, int64_t pos_base, int ib,
                          uint64_t prefix, int plen, int digit_bits, float scaler, uint32_t* hist, void* stream);
/* Compacts entries (value bits << 32 | global position) of this shard whose
 * composite's top plen bits are below prefix into better[] and equal to it
 * into tied[]; counts[0] / counts[1] (device) receive how many there were,
 * entries past a capacity counted but not stored. */
int radik_shard_collect(int dtype, uint32_t flags, const void* val_in, int64_t n, int64_t pos_base, int ib,
                        uint64_t prefix, int plen, float scaler, uint64_t* better, int cap_better, uint64_t* tied,
                        int cap_tied, uint32_t* counts, void* stream);

/* ---- Serving: a continuous-batching request loop.  No RadiK counterpart:
 * RadiK's callers form their own batches and call topKRadixSelectL once per
 * batch.  A server owns a worker thread, batch slots (workspace, output
 * staging, a stream each) and a device-memory budget.  Each request is one
 * row already on the device; its results land in the request's own device
 * buffers.  Requests that arrive while batches run are admitted into the next
 * batch as a slot, the budget and free SMs allow: a batch asks for one engine
 * CTA (one SM) per 2^16 keys (at least 32 when no other batch is in flight),
 * at most three quarters of the device when
 * several slots exist, and starts when that many SMs are free of other
 * batches.  So several batches are in flight at once and their selection
 * kernels run side by side on disjoint SMs.  Each
 * batch is one radik_topk_rows launch over the requests of one (dtype, flags)
 * group; a request's result does not depend on the batch it joined (the
 * selection is exact, ties go to the lowest positions). */
typedef struct radik_server radik_server;

typedef struct {
  int device;              /* CUDA device the server works on */
  int mode;                /* 0: continuous batching; 1: one radik_topk launch per request (baseline) */
  int slots;               /* batches in flight at once (default 3; mode 1 uses 1) */
  int max_batch_rows;      /* requests per batch (default 512) */
  int64_t max_batch_keys;  /* sum of n per batch (default 2^27) */
  int max_n;               /* largest request n (default 2^24) */
  int max_k;               /* largest request k (default 2048) */
  size_t budget_bytes;     /* device bytes of requests in flight (values + results; default 40 GiB) */
} radik_server_config;

typedef struct {
  uint64_t id;        /* as returned by radik_server_submit */
  int32_t status;     /* radik_status of the request's batch */
  int32_t pad;
  double latency_us;  /* submission to completion seen by the worker */
} radik_completion;

typedef struct {
  double arrival_us;   /* offset from the start of the trace */
  int dtype;
  uint32_t flags;      /* RADIK_LARGEST / SORTED / ASCEND / IDX64 */
  const void* values;  /* device, n values */
  int n, k;
  void* val_out;       /* device, k values */
  void* idx_out;       /* device, k indices */
} radik_trace_item;

/* Counters of a server's batches since it was created. */
typedef struct {
  int64_t batches;                /* batches launched */
  int64_t requests;               /* requests in them */
  int64_t batches_beside_others;  /* batches launched while another batch was still in flight */
  int32_t max_batches_in_flight;  /* most batches in flight at once */
  int32_t max_ctas_in_flight;     /* most engine CTAs (SMs) held by batches at once */
  int32_t ctas_total;             /* engine CTAs of the device (one per SM) */
  int32_t ctas_cap;               /* most CTAs one batch may take */
} radik_server_stats;

int radik_server_create(const radik_server_config* cfg, radik_server** server);
/* Queues one request (thread-safe, returns at once).  WITHSCALE / WITHIDXIN
 * requests are not served (RADIK_ENOTSUP). */
int radik_server_submit(radik_server* server, int dtype, uint32_t flags, const void* values, int n, int k,
                        void* val_out, void* idx_out, uint64_t* id);
/* Moves up to max finished requests into out; *count receives how many. */
int radik_server_poll(radik_server* server, radik_completion* out, int max, int* count);
/* Blocks until every submitted request has finished; returns the first error. */
int radik_server_drain(radik_server* server);
/* Copies the server's batch counters into out. */
int radik_server_get_stats(radik_server* server, radik_server_stats* out);
/* Load generator: submits items at their arrival offsets from this host
 * thread (busy-waiting between them), drains, and writes each item's latency
 * (in item order) to latency_us.  No other thread may submit meanwhile. */
int radik_server_run_trace(radik_server* server, const radik_trace_item* items, int count, double* latency_us);
/* Finishes queued work, then frees the server. */
int radik_server_destroy(radik_server* server);

/* Human-readable text of a radik_status code. */
const char* radik_strerror(int status);

/* Text of the last error raised on the calling host thread. */
const char* radik_last_error(void);

/* Library version as 10000 * major + 100 * minor + patch. */
int radik_version(void);

/* ---- Timeline build (libradik_b200_timeline.so, compiled with RADIK_TIMELINE)
 * Engine launches made after this call write, per CTA, 32 slots of 64 bits
 * into `stamps` (a device buffer of at least grid x 32 x 8 bytes, cleared by
 * the caller): %globaltimer nanoseconds at the engine's phase boundaries
 * (kernel start, first sample, consumer / side teams done, finish start and
 * its steps, phase B, end) and, in slot 31, a finishing row's candidate count.
 * radik_b200/timeline.py reads and summarises them.  Pass NULL to detach.
 * The normal library returns RADIK_ENOTSUP. */
int radik_timeline_attach(void* stamps);

#ifdef __cplusplus
}
#endif

#endif /* RADIK_B200_H_ */

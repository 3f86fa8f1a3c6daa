// ref_radik.cu -- C-callable wrapper around the UNMODIFIED reference RadiK
// header library, compiled from the reference's own sources by oracle/Makefile
// into oracle/_ref/libradik_ref.so.
//
// TEST INFRASTRUCTURE ONLY: it lets the GPU parity tests run RadiK itself on
// the same device buffers as the new library, and gives bench.py's reference
// arm RadiK's own code path.  Nothing in radik_b200/ links or loads it.
//
// The entry points forward to
//   getRadixSelectLWorkSpaceSize<ValType>  (radik/RadixSelect/topk_radixselect.h:22-33)
//   topKRadixSelectL<int32_t, LARGEST, ASCEND, WITHSCALE, WITHIDXIN, ValType>
//                                        (radik/RadixSelect/topk_radixselect.h:59-323)
// for ValType in {float, half}; exceptions become return codes.

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <exception>
#include <string>

#include "RadixSelect/topk_radixselect.h"

namespace {

thread_local std::string g_last_error;

template <bool L, bool A, bool S, bool I, typename V>
void call(const void* val_in, const int* idx_in, void* val_out, int* idx_out, void* ws,
          const int* task_len, int task_num, int K, cudaStream_t stream, bool sorted) {
  topKRadixSelectL<int32_t, L, A, S, I>(static_cast<const V*>(val_in), idx_in, static_cast<V*>(val_out),
                                       idx_out, ws, task_len, task_num, K, stream, sorted);
}

template <typename V>
void dispatch(int largest, int ascend, int withscale, int withidxin, const void* val_in, const int* idx_in,
              void* val_out, int* idx_out, void* ws, const int* task_len, int task_num, int K,
              cudaStream_t stream, bool sorted) {
#define RADIK_REF_CASE(L, A, S, I)                                                               \
  if (largest == L && ascend == A && withscale == S && withidxin == I) {                         \
    call<L, A, S, I, V>(val_in, idx_in, val_out, idx_out, ws, task_len, task_num, K, stream,     \
                        sorted);                                                                 \
    return;                                                                                      \
  }
  RADIK_REF_CASE(0, 0, 0, 0) RADIK_REF_CASE(0, 0, 0, 1) RADIK_REF_CASE(0, 0, 1, 0) RADIK_REF_CASE(0, 0, 1, 1)
  RADIK_REF_CASE(0, 1, 0, 0) RADIK_REF_CASE(0, 1, 0, 1) RADIK_REF_CASE(0, 1, 1, 0) RADIK_REF_CASE(0, 1, 1, 1)
  RADIK_REF_CASE(1, 0, 0, 0) RADIK_REF_CASE(1, 0, 0, 1) RADIK_REF_CASE(1, 0, 1, 0) RADIK_REF_CASE(1, 0, 1, 1)
  RADIK_REF_CASE(1, 1, 0, 0) RADIK_REF_CASE(1, 1, 0, 1) RADIK_REF_CASE(1, 1, 1, 0) RADIK_REF_CASE(1, 1, 1, 1)
#undef RADIK_REF_CASE
  throw std::runtime_error("ref_radik: bad flag combination");
}

}  // namespace

extern "C" {

// dtype: 0 = float, 1 = half.
int ref_radik_workspace_size(int dtype, int K, int n_max, int task_num, size_t* bytes) {
  if (!bytes) return -1;
  if (dtype == 0) getRadixSelectLWorkSpaceSize<float>(K, n_max, task_num, bytes);
  else if (dtype == 1) getRadixSelectLWorkSpaceSize<half>(K, n_max, task_num, bytes);
  else return -1;
  return 0;
}

// task_len is a HOST array, as in the reference.  Returns 0 or -1 (message in
// ref_radik_last_error()).
int ref_radik_topk(int dtype, int largest, int ascend, int withscale, int withidxin, int sorted,
                   const void* val_in, const int* idx_in, void* val_out, int* idx_out, void* ws,
                   const int* task_len, int task_num, int K, void* stream) {
  try {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == 0)
      dispatch<float>(largest, ascend, withscale, withidxin, val_in, idx_in, val_out, idx_out, ws, task_len,
                      task_num, K, s, sorted != 0);
    else if (dtype == 1)
      dispatch<half>(largest, ascend, withscale, withidxin, val_in, idx_in, val_out, idx_out, ws, task_len,
                     task_num, K, s, sorted != 0);
    else
      throw std::runtime_error("ref_radik: dtype must be 0 (float) or 1 (half)");
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return -1;
  }
  return 0;
}

const char* ref_radik_last_error(void) { return g_last_error.c_str(); }

}  // extern "C"

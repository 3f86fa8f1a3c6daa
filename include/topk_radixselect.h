/* topk_radixselect.h -- RadiK's C++ entry points over the radik_b200 C ABI.
 *
 * A RadiK caller recompiles unchanged against this header and links
 * libradik_b200.so: the two templates keep RadiK's names, template
 * parameters, argument order and meaning
 * (radik/RadixSelect/topk_radixselect.h:22-33 and :59-70), and throw
 * std::runtime_error where RadiK throws (null workspace, :77-79; CUDA
 * errors, error_check.hpp:14-58).
 *
 * Differences a caller can observe:
 *   - The workspace it sizes is smaller than RadiK's (no copy of the rows).
 *   - Ties at the k-th value resolve to the lowest positions (RadiK: arrival
 *     order), so results are deterministic.
 *   - IdxType may be int32_t or int64_t; ValType float, __half or
 *     __nv_bfloat16 (RadiK declares bf16 but cannot build it).
 *   - Rows shorter than K are allowed in both sorted and unsorted modes
 *     (slots [n, K) get index -1 and value 0).
 * Like RadiK, the call returns with the results complete: it waits for the
 * stream once to read the device status word, so that a failed bounded wait
 * or an internal selection error is thrown here rather than lost.  Define
 * RADIK_B200_ASYNC before including this header to skip that wait (errors are
 * then read with radik_get_status()).
 */
#ifndef RADIK_B200_TOPK_RADIXSELECT_H_
#define RADIK_B200_TOPK_RADIXSELECT_H_

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>

#include "radik_b200.h"

namespace radik_b200_compat {

template <typename T>
struct dtype_of;
template <>
struct dtype_of<float> {
  static constexpr int value = RADIK_F32;
};
template <>
struct dtype_of<__half> {
  static constexpr int value = RADIK_F16;
};
template <>
struct dtype_of<__nv_bfloat16> {
  static constexpr int value = RADIK_BF16;
};

inline void check(int status) {
  if (status != RADIK_OK) {
    const char* msg = radik_last_error();
    throw std::runtime_error(std::string("radix topk: ") + (msg && *msg ? msg : radik_strerror(status)));
  }
}

// RadiK's workspace formula takes (K, n_max, taskNum); the size used for a
// call is recomputed from the same three numbers, with the sort scratch
// included, so any buffer sized by getRadixSelectLWorkSpaceSize fits.
inline size_t workspace_bytes(int dtype, int K, int n_max, int task_num) {
  size_t bytes = 0;
  check(radik_get_workspace_size(dtype, RADIK_SORTED, K, n_max, task_num, &bytes));
  return bytes;
}

}  // namespace radik_b200_compat

/* Workspace bytes for topKRadixSelectL() on taskNum rows of at most n values. */
template <typename ValType>
void getRadixSelectLWorkSpaceSize(const int& K, const int& n, const int& taskNum, size_t* sizeInBytes) {
  if (sizeInBytes == nullptr) throw std::runtime_error("radix topk: sizeInBytes should not be null");
  *sizeInBytes = radik_b200_compat::workspace_bytes(radik_b200_compat::dtype_of<ValType>::value, K, n, taskNum);
}

/* Batched top-k of taskNum rows stored back to back (row lengths in the HOST
 * array taskLen); outputs taskNum x K.  See topk_radixselect.h:36-58 of
 * RadiK for the parameter list. */
template <typename IdxType, bool LARGEST, bool ASCEND, bool WITHSCALE, bool WITHIDXIN = 0, typename ValType,
          bool WITHPACKING = 1>
void topKRadixSelectL(const ValType* valIn, const IdxType* idxIn, ValType* valOut, IdxType* idxOut, void* workSpace,
                      const int* taskLen, const int& taskNum, const int& K, cudaStream_t stream,
                      bool needSorting = true) {
  static_assert(std::is_same<IdxType, int32_t>::value || std::is_same<IdxType, int64_t>::value,
                "radix topk: IdxType must be int32_t or int64_t");
  if (workSpace == nullptr) throw std::runtime_error("radix topk: workspace should not be null");
  constexpr int dtype = radik_b200_compat::dtype_of<ValType>::value;
  uint32_t flags = 0;
  if (LARGEST) flags |= RADIK_LARGEST;
  if (needSorting) flags |= RADIK_SORTED;
  if (ASCEND) flags |= RADIK_ASCEND;
  if (WITHSCALE) flags |= RADIK_WITHSCALE;
  if (WITHIDXIN) flags |= RADIK_WITHIDXIN;
  if (sizeof(IdxType) == 8) flags |= RADIK_IDX64;
  int n_max = 0;
  for (int i = 0; i < taskNum; ++i) n_max = taskLen[i] > n_max ? taskLen[i] : n_max;
  const size_t bytes = radik_b200_compat::workspace_bytes(dtype, K, n_max, taskNum);
  radik_b200_compat::check(radik_topk(dtype, flags, valIn, idxIn, valOut, idxOut, workSpace, bytes, taskLen, taskNum,
                                      K, static_cast<void*>(stream)));
#ifndef RADIK_B200_ASYNC
  if (taskNum > 0 && K > 0) radik_b200_compat::check(radik_get_status(workSpace, static_cast<void*>(stream), nullptr));
#endif
}

#endif /* RADIK_B200_TOPK_RADIXSELECT_H_ */

// radik_cli.cu -- benchmark driver with the command line and output of RadiK's
// test_radik.out (radik/test/test_radik.cu:225-253, :184), so RadiK's
// evaluation scripts (eval/libs/radik.py:22-33) run unchanged against this
// library: point their binary path at radik_b200/bin/test_radik_b200.
//
//   test_radik_b200 BATCH LOG2_N K RANDOM_TASK SCALING [DISTRIBUTION [BATCHED [PADDING [SORTING]]]]
//
// Prints "batchSize: B, K: K", one "[i, len]" line per task and
// "elapsed: <ms> ms" for the timed call(s).  Same defaults as the original
// driver: smallest-k (LARGEST = 0), ascending order, int32 indices, fp32.
// DISTRIBUTION: 0 U(0,1) (cuRAND, seed 1234), 1 U[0.6, 0.7], 2 U[128.6, 128.7]
// (std::uniform_real_distribution, default_random_engine seeded 1), 3 Zipf(len,
// 1.1) ranks scaled by 1/len, 4 all zero.  RANDOM_TASK = 1 draws task lengths
// uniformly in [0.9 N, 1.1 N].  BATCHED = 0 calls once per task.  PADDING
// (RadiK's vectorised-load switch) has no effect here.
// The call goes through include/topk_radixselect.h, RadiK's own entry points.

#include <cuda_runtime.h>
#include <curand.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <numeric>
#include <random>
#include <stdexcept>
#include <thread>
#include <vector>

#include "topk_radixselect.h"

#define CLI_CHECK(x)                                                                                   \
  do {                                                                                                 \
    cudaError_t e_ = (x);                                                                              \
    if (e_ != cudaSuccess) throw std::runtime_error(std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace {

constexpr bool kLargest = false;
constexpr bool kAscend = true;

// Zipf(N, s) integer ranks by rejection from a continuous bounding density
// (Crease, "Rejection sampling the Zipf distribution"): draw x from the
// density proportional to x^-s on [1, N] (with a flat piece on [0, 1]) by
// inverse CDF, take floor(x) + 1, accept with the ratio of the two densities.
class Zipf {
 public:
  Zipf(std::default_random_engine& g, long n, double s)
      : g_(g), s_(s), t_((std::pow((double)n, 1.0 - s) - s) / (1.0 - s)) {}
  long next() {
    std::uniform_real_distribution<double> u(0.0, 1.0);
    while (true) {
      const double p = u(g_);
      const double x = p * t_ <= 1.0 ? p * t_ : std::pow(p * t_ * (1.0 - s_) + s_, 1.0 / (1.0 - s_));
      const long r = (long)(x + 1.0);
      const double bound = r <= 1 ? 1.0 : std::pow(x, -s_);
      if (u(g_) < std::pow((double)r, -s_) / bound) return r;
    }
  }

 private:
  std::default_random_engine& g_;
  double s_, t_;
};

template <bool WITHSCALE>
void run(int batch, int n, int K, int random_task, int distribution, int batched, bool sorting) {
  std::vector<int> len(batch, n);
  if (random_task) {
    std::uniform_real_distribution<float> d((float)(n * 9 / 10), (float)(n * 11 / 10));
    std::default_random_engine g;
    g.seed(1);
    for (int& l : len) l = (int)d(g);
  }
  std::vector<int64_t> off(batch + 1, 0);
  for (int i = 0; i < batch; ++i) off[i + 1] = off[i] + len[i];
  const int64_t total = off[batch];
  const int max_len = *std::max_element(len.begin(), len.end());
  std::cout << "batchSize: " << batch << ", K: " << K << std::endl;
  for (int i = 0; i < batch; ++i) std::cout << "[" << i << ", " << len[i] << "]" << std::endl;

  float* val = nullptr;
  CLI_CHECK(cudaMalloc(&val, sizeof(float) * total));
  std::vector<float> host;
  if (distribution == 0) {
    curandGenerator_t gen;
    if (curandCreateGenerator(&gen, CURAND_RNG_PSEUDO_DEFAULT) != CURAND_STATUS_SUCCESS ||
        curandSetPseudoRandomGeneratorSeed(gen, 1234ULL) != CURAND_STATUS_SUCCESS ||
        curandGenerateUniform(gen, val, total) != CURAND_STATUS_SUCCESS)
      throw std::runtime_error("curand failed");
    curandDestroyGenerator(gen);
  } else if (distribution == 1 || distribution == 2) {
    host.resize(total);
    const float lo = distribution == 1 ? 0.6f : 128.6f, hi = distribution == 1 ? 0.7f : 128.7f;
    std::uniform_real_distribution<float> d(lo, hi);
    std::default_random_engine g;
    g.seed(1);
    for (float& v : host) v = d(g);
  } else if (distribution == 3) {
    host.resize(total);
    std::vector<std::thread> th;
    for (int i = 0; i < batch; ++i) {
      th.emplace_back([&, i] {
        std::default_random_engine g;
        g.seed(1);
        Zipf z(g, len[i], 1.1);
        for (int64_t j = off[i]; j < off[i + 1]; ++j) host[j] = (float)((double)z.next() / len[i]);
      });
    }
    for (auto& t : th) t.join();
  } else if (distribution == 4) {
    CLI_CHECK(cudaMemset(val, 0, sizeof(float) * total));
  } else {
    throw std::runtime_error("Bad distribution");
  }
  if (!host.empty()) CLI_CHECK(cudaMemcpy(val, host.data(), sizeof(float) * total, cudaMemcpyHostToDevice));

  float* vout = nullptr;
  int32_t* iout = nullptr;
  CLI_CHECK(cudaMalloc(&vout, sizeof(float) * (size_t)batch * K));
  CLI_CHECK(cudaMalloc(&iout, sizeof(int32_t) * (size_t)batch * K));
  size_t ws_bytes = 0;
  getRadixSelectLWorkSpaceSize<float>(K, max_len, batched ? batch : 1, &ws_bytes);
  void* ws = nullptr;
  CLI_CHECK(cudaMalloc(&ws, ws_bytes));
  cudaStream_t stream;
  CLI_CHECK(cudaStreamCreate(&stream));
  cudaEvent_t start, end;
  CLI_CHECK(cudaEventCreate(&start));
  CLI_CHECK(cudaEventCreate(&end));
  float ms = 0.f;
  CLI_CHECK(cudaEventRecord(start, stream));
  if (batched) {
    topKRadixSelectL<int32_t, kLargest, kAscend, WITHSCALE>(val, (const int32_t*)nullptr, vout, iout, ws, len.data(),
                                                            batch, K, stream, sorting);
  } else {
    for (int i = 0; i < batch; ++i)
      topKRadixSelectL<int32_t, kLargest, kAscend, WITHSCALE>(val + off[i], (const int32_t*)nullptr, vout + (size_t)K * i,
                                                              iout + (size_t)K * i, ws, len.data() + i, 1, K, stream,
                                                              sorting);
  }
  CLI_CHECK(cudaEventRecord(end, stream));
  CLI_CHECK(cudaEventSynchronize(end));
  CLI_CHECK(cudaEventElapsedTime(&ms, start, end));
  printf("elapsed: %f ms\n", ms);
  cudaEventDestroy(start);
  cudaEventDestroy(end);
  cudaStreamDestroy(stream);
  cudaFree(ws);
  cudaFree(iout);
  cudaFree(vout);
  cudaFree(val);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 6) {
    fprintf(stderr,
            "usage: %s BATCH LOG2_N K RANDOM_TASK SCALING [DISTRIBUTION [BATCHED [PADDING [SORTING]]]]\n", argv[0]);
    return 2;
  }
  const int batch = atoi(argv[1]);
  const int log2n = atoi(argv[2]);
  const int K = atoi(argv[3]);
  const int random_task = atoi(argv[4]);
  const int scaling = atoi(argv[5]);
  const int distribution = argc >= 7 ? atoi(argv[6]) : 0;
  const int batched = argc >= 8 ? atoi(argv[7]) : 1;
  const int sorting = argc >= 10 ? atoi(argv[9]) : 1;
  if (batch <= 0 || log2n < 0 || log2n > 30 || K <= 0) {
    fprintf(stderr, "bad arguments\n");
    return 2;
  }
  try {
    if (scaling)
      run<true>(batch, 1 << log2n, K, random_task, distribution, batched, sorting != 0);
    else
      run<false>(batch, 1 << log2n, K, random_task, distribution, batched, sorting != 0);
  } catch (const std::exception& e) {
    fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}

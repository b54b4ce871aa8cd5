// Host-side packing: copies many small host arrays into one (pinned) staging
// pool on several threads.  A batch of small dense QPs arrives as thousands
// of separate arrays (one CSC value array per matrix); one pass of parallel
// memcpy into the pool that is then copied to the device replaces a Python
// loop over the instances.  Host code only: no CUDA call.
#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

#include "common.cuh"

using namespace qtqp;

extern "C" int qtqp_host_gather(int32_t count, const uint64_t* h_src, const int64_t* h_bytes,
                                const int64_t* h_dst_off, void* h_dst, int32_t threads) {
  if (count < 0) return fail(QTQP_ERR_BAD_ARG, "qtqp_host_gather: negative count");
  if (count == 0) return QTQP_OK;
  if (h_src == nullptr || h_bytes == nullptr || h_dst_off == nullptr || h_dst == nullptr)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_host_gather: null argument");
  int64_t total = 0;
  for (int32_t i = 0; i < count; ++i) {
    if (h_bytes[i] < 0 || h_dst_off[i] < 0 || (h_bytes[i] > 0 && h_src[i] == 0))
      return fail(QTQP_ERR_BAD_ARG, "qtqp_host_gather: bad block " + std::to_string(i));
    total += h_bytes[i];
  }
  char* dst = static_cast<char*>(h_dst);
  auto copy_range = [&](int32_t lo, int32_t hi) {
    for (int32_t i = lo; i < hi; ++i)
      if (h_bytes[i] > 0)
        std::memcpy(dst + h_dst_off[i], reinterpret_cast<const void*>(h_src[i]),
                    size_t(h_bytes[i]));
  };
  int nt = threads > 0 ? threads
                       : int(std::min(16u, std::max(1u, std::thread::hardware_concurrency())));
  if (total < (int64_t(1) << 20)) nt = 1;  // small pools: threads cost more than they save
  nt = std::min<int>(nt, count);
  if (nt <= 1) {
    copy_range(0, count);
    return QTQP_OK;
  }
  // Contiguous ranges of blocks with about total / nt bytes each.
  std::vector<int32_t> cut(nt + 1, count);
  cut[0] = 0;
  int64_t acc = 0;
  int k = 1;
  for (int32_t i = 0; i < count && k < nt; ++i) {
    acc += h_bytes[i];
    if (acc * nt >= total * k) cut[k++] = i + 1;
  }
  std::vector<std::thread> pool;
  pool.reserve(nt - 1);
  for (int t = 1; t < nt; ++t) pool.emplace_back(copy_range, cut[t], cut[t + 1]);
  copy_range(cut[0], cut[1]);
  for (auto& th : pool) th.join();
  return QTQP_OK;
}

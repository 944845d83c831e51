// multi_device.cpp -- one exact permanent sharded over several devices of
// this process.
//
// Restates gpu_perman64_xshared_coalescing_mshared_multigpu
// (gpu_exact_dense.cu:702-775): the Gray range [0, 2^(n-1)) is cut into one
// contiguous range per device, every device computes its starting X directly
// and walks its range, and the host adds the per-device sums.  Here each
// shard runs through perm_exact_dense_ex on its own context in its own host
// thread (the reference runs one OpenMP thread per device), the shard
// boundaries are perm_shard_range's (device-independent), and the 16-byte
// (hi, lo) partials are added in shard order with TwoSum, so the result does
// not depend on which device finished first.  Uses only the public C ABI.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <exception>
#include <string>
#include <thread>
#include <vector>

#include "../../include/perman_b200.h"

namespace {

constexpr int kMaxShards = 64;

// (hi, lo) += (h, l) in double-double (TwoSum on the high parts)
void dd_accumulate(double& hi, double& lo, double h, double l) {
  const double s = hi + h, bb = s - hi;
  const double e = (hi - (s - bb)) + (h - bb);
  hi = s;
  lo += e + l;
}

}  // namespace

extern "C" int perm_exact_dense_multi(const void* mat, int n, int dtype, int variant, int nshards,
                                      const int* devices, perm_result* out) {
  if (!mat || !out || n < 1 || n > PERM_MAX_EXACT_N || nshards < 1 || nshards > kMaxShards) return PERM_EINVAL;
  if (dtype != PERM_F64 && dtype != PERM_F32 && dtype != PERM_I32) return PERM_EINVAL;
  std::vector<perm_result> parts(nshards);
  std::vector<int> rcs(nshards, PERM_OK);
  std::vector<std::string> errs(nshards);
  std::vector<std::thread> threads;
  threads.reserve(nshards);
  for (int s = 0; s < nshards; s++) {
    auto run = [&, s] {
      perm_ctx* ctx = nullptr;
      const int dev = devices ? devices[s] : s;
      rcs[s] = perm_ctx_create(dev, &ctx);
      if (rcs[s] != PERM_OK) {
        errs[s] = "cannot create a context on device " + std::to_string(dev);
        return;
      }
      perm_ctx_set_rel_target(ctx, -1.0);  // one evaluation per shard, no accuracy policy
      rcs[s] = perm_exact_dense_ex(ctx, mat, n, dtype, variant, s, nshards, &parts[s]);
      if (rcs[s] != PERM_OK) errs[s] = perm_ctx_last_error(ctx);
      perm_ctx_destroy(ctx);
    };
    try {
      threads.emplace_back(run);
    } catch (const std::exception& e) {  // no thread for this shard: fail it, keep the started ones
      for (int t = s; t < nshards; t++) {
        rcs[t] = PERM_ENOMEM;
        errs[t] = std::string("cannot start a host thread: ") + e.what();
      }
      break;
    }
  }
  for (auto& t : threads) t.join();
  for (int s = 0; s < nshards; s++) {
    if (rcs[s] != PERM_OK) {
      fprintf(stderr, "perman_b200: shard %d (device %d): %s: %s\n", s, devices ? devices[s] : s,
              perm_status_string(rcs[s]), errs[s].c_str());
      return rcs[s];
    }
  }
  double hi = 0.0, lo = 0.0, steps = 0.0, abs_sum = 0.0, ms = 0.0;
  for (int s = 0; s < nshards; s++) {
    dd_accumulate(hi, lo, parts[s].hi, parts[s].lo);
    steps += parts[s].steps;
    abs_sum += parts[s].abs_term_sum;
    ms = std::max(ms, parts[s].kernel_ms);  // the shards run concurrently
  }
  *out = parts[0];
  out->hi = hi + lo;
  out->lo = lo - (out->hi - hi);
  out->value = out->hi;
  out->steps = steps;
  out->total_steps = std::ldexp(1.0, n - 1);
  out->kernel_ms = ms;
  out->abs_term_sum = abs_sum;  // 0: shards carry no estimate
  out->rel_error_estimate = 0.0;  // not estimated: perm_exact_dense_refine applies the policy
  return PERM_OK;
}

// reference signature: devices 0 .. gpu_num - 1 (at most the visible ones),
// one evaluation; NaN and a message on stderr on failure
template <class T>
static double shim_multigpu(const T* mat, int nov, int gpu_num, int dtype) {
  const int avail = perm_device_count();
  if (avail < 1) {
    fprintf(stderr, "perman_b200: no CUDA device\n");
    return NAN;
  }
  const int g = std::max(1, std::min(gpu_num, std::min(avail, kMaxShards)));
  perm_result r;
  if (perm_exact_dense_multi(mat, nov, dtype, 0, g, nullptr, &r) != PERM_OK) return NAN;
  return r.value;
}

extern "C" {
double gpu_perman64_xshared_coalescing_mshared_multigpu_int(int* mat, int nov, int gpu_num, int, int) {
  return shim_multigpu(mat, nov, gpu_num, PERM_I32);
}
double gpu_perman64_xshared_coalescing_mshared_multigpu_float(float* mat, int nov, int gpu_num, int, int) {
  return shim_multigpu(mat, nov, gpu_num, PERM_F32);
}
double gpu_perman64_xshared_coalescing_mshared_multigpu_double(double* mat, int nov, int gpu_num, int, int) {
  return shim_multigpu(mat, nov, gpu_num, PERM_F64);
}
}  // extern "C"

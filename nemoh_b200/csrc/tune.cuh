// Autotuner of the triangular sweep's tile shape.
//
// Two sweeps solve the same systems (linalg.cuh): the cluster sweep spreads
// the 64-row blocks of one system over a thread-block cluster of csize CTAs
// (1, 2, 4 or 8; a larger cluster puts more SMs on one system's updates but
// adds cluster barriers and distributed-shared-memory copies per step), the
// dataflow sweep (SWEEP_FLOW) spreads the row blocks of all systems over a
// persistent grid that follows ready flags. The fastest choice depends on the
// number of systems in the batch, their order, the precision and the number
// of right-hand sides. The tuner times every candidate once per key (device,
// element type, power-of-two buckets of the order, of the system count and
// of the right-hand sides), after one untimed run of it, on a copy of the
// batch's right-hand sides, keeps
// the fastest for the life of the process, and then solves with it. Under
// stream capture (no timing possible) and before a key has been tuned without
// scratch, trsm_sweep's default decides.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cfloat>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>

#include "linalg.cuh"

namespace nb200 {

struct SweepTuner {
  std::mutex mu;
  std::map<unsigned long long, int> best;   // key -> cluster size
  void* scratch[64] = {};                   // per device: right-hand sides kept while candidates run
  size_t scratch_bytes[64] = {};
  long long tuned = 0;                      // keys tuned so far (diagnostics)
};

inline SweepTuner& sweep_tuner() {
  static SweepTuner t;
  return t;
}

inline int log2_bucket(long long v) {
  int b = 0;
  while ((1LL << b) < v) ++b;
  return b;
}

inline unsigned long long sweep_key(int dev, bool f32, int n, int nsys, int nrhs) {
  return ((unsigned long long)dev << 40) | ((unsigned long long)f32 << 32) |
         ((unsigned long long)log2_bucket(n) << 16) | ((unsigned long long)log2_bucket(nsys) << 8) |
         (unsigned long long)log2_bucket(nrhs);
}

// cluster size cached for this batch's key, 0 if none yet
template <class C2>
inline int sweep_tuned_size(const BatchT<C2>& b, int nsys, int nrhs) {
  int dev = 0;
  cudaGetDevice(&dev);
  SweepTuner& t = sweep_tuner();
  std::lock_guard<std::mutex> lock(t.mu);
  auto it = t.best.find(sweep_key(dev, sizeof(C2) == sizeof(float2), b.n, nsys, nrhs));
  return it == t.best.end() ? 0 : it->second;
}

// trsm_sweep with the tuned cluster size; tunes the key first when it is new
// and the stream is not being captured. X: right-hand sides in, solution out.
// NEMOH_B200_SWEEP=flow or =cluster fixes the choice (tests, diagnosis):
// the dataflow sweep where a workspace is given, or the cluster sweep with
// its SM-count cluster size.
inline int sweep_forced() {
  static const int f = [] {
    const char* e = std::getenv("NEMOH_B200_SWEEP");
    if (!e) return 0;
    if (std::strcmp(e, "flow") == 0) return SWEEP_FLOW;
    if (std::strcmp(e, "cluster") == 0) return -1;
    return 0;
  }();
  return f;
}

// autotuning on (default) or off (nemoh_b200_set_autotune): off, a shape not
// tuned yet takes trsm_sweep's default instead of timing the candidates (a
// server keeps timing runs, and the lock they hold, off its requests' path)
inline std::atomic<bool>& sweep_autotune_flag() {
  static std::atomic<bool> on{true};
  return on;
}
inline void set_sweep_autotune(bool on) { sweep_autotune_flag().store(on); }

template <class C2>
inline cudaError_t trsm_sweep_tuned(BatchT<C2> b, const C2* inv, C2* X, C2* Y, int nsys, int nrhs, cudaStream_t st,
                                    long long& launches, const int* active = nullptr, SweepSync sync = SweepSync()) {
  const int forced = sweep_forced();
  if (forced == -1) return trsm_sweep<C2>(b, inv, X, Y, nsys, nrhs, st, launches, active, 0, SweepSync());
  if (forced == SWEEP_FLOW && sync.ws)
    return trsm_sweep<C2>(b, inv, X, Y, nsys, nrhs, st, launches, active, SWEEP_FLOW, sync);
  int csize = sweep_tuned_size(b, nsys, nrhs);
  if (csize > 0 && (csize != SWEEP_FLOW || sync.ws))
    return trsm_sweep<C2>(b, inv, X, Y, nsys, nrhs, st, launches, active, csize, sync);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (!sweep_autotune_flag().load() || cudaStreamIsCapturing(st, &cap) != cudaSuccess ||
      cap != cudaStreamCaptureStatusNone)
    return trsm_sweep<C2>(b, inv, X, Y, nsys, nrhs, st, launches, active, 0, sync);
  int dev = 0;
  cudaGetDevice(&dev);
  const unsigned long long key = sweep_key(dev, sizeof(C2) == sizeof(float2), b.n, nsys, nrhs);
  const size_t bytes = (size_t)nsys * b.n * nrhs * sizeof(C2);
  SweepTuner& t = sweep_tuner();
  std::lock_guard<std::mutex> lock(t.mu);
  cudaError_t e;
  if (dev < 0 || dev >= 64) return trsm_sweep<C2>(b, inv, X, Y, nsys, nrhs, st, launches, active, 0, sync);
  void*& scratch = t.scratch[dev];
  if (t.scratch_bytes[dev] < bytes) {
    cudaFree(scratch);
    scratch = nullptr;
    t.scratch_bytes[dev] = 0;
    if ((e = cudaMalloc(&scratch, bytes)) != cudaSuccess) return e;
    t.scratch_bytes[dev] = bytes;
  }
  if ((e = cudaMemcpyAsync(scratch, X, bytes, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
  cudaEvent_t ev[2];
  cudaEventCreate(&ev[0]);
  cudaEventCreate(&ev[1]);
  const int nblk = (b.n + TB - 1) / TB;
  float best_ms = FLT_MAX;
  int best_c = 0;
  int cands[5], nc = 0;
  for (int c = 1; c <= 8 && c <= nblk; c *= 2) cands[nc++] = c;
  if (sync.ws) cands[nc++] = SWEEP_FLOW;
  for (int ci = 0; ci < nc; ++ci) {
    const int c = cands[ci];
    long long l = 0;
    // one untimed run first (first-launch setup on the host, cold caches),
    // then the timed one
    cudaMemcpyAsync(X, scratch, bytes, cudaMemcpyDeviceToDevice, st);
    if (trsm_sweep<C2>(b, inv, X, Y, nsys, nrhs, st, l, active, c, sync) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    cudaMemcpyAsync(X, scratch, bytes, cudaMemcpyDeviceToDevice, st);
    cudaEventRecord(ev[0], st);
    e = trsm_sweep<C2>(b, inv, X, Y, nsys, nrhs, st, l, active, c, sync);
    cudaEventRecord(ev[1], st);
    if (e != cudaSuccess) {   // e.g. a cluster that cannot be scheduled: not a candidate
      cudaGetLastError();
      continue;
    }
    float ms = 0.f;
    if (cudaEventSynchronize(ev[1]) != cudaSuccess || cudaEventElapsedTime(&ms, ev[0], ev[1]) != cudaSuccess) continue;
    if (ms < best_ms) {
      best_ms = ms;
      best_c = c;
    }
  }
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  if (!best_c) return cudaErrorLaunchFailure;
  t.best[key] = best_c;
  ++t.tuned;
  if ((e = cudaMemcpyAsync(X, scratch, bytes, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
  return trsm_sweep<C2>(b, inv, X, Y, nsys, nrhs, st, launches, active, best_c, sync);
}

}  // namespace nb200

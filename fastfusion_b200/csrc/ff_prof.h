// Per-stage device timing with CUDA events on the map's stream (internal).
// Off by default; when on, each stage launch is bracketed by two events and
// its algorithmic byte count is recorded; ff_profile_read resolves them.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace ffb {

enum Stage {
  ST_GROW = 0,
  ST_DEDUPE,
  ST_INSERT,
  ST_FINALIZE,
  ST_FUSE,
  ST_MESH_CELLS,
  ST_MESH_COUNT,
  ST_MESH_EMIT,
  ST_CONFIDENCE,  // learned weight: features and the three convolution layers
  ST_COUNT
};

struct Prof {
  bool on = false;
  struct Rec {
    int stage;
    cudaEvent_t a, b;
    double bytes;
  };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  double ms[ST_COUNT] = {0};
  double bytes[ST_COUNT] = {0};
  uint64_t launches[ST_COUNT] = {0};

  cudaEvent_t get() {
    cudaEvent_t e;
    if (!pool.empty()) {
      e = pool.back();
      pool.pop_back();
    } else {
      cudaEventCreate(&e);
    }
    return e;
  }
  int begin(int stage, cudaStream_t s) {
    if (!on) return -1;
    Rec r{stage, get(), get(), 0.0};
    cudaEventRecord(r.a, s);
    recs.push_back(r);
    return (int)recs.size() - 1;
  }
  void end(int idx, double nbytes, cudaStream_t s) {
    if (idx < 0) return;
    recs[idx].bytes = nbytes;
    cudaEventRecord(recs[idx].b, s);
  }
  void set_bytes(int idx, double nbytes) {
    if (idx >= 0 && idx < (int)recs.size()) recs[idx].bytes = nbytes;
  }
  void flush() {
    for (auto &r : recs) {
      cudaEventSynchronize(r.b);
      float t = 0.0f;
      cudaEventElapsedTime(&t, r.a, r.b);
      ms[r.stage] += t;
      bytes[r.stage] += r.bytes;
      launches[r.stage]++;
      pool.push_back(r.a);
      pool.push_back(r.b);
    }
    recs.clear();
  }
  void reset() {
    flush();
    for (int i = 0; i < ST_COUNT; i++) ms[i] = bytes[i] = 0, launches[i] = 0;
  }
  void destroy() {
    flush();
    for (auto e : pool) cudaEventDestroy(e);
    pool.clear();
  }
};

}  // namespace ffb

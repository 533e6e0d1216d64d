// The context object behind glc_ctx*, shared by the translation units that launch traces.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "../../include/glc.h"

struct glc_ctx {
  int device = 0;
  int sm_count = 0;
  glc_policy policy{};
  unsigned char* d_job = nullptr;
  size_t d_job_bytes = 0;
  unsigned char* h_stage = nullptr;
  size_t h_stage_bytes = 0;
  cudaEvent_t stage_free = nullptr;  // recorded after the last staging copy
  bool stage_pending = false;
  unsigned long long* d_queue = nullptr;
  uint32_t* d_cert = nullptr;          // per-tile capture certificates (grow-only)
  size_t d_cert_words = 0;
  uint32_t* d_emap = nullptr;          // packed escape-map nodes (grow-only)
  size_t d_emap_words = 0;
  uint32_t* d_shadow = nullptr;        // shadow-edge list: counter word pair, then u64 entries (grow-only)
  size_t d_shadow_words = 0;
  uint32_t* d_footprint = nullptr;     // surface-footprint pixel list: counter word pair, then u64 entries
  size_t d_footprint_words = 0;
  unsigned char* d_host_ws = nullptr;  // device workspace of glc_trace_host (grow-only)
  unsigned char* d_handoff = nullptr;  // MIXED two-kernel hand-off records (grow-only)
  size_t d_handoff_bytes = 0;
  cudaStream_t host_compute[2] = {};  // glc_trace_host: bands are traced on two streams in turn ...
  cudaStream_t host_copy = nullptr;    // ... and copied back on a third
  cudaEvent_t host_upload = nullptr;   // the job table is on the device
  cudaEvent_t host_band[64] = {};      // band k traced
  cudaEvent_t host_entry = nullptr;    // orders a banded host trace after the legacy stream's work
  size_t d_host_ws_bytes = 0;
  glc_launch_stats stats{};
};

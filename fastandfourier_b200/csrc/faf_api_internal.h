// faf_api_internal.h -- helpers shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include "faf_plan.h"
#include "fastandfourier.h"

namespace fafapi {

int fail(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);
void note_launches(int k);
fafp::DevicePlan* plan_of(const faf_transform* t);
int ptr_is_device(const void* p);

bool is_5_smooth(size_t n);
bool is_7_smooth(size_t n);
bool is_prime(size_t n);
bool is_codelet(size_t n);
bool rader_eligible(size_t n);
size_t next_5_smooth(size_t m);

faf_transform* alloc_transform();
void apply_resolved(faf_transform* t, const faf_config& c);
float norm_scale(faf_norm norm, bool inverse, size_t n);
double norm_scale64(faf_norm norm, bool inverse, size_t n);
bool backend_ok(const faf_config& c, bool fp64_ok = false);

int exec_split_one(const faf_transform* t, void* out_re, void* out_im, const void* in_re,
                   const void* in_im);

// Pipeline op resolution (chirp.cpp) -> device op list; returns the number of
// ops or -1; sets *host_ops when an op needs the host round trip.
int resolve_pipeline_ops(const faf_transform* t, fafk::PipeOp* ops, int cap, bool* host_ops,
                         cudaStream_t st);
// Apply the pipeline's ops on host split-plane bins (host round-trip path).
void apply_ops_host(const faf_transform* t, float* re, float* im, size_t nb);

}  // namespace fafapi

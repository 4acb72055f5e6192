// nrc.h — entry points of the radiance cache shared with the path tracer
// (batch sizes read from a device counter, so no host synchronisation).
#pragma once
#include <cuda_runtime.h>

#include "../../include/strelka_b200.h"

// col[slot] += throughput * max(prediction, 0) for queries [0, *count) (out == NULL),
// or out[3*i + c] = prediction.
int nrc_infer_device(StrelkaNrc* nrc, const StrelkaNrcRecord* recs, const uint32_t* count, uint32_t maxN, float* out,
                     float4* col, uint32_t* status, cudaStream_t st);
// Gradients of the batch [0, *count) into the cache's gradient buffers.
int nrc_gradients_device(StrelkaNrc* nrc, const StrelkaNrcRecord* recs, const uint32_t* count, uint32_t maxN,
                         cudaStream_t st);
// One Adam step with the gradients of a batch of `batch` records (or of
// *count records when count is not NULL).
int nrc_adam_device(StrelkaNrc* nrc, float batch, cudaStream_t st);
int nrc_adam_device_count(StrelkaNrc* nrc, float batch, const uint32_t* count, cudaStream_t st);

// Library-internal entry points of the radiance-cache network (nrc.cu) for
// callers that keep the row count in device memory (the path tracer's queues):
// nothing here synchronises, so a whole frame can be enqueued (or captured)
// without a host round trip.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "illume_gpu.h"

namespace ilm {

// Rows to process: n = min(*dev, cap) (or cap when dev is null); with
// batches > 1, only batch `batch` of the interleaved split: rows r with
// r % batches == batch, which the caller has stored contiguously.
struct NrcCount {
    const unsigned long long* dev;
    uint32_t cap;
    uint32_t batches;
    uint32_t batch;
};

// out[n][3] = network(raw[n][12]) with the inference weights.
cudaError_t nrc_infer_async(ilm_nrc* h, const float* raw, NrcCount n, float* out, cudaStream_t s);
// One Adam step on (raw[n][12], target[n][3]); the loss sum is added to the
// network's loss word.
cudaError_t nrc_train_async(ilm_nrc* h, const float* raw, const float* target, NrcCount n, cudaStream_t s);
// Grows the training buffers to `rows` rows per step, so that later steps of
// at most that many rows allocate nothing (and can be captured in a graph).
cudaError_t nrc_reserve(ilm_nrc* h, uint32_t rows);
// The network's device error word (non-zero after a tensor-core wait timed out).
uint32_t* nrc_error_word(ilm_nrc* h);

}  // namespace ilm

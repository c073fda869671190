// Host-side state of the wavefront path tracer (pt.cu).  Included by
// context.h after DeviceBuffer is defined.
#pragma once
#include <cuda_runtime.h>

#include "illume_gpu.h"

namespace ilm {

// Queues and film, reused across renders of one scene (grown on demand).
struct PtBuffers {
    DeviceBuffer rays[2], beta[2], rng[2], pid[2];   // path queues (double-buffered)
    DeviceBuffer hits;
    DeviceBuffer srays, scontrib, socc;              // shadow queue
    DeviceBuffer counts;
    DeviceBuffer film, out;
    DeviceBuffer ftable, wsum;                       // film filter table and weight sums
    // radiance-cache mode: spread per path, cache queries, training records
    DeviceBuffer spread[2], q_in, q_beta, q_train, q_out, t_rec, t_count, s_train, t_in, t_tg;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // radiance-cache mode: the training branch's stream, fork/join events, and
    // the batch layout (batches, rows per batch) of the kept training samples
    cudaStream_t train_stream = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    uint32_t train_layout[2] = {0, 0};
    ~PtBuffers() {
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
        if (stream) cudaStreamDestroy(stream);
        if (train_stream) cudaStreamDestroy(train_stream);
    }
};

struct PtScene {
    ilm_accel_id accel = 0;
    ilm_pt_scene_desc desc{};
    float bound[6] = {0, 0, 0, 0, 0, 0};   // world bound of the accel (min xyz, max xyz)
    DeviceBuffer d_tri, d_mat, d_lights, d_light_geo;
    uint32_t n_lights = 0;
    PtBuffers buf;
};

}  // namespace ilm

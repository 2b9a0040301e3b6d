// Internal definitions of the C-ABI handles (include/tlno_gpu.h), shared by
// the translation units that implement the entry points.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/tlno_gpu.h"
#include "engine.hpp"
#include "plan.hpp"

namespace tlno_gpu {
// Sets the calling thread's tlno_gpu_last_error() text.
void set_last_error(const std::string& message);
// Resolves (once per device, current device = `device`) the device address
// of the fixed scratch of tlno_gpu_eri_blocks_noalloc.
void noalloc_prepare(int device);

// Auxiliary streams and fork/join events of a build whose class launches
// run on several streams (created on first use, destroyed with the owner).
struct StreamFan {
    int device = 0;
    std::vector<cudaStream_t> aux;
    std::vector<cudaEvent_t> ev;
    void ensure(int n_aux);
    ~StreamFan();
};

struct JkWork {
    DeviceBuffer D, J, K, G, dmax, status;
    DeviceBuffer D32;  // FP32 copy of the density for the FP32 kernels (mixed builds)
};
}  // namespace tlno_gpu

struct tlno_gpu_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    tlno_gpu::Basis basis;
    std::unique_ptr<tlno_gpu::Plan2e> plan;
    tlno_gpu_screening screening{1e-12, 0, 0, 0, 1e-9};
    tlno_gpu::Tuning tune;
    tlno_gpu::OneePlan onee;
    int onee_state = -1;  // screening flag the 1e plan was built with
    double onee_decay_eps = 1e-15, onee_nuclear_eps = 1e-15;
    tlno_gpu::DeviceBuffer d_shell_xyz, d_shell_L, d_shell_nprim, d_shell_prim, d_shell_sph, d_exps, d_crad;
    tlno_gpu::DeviceBuffer d_comp_coef, d_comp_off;
    tlno_gpu::JkWork w;
    tlno_gpu::StreamFan fan;
    tlno_gpu::DeviceBuffer d_S, d_T, d_V;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;

    ~tlno_gpu_context() {
        if (device >= 0) cudaSetDevice(device);
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        if (stream) cudaStreamDestroy(stream);
    }
};

struct tlno_gpu_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<tlno_gpu::Basis> bases;
    tlno_gpu::Plan2e plan;
    tlno_gpu_screening screening{};
    tlno_gpu::Tuning tune;
    tlno_gpu::JkWork w;
    tlno_gpu::StreamFan fan;
    long long total = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    ~tlno_gpu_batch() {
        cudaSetDevice(device);
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        if (stream) cudaStreamDestroy(stream);
    }
};


// pipeline.cuh -- device context and the per-k-block solve pipeline.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "../../include/dvr3d_b200.h"
#include "common.cuh"
#include "host_setup.h"
#include "pes.cuh"

namespace dvr3d {

// Device buffers keyed by name, grown on demand and reused across solves.
class DeviceArena {
  public:
    ~DeviceArena();
    void *get(const std::string &name, size_t bytes);
    template <class T>
    T *get_t(const std::string &name, size_t count) {
        return static_cast<T *>(get(name, count * sizeof(T)));
    }
    size_t bytes_held() const;
    void release_all();

  private:
    struct Buf {
        void *p = nullptr;
        size_t bytes = 0;
    };
    std::map<std::string, Buf> bufs_;
};

struct CudaFail {
    cudaError_t err;
    std::string where;
};

}  // namespace dvr3d

struct dvr3d_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;     // stream all work of this context is issued on
    cudaStream_t own_stream = nullptr; // the stream the context created (destroyed with it)
    std::string last_error;
    dvr3d::PesParams pes{};
    std::vector<double> pes_grid;  // host copy of a tabulated PES
    dvr3d::DeviceArena arena;
    cudaEvent_t ev[8] = {};
    int sm_count = 0;
    int dense_grid = 0;
    std::vector<cudaEvent_t> panel_ev;  // timing pool for the reduction panels
};

namespace dvr3d {

// Solve one k block. Throws HostError / CudaFail.
void solve_block(dvr3d_ctx *ctx, const dvr3d_deck &deck, int kk, const dvr3d_options &opt,
                 dvr3d_result &res);

}  // namespace dvr3d

// Shared helpers of the reference-ABI plugin libraries (device buffers, error mapping).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include "gap_b200/gap_interfaces.hpp"
#include "gapk.h"

namespace gapb200 {

// Throws std::runtime_error, the reference backends' error convention across the dlopen
// boundary (e.g. src/solver/powerflow/gpu/gpu_newton_raphson.cu:125-130).
inline void check(int rc, const char* what) {
    if (rc != GAPK_OK) throw std::runtime_error(std::string(what) + ": " + gapk_last_error());
}
inline void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// Grow-only device buffer.
struct DeviceBuffer {
    void* p = nullptr;
    size_t cap = 0;
    DeviceBuffer() = default;
    DeviceBuffer(DeviceBuffer const&) = delete;
    DeviceBuffer& operator=(DeviceBuffer const&) = delete;
    ~DeviceBuffer() {
        if (p) cudaFree(p);
    }
    void* ensure(size_t bytes) {
        if (bytes > cap) {
            if (p) cudaFree(p);
            p = nullptr;
            cap = 0;
            check_cuda(cudaMalloc(&p, bytes ? bytes : 16), "cudaMalloc");
            cap = bytes;
        }
        return p;
    }
    template <typename T>
    T* upload(std::vector<T> const& v) {
        void* d = ensure(v.size() * sizeof(T));
        if (!v.empty())
            check_cuda(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice),
                       "cudaMemcpy H2D");
        return static_cast<T*>(d);
    }
    template <typename T>
    void download(std::vector<T>& v, size_t n) const {
        v.resize(n);
        if (n) check_cuda(cudaMemcpy(v.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost),
                          "cudaMemcpy D2H");
    }
};

// Bus ID -> position as the reference builds it (src/admittance/cpu/cpu_admittance_matrix.cpp:
// 56-73): sized max_id + 1, later duplicates win, negative IDs never mapped.
inline std::vector<int> id_to_index(gap::NetworkData const& net, int& max_id) {
    max_id = -1;
    for (auto const& b : net.buses) max_id = std::max(max_id, b.id);
    std::vector<int> lut(max_id + 1 > 0 ? max_id + 1 : 0, -1);
    for (size_t i = 0; i < net.buses.size(); ++i) {
        int id = net.buses[i].id;
        if (id >= 0 && id <= max_id) lut[id] = static_cast<int>(i);
    }
    return lut;
}

}  // namespace gapb200

// vt_host.cuh -- host-side helpers shared by the engine and the updateable tessellation:
// grow-only device buffers, CUDA error propagation as C-ABI status codes, the result
// object handed across the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <new>
#include <string>
#include <vector>

#include "../../include/voronota_b200.h"

namespace vt {

// Sets the calling thread's message for vt_last_error().
void set_last_error(const std::string& msg);

struct CudaError {
    int status;
};

#define VT_CUDA(call)                                                                       \
    do {                                                                                    \
        cudaError_t _e = (call);                                                            \
        if (_e != cudaSuccess) {                                                            \
            ::vt::set_last_error(std::string(#call) + ": " + cudaGetErrorString(_e));      \
            throw ::vt::CudaError{_e == cudaErrorMemoryAllocation ? VT_ERR_OOM : VT_ERR_CUDA}; \
        }                                                                                   \
    } while (0)

// Grow-only device buffer; contents are not preserved across growth.
template <typename T>
struct DBuf {
    T* p = nullptr;
    size_t cap = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void ensure(size_t n) {
        if (n <= cap && p) return;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t c = std::max<size_t>(n + n / 4, 64);
        VT_CUDA(cudaMalloc(&p, c * sizeof(T)));
        cap = c;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    void swap(DBuf& o) {
        std::swap(p, o.p);
        std::swap(cap, o.cap);
    }
    // device-to-device copy of the first n elements of `src`
    void copy_from(const DBuf& src, size_t n, cudaStream_t s) {
        if (n == 0) return;
        ensure(n);
        VT_CUDA(cudaMemcpyAsync(p, src.p, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
    }
};

// Runs f() and turns exceptions into status codes (nothing crosses the C ABI).
template <typename F>
int guarded(F&& f) {
    try {
        return f();
    } catch (const CudaError& e) {
        return e.status;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return VT_ERR_OOM;
    } catch (...) {
        set_last_error("unexpected exception");
        return VT_ERR_CUDA;
    }
}

// Page-locked host blocks for results, recycled through a process-wide pool so that a
// result is copied from the device by DMA without a bounce buffer or a zero-fill.
// Falls back to malloc when page-locked memory is not available.
void* host_block_acquire(size_t bytes, size_t* cap, bool* pinned);
void host_block_release(void* p, size_t cap, bool pinned);

// Uninitialised host array in a pooled block (resize discards the contents).
template <typename T>
struct HostArr {
    T* p = nullptr;
    size_t n = 0, capb = 0;
    bool pinned = false;
    HostArr() = default;
    HostArr(const HostArr&) = delete;
    HostArr& operator=(const HostArr&) = delete;
    ~HostArr() { release(); }
    void release() {
        if (p) host_block_release(p, capb, pinned);
        p = nullptr;
        n = capb = 0;
    }
    void resize(size_t m) {
        if (m * sizeof(T) > capb || !p) {
            release();
            p = (T*)host_block_acquire(std::max<size_t>(m, 1) * sizeof(T), &capb, &pinned);
            if (!p) throw std::bad_alloc();
        }
        n = m;
    }
    T* data() { return p; }
    const T* data() const { return p; }
    size_t size() const { return n; }
};

}  // namespace vt

// Host copy of a tessellation result (TessellationResult, types.rs:69-95).
struct vt_result {
    uint64_t num_balls = 0;
    vt::HostArr<uint32_t> a, b;
    vt::HostArr<double> area, arc;
    vt::HostArr<uint8_t> central;
    vt::HostArr<uint32_t> cell_index;
    vt::HostArr<double> cell_sas, cell_vol;
    double totals[3] = {0, 0, 0};
    // tessellation network (with_cell_vertices): 4 / 3 ids per vertex / edge
    bool has_network = false;
    vt::HostArr<uint32_t> net_vid, net_eid;
    vt::HostArr<double> net_vxyz, net_elen;
};

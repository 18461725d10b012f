// smem_attr.cuh -- the dynamic shared-memory limit of a kernel, set once per
// device.  The attribute belongs to the kernel as loaded in one device's
// context, so a process that drives several GPUs (or creates handles on
// another device later) sets it on each; the per-call-site bit mask makes the
// check one atomic load after the first launch on a device.
#pragma once

#include <cuda_runtime.h>

#include <atomic>

namespace mhd3d {

inline cudaError_t smem_attr_once(std::atomic<unsigned long long>& done, const void* fn, size_t bytes)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

}  // namespace mhd3d

// emu_runtime.cpp -- host stand-ins for the CUDA runtime calls that
// emu_shim.h renames, the thread-index registers the shim's sequential
// launcher sets, and the members of mn::CudaDevice
// (Mine/system/CudaDevice/CudaDevice.h) that the reference's host code
// reaches (its device queries and occupancy-based block sizes have no
// meaning when every kernel runs one thread at a time).
//
// TEST INFRASTRUCTURE ONLY (oracle/ref/Makefile.refemu).
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "system/CudaDevice/CudaDevice.h"

uint3 threadIdx;
uint3 blockIdx;
dim3 blockDim;
dim3 gridDim;
int warpSize = 32;

extern "C" {
// Fresh allocations are zero-filled, as fresh device pages are.
cudaError_t emu_cudaMalloc(void **p, size_t n) {
    *p = std::calloc(n ? n : 1, 1);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t emu_cudaFree(void *p) {
    std::free(p);
    return cudaSuccess;
}
cudaError_t emu_cudaMemcpy(void *dst, const void *src, size_t n, enum cudaMemcpyKind) {
    if (n) std::memmove(dst, src, n);
    return cudaSuccess;
}
cudaError_t emu_cudaMemset(void *p, int v, size_t n) {
    if (n) std::memset(p, v, n);
    return cudaSuccess;
}
cudaError_t emu_cudaMemGetInfo(size_t *free_b, size_t *total_b) {
    *free_b = *total_b = (size_t)1 << 34;
    return cudaSuccess;
}
cudaError_t emu_cudaDeviceSynchronize(void) { return cudaSuccess; }
cudaError_t emu_cudaGetLastError(void) { return cudaSuccess; }
cudaError_t emu_cudaPeekAtLastError(void) { return cudaSuccess; }
}

namespace mn {
cudaDeviceProp *CudaDevice::_akDeviceProps = nullptr;
int CudaDevice::_iDevID = 0;
std::unordered_map<std::string, CudaDevice::KernelConfig> CudaDevice::_kFuncTable;

CudaDevice::KernelConfig::KernelConfig(KernelFunc f, cudaFuncCache cacheConfig, bool isWave)
    : func(f), cachePreference(cacheConfig), waveFashion(isWave), maxOccBlockSize(256) {
    std::memset(&attribs, 0, sizeof(attribs));
}
CudaDevice::CudaDevice() { std::printf("# host emulation: kernels run one thread at a time\n"); }
CudaDevice::~CudaDevice() {}
int CudaDevice::generalGridSize(int &threadNum, int &blockSize) const {
    return (threadNum + blockSize - 1) / blockSize;
}
int CudaDevice::waveGridSize(int &threadNum, int &blockSize) const { return generalGridSize(threadNum, blockSize); }
int CudaDevice::evalOptimalBlockSize(cudaFuncAttributes, cudaFuncCache, size_t) { return 256; }
ExecutionPolicy CudaDevice::launchConfig(const std::string &, int threadNum, bool sync, size_t smemSize,
                                         cudaStream_t) const {
    int bs = 256;
    return {generalGridSize(threadNum, bs), bs, smemSize, sync};
}
void CudaDevice::registerKernel(const std::string &tag, KernelFunc f, cudaFuncCache cacheConfig, bool waveFashion) {
    _kFuncTable.emplace(tag, KernelConfig(f, cacheConfig, waveFashion));
}
const CudaDevice::KernelConfig &CudaDevice::findKernel(const std::string &tag) { return _kFuncTable[tag]; }
}  // namespace mn

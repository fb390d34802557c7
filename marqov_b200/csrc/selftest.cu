// Philox self test: the engine's Philox4x32-10 against cuRAND's
// Philox4_32_10 generator, both evaluated on the device.  cuRAND is only
// called (curand_init / curand4), never restated: a state initialised with
// (seed, subsequence = c2 | c3 << 32, offset = 4 * (c0 | c1 << 32)) yields the
// Philox block of counter (c0, c1, c2, c3) under key (lo32 seed, hi32 seed).
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include "engine.h"

namespace mqv {

__global__ void selftest_philox_kernel(uint64_t seed, uint32_t c1, uint32_t c2, uint32_t c3, int n,
                                       uint32_t* __restrict__ eng, uint32_t* __restrict__ cur)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint4 e = philox((uint32_t)i, c1, c2, c3, make_key(seed));
    eng[4 * i + 0] = e.x;
    eng[4 * i + 1] = e.y;
    eng[4 * i + 2] = e.z;
    eng[4 * i + 3] = e.w;
    curandStatePhilox4_32_10_t st;
    const unsigned long long sub = (unsigned long long)c2 | ((unsigned long long)c3 << 32);
    const unsigned long long off = 4ull * ((unsigned long long)(uint32_t)i | ((unsigned long long)c1 << 32));
    curand_init(seed, sub, off, &st);
    const uint4 c = curand4(&st);
    cur[4 * i + 0] = c.x;
    cur[4 * i + 1] = c.y;
    cur[4 * i + 2] = c.z;
    cur[4 * i + 3] = c.w;
}

cudaError_t launch_selftest_philox(uint64_t seed, uint32_t c1, uint32_t c2, uint32_t c3, int n, uint32_t* d_eng,
                                   uint32_t* d_cur, cudaStream_t st)
{
    selftest_philox_kernel<<<(n + 127) / 128, 128, 0, st>>>(seed, c1, c2, c3, n, d_eng, d_cur);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e;
}

}  // namespace mqv

// External-potential evaluation that allocates no device memory.
//
// nbExtAccelerationCUDA stages the caller's host positions and results through device
// buffers it allocates and frees on every call.  cudaFree waits for all work on the device
// to finish and cudaMalloc can fail under a fixed memory budget, so callers that evaluate the
// potential at a few points inside a tight stepping loop -- an orbit integrator advancing one
// particle, a host process that shares the GPU with a running simulation or holds the device
// memory through its own allocator, a volunteer client held to a fixed device-memory share --
// cannot use it.  nbExtAccelerationNoAllocCUDA does the same arithmetic through a fixed
// staging area that lives in this file as a static device array (NB_NOALLOC_MAX_POINTS
// points, 2 x 3 doubles each = 3 MiB), which every device that loads the library keeps until
// the process exits.
#include <mutex>
#include <string>

#include "nb_common.cuh"
#include "nb_potential.cuh"

#define NB_NOALLOC_MAX_POINTS 65536

// positions of up to NB_NOALLOC_MAX_POINTS points, then their accelerations
static __device__ __align__(256) double g_extScratch[2 * 3 * NB_NOALLOC_MAX_POINTS];

NbPot nb_pot_from(const NBodyCudaCtx* c);
NBodyCudaStatus nb_check_ctx(const NBodyCudaCtx* c, std::string& why);
extern thread_local std::string g_lastError;

__global__ void k_ext_scratch(double* __restrict__ scratch, int n, NbPot pot)
{
    const double* pos = scratch;
    double* acc = scratch + 3 * NB_NOALLOC_MAX_POINTS;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double ex, ey, ez;
        nb_ext_accel(pot, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], ex, ey, ez);
        acc[3 * i] = ex; acc[3 * i + 1] = ey; acc[3 * i + 2] = ez;
    }
}

// Device address of g_extScratch, looked up once per device with that device current and kept
// for the life of the process (a device reset unloads the array; calls after one are not
// supported).
static std::mutex g_scratchLock;
static double* g_scratchPtr[64];

static cudaError_t nb_scratch_for(int device, double** out)
{
    if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> guard(g_scratchLock);
    if (!g_scratchPtr[device]) {
        double* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void**) &p, g_extScratch);
        if (e != cudaSuccess) return e;
        g_scratchPtr[device] = p;
    }
    *out = g_scratchPtr[device];
    return cudaSuccess;
}

extern "C" NBodyCudaStatus nbExtAccelerationNoAllocCUDA(const NBodyCudaPotential* pot,
                                                        const double* pos, double* acc, int n,
                                                        int device)
{
    if (!pot || n < 0 || (n && (!pos || !acc))) return NBODY_USER_ERROR;
    if (n > NB_NOALLOC_MAX_POINTS) {
        g_lastError = "nbExtAccelerationNoAllocCUDA: " + std::to_string(n) +
                      " points exceed the fixed staging area of " +
                      std::to_string(NB_NOALLOC_MAX_POINTS) + " points";
        return NBODY_USER_ERROR;
    }
    NBodyCudaCtx c{};
    c.potentialType = NBCUDA_POTENTIAL_DEFAULT;
    c.pot = *pot;
    std::string why;
    NBodyCudaStatus rc = nb_check_ctx(&c, why);
    if (rc) { g_lastError = why; return rc; }
    if (!n) return NBODY_SUCCESS;
    cudaError_t e = cudaSetDevice(device);
    double* scratch = nullptr;
    if (e == cudaSuccess) e = nb_scratch_for(device, &scratch);
    if (e == cudaSuccess)
        e = cudaMemcpy(scratch, pos, 3 * sizeof(double) * (size_t) n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_ext_scratch<<<(n + 255) / 256, 256>>>(scratch, n, nb_pot_from(&c));
        nb_count_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(acc, scratch + 3 * NB_NOALLOC_MAX_POINTS, 3 * sizeof(double) * (size_t) n,
                       cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        g_lastError = std::string("nbExtAccelerationNoAllocCUDA: ") + cudaGetErrorString(e);
        return NBODY_CUDA_ERROR;
    }
    return NBODY_SUCCESS;
}

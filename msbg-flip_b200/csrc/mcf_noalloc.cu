// Mean-curvature flow without any allocation by the library.
//
// Some callers of the smoother cannot let a library allocate device memory:
// simulation codes that reserve the whole device memory up front with their
// own pool allocator (a cudaMalloc from the library then fails or fragments
// that pool), and host threads that must not block in the CUDA allocator's
// device-wide synchronisation in the middle of a time step.  For them this
// file provides msbg_gpu_pde_mcf_noalloc: the caller passes device pointers
// for its block pool and slot map, and the only scratch the smoother needs
// (the block list regrouped by colour and the error flag of the bounded
// waits) lives in a fixed file-scope device array instead of cudaMalloc'd
// memory.  It needs no context either, because creating one allocates.
#include <cuda_runtime.h>

#include <mutex>

#include "common.cuh"
#include "msbg_gpu.h"

namespace {

constexpr int MAXB = MSBG_MCF_NOALLOC_MAX_BLOCKS;
// Layout: [0, MAXB) the caller's list as received, [MAXB, 2*MAXB) the list
// regrouped by colour, [2*MAXB, 2*MAXB+8) per-colour cursors, [2*MAXB+8] the
// error flag.  One copy per device, held until the process exits.
__device__ __align__(256) int g_mcf_scratch[2 * MAXB + 16];

// Device address of g_mcf_scratch per device, looked up once per device.
void* g_scratch_ptr[64];
bool g_scratch_ready[64];
std::mutex g_scratch_mutex;

__global__ void k_group_by_colour(const int* __restrict__ raw, int n, int nbx, int nby,
                                  int4 startLo, int4 startHi, int* __restrict__ cursor,
                                  int* __restrict__ grouped) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int b = raw[i];
  const int bx = b % nbx, by = (b / nbx) % nby, bz = b / (nbx * nby);
  const int c = (bx & 1) + 2 * (by & 1) + 4 * (bz & 1);
  const int start[8] = {startLo.x, startLo.y, startLo.z, startLo.w,
                        startHi.x, startHi.y, startHi.z, startHi.w};
  // the order inside a colour does not change the result: same-colour
  // blocks never touch each other's halo
  grouped[start[c] + atomicAdd(&cursor[c], 1)] = b;
}

int scratch_for_current_device(int** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return MSBG_ENODEV;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ready[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_mcf_scratch) != cudaSuccess || !p) return MSBG_ERROR;
    g_scratch_ptr[dev] = p;
    g_scratch_ready[dev] = true;
  }
  *out = static_cast<int*>(g_scratch_ptr[dev]);
  return MSBG_OK;
}

}  // namespace

extern "C" int msbg_gpu_pde_mcf_noalloc(float* pool, const int* slotOf, const int* blockList,
                                        int n, int nbx, int nby, int nbz, int bsx,
                                        float emptyVal, float fullVal, int numIter, float dt,
                                        int clamp01, void* stream, int* timedOut) {
  if (!pool || !slotOf || (n > 0 && !blockList) || n < 0 || numIter < 0) return MSBG_EINVARG;
  if (n > MAXB) return MSBG_EINVARG;  // beyond the fixed scratch: see the header
  if (reinterpret_cast<uintptr_t>(pool) % 8) return MSBG_EINVARG;  // voxel pairs are copied whole
  if (!(bsx == 8 || bsx == 16 || bsx == 32) || nbx <= 0 || nby <= 0 || nbz <= 0)
    return MSBG_EINVARG;
  const long long nb = (long long)nbx * nby * nbz;
  int cnt[8] = {0};
  for (int i = 0; i < n; i++) {
    const int b = blockList[i];
    if (b < 0 || b >= nb) return MSBG_EINVARG;
    const int bx = b % nbx, by = (b / nbx) % nby, bz = b / (nbx * nby);
    cnt[(bx & 1) + 2 * (by & 1) + 4 * (bz & 1)]++;
  }
  int start[9] = {0};
  for (int c = 0; c < 8; c++) start[c + 1] = start[c] + cnt[c];
  int* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  int* raw = scratch;
  int* grouped = scratch + MAXB;
  int* cursor = scratch + 2 * MAXB;
  int* errFlag = scratch + 2 * MAXB + 8;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the array keeps the previous call's contents: reset cursors and flag
  if (cudaMemsetAsync(cursor, 0, sizeof(int) * 9, st) != cudaSuccess) return MSBG_ERROR;
  if (n > 0) {
    if (cudaMemcpyAsync(raw, blockList, sizeof(int) * n, cudaMemcpyHostToDevice, st) !=
        cudaSuccess)
      return MSBG_ERROR;
    k_group_by_colour<<<(n + 255) / 256, 256, 0, st>>>(
        raw, n, nbx, nby, make_int4(start[0], start[1], start[2], start[3]),
        make_int4(start[4], start[5], start[6], start[7]), cursor, grouped);
  }
  const int nIter = numIter + (numIter & 1);  // src/msbg4.cpp:150-152
  if (msbg::launch_mcf(pool, slotOf, grouped, start, nbx, nby, nbz, bsx, emptyVal, fullVal,
                       nIter, dt, clamp01, errFlag, st) != cudaSuccess)
    return MSBG_ERROR;
  if (timedOut) {
    int h = 0;
    if (cudaStreamSynchronize(st) != cudaSuccess ||
        cudaMemcpy(&h, errFlag, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
      return MSBG_ERROR;
    *timedOut = (h & msbg::ERR_WAIT_TIMEOUT) ? 1 : 0;
    if (h & msbg::MCF_ERR_NOT_VALUE) return MSBG_EINVARG;  // that block was skipped
    if (h) return MSBG_ETIMEOUT;
  }
  return MSBG_OK;
}

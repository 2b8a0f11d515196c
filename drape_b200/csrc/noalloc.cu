// Block-Jacobi PCG for callers that cannot allocate GPU memory.
//
// Some callers of this library run where cudaMalloc is not theirs to call: inside a host application that owns
// every device allocation through its own pool (a game engine or a render service embedding the cloth solve),
// inside code that must never block on the driver's allocator in the middle of a frame, or inside a plugin whose
// host forbids new device allocations after start-up. They hold the matrix, the right-hand side and the solution
// buffer already; what they cannot provide is the solver's work space. drape_pcg_noalloc gives them the same
// solver as drape_pcg with its work space in one fixed, file-scope device array instead of allocations.
//
// The array is sized for kNoAllocMaxRows block rows (about 3.4 MB) and every GPU that loads the library keeps it
// until the process exits. In host code `g_noalloc_scratch` names a host-side stand-in, not device memory: every
// call looks up the device address with cudaGetSymbolAddress while the caller's device is current (a lookup in
// the loaded module, no allocation), and only that address is handed to kernels. Looking it up on every call
// instead of caching it keeps the address valid after cudaDeviceReset or when the caller makes another context
// current on the same device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>

#include "../../include/drape_b200.h"
#include "kernels.h"

namespace drape {
void set_global_error(const std::string& message);  // capi.cpp: the message drape_last_error(NULL) returns
}

namespace {

constexpr int kNoAllocMaxRows = DRAPE_NOALLOC_MAX_ROWS;
constexpr int kNoAllocMaxGrid = 1024;  // one reduction word per CTA thread of the 1024-thread launch
constexpr int kThreads = 1024, kLanes = 8;

// Layout of the scratch array (byte offsets, all 256-aligned):
//   z, p0, p1        float4 [kNoAllocMaxRows] each
//   diag_pos         int    [kNoAllocMaxRows]
//   flags            int    [64]              flags[0]: a row without a diagonal block
//   sync             PcgSyncHeader + 2 parities x 2 values x kNoAllocMaxGrid words
constexpr size_t kVec = size_t(kNoAllocMaxRows) * 16;
constexpr size_t kOffZ = 0, kOffP0 = kVec, kOffP1 = 2 * kVec, kOffDiag = 3 * kVec;
constexpr size_t kOffFlags = kOffDiag + size_t(kNoAllocMaxRows) * 4;
constexpr size_t kOffSync = kOffFlags + 256;
constexpr size_t kSyncBytes = sizeof(drape::PcgSyncHeader) + 32 * size_t(kNoAllocMaxGrid);
constexpr size_t kScratchBytes = (kOffSync + kSyncBytes + 255) / 256 * 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Position of each row's diagonal block; flags[0] = 1 when a row has none.
__global__ void find_diagonal(int R, const int* row_ptr, const int* col_idx, int* diag_pos, int* flags) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  int pos = -1;
  for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k)
    if (col_idx[k] == r) {
      pos = k;
      break;
    }
  diag_pos[r] = pos < 0 ? row_ptr[r] : pos;  // an in-range index even when missing; the host rejects the call
  if (pos < 0) flags[0] = 1;
}

drape_status fail(const std::string& m, drape_status code) {
  drape::set_global_error(m);
  return code;
}

}  // namespace

extern "C" drape_status drape_pcg_noalloc(int32_t rows, const int32_t* row_ptr, const int32_t* col_idx,
                                          const float* a0, const float* a1, const float* a2, const float* rhs,
                                          float* x, double rtol, int32_t max_iterations, void* stream,
                                          int32_t* info, double* relative) {
  if (rows < 1 || rows > kNoAllocMaxRows)
    return fail("drape_pcg_noalloc: " + std::to_string(rows) + " block rows; this entry point holds work space for 1 to " +
                    std::to_string(kNoAllocMaxRows),
                DRAPE_E_ARG);
  if (!row_ptr || !col_idx || !a0 || !a1 || !a2 || !rhs || !x || !(rtol > 0) || max_iterations < 1)
    return fail("drape_pcg_noalloc: null device pointer or invalid tolerance / iteration cap", DRAPE_E_ARG);
  if ((reinterpret_cast<uintptr_t>(a0) | reinterpret_cast<uintptr_t>(a1) | reinterpret_cast<uintptr_t>(rhs) |
       reinterpret_cast<uintptr_t>(x)) % 16)
    return fail("drape_pcg_noalloc: a0, a1, rhs and x must be 16-byte aligned", DRAPE_E_ARG);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail("drape_pcg_noalloc: no current device", DRAPE_E_CUDA);
  unsigned char* base = nullptr;
  {
    // The device address of the file-scope array in the current context (on the first call on a device this
    // also loads the library's device code there, which is why that call should come before any stream capture).
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(std::string("drape_pcg_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e), DRAPE_E_CUDA);
    base = static_cast<unsigned char*>(p);
  }
  // Launch shape: as the context's, with the matrix read from global memory (no per-CTA block capacity needed).
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int groups = kThreads / kLanes;
  int grid = std::max(1, std::min({sms, (rows + groups - 1) / groups, kNoAllocMaxGrid, rows}));
  int cap_rows = (rows + grid - 1) / grid + 1;
  drape::PcgLaunch cfg;
  cfg.threads = kThreads;
  cfg.lanes_per_row = kLanes;
  cfg.matrix_in_smem = false;
  cfg.smem = drape::pcg_smem_bytes(cap_rows, 0, false);
  // Fewer CTAs hold more rows each and so need more shared memory, which can lower the co-resident count again:
  // shrink until the grid fits the occupancy at its own shared-memory size.
  for (;;) {
    const int fit = drape::pcg_max_grid(kThreads, kLanes, cfg.smem, false);
    if (fit <= 0) return fail("drape_pcg_noalloc: the PCG kernel does not fit on this device", DRAPE_E_CUDA);
    if (grid <= fit) break;
    grid = fit;
    cap_rows = (rows + grid - 1) / grid + 1;
    cfg.smem = drape::pcg_smem_bytes(cap_rows, 0, false);
  }
  cfg.grid = grid;

  auto* head = reinterpret_cast<drape::PcgSyncHeader*>(base + kOffSync);
  int* flags = reinterpret_cast<int*>(base + kOffFlags);
  int* diag = reinterpret_cast<int*>(base + kOffDiag);
  // Clear what must start at zero (the array keeps the previous call's contents): flags and reduction words.
  cudaError_t e = cudaMemsetAsync(base + kOffFlags, 0, kOffSync - kOffFlags + sizeof(drape::PcgSyncHeader) + 32 * size_t(grid), s);
  if (e == cudaSuccess) {
    find_diagonal<<<(rows + 255) / 256, 256, 0, s>>>(rows, row_ptr, col_idx, diag, flags);
    e = cudaGetLastError();
  }
  int missing = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&missing, flags, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(std::string("drape_pcg_noalloc: ") + cudaGetErrorString(e), DRAPE_E_CUDA);
  if (missing) return fail("drape_pcg_noalloc: a row has no diagonal block", DRAPE_E_ARG);

  drape::PcgArgs a{};
  a.R = rows;
  a.row_ptr = row_ptr;
  a.col_idx = col_idx;
  a.diag_pos = diag;
  a.A = drape::DevBsr{reinterpret_cast<float4*>(const_cast<float*>(a0)), reinterpret_cast<float4*>(const_cast<float*>(a1)),
                      const_cast<float*>(a2)};
  a.b = reinterpret_cast<const float4*>(rhs);
  a.x = reinterpret_cast<float4*>(x);
  a.z = reinterpret_cast<float4*>(base + kOffZ);
  a.p0 = reinterpret_cast<float4*>(base + kOffP0);
  a.p1 = reinterpret_cast<float4*>(base + kOffP1);
  a.state = &head->state;
  a.error = &head->error;
  a.bcast = head->bcast;
  a.slots = reinterpret_cast<unsigned long long*>(head + 1);
  a.cap_rows = cap_rows;
  a.cap_blocks = 0;
  a.tol2 = float(rtol * rtol);
  a.max_iterations = max_iterations;
  a.spin_limit = 4000000000LL;
  a.timing = nullptr;
  e = drape::launch_pcg(a, cfg, s);
  drape::PcgSyncHeader h{};
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, head, sizeof h, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(std::string("drape_pcg_noalloc: ") + cudaGetErrorString(e), DRAPE_E_CUDA);
  if (h.error) return fail("drape_pcg_noalloc: a grid-wide wait gave up", DRAPE_E_TIMEOUT);
  if (info) {
    info[0] = h.state.iterations;
    info[1] = h.state.status;
    info[2] = h.state.replacements;
  }
  if (relative) *relative = h.state.rr0 > 0 ? std::sqrt(double(h.state.rr) / double(h.state.rr0)) : 0.0;
  return DRAPE_OK;
}

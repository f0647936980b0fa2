// Jacobian combination with homogeneous Dirichlet conditions whose scratch
// lives in a fixed device array of this library instead of allocations.
//
// Scratch layout (g_noalloc_scratch, one copy per device):
//   [0, 256)                      the "first non-zero diagonal" word of the
//                                 Dirichlet scale (written before use)
//   [256, 256 + 8 * MAX_BC)       the caller's Dirichlet node list (int64)
//   [.., + MAX_NDOF)              the DOF mask (uint8), cleared on every call
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "internal.h"

namespace hoefem {

constexpr long long NOALLOC_MAX_NDOF = 1LL << 22;     // 4,194,304 DOFs
constexpr long long NOALLOC_MAX_BC_NODES = 1LL << 18;  // 262,144 Dirichlet nodes
constexpr size_t NOALLOC_NODES_OFF = 256;
constexpr size_t NOALLOC_MASK_OFF = NOALLOC_NODES_OFF + 8 * NOALLOC_MAX_BC_NODES;
constexpr size_t NOALLOC_BYTES = NOALLOC_MASK_OFF + NOALLOC_MAX_NDOF;

namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

__global__ void k_mark_bc_nodes(const long long* __restrict__ nodes, long long count, unsigned char* __restrict__ mask) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < count;
       k += (long long)gridDim.x * blockDim.x) {
    const long long a = nodes[k];
    mask[3 * a] = 1;
    mask[3 * a + 1] = 1;
    mask[3 * a + 2] = 1;
  }
}

constexpr int MAX_DEVICES = 64;
std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_ptr[MAX_DEVICES] = {};

// Device address of the scratch on device `dev`, looked up once per device
// with that device current (the caller makes it current).
unsigned char* noalloc_scratch(int dev) {
  HOEFEM_REQUIRE(dev >= 0 && dev < MAX_DEVICES, HOEFEM_ERR_INVALID_ARGUMENT, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    HOEFEM_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
  }
  return g_noalloc_ptr[dev];
}

// Makes `dev` current for the lifetime of the object and restores the
// previous current device afterwards.
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int dev) {
    HOEFEM_CUDA(cudaGetDevice(&prev));
    if (prev != dev) HOEFEM_CUDA(cudaSetDevice(dev));
    else prev = -1;
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

void jacobian_combination_noalloc(Model& m, double ck, const double* K, double cm, const double* M,
                                  const long long* bc_nodes, long long num_bc, double* out) {
  HOEFEM_REQUIRE(m.finalized && m.on_device, HOEFEM_ERR_NOT_FINALIZED,
                 "model is not resident on the device (run any compute entry point on it first)");
  HOEFEM_REQUIRE(m.ndof <= NOALLOC_MAX_NDOF, HOEFEM_ERR_INVALID_ARGUMENT,
                 "model exceeds the 4,194,304 DOFs of the preallocated scratch");
  HOEFEM_REQUIRE(num_bc >= 0 && num_bc <= NOALLOC_MAX_BC_NODES, HOEFEM_ERR_INVALID_ARGUMENT,
                 "more than 262,144 Dirichlet nodes for the preallocated scratch");
  HOEFEM_REQUIRE(out && (bc_nodes || num_bc == 0), HOEFEM_ERR_INVALID_ARGUMENT, "null array");
  for (long long k = 0; k < num_bc; ++k)
    HOEFEM_REQUIRE(bc_nodes[k] >= 0 && bc_nodes[k] < m.nv, HOEFEM_ERR_INVALID_ARGUMENT,
                   "Dirichlet node out of range");
  // the scratch, the stream and the model's buffers all belong to m.device
  DeviceScope scope(m.device);
  unsigned char* scratch = noalloc_scratch(m.device);
  cudaStream_t s = m.stream;
  unsigned char* mask = nullptr;
  if (num_bc > 0) {
    long long* nodes = reinterpret_cast<long long*>(scratch + NOALLOC_NODES_OFF);
    mask = scratch + NOALLOC_MASK_OFF;
    HOEFEM_CUDA(cudaMemsetAsync(mask, 0, (size_t)m.ndof, s));
    HOEFEM_CUDA(cudaMemcpyAsync(nodes, bc_nodes, sizeof(long long) * num_bc, cudaMemcpyHostToDevice, s));
    const int grid = (int)std::min<long long>((num_bc + 255) / 256, (long long)device_sms() * 8);
    (note_launch(), k_mark_bc_nodes<<<grid, 256, 0, s>>>(nodes, num_bc, mask));
    HOEFEM_CUDA(cudaGetLastError());
  }
  jacobian_combination(m, ck, K, cm, M, mask, out, reinterpret_cast<double*>(scratch), s);
  HOEFEM_CUDA(cudaStreamSynchronize(s));
}

}  // namespace hoefem

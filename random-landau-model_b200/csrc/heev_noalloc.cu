// Allocation-free entry point of the batched eigensolver.
//
// Some callers cannot allocate device memory: a process whose device memory is already
// reserved in full by another allocator (a framework's caching pool, or a job running
// under a fixed device-memory budget), and callers that must not take cudaMalloc /
// cudaFree's implicit device synchronisation in the middle of their own work.  For them
// rlmb_heevd_batched_noalloc runs the double-precision kernels of rlmb_heevd_batched (always
// FP64, never the mixed mode's refinement, whatever precision other callers' contexts use),
// but on scratch that lives in the file-scope device array below instead of a context
// workspace.
#include <mutex>

#include "common.cuh"

namespace rlmb {
size_t heev_scratch_bytes_per_matrix(int n);
size_t heev_max_chunk(int n);
int heev_chunk_on_scratch(cudaStream_t st, cplx* A, double* W, int* info, int n, int nb,
                          void* scratch, long long* launches);
}  // namespace rlmb

// The scratch: RLMB_NOALLOC_SCRATCH_BYTES of device memory that every GPU which loads this
// library holds until the process exits.  All calls share it and it keeps the last call's
// contents; no part of it needs to start at zero, because every kernel writes each scratch
// region before any kernel reads it.  Calls whose GPU work overlaps in time (other streams,
// other host threads) race on it.
static __device__ __align__(256) unsigned char g_heev_scratch[RLMB_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once per device.
// In host code g_heev_scratch names a host-side stand-in, not device memory, so kernels
// must be given this address instead.
int scratch_address(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return RLMB_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_heev_scratch);
        if (e != cudaSuccess || !p) {
            fprintf(stderr, "rlmb: cudaGetSymbolAddress of the eigensolver scratch failed: %s\n",
                    cudaGetErrorString(e));
            return RLMB_ERR_CUDA;
        }
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return RLMB_OK;
}
}  // namespace

extern "C" int rlmb_heevd_batched_noalloc(double* d_a, double* d_w, int n, int batch, int* d_info,
                                          void* stream) {
    if (!d_a || !d_w || n <= 0 || batch < 0) return RLMB_ERR_ARG;
    const size_t per = rlmb::heev_scratch_bytes_per_matrix(n);
    if (per > RLMB_NOALLOC_SCRATCH_BYTES) {
        fprintf(stderr,
                "rlmb_heevd_batched_noalloc: a matrix of order %d needs %zu bytes of scratch, more "
                "than the fixed %zu-byte array of this entry point; use rlmb_heevd_batched\n",
                n, per, (size_t)RLMB_NOALLOC_SCRATCH_BYTES);
        return RLMB_ERR_TOO_LARGE;
    }
    if (batch == 0) return RLMB_OK;
    // a launch error the caller left pending is reported, not consumed (this call's own
    // launch checks would otherwise take it as theirs)
    if (cudaPeekAtLastError() != cudaSuccess) return RLMB_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the scratch address is the current device's: the stream must belong to that device
    if (st) {
        int cur = 0, sdev = 0;
        if (cudaGetDevice(&cur) != cudaSuccess || cudaStreamGetDevice(st, &sdev) != cudaSuccess) return RLMB_ERR_CUDA;
        if (sdev != cur) {
            fprintf(stderr, "rlmb_heevd_batched_noalloc: the stream belongs to device %d, the current device is %d\n",
                    sdev, cur);
            return RLMB_ERR_ARG;
        }
    }
    void* scratch = nullptr;
    if (int rc = scratch_address(&scratch)) return rc;
    // chunks: as many matrices as the array holds, within the grid limits of the per-matrix
    // launches, and equal in size (a short last chunk would leave most SMs idle)
    size_t cap = std::min<size_t>((size_t)batch, RLMB_NOALLOC_SCRATCH_BYTES / per);
    cap = std::max<size_t>(1, std::min(cap, rlmb::heev_max_chunk(n)));
    const size_t nchunks = ((size_t)batch + cap - 1) / cap;
    const int chunk = (int)(((size_t)batch + nchunks - 1) / nchunks);
    long long launches = 0;
    const size_t nn = (size_t)n * n;
    for (int b0 = 0; b0 < batch; b0 += chunk) {
        const int nb = std::min(chunk, batch - b0);
        if (int rc = rlmb::heev_chunk_on_scratch(st, reinterpret_cast<rlmb::cplx*>(d_a) + (size_t)b0 * nn,
                                                 d_w + (size_t)b0 * n, d_info ? d_info + b0 : nullptr, n, nb,
                                                 scratch, &launches))
            return rc;
    }
    return RLMB_OK;
}

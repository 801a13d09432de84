// noalloc.cu -- lbgpu_get_macros_noalloc: the density/velocity read-out of lbgpu_get_macros
// without any device allocation.
//
// Who needs it: callers that must not call cudaMalloc/cudaFree while the solver runs.  A
// serving loop that reads one simulation's fields while other simulations step on other
// streams cannot afford them (cudaMalloc and cudaFree synchronize with the device and stall
// every stream), and a host application whose device memory is reserved up front by another
// allocator (a framework's caching allocator, a fixed per-process budget) may have none left
// to hand out.  lbgpu_get_macros allocates a lattice-sized device buffer on every call; this
// variant uses a fixed device array instead.
//
// The scratch: a file-scope __device__ array of 3 x 262,144 doubles (6 MiB).  Every GPU that
// loads the library holds it until the process exits.  Lattices with more than 262,144
// interior nodes are rejected with LB_ERR_CAPACITY (use lbgpu_get_macros for those).
//
// Set-up: the first call on each device looks up the array's device address with
// cudaGetSymbolAddress while that device is current; make that first call before any stream
// capture.  Calls made while the lattice's stream is not capturing look the address up again
// (a host application that resets the device with cudaDeviceReset reloads the library's device
// code, and the array with it, at a new address); calls made during a capture use the address
// the last uncaptured call found.  Host code never uses the array's name as an address: on the
// host it names a stand-in, not device memory.
//
// Sharing: all calls use the same array, which keeps the last call's contents.  Nothing in it
// has to start at zero: every element a call copies back was written by that same call.  Calls
// that overlap on the GPU (different threads, different lattices on one device) race on the
// array; callers serialize them.
#include <mutex>
#include "lattice.h"
#include "lbgpu.h"

namespace {

constexpr size_t kMaxNodes = (size_t)1 << 18;
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_macros_scratch[3 * kMaxNodes];

double *g_scratch_addr[kMaxDevices];
std::mutex g_scratch_mu;

// Device address of g_macros_scratch on the current device: looked up afresh unless `stream`
// is capturing, in which case the address of the last uncaptured call on the device is used.
int scratch_address(int dev, cudaStream_t stream, double **out)
{
    if (dev < 0 || dev >= kMaxDevices)
        return lbgpu::set_error(LB_ERR_CAPACITY, "lbgpu_get_macros_noalloc: device %d beyond %d",
                                dev, kMaxDevices);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (int rc = lbgpu::cuda_error(cudaStreamIsCapturing(stream, &cap), "cudaStreamIsCapturing"))
        return rc;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (cap != cudaStreamCaptureStatusNone && !g_scratch_addr[dev])
        return lbgpu::set_error(LB_ERR_STATE, "lbgpu_get_macros_noalloc: the first call on device "
                                "%d must come before any stream capture", dev);
    if (cap == cudaStreamCaptureStatusNone) {
        void *p = nullptr;
        if (int rc = lbgpu::cuda_error(cudaGetSymbolAddress(&p, g_macros_scratch),
                                       "cudaGetSymbolAddress(macros scratch)"))
            return rc;
        g_scratch_addr[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_addr[dev];
    return LB_OK;
}

}  // namespace

extern "C" int lbgpu_get_macros_noalloc(lbgpu_lattice *h, double *rho, double *ux, double *uy)
{
    if (!h) return lbgpu::set_error(LB_ERR_ARG, "lbgpu_get_macros_noalloc: null lattice");
    lbgpu::Lattice &L = h->L;
    const size_t nodes = (size_t)L.lx * (size_t)L.ly;
    if (nodes > kMaxNodes)
        return lbgpu::set_error(LB_ERR_CAPACITY,
                                "lbgpu_get_macros_noalloc: %d x %d = %zu nodes exceed the %zu-node "
                                "fixed scratch (use lbgpu_get_macros)",
                                L.lx, L.ly, nodes, kMaxNodes);
    int prev = -1;
    if (int rc = lbgpu::cuda_error(cudaGetDevice(&prev), "cudaGetDevice")) return rc;
    if (prev != L.device)
        if (int rc = lbgpu::cuda_error(cudaSetDevice(L.device), "cudaSetDevice")) return rc;
    double *s = nullptr;
    int rc = scratch_address(L.device, L.stream, &s);
    if (rc == LB_OK) {
        int v, par;
        L.view(v, par);
        lbgpu::launch_macros(L.d, v, L.cur, par, s, s + nodes, s + 2 * nodes, L.stream);
        rc = L.check("lbgpu_get_macros_noalloc");
    }
    double *dst[3] = {rho, ux, uy};
    for (int k = 0; k < 3 && rc == LB_OK; ++k)
        if (dst[k])
            rc = lbgpu::cuda_error(cudaMemcpyAsync(dst[k], s + k * nodes, nodes * sizeof(double),
                                                   cudaMemcpyDeviceToHost, L.stream),
                                   "lbgpu_get_macros_noalloc");
    if (rc == LB_OK) rc = lbgpu::cuda_error(cudaStreamSynchronize(L.stream), "lbgpu_get_macros_noalloc");
    if (prev != L.device) cudaSetDevice(prev);
    return rc;
}

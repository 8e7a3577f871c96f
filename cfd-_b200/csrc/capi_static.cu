// capi_static.cu - pressure solve whose scratch lives in a static device array.
//
// cfd2d_pressure_solve needs the caller to hand it a workspace (cfd2d_poisson.work)
// when it runs the grid-persistent solver. Some callers cannot provide one: a C or
// ctypes host that owns no device allocator, or a caller between the steps of a
// time loop that must not call cudaMalloc/cudaFree (both can synchronise the whole
// device). cfd2d_pressure_solve_static runs the same grid-persistent kernel with its
// workspace taken from kScratch below, so it allocates no device memory at all.

#include <atomic>

#include "../../include/cfd2d_b200.h"
#include "pcg.cuh"

namespace cfd {
namespace {

// Workspace of the grid-persistent solver (pcg_grid_workspace_doubles) for the
// largest grid this entry point accepts: R, P0, P1 (one double per cell each),
// three partial-sum arrays of (4 + CFD2D_MAX_COMPONENTS) doubles for up to
// 148 * 32 CTAs (a B200's SMs times the CTAs an SM holds; on a device with more SMs
// the capacity check below refuses the call), and two barrier words. 8.2 MiB of
// device memory per device, reserved when the library's module is loaded.
constexpr size_t kScratchDoubles =
    (size_t)3 * CFD2D_STATIC_MAX_CELLS + (size_t)3 * 148 * 32 * (4 + CFD2D_MAX_COMPONENTS) + 8;

// Nothing in it has to start at zero: the solver writes R, P0, P1 and its partial
// sums before reading them, and the launcher clears the two barrier words with
// cudaMemsetAsync on the caller's stream before every launch.
static __device__ __align__(256) double kScratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::atomic<double*> g_scratch[kMaxDevices];

// Address of kScratch on the current device, looked up once per device. The first
// lookup can load the module on that device, so it must not run inside a stream
// capture.
cudaError_t scratch_of_current_device(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < kMaxDevices) {
        double* p = g_scratch[dev].load(std::memory_order_acquire);
        if (p) { *out = p; return cudaSuccess; }
    }
    double* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, kScratch);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < kMaxDevices) g_scratch[dev].store(p, std::memory_order_release);
    *out = p;
    return cudaSuccess;
}

}  // namespace
}  // namespace cfd

extern "C" int cfd2d_pressure_solve_static(const cfd2d_poisson* op, const double* rhs, double* p, double rtol,
                                           int maxiter, int32_t* iters_out, int32_t* status_out, void* stream) {
    using namespace cfd;
    if (!op || !rhs || !p || maxiter < 0 || op->nx < 4 || op->ny < 4) return CFD2D_E_ARG;
    if ((long long)op->nx * op->ny > CFD2D_STATIC_MAX_CELLS) return CFD2D_E_CAPACITY;
    if (op->ncomp > CFD2D_MAX_COMPONENTS) return CFD2D_E_CAPACITY;
    if (pcg_grid_workspace_doubles(op->nx, op->ny) > kScratchDoubles) return CFD2D_E_CAPACITY;
    double* scratch = nullptr;
    if (scratch_of_current_device(&scratch) != cudaSuccess) {
        cudaGetLastError();
        return CFD2D_E_CUDA;
    }
    PcgLaunch L = {};
    L.op = *op;
    L.op.cluster = 0;    // the grid-persistent solver, the variant that uses scratch,
    L.op.grid_ctas = 0;  // as a cooperative launch over every SM (never the 16-CTA form)
    L.op.work = scratch;
    L.op.work_bytes = kScratchDoubles * sizeof(double);
    L.rhs_mode = 0;
    L.rhs = rhs;
    L.rtol = rtol;
    L.maxiter = maxiter;
    L.p_out = p;
    L.p_padded = 0;
    L.iters_out = iters_out;
    L.status_out = status_out;
    return pcg_launch(L, reinterpret_cast<cudaStream_t>(stream)) == cudaSuccess ? CFD2D_OK : CFD2D_E_CUDA;
}

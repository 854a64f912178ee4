// CG field solve that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the point where they need a solve: a host
// framework that owns every device allocation through its own pool, a loop that must not
// take the device-wide synchronisation an allocation can imply, or code that runs while
// allocation is forbidden by its host. mzb_conj_grad_noalloc serves them: the caller
// passes its own device buffers for b, x0 and x, and the solver's work arrays (r, the two
// search-direction buffers, A p, the reduction partials and the grid-barrier words) live
// in one file-scope __device__ array of fixed size below. That array exists in every
// device that loads this library and stays allocated until the process exits.
#include "engine.cuh"

namespace mzb {
namespace {

// Largest grid side n the static work area serves (n^3 points per work array).
constexpr int kNoAllocMaxN = 64;
constexpr long kNoAllocGrid = (long)kNoAllocMaxN * kNoAllocMaxN * kNoAllocMaxN;
constexpr long kNoAllocPartials = 4096;  // doubles for the per-block reduction partials
// r, p0, p1, Ap (n^3 each), partials, then barrier + result words: about 8.4 MB
constexpr long kNoAllocDoubles = 4 * kNoAllocGrid + kNoAllocPartials + 16;

static __device__ __align__(256) double g_noalloc_work[kNoAllocDoubles];

// Device address of g_noalloc_work, looked up once per device. In host code the array's
// name is only a host-side stand-in, never a device address.
constexpr int kMaxDevices = 64;
double* g_noalloc_addr[kMaxDevices] = {};

}  // namespace
}  // namespace mzb

using namespace mzb;

// Solve L x = b (the reference's conj_grad, library/src/plcg.c:28-90, or its Jacobi form
// with precond = 1) on an n^3 grid with 2 <= n <= 64, on device buffers the caller owns.
// No device memory is allocated or freed by this call.
//
//  * b, x0, x: device pointers to n^3 doubles on the current device (x may equal x0);
//    stream: the cudaStream_t to run on (NULL = the default stream).
//  * Synchronous: the call waits for the solve on `stream` and copies the result word to
//    the host, so it must not be called while `stream` (or, in global capture mode, any
//    stream) is being captured into a CUDA graph.
//  * Returns the reference's value (0-based iteration of convergence, or -1 when not
//    converged), -2 for arguments it cannot serve (n outside [2, 64], precond not 0/1,
//    null pointers or pointers that are not memory of the current device), -3 when the
//    solver aborted, -4 when the work area's address could not be obtained, -5 when the
//    CUDA context already holds an error or the copy or synchronisation of the result
//    fails (the message is printed). A kernel that cannot be launched ends the process,
//    as in every other entry point of this library.
//  * The first call on each device looks up the work area's device address
//    (cudaGetSymbolAddress) and sets kernel attributes.
//  * Every call shares the one work area, which keeps the last call's contents; the
//    solver clears what must start at zero (the barrier words) itself. Calls that overlap
//    on the GPU -- on different streams or threads -- race on it and must not be issued.
extern "C" int mzb_conj_grad_noalloc(const double* b, const double* x0, double* x, double tol, int n,
                                     int precond, void* stream) {
    if (n < 2 || n > kNoAllocMaxN) {
        fprintf(stderr, "mzb_conj_grad_noalloc: n = %d is outside [2, %d], the size its static work area serves\n",
                n, kNoAllocMaxN);
        return -2;
    }
    if (precond != 0 && precond != 1) {
        fprintf(stderr, "mzb_conj_grad_noalloc: precond must be 0 (implicit Jacobi) or 1 (Jacobi)\n");
        return -2;
    }
    if (b == nullptr || x0 == nullptr || x == nullptr) {
        fprintf(stderr, "mzb_conj_grad_noalloc: null buffer\n");
        return -2;
    }
    const cudaError_t sticky = cudaPeekAtLastError();
    if (sticky != cudaSuccess) {
        fprintf(stderr, "mzb_conj_grad_noalloc: CUDA error before the call: %s\n", cudaGetErrorString(sticky));
        return -5;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return -4;
    for (const void* ptr : {static_cast<const void*>(b), static_cast<const void*>(x0), static_cast<const void*>(x)}) {
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess || at.device != dev ||
            (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)) {
            cudaGetLastError();  // clear the lookup's error, if any
            fprintf(stderr, "mzb_conj_grad_noalloc: %p is not memory of device %d\n", ptr, dev);
            return -2;
        }
    }
    if (g_noalloc_addr[dev] == nullptr) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_work);
        if (e != cudaSuccess || p == nullptr) {
            fprintf(stderr, "mzb_conj_grad_noalloc: cannot get the work area's address: %s\n", cudaGetErrorString(e));
            return -4;
        }
        g_noalloc_addr[dev] = static_cast<double*>(p);
    }
    if ((long)engine_grid_blocks() * 16 > kNoAllocPartials) {
        fprintf(stderr, "mzb_conj_grad_noalloc: this device has more SMs than the work area serves\n");
        return -2;
    }
    double* w = g_noalloc_addr[dev];
    const long m = (long)n * n * n;
    EngineArgs a{};
    a.prog = precond == 0 ? PROG_CG : PROG_PCG;
    a.precond = precond;
    a.n = n;
    a.tol = tol;
    a.b = b;
    a.x0 = x0;
    a.x = x;
    a.r = w;
    a.p0 = w + m;
    a.p1 = w + 2 * m;
    a.Ap = w + 3 * m;
    a.partials = w + 4 * kNoAllocGrid;
    a.bar = reinterpret_cast<GridBarrier*>(w + 4 * kNoAllocGrid + kNoAllocPartials);
    a.result = reinterpret_cast<int*>(w + 4 * kNoAllocGrid + kNoAllocPartials + 4);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!cg_fast_launch(a, s)) engine_launch(a, s);
    int res[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(res, a.result, sizeof(res), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        fprintf(stderr, "mzb_conj_grad_noalloc: %s\n", cudaGetErrorString(e));
        return -5;
    }
    if (res[1] != 0) return -3;
    return res[0];
}

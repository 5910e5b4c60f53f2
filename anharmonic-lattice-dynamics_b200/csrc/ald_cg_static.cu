// ald_cg_quadratic_static: the conjugate-gradient solve of cg_quadratic for
// callers that must not allocate device memory.
//
// Who needs this: a host whose device memory all comes from its own pool --
// a Fortran or C code that sets up every device array once and hands out
// slices, or a solver running inside another framework's caching allocator
// and memory budget.  For such callers a cudaMalloc inside the library breaks
// their accounting (it can fail even though the pool has room), and a
// cudaFree synchronises the whole device and stalls their other streams.
// They already hold the matrix, the right-hand side and the solution vector
// in device memory; this entry point takes those device pointers and keeps
// every CG work vector in one file-scope __device__ array instead of
// allocating.
//
// The scratch array is sized for n <= ALD_CG_STATIC_MAX_N unknowns (about
// 0.8 MB) and stays resident on every device that loads the library until the
// process exits.  The first call on a device looks up the array's device
// address (cudaGetSymbolAddress, with that device current) and keeps it for
// the life of the process; make that first call before any stream capture.
// A cudaDeviceReset by the host discards the module that holds the array, so
// the kept address is no longer valid after one: do not reset a device
// between calls.  All calls share the array: two calls whose
// kernels overlap on the same device (different streams, or different host
// threads) race on it.  Every value a call reads from it is written earlier in
// the same call, so the contents left by a previous call never leak into a
// result.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "../../include/ald.h"

namespace ald {
namespace capi {
int fail(int code, const std::string& msg);  // records the message for ald_last_error
}
}  // namespace ald

namespace {

constexpr int kMaxN = ALD_CG_STATIC_MAX_N;
constexpr int kRows = 32;                      // rows per gemv block (one per lane)
constexpr int kColGroups = 8;                  // warps per gemv block, each a slice of the columns
constexpr int kMaxParts = (kMaxN + kRows - 1) / kRows;
constexpr int kVecThreads = 1024;
constexpr int kMaxDevices = 64;

struct CgState {
  double bnorm, err, fmin;
  int done, iters;
};

// Scratch layout (doubles): grad | conj | aux | partial | state.
constexpr size_t kOffGrad = 0;
constexpr size_t kOffConj = kOffGrad + kMaxN;
constexpr size_t kOffAux = kOffConj + kMaxN;
constexpr size_t kOffPart = kOffAux + kMaxN;
constexpr size_t kOffState = kOffPart + kMaxParts;
constexpr size_t kScratchDoubles = kOffState + (sizeof(CgState) + sizeof(double) - 1) / sizeof(double);

static __device__ __align__(256) double g_cg_scratch[kScratchDoubles];

// y = A x with A column-major (the reference's a(n,n)), so the 32 lanes of a
// warp read 32 consecutive rows of one column: 256 coalesced bytes.  Warp w of
// the block sums columns j = w, w+8, ...; the eight partial sums are added in
// a fixed order, so the result does not depend on scheduling.  partial[blk]
// receives sum over the block's rows of y_i * x_i (the CG denominator).
__global__ void __launch_bounds__(kRows * kColGroups)
    gemv_cm_kernel(int n, const double* __restrict__ A, const double* __restrict__ x, double* __restrict__ y,
                   double* __restrict__ partial, const CgState* st) {
  if (st && st->done) return;
  __shared__ double part[kColGroups][kRows];
  const int lane = threadIdx.x & 31, grp = threadIdx.x >> 5;
  const int row = blockIdx.x * kRows + lane;
  double s = 0.0;
  if (row < n)
    for (int j = grp; j < n; j += kColGroups) s += A[(size_t)j * n + row] * x[j];
  part[grp][lane] = s;
  __syncthreads();
  if (grp == 0) {
    double t = 0.0;
    for (int g = 0; g < kColGroups; ++g) t += part[g][lane];
    double d = 0.0;
    if (row < n) {
      y[row] = t;
      d = t * x[row];
    }
    for (int o = 16; o > 0; o >>= 1) d += __shfl_down_sync(0xffffffffu, d, o);
    if (lane == 0 && partial) partial[blockIdx.x] = d;
  }
}

__device__ double block_sum(double v) {
  __shared__ double red[kVecThreads / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) red[0] = t;
  }
  __syncthreads();
  double r = red[0];
  __syncthreads();
  return r;
}

// grad = A x - b, conj = -grad (cg.f90:30-34); resets the shared state
__global__ void cg_start_kernel(int n, const double* Ax, const double* b, double* grad, double* conj, CgState* st) {
  double bb = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double g = Ax[i] - b[i];
    grad[i] = g;
    conj[i] = -g;
    bb += b[i] * b[i];
  }
  bb = block_sum(bb);
  if (threadIdx.x == 0) {
    st->bnorm = sqrt(bb);
    st->err = 9999.0;
    st->fmin = 0.0;
    st->done = 0;
    st->iters = 0;
  }
}

// One iteration after aux = A conj (cg.f90:37-55): step length from
// grad.conj / conj.A.conj, update x and grad, stop when
// (num/den)^2 |conj|^2 / |x|^2 < tol, else the Fletcher-Reeves direction.
__global__ void cg_iter_kernel(int n, const double* aux, const double* partial, int nparts, double* grad,
                               double* conj, double* x, CgState* st, double tol) {
  if (st->done) return;
  double num = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) num += grad[i] * conj[i];
  num = block_sum(num);
  double den = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) den += partial[i];
  den = block_sum(den);
  const double alpha = num / den;
  double xx = 0.0, cc = 0.0, gg = 0.0, g0 = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double gi = grad[i], ci = conj[i];
    const double xi = x[i] - alpha * ci;
    const double gn = gi - alpha * aux[i];
    x[i] = xi;
    grad[i] = gn;
    xx += xi * xi;
    cc += ci * ci;
    gg += gn * gn;
    g0 += gi * gi;
  }
  xx = block_sum(xx);
  cc = block_sum(cc);
  gg = block_sum(gg);
  g0 = block_sum(g0);
  const double err = (num * num / den / den) * cc / xx;
  const bool stop = err < tol;
  if (!stop) {
    const double beta = gg / g0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) conj[i] = -grad[i] + beta * conj[i];
  }
  if (threadIdx.x == 0) {
    st->iters += 1;
    st->err = err;
    if (stop) st->done = 1;
  }
}

// funcmin = 1/2 x.A.x - b.x (cg.f90:57)
__global__ void cg_value_kernel(int n, const double* x, const double* Ax, const double* b, CgState* st) {
  double s1 = 0.0, s2 = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    s1 += x[i] * Ax[i];
    s2 += x[i] * b[i];
  }
  s1 = block_sum(s1);
  s2 = block_sum(s2);
  if (threadIdx.x == 0) st->fmin = 0.5 * s1 - s2;
}

// Device address of g_cg_scratch, looked up once per device.  In host code
// the name g_cg_scratch is only a host-side handle, never a device address.
std::mutex g_addr_mutex;
double* g_addr[kMaxDevices] = {nullptr};

int scratch_address(int dev, double** out, std::string& msg) {
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  if (!g_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_cg_scratch);
    if (e != cudaSuccess || !p) {
      msg = std::string("cg_static: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
      return ALD_ERR_CUDA;
    }
    g_addr[dev] = static_cast<double*>(p);
  }
  *out = g_addr[dev];
  return ALD_OK;
}

bool on_device(const void* p, int dev) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) && at.device == dev;
}

// The driver's cuMemGetAddressRange, reached through the runtime (the library
// links only cudart): the allocation that holds a device address.  Declared
// with plain types: CUdeviceptr is a 64-bit integer and CUresult an int.
using AddrRangeFn = int (*)(unsigned long long* base, size_t* size, unsigned long long ptr);

AddrRangeFn addr_range_fn() {
  static AddrRangeFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      f = nullptr;
    }
    return reinterpret_cast<AddrRangeFn>(f);
  }();
  return fn;
}

// false when the allocation holding p is known to end before p + bytes (a
// caller's slice too short for what the call reads or writes); true when it
// covers them or when its extent cannot be queried
bool covers(const void* p, size_t bytes) {
  AddrRangeFn fn = addr_range_fn();
  if (!fn) return true;
  unsigned long long base = 0;
  size_t size = 0;
  const unsigned long long q = reinterpret_cast<unsigned long long>(p);
  if (fn(&base, &size, q) != 0) return true;
  return q >= base && q - base <= size && bytes <= size - (size_t)(q - base);
}

using ald::capi::fail;

}  // namespace

extern "C" int ald_cg_quadratic_static(int n, const double* a, const double* b, double* vmin, double* funcmin,
                                       int max_iter, int n_dig_accur, int* iters, void* stream) {
  if (n <= 0 || !a || !b || !vmin) return fail(ALD_ERR_ARG, "cg_static: bad argument");
  if (n > kMaxN)
    return fail(ALD_ERR_ARG, "cg_static: n = " + std::to_string(n) + " exceeds ALD_CG_STATIC_MAX_N = " +
                                 std::to_string(kMaxN) + "; use ald_cg_quadratic");
  if (max_iter < 0) return fail(ALD_ERR_ARG, "cg_static: max_iter < 0");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(ALD_ERR_CUDA, std::string("cg_static: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(ALD_ERR_UNSUPPORTED, "cg_static: device ordinal out of range");
  if (!on_device(a, dev) || !on_device(b, dev) || !on_device(vmin, dev))
    return fail(ALD_ERR_ARG, "cg_static: a, b and vmin must be device memory of the current device");
  if (!covers(a, (size_t)n * n * sizeof(double)) || !covers(b, (size_t)n * sizeof(double)) ||
      !covers(vmin, (size_t)n * sizeof(double)))
    return fail(ALD_ERR_ARG, "cg_static: a holds fewer than n*n doubles, or b or vmin fewer than n, in its allocation");
  double* base = nullptr;
  std::string msg;
  int r = scratch_address(dev, &base, msg);
  if (r) return fail(r, msg);
  double* grad = base + kOffGrad;
  double* conj = base + kOffConj;
  double* aux = base + kOffAux;
  double* part = base + kOffPart;
  CgState* st = reinterpret_cast<CgState*>(base + kOffState);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nblk = (n + kRows - 1) / kRows;
  const double tol = 1.0 / std::pow(10.0, 2 * n_dig_accur);

  gemv_cm_kernel<<<nblk, kRows * kColGroups, 0, s>>>(n, a, vmin, aux, nullptr, nullptr);
  cg_start_kernel<<<1, kVecThreads, 0, s>>>(n, aux, b, grad, conj, st);
  // every 8 iterations the host reads the stop flag (into a stack copy, no
  // allocation) and stops launching once the stop rule has fired; the
  // iterations launched past it return at once
  CgState h;
  for (int it = 0; it < max_iter; ++it) {
    gemv_cm_kernel<<<nblk, kRows * kColGroups, 0, s>>>(n, a, conj, aux, part, st);
    cg_iter_kernel<<<1, kVecThreads, 0, s>>>(n, aux, part, nblk, grad, conj, vmin, st, tol);
    if ((it & 7) == 7 && it + 1 < max_iter) {
      e = cudaMemcpyAsync(&h, st, sizeof h, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) return fail(ALD_ERR_CUDA, std::string("cg_static: ") + cudaGetErrorString(e));
      if (h.done) break;
    }
  }
  gemv_cm_kernel<<<nblk, kRows * kColGroups, 0, s>>>(n, a, vmin, aux, nullptr, nullptr);
  cg_value_kernel<<<1, kVecThreads, 0, s>>>(n, vmin, aux, b, st);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, st, sizeof h, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(ALD_ERR_CUDA, std::string("cg_static: ") + cudaGetErrorString(e));
  if (funcmin) *funcmin = h.fmin;
  if (iters) *iters = h.iters;
  return h.done ? ALD_OK : ALD_WARN_CG_MAXITER;
}

/* dqmc_udv_green_noalloc: G = (1 + U diag(D) T)^{-1} without allocating.
 *
 * Same computation and arguments as dqmc_udv_green (host arrays in and
 * out), for callers that must not allocate device memory: a host
 * application whose device memory is owned by its own allocator (a
 * framework's caching pool that has reserved the GPU, where an outside
 * cudaMalloc fails or fragments its pool).  Every buffer the kernel needs
 * (the caller's U, D, T staged on the device, the positive-D UDV slot, the
 * QR workspaces, G and the sign) lives in one file-scope __device__ array
 * of fixed size for n <= DQMC_NOALLOC_MAX_N (128), about 1.1 MB.
 *
 * When that memory is taken: CUDA loads a module lazily (the default since
 * CUDA 12.2), so the array and this file's kernel are placed on a device by
 * the first call on that device, in its set-up (cudaGetSymbolAddress with
 * the device current, and the kernel's shared-memory limit).  That first
 * call can therefore fail for lack of device memory; make it before the
 * caller's allocator reserves the device, and before any stream capture on
 * the device.  Later calls take no device memory; the array stays until the
 * process exits.
 *
 * The call selects `device`, runs on that device's legacy default stream
 * with synchronous copies, returns only after the result has been copied
 * back, and restores the caller's current device before it returns.  All
 * calls share the one array and a call leaves its contents behind: the sign
 * slot is cleared at the start of every call and everything else is written
 * before it is read.  Two calls that overlap on the GPU (from two host
 * threads, for example) race on the array and must be serialized by the
 * caller.  No cudaMalloc, cudaFree or allocating library routine is called,
 * on the device or on the host.
 */
#define DQMC_NS dqn
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/dqmc_gpu.h"
#include "dqmc_device.cuh"

namespace {

constexpr int NMAX = DQMC_NOALLOC_MAX_N;
constexpr size_t NN = (size_t)NMAX * NMAX;
constexpr size_t TWSZ = (size_t)((NMAX + DQMC_QNB - 1) / DQMC_QNB) * DQMC_QNB * DQMC_QNB;
/* layout of the array, in doubles */
constexpr size_t OFF_U = 0;
constexpr size_t OFF_D = OFF_U + NN;
constexpr size_t OFF_T = OFF_D + NMAX;
constexpr size_t OFF_SLOT = OFF_T + NN;
constexpr size_t OFF_WS = OFF_SLOT + DQMC_UDV_SIZE(NMAX);
constexpr size_t OFF_G = OFF_WS + 3 * NN + TWSZ;
constexpr size_t OFF_SIGN = OFF_G + NN;
constexpr size_t TOTAL = OFF_SIGN + 8;

}  // namespace

static __device__ __align__(256) double g_udv_scratch[TOTAL];

namespace {

/* One CTA: sign of det U by a QR of a copy of U, the positive-D slot
 * (U columns times sign(D), log|D|, T), then udv_green into G. */
__global__ void __launch_bounds__(DQMC_NT, 1) k_udv_green_static(int n, double *base)
{
    extern __shared__ __align__(16) double smraw[];
    __shared__ int flag;
    using namespace dqn;
    if (threadIdx.x == 0) flag = 0;
    __syncthreads();
    Smem s = carve(smraw, n, 1);
    const double *U = base + OFF_U, *D = base + OFF_D, *T = base + OFF_T;
    double *ws = base + OFF_WS, *tw = ws + 3 * NN;
    int *sign_out = (int *)(base + OFF_SIGN);
    for (int e = threadIdx.x; e < n * n; e += NT) ws[e] = U[e];
    __syncthreads();
    const int nt = qr_factor(n, ws, tw, s, &flag);
    const int rs = qr_diag(n, ws, s, &flag);
    double negD = 0.0;
    for (int j = threadIdx.x; j < n; j += NT) negD += D[j] < 0.0 ? 1.0 : 0.0;
    negD = block_reduce<false>(negD, s.red);
    const double detU = ((nt & 1) ? -1.0 : 1.0) * rs * ((((long long)negD) & 1) ? -1.0 : 1.0);
    Udv u = udv_at(base + OFF_SLOT, n);
    for (int e = threadIdx.x; e < n * n; e += NT) {
        const int j = e / n;
        u.U[e] = D[j] < 0.0 ? -U[e] : U[e];
        u.T[e] = T[e];
    }
    for (int j = threadIdx.x; j < n; j += NT) u.ell[j] = log(fabs(D[j]));
    if (threadIdx.x == 0) *u.det = detU;
    __syncthreads();
    const Scr w{ws, ws + NN, ws + 2 * NN, tw};
    const int ds = udv_green(n, u, base + OFF_G, w, s, &flag);
    __syncthreads();
    if (threadIdx.x == 0) *sign_out = flag ? 0 : ds;
}

std::mutex g_setup_mutex;
double *g_base[64];
bool g_ready[64];

}  // namespace

extern "C" int dqmc_udv_green_noalloc(int device, int n, const double *U, const double *D,
                                      const double *T, double *G, int *det_sign);

namespace dqmc_internal {
void set_error(const char *msg);   /* dqmc_last_error() text, dqmc_engine.cu */
}

static int noalloc_fail(const char *msg, cudaError_t e)
{
    char buf[256];
    std::snprintf(buf, sizeof buf, "dqmc_udv_green_noalloc: %s%s%s", msg,
                  e != cudaSuccess ? ": " : "", e != cudaSuccess ? cudaGetErrorString(e) : "");
    dqmc_internal::set_error(buf);
    return 1;
}

/* Selects a device for the duration of one call and restores the caller's
 * current device on every return path. */
struct DeviceGuard {
    int prev = -1;
    ~DeviceGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

static int noalloc_call(int device, int n, const double *U, const double *D, const double *T,
                        double *G, int *det_sign);

extern "C" int dqmc_udv_green_noalloc(int device, int n, const double *U, const double *D,
                                      const double *T, double *G, int *det_sign)
{
    DeviceGuard guard;
    if (cudaGetDevice(&guard.prev) != cudaSuccess) guard.prev = -1;
    return noalloc_call(device, n, U, D, T, G, det_sign);
}

static int noalloc_call(int device, int n, const double *U, const double *D, const double *T,
                        double *G, int *det_sign)
{
    if (!U || !D || !T || !G || !det_sign) return noalloc_fail("null argument", cudaSuccess);
    if (n <= 0 || n > NMAX) {
        char msg[96];
        std::snprintf(msg, sizeof msg, "n=%d outside 1..%d (the fixed scratch limit)", n, NMAX);
        return noalloc_fail(msg, cudaSuccess);
    }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return noalloc_fail("no CUDA device", e);
    if (device < 0 || device >= ndev || device >= 64)
        return noalloc_fail("device out of range", cudaSuccess);
    if ((e = cudaSetDevice(device)) != cudaSuccess) return noalloc_fail("cudaSetDevice", e);
    const size_t smem = dqn::smem_doubles(NMAX, 1) * sizeof(double);
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_ready[device]) {
            void *p = nullptr;
            if ((e = cudaGetSymbolAddress(&p, g_udv_scratch)) != cudaSuccess)
                return noalloc_fail("cudaGetSymbolAddress", e);
            if ((e = cudaFuncSetAttribute(k_udv_green_static,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem)) != cudaSuccess)
                return noalloc_fail("cudaFuncSetAttribute", e);
            g_base[device] = (double *)p;
            g_ready[device] = true;
        }
    }
    double *base = g_base[device];
    const size_t bytes = (size_t)n * n * sizeof(double);
    if ((e = cudaMemcpy(base + OFF_U, U, bytes, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(base + OFF_D, D, (size_t)n * sizeof(double), cudaMemcpyHostToDevice)) !=
            cudaSuccess ||
        (e = cudaMemcpy(base + OFF_T, T, bytes, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(base + OFF_SIGN, 0, sizeof(double))) != cudaSuccess)
        return noalloc_fail("staging the inputs", e);
    k_udv_green_static<<<1, DQMC_NT, smem>>>(n, base);
    if ((e = cudaGetLastError()) != cudaSuccess) return noalloc_fail("launch", e);
    if ((e = cudaMemcpy(G, base + OFF_G, bytes, cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (e = cudaMemcpy(det_sign, base + OFF_SIGN, sizeof(int), cudaMemcpyDeviceToHost)) !=
            cudaSuccess)
        return noalloc_fail("reading the result", e);
    return 0;
}

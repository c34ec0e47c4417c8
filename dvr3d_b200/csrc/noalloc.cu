// noalloc.cu -- batched symmetric eigensolver entry point that allocates no device memory.
//
// Who needs it: callers that are not allowed to allocate device memory themselves or to let
// a library do so behind their back -- a host running inside a framework whose memory pool
// already owns (nearly) all of the GPU's memory and forbids foreign cudaMalloc calls, or a
// latency-critical loop where cudaMalloc/cudaFree (which can synchronise the whole device)
// must not occur. dvr3d_b200_diag_batched keeps its scratch in a per-context arena that grows
// with cudaMalloc; this variant runs the same kernels with all scratch taken from one
// fixed-size array compiled into the library.
//
// Properties a user must know:
//  * the scratch is a file-scope __device__ array of DVR3D_NOALLOC_SCRATCH_BYTES (64 MiB);
//    every GPU that loads this library holds it for the life of the process;
//  * its device address is looked up once per device (cudaGetSymbolAddress, with that device
//    current) by the first call on that device; make that first call before any stream
//    capture is started on the device;
//  * every call uses the same array: calls that can overlap on the GPU (different streams,
//    or different host threads on the same device) race on it and must be serialised by
//    the caller. Whatever must start at zero is cleared by each call;
//  * a request whose scratch exceeds the array fails with DVR3D_ERR_SCRATCH before any work.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "../../include/dvr3d_b200.h"
#include "common.cuh"
#include "eig_batched.cuh"

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[DVR3D_NOALLOC_SCRATCH_BYTES];

std::mutex g_scratch_mu;
constexpr int kMaxDevices = 64;
void *g_scratch_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (looked up once per device).
cudaError_t scratch_address(void **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return cudaSuccess;
}

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Blocks per call: the copy-in and symmetrisation launches put the block index in blockIdx.y.
constexpr int kMaxNoallocBlocks = 65535;

// Offsets of every block inside the scratch regions (one thread; nblk is small).
__global__ void noalloc_plan_kernel(int nblk, const int *n, long long *voff, long long *asz,
                                    long long *wkoff) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    long long v = 0, a = 0, w = 0;
    for (int b = 0; b < nblk; ++b) {
        const long long nb = n[b];
        voff[b] = v;
        asz[b] = a;
        wkoff[b] = w;
        v += nb;
        a += nb * nb;
        w += 5 * nb * (nb < 128 ? nb : 128) + nb * nb;
    }
}

// Copy the caller's blocks (at off[b], leading dimension n[b]) into the scratch copies.
__global__ void noalloc_copy_in_kernel(const int *n, const long long *off, const long long *asz,
                                       const double *a, double *acopy) {
    const int b = blockIdx.y;
    const long long nn = (long long)n[b] * n[b];
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += (long long)gridDim.x * blockDim.x)
        acopy[asz[b] + i] = a[off[b] + i];
}

// Eigenvalues to the caller's output (w + woff[b]).
__global__ void noalloc_copy_w_kernel(const int *n, const long long *voff, const long long *woff,
                                      const double *wsrc, double *wdst) {
    const int b = blockIdx.x;
    for (int i = threadIdx.x; i < n[b]; i += blockDim.x) wdst[woff[b] + i] = wsrc[voff[b] + i];
}

}  // namespace

extern "C" int dvr3d_b200_diag_batched_noalloc(void *stream, int nblk, const int *n_host,
                                                const long long *off_host, const long long *woff_host,
                                                double *a_dev, double *w_dev, int vecs) {
    if (nblk <= 0 || !n_host || !off_host || !woff_host || !a_dev || !w_dev) return DVR3D_ERR_ARG;
    if (nblk > kMaxNoallocBlocks) return DVR3D_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    // size the request with host arithmetic only
    int nmax = 0;
    size_t sum_n = 0, sum_n2 = 0, sum_work = 0;
    for (int b = 0; b < nblk; ++b) {
        const int nb = n_host[b];
        if (nb < 1 || nb > 1024) return DVR3D_ERR_ARG;
        nmax = std::max(nmax, nb);
        sum_n += (size_t)nb;
        sum_n2 += (size_t)nb * nb;
        sum_work += 5 * (size_t)nb * std::min(nb, 128) + (size_t)nb * nb;
    }
    const size_t meta =
        align256(sizeof(int) * nblk) * 2 + align256(sizeof(int)) + align256(sizeof(long long) * nblk) * 5 + 256;
    const size_t need = meta + align256(sizeof(double) * sum_n) * 4 + align256(sizeof(double) * sum_n2) +
                        (vecs ? align256(sizeof(double) * sum_work) : 0);
    if (need > (size_t)DVR3D_NOALLOC_SCRATCH_BYTES) return DVR3D_ERR_SCRATCH;
    void *base = nullptr;
    if (scratch_address(&base) != cudaSuccess) {
        cudaGetLastError();
        return DVR3D_ERR_CUDA;
    }
    // carve the fixed array
    unsigned char *p = static_cast<unsigned char *>(base);
    auto take = [&](size_t bytes) {
        unsigned char *q = p;
        p += align256(bytes);
        return q;
    };
    int *d_n = reinterpret_cast<int *>(take(sizeof(int) * nblk));
    int *d_cnt = reinterpret_cast<int *>(take(sizeof(int) * nblk));
    int *d_err = reinterpret_cast<int *>(take(sizeof(int)));
    long long *d_off = reinterpret_cast<long long *>(take(sizeof(long long) * nblk));
    long long *d_woff = reinterpret_cast<long long *>(take(sizeof(long long) * nblk));
    long long *d_voff = reinterpret_cast<long long *>(take(sizeof(long long) * nblk));
    long long *d_asz = reinterpret_cast<long long *>(take(sizeof(long long) * nblk));
    long long *d_wk = reinterpret_cast<long long *>(take(sizeof(long long) * nblk));
    double *d_d = reinterpret_cast<double *>(take(sizeof(double) * sum_n));
    double *d_e = reinterpret_cast<double *>(take(sizeof(double) * sum_n));
    double *d_tau = reinterpret_cast<double *>(take(sizeof(double) * sum_n));
    double *d_w = reinterpret_cast<double *>(take(sizeof(double) * sum_n));
    double *d_acopy = reinterpret_cast<double *>(take(sizeof(double) * sum_n2));
    double *d_work = vecs ? reinterpret_cast<double *>(take(sizeof(double) * sum_work)) : nullptr;
    cudaError_t e = cudaSuccess;
    auto ck = [&](cudaError_t x) {
        if (e == cudaSuccess && x != cudaSuccess) e = x;
    };
    ck(cudaMemcpyAsync(d_n, n_host, sizeof(int) * nblk, cudaMemcpyHostToDevice, st));
    ck(cudaMemcpyAsync(d_off, off_host, sizeof(long long) * nblk, cudaMemcpyHostToDevice, st));
    ck(cudaMemcpyAsync(d_woff, woff_host, sizeof(long long) * nblk, cudaMemcpyHostToDevice, st));
    ck(cudaMemsetAsync(d_err, 0, sizeof(int), st));  // the error flag starts at zero
    // Stop before anything is written to the caller's a_dev / w_dev when a launch fails: the
    // caller's blocks must survive a failed call, as they do with dvr3d_b200_diag_batched.
    auto bail = [&]() {
        cudaStreamSynchronize(st);
        cudaGetLastError();
        return DVR3D_ERR_CUDA;
    };
    if (e != cudaSuccess) return bail();
    noalloc_plan_kernel<<<1, 32, 0, st>>>(nblk, d_n, d_voff, d_asz, d_wk);
    ck(cudaGetLastError());
    noalloc_copy_in_kernel<<<dim3(64, nblk), 256, 0, st>>>(d_n, d_off, d_asz, a_dev, d_acopy);
    ck(cudaGetLastError());
    DVR3D_COUNT_LAUNCH(2);
    if (e != cudaSuccess) return bail();
    const dvr3d::BatchDesc bd{nblk, d_n, d_asz, d_voff};
    dvr3d::launch_symmetrize_lower(bd, d_acopy, nmax, st);
    ck(cudaGetLastError());
    dvr3d::launch_tridiag_batched(bd, d_acopy, d_d, d_e, d_tau, nmax, st);
    ck(cudaGetLastError());
    dvr3d::launch_eigvals_batched(bd, d_d, d_e, d_w, d_cnt, 0, 0.0, st);  // all eigenvalues
    ck(cudaGetLastError());
    if (e != cudaSuccess) return bail();
    noalloc_copy_w_kernel<<<nblk, 128, 0, st>>>(d_n, d_voff, d_woff, d_w, w_dev);
    DVR3D_COUNT_LAUNCH(1);
    ck(cudaGetLastError());
    if (vecs && e == cudaSuccess) {
        // eigenvectors of all eigenvalues written over the caller's blocks (ld = n)
        dvr3d::launch_eigvecs_batched(bd, d_acopy, d_d, d_e, d_tau, d_w, d_n, d_off, d_n, a_dev, d_work, d_wk,
                                      nmax, d_err, st);
        ck(cudaGetLastError());
    }
    int err_host = 0;
    if (vecs) ck(cudaMemcpyAsync(&err_host, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    ck(cudaStreamSynchronize(st));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return DVR3D_ERR_CUDA;
    }
    if (err_host != 0) return DVR3D_ERR_NOCONV;  // inverse iteration failed its growth test
    return DVR3D_OK;
}

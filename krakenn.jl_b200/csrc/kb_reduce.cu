// kb_reduce.cu -- FP64 reductions (mass, steady residual) with a device
// workspace for the per-block partial sums.
//
// Two passes.  Pass 1: a grid-stride loop in which every thread keeps a
// compensated (Neumaier) FP64 sum of its elements, then a warp-shuffle tree
// and a shared-memory tree inside the block; each block writes one partial
// (sum, compensation) pair.  Pass 2: one block adds the partials the same
// way and writes the result, which is copied to the host.  A non-finite
// input sets a flag that the host reads with the sums.
#include <cstring>

#include "kb_common.cuh"

namespace kb {
namespace red {

constexpr int RT = 256;  // threads per block in both passes

struct KSum {
    double s, c;
    __device__ __forceinline__ void add(double x) {
        const double t = s + x;
        if (fabs(s) >= fabs(x)) c += (s - t) + x;
        else c += (x - t) + s;
        s = t;
    }
    __device__ __forceinline__ void add(const KSum &o) { add(o.s); add(o.c); }
    __device__ __forceinline__ double value() const { return s + c; }
};

__device__ __forceinline__ KSum shfl_down(KSum v, int o) {
    KSum r;
    r.s = __shfl_down_sync(0xffffffffu, v.s, o);
    r.c = __shfl_down_sync(0xffffffffu, v.c, o);
    return r;
}

// Block-wide combine of NV independent compensated sums; thread 0 gets them.
template <int NV>
__device__ __forceinline__ void block_combine(KSum *v) {
    __shared__ KSum sh[NV][RT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int a = 0; a < NV; ++a) v[a].add(shfl_down(v[a], o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int a = 0; a < NV; ++a) sh[a][warp] = v[a];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int a = 0; a < NV; ++a) {
            v[a] = lane < RT / 32 ? sh[a][lane] : KSum{0.0, 0.0};
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[a].add(shfl_down(v[a], o));
        }
    }
}

template <typename R>
__device__ __forceinline__ double ldd(const R *p, size_t m) { return (double)p[m]; }
template <>
__device__ __forceinline__ double ldd<__half>(const __half *p, size_t m) { return (double)__half2float(p[m]); }
template <>
__device__ __forceinline__ double ldd<__nv_bfloat16>(const __nv_bfloat16 *p, size_t m) {
    return (double)__bfloat162float(p[m]);
}

// Pass 1 of the mass sum.  `dev` adds w_q back for deviation storages.
template <typename R>
__global__ void __launch_bounds__(RT) mass_pass1(const R *__restrict__ f, int Q, size_t n, bool dev,
                                                  KSum *__restrict__ part, int *__restrict__ bad) {
    KSum v[1] = {{0.0, 0.0}};
    bool nonfinite = false;
    const size_t total = (size_t)Q * n;
    for (size_t m = (size_t)blockIdx.x * RT + threadIdx.x; m < total; m += (size_t)gridDim.x * RT) {
        double x = ldd(f, m);
        if (!isfinite(x)) nonfinite = true;
        if (dev) {
            const int q = (int)(m / n);
            x += Q == 9 ? w9(q) : w19(q);
        }
        v[0].add(x);
    }
    if (nonfinite) atomicOr(bad, 1);
    block_combine<1>(v);
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

// Pass 1 of the residual: sums of |u - u_prev|^2 and |u|^2 over fluid nodes.
template <typename R>
__global__ void __launch_bounds__(RT) resid_pass1(const R *__restrict__ ux, const R *__restrict__ uy,
                                                   const R *__restrict__ uz, const R *__restrict__ uxp,
                                                   const R *__restrict__ uyp, const R *__restrict__ uzp,
                                                   const uint8_t *__restrict__ solid, size_t n,
                                                   KSum *__restrict__ part, int *__restrict__ bad) {
    KSum v[2] = {{0.0, 0.0}, {0.0, 0.0}};
    bool nonfinite = false;
    for (size_t m = (size_t)blockIdx.x * RT + threadIdx.x; m < n; m += (size_t)gridDim.x * RT) {
        if (solid && solid[m]) continue;
        const double a = ldd(ux, m), b = ldd(uy, m);
        const double da = a - ldd(uxp, m), db = b - ldd(uyp, m);
        double d = da * da + db * db, s = a * a + b * b;
        if (uz) {
            const double c = ldd(uz, m), dc = c - ldd(uzp, m);
            d += dc * dc;
            s += c * c;
        }
        if (!isfinite(d) || !isfinite(s)) nonfinite = true;
        v[0].add(d);
        v[1].add(s);
    }
    if (nonfinite) atomicOr(bad, 1);
    block_combine<2>(v);
    if (threadIdx.x == 0) { part[2 * blockIdx.x] = v[0]; part[2 * blockIdx.x + 1] = v[1]; }
}

// Pass 2: NV sums, partials laid out [block][NV]; out[a] = total a.
template <int NV>
__global__ void __launch_bounds__(RT) pass2(const KSum *__restrict__ part, int nblocks,
                                             double *__restrict__ out) {
    KSum v[NV];
#pragma unroll
    for (int a = 0; a < NV; ++a) v[a] = KSum{0.0, 0.0};
    for (int b = threadIdx.x; b < nblocks; b += RT)
#pragma unroll
        for (int a = 0; a < NV; ++a) v[a].add(part[NV * b + a]);
    block_combine<NV>(v);
    if (threadIdx.x == 0)
#pragma unroll
        for (int a = 0; a < NV; ++a) out[a] = v[a].value();
}

}  // namespace red

// ----------------------------------------------------------------- workspace
// Per-device grow-only buffer for the partials: [int flag | pad][double out[4]]
// [KSum partials...].  Allocated on the first call of a device (cudaMalloc,
// which also synchronises the device).
namespace {

struct Workspace {
    void *ptr = nullptr;
    size_t cap = 0;
};

void *reduce_workspace(size_t bytes, int *err) {
    static Workspace ws[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        *err = KB_ERR_CUDA;
        return nullptr;
    }
    Workspace &w = ws[dev];
    if (w.cap < bytes) {
        if (w.ptr) cudaFree(w.ptr);
        w.ptr = nullptr; w.cap = 0;
        if (cudaMalloc(&w.ptr, bytes) != cudaSuccess) {
            cudaGetLastError();
            *err = KB_ERR_NOMEM;
            return nullptr;
        }
        w.cap = bytes;
    }
    *err = KB_OK;
    return w.ptr;
}

constexpr size_t kHead = 64;  // flag + 4 result doubles, rounded to 64 B

int reduction_blocks(size_t items) {
    size_t b = (items + red::RT - 1) / red::RT;
    const size_t cap = (size_t)sm_count() * 4;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

// Read flag and results back (synchronises the stream through the copy).
int finish(const char *what, void *ws, int nres, double *res, int *bad, cudaStream_t s) {
    char head[kHead];
    cudaError_t e = cudaMemcpyAsync(head, ws, kHead, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_error(KB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    int flag;
    memcpy(&flag, head, sizeof(int));
    memcpy(res, head + 16, sizeof(double) * nres);
    *bad = flag;
    return KB_OK;
}

// ------------------------------------------------------- static scratch --
// Scratch of kb_mass_static: a fixed array in device memory that exists as
// soon as the library is loaded on a device, so that entry point never
// allocates.  Layout: [head: int flag @0, double result @16 | 64 B]
// [partial sums, one KSum per block].  Every GPU that loads the library
// holds these bytes until the process exits.
constexpr size_t kStaticScratchBytes = 256 * 1024;
constexpr size_t kStaticMaxPartials = (kStaticScratchBytes - kHead) / sizeof(red::KSum);
// Each thread of kb_mass_static adds up to 256 populations, so one block
// (256 threads) covers 65536 and one partial sum stands for 65536 items.
constexpr size_t kStaticItemsPerBlock = 256 * (size_t)red::RT;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// Device address of g_static_scratch on the current device, looked up once
// per device (host code may not use the symbol's name as an address).  The
// cached address belongs to the device's current context: after a
// cudaDeviceReset it is stale, and the process must not call
// kb_mass_static on that device again.
int static_scratch(char **out) {
    static char *addr[64] = {nullptr};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64)
        return set_error(KB_ERR_CUDA, "kb_mass_static: no current device");
    if (!addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p)
            return set_error(KB_ERR_CUDA, "kb_mass_static: cudaGetSymbolAddress failed: %s",
                             cudaGetErrorString(e));
        addr[dev] = (char *)p;
    }
    *out = addr[dev];
    return KB_OK;
}

}  // namespace
}  // namespace kb

extern "C" {

int kb_mass(const void *f, int lattice_q, size_t n_nodes, int dtype, double *out_host,
            void *stream) {
    using namespace kb;
    KB_REQUIRE(f && out_host, "kb_mass: null pointer");
    KB_REQUIRE(lattice_q == 9 || lattice_q == 19, "kb_mass: lattice_q must be 9 or 19");
    KB_REQUIRE(n_nodes > 0, "kb_mass: n_nodes must be positive");
    KB_REQUIRE(dtype_bytes(dtype), "kb_mass: unknown dtype %d", dtype);
    KB_REQUIRE(n_nodes <= SIZE_MAX / (size_t)lattice_q,
               "kb_mass: lattice_q * n_nodes overflows size_t (n_nodes = %zu)", n_nodes);
    const int nb = reduction_blocks((size_t)lattice_q * n_nodes);
    int err;
    char *ws = (char *)reduce_workspace(kHead + sizeof(red::KSum) * nb, &err);
    if (!ws) return set_error(err, "kb_mass: cannot allocate the reduction workspace");
    cudaStream_t s = as_stream(stream);
    int *bad = (int *)ws;
    double *out = (double *)(ws + 16);
    red::KSum *part = (red::KSum *)(ws + kHead);
    if (cudaMemsetAsync(ws, 0, kHead, s) != cudaSuccess)
        return set_error(KB_ERR_CUDA, "kb_mass: memset failed");
    dtype = storage_format(dtype);  // the stochastic-rounding storages share the format
    const bool dev = dtype == KB_F32_DEV || dtype == KB_F16_DEV || dtype == KB_BF16_DEV;
    switch (dtype) {
        case KB_F64: red::mass_pass1<double><<<nb, red::RT, 0, s>>>((const double *)f, lattice_q, n_nodes, dev, part, bad); break;
        case KB_F32:
        case KB_F32_DEV: red::mass_pass1<float><<<nb, red::RT, 0, s>>>((const float *)f, lattice_q, n_nodes, dev, part, bad); break;
        case KB_F16_DEV: red::mass_pass1<__half><<<nb, red::RT, 0, s>>>((const __half *)f, lattice_q, n_nodes, dev, part, bad); break;
        default: red::mass_pass1<__nv_bfloat16><<<nb, red::RT, 0, s>>>((const __nv_bfloat16 *)f, lattice_q, n_nodes, dev, part, bad); break;
    }
    red::pass2<1><<<1, red::RT, 0, s>>>(part, nb, out);
    if (int e = check_launch("kb_mass")) return e;
    int flag = 0;
    if (int e = finish("kb_mass", ws, 1, out_host, &flag, s)) return e;
    if (flag) return set_error(KB_ERR_NONFINITE, "kb_mass: non-finite population found");
    return KB_OK;
}

int kb_residual(const void *ux, const void *uy, const void *uz, const void *ux_prev,
                const void *uy_prev, const void *uz_prev, const uint8_t *is_solid,
                size_t n_nodes, int dtype, double *out_host, void *stream) {
    using namespace kb;
    KB_REQUIRE(ux && uy && ux_prev && uy_prev && out_host, "kb_residual: null pointer");
    KB_REQUIRE((uz == nullptr) == (uz_prev == nullptr), "kb_residual: uz and uz_prev must both be set or both NULL");
    KB_REQUIRE(n_nodes > 0, "kb_residual: n_nodes must be positive");
    KB_REQUIRE(dtype_bytes(dtype), "kb_residual: unknown dtype %d", dtype);
    const int nb = reduction_blocks(n_nodes);
    int err;
    char *ws = (char *)reduce_workspace(kHead + 2 * sizeof(red::KSum) * nb, &err);
    if (!ws) return set_error(err, "kb_residual: cannot allocate the reduction workspace");
    cudaStream_t s = as_stream(stream);
    int *bad = (int *)ws;
    double *out = (double *)(ws + 16);
    red::KSum *part = (red::KSum *)(ws + kHead);
    if (cudaMemsetAsync(ws, 0, kHead, s) != cudaSuccess)
        return set_error(KB_ERR_CUDA, "kb_residual: memset failed");
    if (dtype == KB_F64)
        red::resid_pass1<double><<<nb, red::RT, 0, s>>>((const double *)ux, (const double *)uy, (const double *)uz,
            (const double *)ux_prev, (const double *)uy_prev, (const double *)uz_prev, is_solid, n_nodes, part, bad);
    else
        red::resid_pass1<float><<<nb, red::RT, 0, s>>>((const float *)ux, (const float *)uy, (const float *)uz,
            (const float *)ux_prev, (const float *)uy_prev, (const float *)uz_prev, is_solid, n_nodes, part, bad);
    red::pass2<2><<<1, red::RT, 0, s>>>(part, nb, out);
    if (int e = check_launch("kb_residual")) return e;
    double sums[2];
    int flag = 0;
    if (int e = finish("kb_residual", ws, 2, sums, &flag, s)) return e;
    *out_host = sqrt(sums[0] / sums[1]);
    if (flag) return set_error(KB_ERR_NONFINITE, "kb_residual: non-finite velocity found");
    return KB_OK;
}

// Allocation-free variant of kb_mass: the partial sums live in the library's
// fixed device array instead of a cudaMalloc'ed workspace.
int kb_mass_static(const void *f, int lattice_q, size_t n_nodes, int dtype, double *out_host,
                   void *stream) {
    using namespace kb;
    KB_REQUIRE(f && out_host, "kb_mass_static: null pointer");
    KB_REQUIRE(lattice_q == 9 || lattice_q == 19, "kb_mass_static: lattice_q must be 9 or 19");
    KB_REQUIRE(n_nodes > 0, "kb_mass_static: n_nodes must be positive");
    KB_REQUIRE(dtype_bytes(dtype), "kb_mass_static: unknown dtype %d", dtype);
    // (a product that wrapped around would pass the limit check below)
    KB_REQUIRE(n_nodes <= SIZE_MAX / (size_t)lattice_q,
               "kb_mass_static: lattice_q * n_nodes overflows size_t (n_nodes = %zu)", n_nodes);
    const size_t items = (size_t)lattice_q * n_nodes;
    const size_t nb = (items + kStaticItemsPerBlock - 1) / kStaticItemsPerBlock;
    if (nb > kStaticMaxPartials)
        return set_error(KB_ERR_ARG,
                         "kb_mass_static: %zu populations exceed the static scratch limit of %zu "
                         "(%zu KiB); use kb_mass", items, kStaticMaxPartials * kStaticItemsPerBlock,
                         kStaticScratchBytes / 1024);
    char *ws = nullptr;
    if (int e = static_scratch(&ws)) return e;
    cudaStream_t s = as_stream(stream);
    int *bad = (int *)ws;
    double *out = (double *)(ws + 16);
    red::KSum *part = (red::KSum *)(ws + kHead);
    // the flag and the result must start at zero; the partials are all written
    if (cudaMemsetAsync(ws, 0, kHead, s) != cudaSuccess)
        return set_error(KB_ERR_CUDA, "kb_mass_static: memset failed");
    dtype = storage_format(dtype);  // the stochastic-rounding storages share the format
    const bool dev = dtype == KB_F32_DEV || dtype == KB_F16_DEV || dtype == KB_BF16_DEV;
    const int blocks = (int)nb;
    switch (dtype) {
        case KB_F64: red::mass_pass1<double><<<blocks, red::RT, 0, s>>>((const double *)f, lattice_q, n_nodes, dev, part, bad); break;
        case KB_F32:
        case KB_F32_DEV: red::mass_pass1<float><<<blocks, red::RT, 0, s>>>((const float *)f, lattice_q, n_nodes, dev, part, bad); break;
        case KB_F16_DEV: red::mass_pass1<__half><<<blocks, red::RT, 0, s>>>((const __half *)f, lattice_q, n_nodes, dev, part, bad); break;
        default: red::mass_pass1<__nv_bfloat16><<<blocks, red::RT, 0, s>>>((const __nv_bfloat16 *)f, lattice_q, n_nodes, dev, part, bad); break;
    }
    red::pass2<1><<<1, red::RT, 0, s>>>(part, blocks, out);
    if (int e = check_launch("kb_mass_static")) return e;
    int flag = 0;
    if (int e = finish("kb_mass_static", ws, 1, out_host, &flag, s)) return e;
    if (flag) return set_error(KB_ERR_NONFINITE, "kb_mass_static: non-finite population found");
    return KB_OK;
}

}  // extern "C"

// kb_surrogate.cu -- the warm-start network: a 4-level convolutional
// encoder-decoder (U-Net) with BF16 weights and activations and FP32
// accumulation, trained and evaluated entirely by this library's kernels.
//
// Every 3x3 convolution (forward, data gradient, weight gradient) runs on the
// tcgen05 mainloop of kb_umma.cuh as an implicit GEMM over NHWC activations:
//   forward   D[pixel, cout]      = sum_(tap,cin) X(pixel+tap, cin) W[cout, tap, cin]
//   data grad D[pixel, cin]       = sum_(tap,cout) dY(pixel+tap, cout) W[cout, 8-tap, cin]
//   weight    D[(tap,cin), cout]  = sum_pixel X(pixel+tap, cin) dY(pixel, cout)  (+ bias row)
// The decoder's nearest-neighbour upsampling and skip concatenation are
// folded into the operand loader (ActView), so neither is materialised.
//
// Network (C = base channels, resolution H x W at level 0):
//   enc1a 8->C, enc1b C->C | pool | enc2a C->2C, enc2b | pool | enc3a 2C->4C,
//   enc3b | pool | bott_a 4C->8C, bott_b 8C->8C | dec3a [up(8C), 4C]->4C, dec3b |
//   dec2a [up(4C), 2C]->2C, dec2b | dec1a [up(2C), C]->C, dec1b | head C->16
// ReLU after every convolution except the head; 2x2 average pooling.  The
// head's channels 0..2 are the normalised (rho, ux, uy); 3..15 are unused.
//
// Parameters are one flat FP32 array: per layer W[cout][9*cin] (k = tap*cin +
// c, tap = (dy+1)*3 + (dx+1)) followed by b[cout].  Adam keeps FP32 moments;
// the BF16 operand copies (forward and transposed-flipped) are repacked after
// every update.
#include <algorithm>
#include <cmath>
#include <vector>

#include "kb_common.cuh"
#include "kb_umma_tma.cuh"

namespace kb {
namespace sur {

using bf16 = __nv_bfloat16;
using umma::ActView;

enum {
    T_IN, T_E1A, T_E1B, T_P1, T_E2A, T_E2B, T_P2, T_E3A, T_E3B, T_P3,
    T_BA, T_BB, T_D3A, T_D3B, T_D2A, T_D2B, T_D1A, T_D1B, T_OUT, T_COUNT
};
constexpr int IN_CH = 8, OUT_CH = 16, N_LAYERS = 15;

struct LayerSpec { int in1, in2, out, relu, pooled_in; };
constexpr LayerSpec kLayers[N_LAYERS] = {
    {T_IN, -1, T_E1A, 1, 0},  {T_E1A, -1, T_E1B, 1, 0}, {T_P1, -1, T_E2A, 1, 1},
    {T_E2A, -1, T_E2B, 1, 0}, {T_P2, -1, T_E3A, 1, 1},  {T_E3A, -1, T_E3B, 1, 0},
    {T_P3, -1, T_BA, 1, 1},   {T_BA, -1, T_BB, 1, 0},   {T_BB, T_E3B, T_D3A, 1, 0},
    {T_D3A, -1, T_D3B, 1, 0}, {T_D3B, T_E2B, T_D2A, 1, 0}, {T_D2A, -1, T_D2B, 1, 0},
    {T_D2B, T_E1B, T_D1A, 1, 0}, {T_D1A, -1, T_D1B, 1, 0}, {T_D1B, -1, T_OUT, 0, 0},
};

// channels (as a multiple of C, or absolute when negative) and level of each tensor
struct TensorSpec { int mult, level; };
constexpr TensorSpec kTensors[T_COUNT] = {
    {-IN_CH, 0}, {1, 0}, {1, 0}, {1, 1}, {2, 1}, {2, 1}, {2, 2}, {4, 2}, {4, 2}, {4, 3},
    {8, 3}, {8, 3}, {4, 2}, {4, 2}, {2, 1}, {2, 1}, {1, 0}, {1, 0}, {-OUT_CH, 0},
};

__host__ __device__ inline int round_up(int a, int b) { return (a + b - 1) / b * b; }

// ------------------------------------------------------------------ kernels

// 2x2 average pooling, NHWC BF16, 8 channels per thread.
__global__ void pool_k(bf16 *__restrict__ out, const bf16 *__restrict__ in, int B, int Ho, int Wo,
                       int C) {
    const int cc = C / 8;
    const unsigned n = (unsigned)B * Ho * Wo * cc;  // < 2^31 (kb_surrogate_create)
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const unsigned p = t / cc;
        const int c = (int)(t - p * cc) * 8;
        const unsigned r = p / Wo, b = r / Ho;
        const int w = (int)(p - r * Wo), h = (int)(r - b * Ho);
        float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                const size_t q = (((size_t)b * 2 * Ho + 2 * h + dy) * 2 * Wo + 2 * w + dx) * C + c;
                const uint4 v = *reinterpret_cast<const uint4 *>(in + q);
                const bf16 *e = reinterpret_cast<const bf16 *>(&v);
#pragma unroll
                for (int i = 0; i < 8; ++i) s[i] += __bfloat162float(e[i]);
            }
        __align__(16) bf16 o[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) o[i] = __float2bfloat16_rn(0.25f * s[i]);
        *reinterpret_cast<uint4 *>(out + (size_t)p * C + c) = *reinterpret_cast<const uint4 *>(o);
    }
}

// Nearest upsampling, NHWC BF16, 8 channels per thread: dst [B][H][W][C] from
// src [B][H/2][W/2][C] (the decoder input that the TMA engine copies by boxes).
__global__ void upsample_k(bf16 *__restrict__ dst, const bf16 *__restrict__ src, int B, int H, int W,
                           int C) {
    const int cc = C / 8;
    const unsigned n = (unsigned)B * H * W * cc;  // < 2^31 (kb_surrogate_create)
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const unsigned p = t / cc;
        const int c = (int)(t - p * cc) * 8;
        const unsigned r = p / W, b = r / H;
        const int w = (int)(p - r * W), h = (int)(r - b * H);
        const size_t q = (((size_t)b * (H / 2) + h / 2) * (W / 2) + w / 2) * C + c;
        *reinterpret_cast<uint4 *>(dst + (size_t)p * C + c) = *reinterpret_cast<const uint4 *>(src + q);
    }
}

// Gradient of nearest upsampling: dst (low resolution, Cl channels) = sum of
// the 2x2 children of src channels [0, Cl) (src has Cs channels).
__global__ void upsum_k(bf16 *__restrict__ dst, const bf16 *__restrict__ src, int B, int Hl, int Wl,
                        int Cl, int Cs) {
    const int cc = Cl / 8;
    const unsigned n = (unsigned)B * Hl * Wl * cc;  // < 2^31 (kb_surrogate_create)
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const unsigned p = t / cc;
        const int c = (int)(t - p * cc) * 8;
        const unsigned r = p / Wl, b = r / Hl;
        const int w = (int)(p - r * Wl), h = (int)(r - b * Hl);
        float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                const size_t q = (((size_t)b * 2 * Hl + 2 * h + dy) * 2 * Wl + 2 * w + dx) * Cs + c;
                const uint4 v = *reinterpret_cast<const uint4 *>(src + q);
                const bf16 *e = reinterpret_cast<const bf16 *>(&v);
#pragma unroll
                for (int i = 0; i < 8; ++i) s[i] += __bfloat162float(e[i]);
            }
        __align__(16) bf16 o[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) o[i] = __float2bfloat16_rn(s[i]);
        *reinterpret_cast<uint4 *>(dst + (size_t)p * Cl + c) = *reinterpret_cast<const uint4 *>(o);
    }
}

// Gradient of a skip tensor S (C channels, H x W) used by a decoder concat
// (channels [off, off+C) of dcat, Cc channels, already masked) and by a 2x2
// average pool (dpool at H/2 x W/2, not masked):
//   dS = dcat[.., off + c] + (S > 0) * dpool(parent) / 4
__global__ void skip_grad_k(bf16 *__restrict__ dst, const bf16 *__restrict__ dcat,
                            const bf16 *__restrict__ dpool, const bf16 *__restrict__ S, int B, int H,
                            int W, int C, int Cc, int off) {
    const int cc = C / 8;
    const unsigned n = (unsigned)B * H * W * cc;  // < 2^31 (kb_surrogate_create)
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const unsigned p = t / cc;
        const int c = (int)(t - p * cc) * 8;
        const unsigned r = p / W, b = r / H;
        const int w = (int)(p - r * W), h = (int)(r - b * H);
        const size_t pp = (((size_t)b * (H / 2) + h / 2) * (W / 2) + w / 2) * C + c;
        const uint4 a = *reinterpret_cast<const uint4 *>(dcat + (size_t)p * Cc + off + c);
        const uint4 g = *reinterpret_cast<const uint4 *>(dpool + pp);
        const uint4 s = *reinterpret_cast<const uint4 *>(S + (size_t)p * C + c);
        const bf16 *ea = reinterpret_cast<const bf16 *>(&a);
        const bf16 *eg = reinterpret_cast<const bf16 *>(&g);
        const bf16 *es = reinterpret_cast<const bf16 *>(&s);
        __align__(16) bf16 o[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            float v = __bfloat162float(ea[i]);
            if (__bfloat162float(es[i]) > 0.f) v += 0.25f * __bfloat162float(eg[i]);
            o[i] = __float2bfloat16_rn(v);
        }
        *reinterpret_cast<uint4 *>(dst + (size_t)p * C + c) = *reinterpret_cast<const uint4 *>(o);
    }
}

// Loss over channels 0..2 of the head against the normalised target
// ((t - offset) * scale, target planar [n][3][H][W]), with e = pred - target:
//   L = 1/(3M) sum_{pixels, c} [ e_c^2 + gw * ((e_c(x+1) - e_c(x))^2 + (e_c(y+1) - e_c(y))^2) ]
// The gradient term (an H1 seminorm; gw = 0 gives the mean-squared error)
// weights an error of wavenumber k by about 1 + gw k^2, so it penalises
// grid-scale error, which the plain method's slow wall mode picks up, far
// more than smooth error.  Differences are taken only between pixels of the
// same image.  Writes dL/dpred (BF16, OUT_CH channels, zero beyond 2) and adds
// L to *loss.
struct Norm { float scale[3], offset[3]; };

// One block per tile of LTX x LTY pixels of one image (grid x, y, image): the
// errors of the tile and its one-pixel halo are computed once into shared
// memory, then each pixel forms its loss terms and gradient from them.
constexpr int LTX = 32, LTY = 8;
__global__ void __launch_bounds__(LTX *LTY) loss_k(bf16 *__restrict__ grad, float *__restrict__ loss,
                                                   const float *__restrict__ pred,
                                                   const float *__restrict__ target, Norm nm, int M, int H,
                                                   int W, float gw) {
    __shared__ float E[3][LTY + 2][LTX + 2];
    __shared__ float red[LTX * LTY / 32];
    const int HW = H * W, b = blockIdx.z;
    const int x0 = blockIdx.x * LTX, y0 = blockIdx.y * LTY;
    const float gs = 2.0f / (3.0f * (float)M);
    for (int u = threadIdx.x; u < (LTX + 2) * (LTY + 2); u += LTX * LTY) {
        const int ly = u / (LTX + 2), lx = u - ly * (LTX + 2);
        const int x = x0 + lx - 1, y = y0 + ly - 1;
        float e0 = 0.f, e1 = 0.f, e2 = 0.f;
        if (x >= 0 && x < W && y >= 0 && y < H) {
            const int p = y * W + x;
            const float4 pr = *reinterpret_cast<const float4 *>(pred + ((size_t)b * HW + p) * OUT_CH);
            const float *tg = target + (size_t)b * 3 * HW + p;
            e0 = pr.x - (tg[0] - nm.offset[0]) * nm.scale[0];
            e1 = pr.y - (tg[HW] - nm.offset[1]) * nm.scale[1];
            e2 = pr.z - (tg[2 * HW] - nm.offset[2]) * nm.scale[2];
        }
        E[0][ly][lx] = e0;
        E[1][ly][lx] = e1;
        E[2][ly][lx] = e2;
    }
    __syncthreads();
    const int tx = threadIdx.x % LTX, ty = threadIdx.x / LTX;
    const int x = x0 + tx, y = y0 + ty;
    float acc = 0.f;
    if (x < W && y < H) {
        __align__(16) bf16 g[OUT_CH];
#pragma unroll
        for (int c = 0; c < OUT_CH; ++c) g[c] = __float2bfloat16_rn(0.f);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float e = E[c][ty + 1][tx + 1];
            acc += e * e;
            float d = e;
            if (gw != 0.f) {
                // forward differences owned by this pixel enter the loss; the
                // gradient collects the differences with all four neighbours
                float lap = 0.f;
                if (x + 1 < W) {
                    const float en = E[c][ty + 1][tx + 2];
                    acc += gw * (en - e) * (en - e);
                    lap += e - en;
                }
                if (y + 1 < H) {
                    const float en = E[c][ty + 2][tx + 1];
                    acc += gw * (en - e) * (en - e);
                    lap += e - en;
                }
                if (x > 0) lap += e - E[c][ty + 1][tx];
                if (y > 0) lap += e - E[c][ty][tx + 1];
                d += gw * lap;
            }
            g[c] = __float2bfloat16_rn(gs * d);
        }
        uint4 *dst = reinterpret_cast<uint4 *>(grad + ((size_t)b * HW + (size_t)y * W + x) * OUT_CH);
        dst[0] = reinterpret_cast<const uint4 *>(g)[0];
        dst[1] = reinterpret_cast<const uint4 *>(g)[1];
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float sum = 0.f;
        for (int i = 0; i < LTX * LTY / 32; ++i) sum += red[i];
        atomicAdd(loss, sum / (3.0f * (float)M));
    }
}

// Head output (normalised, [M][OUT_CH]) -> physical planar [n][3][H][W].
__global__ void unpack_k(float *__restrict__ out, const float *__restrict__ pred, Norm nm, int M, int HW) {
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
        const int b = m / HW, p = m - b * HW;
#pragma unroll
        for (int c = 0; c < 3; ++c)
            out[((size_t)b * 3 + c) * HW + p] = pred[(size_t)m * OUT_CH + c] / nm.scale[c] + nm.offset[c];
    }
}

// Sum the split-K partials of the weight gradients of all layers into the
// flat gradient array, in a fixed order, in two launches for the whole
// network (the gradients are needed only after the backward pass).  Job k:
// part [splits][Rp+1][Cout] (Rp = 9 Cp, E = (Rp+1) Cout elements) ->
// gW[cout][9 Cs], gb[cout] (row Rp).  A job with many splits first sums groups
// of `per` consecutive splits into tmp [groups][E] (wgrad_group_all_k), and
// the final pass sums the groups.  Cp > Cs: the partials carry zero-padded
// input channels c >= Cs, which are dropped.
struct RJob {
    const float *part;
    float *tmp, *gW, *gb;
    int splits, groups, per, E, Cp, Cs, cout;
    long long g_start, r_start;  // first work item of the job in each pass
};
constexpr int N_LAYERS_MAX = 16;  // >= N_LAYERS
static_assert(N_LAYERS <= N_LAYERS_MAX, "job tables hold every layer");
struct RJobs {
    RJob j[N_LAYERS_MAX];
    int n;
    long long g_total, r_total;
};

__global__ void wgrad_group_all_k(const RJobs J) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < J.g_total;
         t += (long long)gridDim.x * blockDim.x) {
        int k = 0;
        while (k + 1 < J.n && t >= J.j[k + 1].g_start) ++k;
        const RJob &b = J.j[k];
        const int u = (int)(t - b.g_start), g = u / b.E, e = u - g * b.E;
        const int z0 = g * b.per, z1 = min(b.splits, z0 + b.per);
        float s = 0.f;
        for (int z = z0; z < z1; ++z) s += b.part[(size_t)z * b.E + e];
        b.tmp[(size_t)g * b.E + e] = s;
    }
}

__global__ void wgrad_reduce_all_k(const RJobs J) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < J.r_total;
         t += (long long)gridDim.x * blockDim.x) {
        int k = 0;
        while (k + 1 < J.n && t >= J.j[k + 1].r_start) ++k;
        const RJob &b = J.j[k];
        const int e = (int)(t - b.r_start);
        const float *src = b.groups > 1 ? b.tmp : b.part;
        const int nz = b.groups > 1 ? b.groups : b.splits;
        float s = 0.f;
        for (int z = 0; z < nz; ++z) s += src[(size_t)z * b.E + e];
        const int Rp = 9 * b.Cp, r = e / b.cout, co = e - r * b.cout;
        if (r == Rp) {
            b.gb[co] = s;
        } else {
            const int tap = r / b.Cp, c = r - tap * b.Cp;
            if (c < b.Cs) b.gW[((size_t)co * 9 + tap) * b.Cs + c] = s;
        }
    }
}

__global__ void adam_k(float *__restrict__ p, float *__restrict__ m, float *__restrict__ v,
                       const float *__restrict__ g, long long n, float lr_t, float b1, float b2,
                       float eps_t) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr_t * mi / (sqrtf(vi) + eps_t);
    }
}

// W [Cout][9 Cin] FP32 -> wb [Cout][Kp] and wt [Cin][Kpt] BF16 (zero padded):
//   wt[ci][t*Cout + co] = W[co][(8 - t)*Cin + ci]
// The BF16 operand copies of every layer's weights in one launch.  Job k:
// W [Cout][9 Cin] FP32 -> wb [Cout][Kp] and wt [Cin][Kpt] (zero padded):
//   wt[ci][t*Cout + co] = W[co][(8 - t)*Cin + ci]
// or, for a padded job (pad = Cp > Cin input channels, no wt):
//   wb[co][t*Cp + c] = W[co][t*Cin + c] (0 for c >= Cin).
struct PJob {
    bf16 *wb, *wt;
    const float *W;
    int Cin, Cout, Kp, Kpt, pad;
    long long start;
};
struct PJobs {
    PJob j[N_LAYERS_MAX + 1];
    int n;
    long long total;
};
__global__ void pack_all_k(const PJobs J) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < J.total;
         t += (long long)gridDim.x * blockDim.x) {
        int k = 0;
        while (k + 1 < J.n && t >= J.j[k + 1].start) ++k;
        const PJob &b = J.j[k];
        const int u0 = (int)(t - b.start), n1 = b.Cout * b.Kp;
        if (b.pad) {
            const int co = u0 / b.Kp, kk = u0 - co * b.Kp;
            float x = 0.f;
            if (kk < 9 * b.pad) {
                const int tap = kk / b.pad, c = kk - tap * b.pad;
                if (c < b.Cin) x = b.W[((size_t)co * 9 + tap) * b.Cin + c];
            }
            b.wb[u0] = __float2bfloat16_rn(x);
        } else if (u0 < n1) {
            const int co = u0 / b.Kp, kk = u0 - co * b.Kp;
            b.wb[u0] = __float2bfloat16_rn(kk < 9 * b.Cin ? b.W[(size_t)co * 9 * b.Cin + kk] : 0.f);
        } else {
            const int u = u0 - n1, ci = u / b.Kpt, kk = u - ci * b.Kpt;
            float x = 0.f;
            if (kk < 9 * b.Cout) {
                const int tap = kk / b.Cout, co = kk - tap * b.Cout;
                x = b.W[(size_t)co * 9 * b.Cin + (8 - tap) * b.Cin + ci];
            }
            b.wt[u] = __float2bfloat16_rn(x);
        }
    }
}

// Network input of n lid-driven cavities at H x W (NHWC BF16, IN_CH channels):
// 0 wall mask (x = 0, x = W-1, y = 0), 1 lid row (y = H-1), 2 (ln Re - ln 100)/ln 32,
// 3 N/512, 4 x in (-1, 1), 5 y in (-1, 1), 6-7 zero.
__global__ void cavity_inputs_k(bf16 *__restrict__ in, const float *__restrict__ re, int n, int H,
                                int W, float n_norm) {
    const long long total = (long long)n * H * W;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int w = (int)(t % W), h = (int)((t / W) % H), b = (int)(t / ((long long)W * H));
        __align__(16) bf16 o[IN_CH];
        o[0] = __float2bfloat16_rn((w == 0 || w == W - 1 || h == 0) ? 1.f : 0.f);
        o[1] = __float2bfloat16_rn(h == H - 1 ? 1.f : 0.f);
        o[2] = __float2bfloat16_rn((logf(re[b]) - 4.605170186f) / 3.465735903f);
        o[3] = __float2bfloat16_rn(n_norm);
        o[4] = __float2bfloat16_rn(2.f * (w + 0.5f) / W - 1.f);
        o[5] = __float2bfloat16_rn(2.f * (h + 0.5f) / H - 1.f);
        o[6] = o[7] = __float2bfloat16_rn(0.f);
        *reinterpret_cast<uint4 *>(in + (size_t)t * IN_CH) = *reinterpret_cast<const uint4 *>(o);
    }
}

// The network input (IN_CH = 8 channels) zero-padded to PAD_CH = 16 channels
// per pixel, the narrowest channel run a swizzled TMA box copies.
constexpr int PAD_CH = 16;
__global__ void pad_input_k(bf16 *__restrict__ dst, const bf16 *__restrict__ src, long long npix) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix;
         p += (long long)gridDim.x * blockDim.x) {
        uint4 *d = reinterpret_cast<uint4 *>(dst + p * PAD_CH);
        d[0] = *reinterpret_cast<const uint4 *>(src + p * IN_CH);
        d[1] = make_uint4(0, 0, 0, 0);
    }
}

inline dim3 ew_grid(long long n) {
    long long b = (n + 255) / 256;
    const long long cap = (long long)kb::sm_count() * 16;
    return dim3((unsigned)(b < 1 ? 1 : (b > cap ? cap : b)));
}

// ------------------------------------------------------------------ network

struct Layer {
    int cin1, cin2, up1, cin, cout, level, relu, pooled_in, in1, in2, out;
    int Kp, Kpt, bn_f, bn_d, bn_w;
    long long w_off, b_off;
    bf16 *wb = nullptr, *wt = nullptr;
    bf16 *dx = nullptr;  // data-gradient output (own buffer for concat inputs)
    bf16 *up = nullptr;  // decoder layers: in1 upsampled to this level (TMA engine)
    size_t part_off = 0, tmp_off = 0;  // this layer's regions of the weight-gradient buffers
};

// The TMA engine's operations of one layer for a batch of n images (the maps
// bound the image index by n, so images beyond the batch read as zeros).
// f / d / w: how the forward, data-gradient and weight-gradient operations
// run -- row strips where rows are wide enough and one output-channel tile
// holds the layer, else per-tap boxes where the shapes tile into boxes, else
// the one-CTA-per-tile engine.
struct TmaPlan {
    int n = -1;
    int f = 0, d = 0, w = 0;  // 0: per-tile engine, 1: TMA per-tap boxes, 2: TMA row strips
    int wsplits = 0, wgroups = 1;
    int cp = 0;               // input channels of the weight-gradient partials (padded first layer: PAD_CH)
    kb::umma::ConvTma fwd, dgr;
    kb::umma::ConvStrip sfwd, sdgr;
    kb::umma::WgradTma wg;
    kb::umma::WgradStrip swg;
};

}  // namespace sur
}  // namespace kb

using namespace kb::sur;

struct kb_surrogate {
    int Bmax, H, W, C;
    std::vector<Layer> L;
    int tch[T_COUNT];
    bf16 *act[T_COUNT] = {};
    bf16 *grad[T_COUNT] = {};
    float *out_f32 = nullptr;           // head output [Bmax*H*W][OUT_CH]
    float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    long long n_params = 0;
    float *part = nullptr;              // split-K partials
    size_t part_floats = 0;
    float *tmp = nullptr;               // grouped sums of the partials
    size_t tmp_floats = 0;
    int *err = nullptr;
    float *loss = nullptr;
    Norm norm{{1.f, 1.f, 1.f}, {0.f, 0.f, 0.f}};
    float grad_weight = 0.f;  // weight of the gradient (H1) term of the loss
    std::vector<TmaPlan> tp;            // per layer, TMA engine
    bf16 *ones = nullptr;               // [72][64] BF16, column 0 = 1: the bias row's A block
    int up_batch = -1;                  // batch of the decoder inputs last upsampled
    bf16 *in_pad = nullptr;             // [Bmax*H*W][PAD_CH]: the input padded for the TMA engine
    bf16 *wb_pad = nullptr;             // [cout][Kp_pad]: first layer's weights for PAD_CH channels
    int Kp_pad = 0;
    int pad_batch = -1;                 // batch of the input last padded
    std::vector<void *> allocs;
    int H_at(int level) const { return H >> level; }
    int W_at(int level) const { return W >> level; }
};

namespace {

int alloc(kb_surrogate *s, void **p, size_t bytes) {
    if (cudaMalloc(p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return kb::set_error(KB_ERR_NOMEM, "kb_surrogate_create: cudaMalloc of %zu bytes failed", bytes);
    }
    s->allocs.push_back(*p);
    return 0;
}

ActView view_of(const kb_surrogate *s, const Layer &l, int n) {
    ActView v{};
    v.s1 = s->act[l.in1];
    v.c1 = l.cin1;
    v.up1 = l.up1;
    v.s2 = l.in2 >= 0 ? s->act[l.in2] : nullptr;
    v.c2 = l.cin2;
    v.B = n;
    v.H = s->H_at(l.level);
    v.W = s->W_at(l.level);
    return v;
}

// Upper bound of the split count of a layer's weight gradient (any batch).
int max_wgrad_splits(const Layer &l) {
    const int R = 9 * l.cin;
    const int tiles = ((R + 1 + kb::umma::BM - 1) / kb::umma::BM) * (l.cout / l.bn_w);
    const int want = (2 * kb::sm_count() + tiles - 1) / tiles;
    return want < 1 ? 1 : want;
}

// Splits of the pixel (K) range so that about two CTAs per SM run; every
// split gets at least one K step and the count never exceeds the bound above.
int wgrad_splits(const Layer &l, int M, int &steps_per_split) {
    const int nsteps = (M + kb::umma::BK - 1) / kb::umma::BK;
    int want = max_wgrad_splits(l);
    if (want > nsteps) want = nsteps;
    steps_per_split = (nsteps + want - 1) / want;
    return (nsteps + steps_per_split - 1) / steps_per_split;
}

// Decoder input in1 of layer l upsampled to the layer's level (l.up).
void upsample(kb_surrogate *s, const Layer &l, int n, cudaStream_t st) {
    const int H = s->H_at(l.level), W = s->W_at(l.level);
    upsample_k<<<ew_grid((long long)n * H * W * (l.cin1 / 8)), 256, 0, st>>>(l.up, s->act[l.in1], n, H,
                                                                              W, l.cin1);
}

// Row-strip weight gradient of a layer (input channels cin1 + cin2 in
// chunks of ea): the chunks per tile (cpt, a divisor of the chunk count)
// with the most MMA issuers per SM, the TMEM columns of a tile's
// accumulators (all taps of its chunks plus the bias row) and the fit
// (CTAs per SM); false when the layer does not take that form.
struct StripWgradPlan { int ea, cpt, sr; uint32_t cols, strip, stage; kb::umma::TmaBase fit; };
bool plan_strip_wgrad(const Layer &l, int W, int cin1, StripWgradPlan &P) {
    using namespace kb::umma;
    const int ea = chunk_of(cin1, l.cin2), bn = l.bn_w;
    if (!ea || !chunk_of(bn) || W % BK || l.cout != bn || (bn & (bn - 1))) return false;
    const int nck = (cin1 + l.cin2) / ea, mtp = ea == 64 ? 2 : 1;
    const int sr = BK + (BM / ea - 1 > 3 ? BM / ea - 1 : 3);  // strip rows
    const uint32_t strip = round1k((uint32_t)(sr * 2 * ea));
    bool found = false;
    for (int cpt = nck; cpt >= 1; --cpt) {
        if (nck % cpt) continue;
        const uint32_t need = (uint32_t)((3 * cpt * mtp + 1) * bn);
        uint32_t cols = 32;
        while (cols < need) cols <<= 1;
        if (cols > 512) continue;
        TmaBase b{};
        b.a_bytes = 3u * (uint32_t)cpt * strip;
        b.b_bytes = round1k((uint32_t)(bn * BK * 2));
        b.res_bytes = (uint32_t)(72 * 2 * ea);
        b.acc_cols = cols;
        b.nbuf = 1;
        // one CTA per SM (512 accumulator columns) measured slower than the
        // per-tap boxes: take this form only where CTAs share the SM
        if ((b.cps = tma_fit(b)) < 2) continue;
        if (!found || b.cps > P.fit.cps) {
            P = StripWgradPlan{ea, cpt, sr, cols, strip, b.a_bytes + b.b_bytes, b};
            found = true;
        }
    }
    return found;
}

// Row-strip convolution (forward or data gradient): input channels c1 + c2
// in chunks of e, weights [Nout][Kp] resident, Nout one tile of bn.
int conv_strip(kb::umma::ConvStrip &c, const bf16 *x1, int c1, const bf16 *x2, int c2, const bf16 *wmat,
               int Kp, int bn, int e, int H, int W, int n, const char *what) {
    using namespace kb::umma;
    int rc;
    const PixBox strip{BM + 2, 1, 1};
    if ((rc = nhwc_map(&c.x1, x1, c1, W, H, n, e, strip, what))) return rc;
    if (x2 && (rc = nhwc_map(&c.x2, x2, c2, W, H, n, e, strip, what))) return rc;
    if (!x2) c.x2 = c.x1;
    const cuuint64_t d[2] = {(cuuint64_t)Kp, (cuuint64_t)bn}, sd[1] = {(cuuint64_t)Kp * 2};
    const cuuint32_t bx[2] = {(cuuint32_t)e, (cuuint32_t)bn};
    if ((rc = bf16_map(&c.w, wmat, 2, d, sd, bx, 2 * e, what))) return rc;
    const int C = c1 + c2;
    c.e = e;
    c.c1 = c1;
    c.C = C;
    c.H = H;
    c.W = W;
    c.nck = C / e;
    c.strip_bytes = round1k((uint32_t)((BM + 2) * 2 * e));
    c.acc_cols = tmem_cols(bn);
    c.nbuf = 2;
    c.ncols = bn;
    // resident weights, or streamed ones where that at least doubles the CTAs
    // per SM (96-channel decoder input: 2 -> 4, 130 against 151 us; 3 -> 4
    // measured slower: copying the weights per stage costs more)
    c.streamed = 0;
    c.tx = (uint32_t)(c.nck * (BM + 2) * 2 * e);
    c.a_bytes = (uint32_t)c.nck * c.strip_bytes;
    c.b_bytes = 0;
    c.res_bytes = (uint32_t)(9 * c.nck * bn * 2 * e);
    const int cps_res = tma_fit(c);
    ConvStrip t = c;
    t.streamed = 1;
    t.tx = (uint32_t)((BM + 2) * 2 * e + 3 * bn * 2 * e);
    t.a_bytes = c.strip_bytes;
    t.b_bytes = round1k((uint32_t)(3 * bn * 2 * e));
    t.res_bytes = 0;
    const int cps_str = tma_fit(t);
    if (cps_str >= 2 * cps_res) c = t;
    c.cps = c.streamed ? cps_str : cps_res;
    return c.cps ? 0 : kb::set_error(KB_ERR_ARG, "%s: row-strip convolution does not fit", what);
}

// Whether a row-strip convolution of these shapes fits the engine.
bool conv_strip_fits(int C, int e, int bn, int W) {
    using namespace kb::umma;
    if (!e || W % BM) return false;
    TmaBase b{};
    const int nck = C / e;
    b.a_bytes = (uint32_t)nck * round1k((uint32_t)((BM + 2) * 2 * e));
    b.res_bytes = (uint32_t)(9 * nck * bn * 2 * e);
    b.acc_cols = tmem_cols(bn);
    b.nbuf = 2;
    TmaBase t = b;  // streamed weights
    t.a_bytes = round1k((uint32_t)((BM + 2) * 2 * e));
    t.b_bytes = round1k((uint32_t)(3 * bn * 2 * e));
    t.res_bytes = 0;
    return tma_fit(b) > 0 || tma_fit(t) > 0;
}

// The network input (s->act[T_IN]) padded to PAD_CH channels (s->in_pad).
void pad_input(kb_surrogate *s, int n, cudaStream_t st) {
    const long long npix = (long long)n * s->H * s->W;
    pad_input_k<<<ew_grid(npix), 256, 0, st>>>(s->in_pad, s->act[T_IN], npix);
}

// Build (or keep) the TMA engine's operations of layer i for n images.
int prepare_tma(kb_surrogate *s, int i, int n) {
    using namespace kb::umma;
    const Layer &l = s->L[i];
    TmaPlan &p = s->tp[i];
    if (p.n == n) return 0;
    p.n = -1;
    p.f = p.d = p.w = 0;
    const char *what = "kb_surrogate (TMA engine)";
    const int H = s->H_at(l.level), W = s->W_at(l.level), M = n * H * W;
    // the first layer reads the input padded to PAD_CH channels
    const bool padded = l.in1 == T_IN && l.cin1 % 16;
    const int cin1 = padded ? PAD_CH : l.cin1, cin = cin1 + l.cin2;
    const bf16 *x1 = padded ? s->in_pad : (l.in2 >= 0 ? l.up : s->act[l.in1]);
    const bf16 *x2 = l.in2 >= 0 ? s->act[l.in2] : nullptr;
    const bf16 *wb = padded ? s->wb_pad : l.wb;
    const int Kp = padded ? s->Kp_pad : l.Kp;
    p.cp = cin;
    PixBox b128{}, b64{};
    const bool g128 = pix_box(BM, H, W, b128), g64 = pix_box(BK, H, W, b64);
    int rc = 0;
    // forward: row strips, or boxes of e input channels x 128 pixels (weights e x bn_f)
    const int ef = chunk_of(cin1, l.cin2);
    if (ef && l.cout == l.bn_f && conv_strip_fits(cin, ef, l.bn_f, W)) {
        ConvStrip &c = p.sfwd;
        c = ConvStrip{};
        if ((rc = conv_strip(c, x1, cin1, x2, l.cin2, wb, Kp, l.bn_f, ef, H, W, n, what))) return rc;
        c.bias = s->params + l.b_off;
        c.mask.s1 = nullptr;
        c.out = l.out == T_OUT ? (void *)s->out_f32 : (void *)s->act[l.out];
        c.M = M;
        c.Nout = l.cout;
        c.bn = l.bn_f;
        c.relu = l.relu;
        c.out_f32 = l.out == T_OUT;
        c.store_cols = l.out == T_OUT ? 8 : 0;  // the head: the loss and unpacking read channels 0-2
        p.f = 2;
    } else if (ef && g128) {
        ConvTma &c = p.fwd;
        c = ConvTma{};
        if ((rc = nhwc_map(&c.x1, x1, cin1, W, H, n, ef, b128, what))) return rc;
        if (x2 && (rc = nhwc_map(&c.x2, x2, l.cin2, W, H, n, ef, b128, what))) return rc;
        if (!x2) c.x2 = c.x1;
        const cuuint64_t d[2] = {(cuuint64_t)Kp, (cuuint64_t)l.cout}, sd[1] = {(cuuint64_t)Kp * 2};
        const cuuint32_t bx[2] = {(cuuint32_t)ef, (cuuint32_t)l.bn_f};
        if ((rc = bf16_map(&c.w, wb, 2, d, sd, bx, 2 * ef, what))) return rc;
        c.e = ef;
        c.c1 = cin1;
        c.C = cin;
        c.H = H;
        c.W = W;
        c.nck = cin / ef;
        c.a_bytes = round1k((uint32_t)(BM * 2 * ef));
        c.b_bytes = round1k((uint32_t)(l.bn_f * 2 * ef));
        c.res_bytes = 0;
        c.acc_cols = tmem_cols(l.bn_f);
        c.nbuf = 2;
        c.ncols = l.bn_f;
        c.cps = tma_fit(c);
        c.tx = (uint32_t)(BM * 2 * ef + l.bn_f * 2 * ef);
        c.bias = s->params + l.b_off;
        c.mask.s1 = nullptr;
        c.out = l.out == T_OUT ? (void *)s->out_f32 : (void *)s->act[l.out];
        c.M = M;
        c.Nout = l.cout;
        c.bn = l.bn_f;
        c.relu = l.relu;
        c.out_f32 = l.out == T_OUT;
        c.store_cols = l.out == T_OUT ? 8 : 0;  // the head: the loss and unpacking read channels 0-2
        p.f = c.cps ? 1 : 0;
    }
    // data gradient: row strips, or boxes of e output-gradient channels
    // (weights wt [cin][Kpt])
    const int ed = chunk_of(l.cout);
    if (i > 0 && ed && l.cin == l.bn_d && conv_strip_fits(l.cout, ed, l.bn_d, W)) {
        ConvStrip &c = p.sdgr;
        c = ConvStrip{};
        if ((rc = conv_strip(c, s->grad[l.out], l.cout, nullptr, 0, l.wt, l.Kpt, l.bn_d, ed, H, W, n, what)))
            return rc;
        c.bias = nullptr;
        if (l.pooled_in) c.mask.s1 = nullptr;
        else c.mask = view_of(s, l, n);
        c.out = l.dx;
        c.M = M;
        c.Nout = l.cin;
        c.bn = l.bn_d;
        c.relu = 0;
        c.out_f32 = 0;
        p.d = 2;
    } else if (i > 0 && ed && g128) {
        ConvTma &c = p.dgr;
        c = ConvTma{};
        if ((rc = nhwc_map(&c.x1, s->grad[l.out], l.cout, W, H, n, ed, b128, what))) return rc;
        c.x2 = c.x1;
        const cuuint64_t d[2] = {(cuuint64_t)l.Kpt, (cuuint64_t)l.cin}, sd[1] = {(cuuint64_t)l.Kpt * 2};
        const cuuint32_t bx[2] = {(cuuint32_t)ed, (cuuint32_t)l.bn_d};
        if ((rc = bf16_map(&c.w, l.wt, 2, d, sd, bx, 2 * ed, what))) return rc;
        c.e = ed;
        c.c1 = l.cout;
        c.C = l.cout;
        c.H = H;
        c.W = W;
        c.nck = l.cout / ed;
        c.a_bytes = round1k((uint32_t)(BM * 2 * ed));
        c.b_bytes = round1k((uint32_t)(l.bn_d * 2 * ed));
        c.res_bytes = 0;
        c.acc_cols = tmem_cols(l.bn_d);
        c.nbuf = 2;
        c.ncols = l.bn_d;
        c.cps = tma_fit(c);
        c.tx = (uint32_t)(BM * 2 * ed + l.bn_d * 2 * ed);
        c.bias = nullptr;
        if (l.pooled_in) c.mask.s1 = nullptr;
        else c.mask = view_of(s, l, n);
        c.out = l.dx;
        c.M = M;
        c.Nout = l.cin;
        c.bn = l.bn_d;
        c.relu = 0;
        c.out_f32 = 0;
        p.d = c.cps ? 1 : 0;
    }
    // weight gradient: row strips (whole gradient per pixel split), or blocks
    // of ea input channels / eb output-gradient channels x 64 pixels
    const int ea = chunk_of(cin1, l.cin2), eb = chunk_of(l.bn_w);
    StripWgradPlan sp{};
    if (eb && plan_strip_wgrad(l, W, cin1, sp)) {
        WgradStrip &w = p.swg;
        w = WgradStrip{};
        const PixBox strip{sp.sr, 1, 1};
        if ((rc = nhwc_map(&w.x1, x1, cin1, W, H, n, ea, strip, what))) return rc;
        if (x2 && (rc = nhwc_map(&w.x2, x2, l.cin2, W, H, n, ea, strip, what))) return rc;
        if (!x2) w.x2 = w.x1;
        const cuuint64_t d[2] = {(cuuint64_t)ea, 72}, sd[1] = {128};
        const cuuint32_t bx[2] = {(cuuint32_t)ea, 72};
        if ((rc = bf16_map(&w.ones, s->ones, 2, d, sd, bx, 2 * ea, what))) return rc;
        if ((rc = nhwc_map(&w.dy, s->grad[l.out], l.cout, W, H, n, eb, b64, what))) return rc;
        const int ngroups = cin / ea / sp.cpt;
        const int nsteps = (M + BK - 1) / BK;
        // about one tile (chunk group, pixel split) per CTA
        int want = (kb::sm_count() * sp.fit.cps + ngroups - 1) / ngroups;
        if (want > nsteps) want = nsteps;
        const int sps = (nsteps + want - 1) / want;
        p.wsplits = (nsteps + sps - 1) / sps;
        p.wgroups = ngroups;
        w.part = s->part + l.part_off;
        w.bn = l.bn_w;
        w.ea = ea;
        w.eb = eb;
        w.c1 = cin1;
        w.C = cin;
        w.H = H;
        w.W = W;
        w.Nout = l.cout;
        w.steps_per_split = sps;
        w.nsteps = nsteps;
        w.cpt = sp.cpt;
        w.mtp = ea == 64 ? 2 : 1;
        w.nb = l.bn_w / eb;
        w.nmt = 3 * sp.cpt * w.mtp;
        w.ea_shift = ea == 64 ? 6 : (ea == 32 ? 5 : 4);
        w.bn_shift = 31 - __builtin_clz((unsigned)l.bn_w);
        w.strip_bytes = sp.strip;
        w.tx = (uint32_t)(3 * sp.cpt * sp.sr * 2 * ea + l.bn_w * BK * 2);
        w.a_bytes = sp.fit.a_bytes;
        w.b_bytes = sp.fit.b_bytes;
        w.res_bytes = sp.fit.res_bytes;
        w.acc_cols = sp.cols;
        w.nbuf = 1;  // about one tile per CTA: nothing to overlap the epilogue with
        w.ncols = (w.nmt + 1) * l.bn_w;
        w.cps = tma_fit(w);
        p.w = w.cps ? 2 : 0;
    } else if (ea && eb && g64) {
        WgradTma &w = p.wg;
        w = WgradTma{};
        if ((rc = nhwc_map(&w.x1, x1, cin1, W, H, n, ea, b64, what))) return rc;
        if (x2 && (rc = nhwc_map(&w.x2, x2, l.cin2, W, H, n, ea, b64, what))) return rc;
        if (!x2) w.x2 = w.x1;
        const cuuint64_t d[2] = {(cuuint64_t)ea, 64}, sd[1] = {128};
        const cuuint32_t bx[2] = {(cuuint32_t)ea, 64};
        if ((rc = bf16_map(&w.ones, s->ones, 2, d, sd, bx, 2 * ea, what))) return rc;
        if ((rc = nhwc_map(&w.dy, s->grad[l.out], l.cout, W, H, n, eb, b64, what))) return rc;
        int sps = 0;
        p.wsplits = wgrad_splits(l, M, sps);
        w.part = s->part + l.part_off;
        w.bn = l.bn_w;
        w.ea = ea;
        w.eb = eb;
        w.c1 = cin1;
        w.C = cin;
        w.H = H;
        w.W = W;
        w.Nout = l.cout;
        w.steps_per_split = sps;
        w.nsteps = (M + BK - 1) / BK;
        w.py = W < BK && H * W >= BK ? BK / W : 0;
        w.pb = H * W < BK ? BK / (H * W) : 0;
        w.na = BM / ea;
        w.nb = l.bn_w / eb;
        w.a_bytes = BM * BK * 2;
        w.b_bytes = round1k((uint32_t)(l.bn_w * BK * 2));
        w.res_bytes = 0;
        w.acc_cols = tmem_cols(l.bn_w);
        w.nbuf = 2;
        w.ncols = l.bn_w;
        w.cps = tma_fit(w);
        p.w = w.cps ? 1 : 0;
    }
    p.n = n;
    return 0;
}

int forward(kb_surrogate *s, const void *input, int n, cudaStream_t st) {
    using namespace kb::umma;
    s->act[T_IN] = (bf16 *)input;
    const bool tma = engine() == 2;
    if (tma) pad_input(s, n, st);
    for (int i = 0; i < N_LAYERS; ++i) {
        const Layer &l = s->L[i];
        // pooled inputs are produced just before their consumer
        if (l.pooled_in) {
            const Layer &src = s->L[i - 1];
            const int Ho = s->H_at(l.level), Wo = s->W_at(l.level);
            pool_k<<<ew_grid((long long)n * Ho * Wo * (src.cout / 8)), 256, 0, st>>>(
                s->act[l.in1], s->act[src.out], n, Ho, Wo, src.cout);
        }
        const int M = n * s->H_at(l.level) * s->W_at(l.level);
        const dim3 grid((M + BM - 1) / BM, l.cout / l.bn_f);
        if (tma) {
            if (l.in2 >= 0) upsample(s, l, n, st);
            if (int rc = prepare_tma(s, i, n)) return rc;
            const TmaPlan &tp = s->tp[i];
            if (tp.f) {
                if (int rc = tp.f == 2 ? launch_tma(tp.sfwd, grid, s->err, st)
                                       : launch_tma(tp.fwd, grid, s->err, st))
                    return rc;
                continue;
            }
        }
        ConvOp op{};
        op.x = view_of(s, l, n);
        op.wt = l.wb;
        op.bias = s->params + l.b_off;
        op.mask.s1 = nullptr;
        op.out = l.out == T_OUT ? (void *)s->out_f32 : (void *)s->act[l.out];
        op.M = M;
        op.Nout = l.cout;
        op.Kp = l.Kp;
        op.bn = l.bn_f;
        op.relu = l.relu;
        op.out_f32 = l.out == T_OUT;
        op.nsteps = l.Kp / BK;
        if (int rc = launch(op, grid, s->err, st)) return rc;
    }
    s->up_batch = tma ? n : -1;
    return kb::check_launch("kb_surrogate forward");
}

// Queue the reduction of layer l's split partials (input channels Cp in the
// partials) into its gradient; run_reduce_jobs runs the queue.
void add_reduce_job(kb_surrogate *s, RJobs &J, const Layer &l, int splits, int Cp) {
    const long long E = (long long)(9 * Cp + 1) * l.cout;
    int groups = 1, per = splits;
    if (splits >= 16) {
        groups = (int)((300000 + E - 1) / E);
        groups = std::min(groups, splits / 8);
        groups = std::max(groups, 1);
        per = (splits + groups - 1) / groups;
        groups = (splits + per - 1) / per;
    }
    RJob &b = J.j[J.n++];
    b.part = s->part + l.part_off;
    b.tmp = s->tmp + l.tmp_off;  // holds 300000 + E floats >= groups E
    b.gW = s->grads + l.w_off;
    b.gb = s->grads + l.b_off;
    b.splits = splits;
    b.groups = groups;
    b.per = per;
    b.E = (int)E;
    b.Cp = Cp;
    b.Cs = l.cin;
    b.cout = l.cout;
    b.g_start = J.g_total;
    b.r_start = J.r_total;
    if (groups > 1) J.g_total += groups * E;
    J.r_total += E;
}

void run_reduce_jobs(const RJobs &J, cudaStream_t st) {
    if (J.g_total) wgrad_group_all_k<<<ew_grid(J.g_total), 256, 0, st>>>(J);
    if (J.r_total) wgrad_reduce_all_k<<<ew_grid(J.r_total), 256, 0, st>>>(J);
}

int backward(kb_surrogate *s, int n, cudaStream_t st) {
    using namespace kb::umma;
    const bool tma = engine() == 2;
    RJobs jobs{};
    if (tma && s->up_batch != n) {
        // the forward pass ran on another engine: upsample the decoder inputs
        // and pad the network input
        for (const Layer &l : s->L)
            if (l.in2 >= 0) upsample(s, l, n, st);
        pad_input(s, n, st);
        s->up_batch = n;
    }
    for (int i = N_LAYERS - 1; i >= 0; --i) {
        const Layer &l = s->L[i];
        const int Hl = s->H_at(l.level), Wl = s->W_at(l.level);
        const int M = n * Hl * Wl;
        const ActView xv = view_of(s, l, n);
        if (tma)
            if (int rc = prepare_tma(s, i, n)) return rc;
        const TmaPlan &tp = s->tp[i];
        const int R = 9 * l.cin;
        // weight gradient (split over pixels) and its reduction; the TMA
        // engine's partials carry tp.cp input channels (the padded input's
        // PAD_CH for the first layer)
        int sps = 0;
        int splits = wgrad_splits(l, M, sps);
        if (tma && tp.w == 2) {
            splits = tp.wsplits;
            if (int rc = launch_tma(tp.swg, dim3(tp.wgroups, 1, splits), s->err, st)) return rc;
        } else if (tma && tp.w == 1) {
            splits = tp.wsplits;
            const dim3 wg((9 * tp.cp + 1 + BM - 1) / BM, l.cout / l.bn_w, splits);
            if (int rc = launch_tma(tp.wg, wg, s->err, st)) return rc;
        } else {
            WgradOp wo{};
            wo.x = xv;
            wo.dy = s->grad[l.out];
            wo.part = s->part + l.part_off;
            wo.M = M;
            wo.Nout = l.cout;
            wo.bn = l.bn_w;
            wo.steps_per_split = sps;
            wo.nsteps = (M + BK - 1) / BK;
            const dim3 wg((R + 1 + BM - 1) / BM, l.cout / l.bn_w, splits);
            if (int rc = launch(wo, wg, s->err, st)) return rc;
        }
        add_reduce_job(s, jobs, l, splits, (tma && tp.w) ? tp.cp : l.cin);
        if (i == 0) break;
        // data gradient
        const dim3 grid((M + BM - 1) / BM, l.cin / l.bn_d);
        if (tma && tp.d) {
            if (int rc = tp.d == 2 ? launch_tma(tp.sdgr, grid, s->err, st) : launch_tma(tp.dgr, grid, s->err, st))
                return rc;
        } else {
            ConvOp op{};
            op.x.s1 = s->grad[l.out];
            op.x.c1 = l.cout;
            op.x.up1 = 0;
            op.x.s2 = nullptr;
            op.x.c2 = 0;
            op.x.B = n;
            op.x.H = Hl;
            op.x.W = Wl;
            op.wt = l.wt;
            op.bias = nullptr;
            if (l.pooled_in) op.mask.s1 = nullptr;
            else op.mask = xv;
            op.out = l.dx;
            op.M = M;
            op.Nout = l.cin;
            op.Kp = l.Kpt;
            op.bn = l.bn_d;
            op.relu = 0;
            op.out_f32 = 0;
            op.nsteps = l.Kpt / BK;
            if (int rc = launch(op, grid, s->err, st)) return rc;
        }
        // route the concat's gradient: the upsampled part to the low-resolution tensor
        if (l.in2 >= 0) {
            const Layer &lo = s->L[i - 1];  // producer of in1 (bott_b / dec3b / dec2b)
            const int Hlo = s->H_at(lo.level), Wlo = s->W_at(lo.level);
            upsum_k<<<ew_grid((long long)n * Hlo * Wlo * (l.cin1 / 8)), 256, 0, st>>>(
                s->grad[l.in1], l.dx, n, Hlo, Wlo, l.cin1, l.cin);
        }
        // a pooled input: finish the skip tensor's gradient (concat part + pool part)
        if (l.pooled_in) {
            const int skip = s->L[i - 1].out;  // enc1b / enc2b / enc3b
            const Layer *dec = nullptr;
            for (const Layer &d : s->L)
                if (d.in2 == skip) dec = &d;
            const int Hs = s->H_at(s->L[i - 1].level), Ws = s->W_at(s->L[i - 1].level);
            const int Cs = s->L[i - 1].cout;
            skip_grad_k<<<ew_grid((long long)n * Hs * Ws * (Cs / 8)), 256, 0, st>>>(
                s->grad[skip], dec->dx, s->grad[l.in1], s->act[skip], n, Hs, Ws, Cs, dec->cin,
                dec->cin1);
        }
    }
    run_reduce_jobs(jobs, st);
    return kb::check_launch("kb_surrogate backward");
}

int repack(kb_surrogate *s, cudaStream_t st) {
    PJobs J{};
    for (int i = 0; i < N_LAYERS; ++i) {
        const Layer &l = s->L[i];
        PJob &b = J.j[J.n++];
        b.wb = l.wb;
        b.wt = l.wt;
        b.W = s->params + l.w_off;
        b.Cin = l.cin;
        b.Cout = l.cout;
        b.Kp = l.Kp;
        b.Kpt = l.Kpt;
        b.pad = 0;
        b.start = J.total;
        J.total += (long long)l.cout * l.Kp + (l.wt ? (long long)l.cin * l.Kpt : 0);
    }
    // the first layer's weights for the input padded to PAD_CH channels
    const Layer &l0 = s->L[0];
    PJob &b = J.j[J.n++];
    b.wb = s->wb_pad;
    b.wt = nullptr;
    b.W = s->params + l0.w_off;
    b.Cin = l0.cin;
    b.Cout = l0.cout;
    b.Kp = s->Kp_pad;
    b.Kpt = 0;
    b.pad = PAD_CH;
    b.start = J.total;
    J.total += (long long)l0.cout * s->Kp_pad;
    pack_all_k<<<ew_grid(J.total), 256, 0, st>>>(J);
    return kb::check_launch("kb_surrogate repack");
}

uint64_t splitmix(uint64_t &x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace

extern "C" {

int kb_surrogate_create(kb_surrogate **out, int max_batch, int H, int W, int base_channels,
                        unsigned long long seed, void *stream) {
    KB_REQUIRE(out, "kb_surrogate_create: null handle pointer");
    *out = nullptr;
    KB_REQUIRE(max_batch > 0, "kb_surrogate_create: max_batch=%d must be positive", max_batch);
    KB_REQUIRE(H >= 8 && W >= 8 && H % 8 == 0 && W % 8 == 0,
               "kb_surrogate_create: H=%d and W=%d must be multiples of 8 (three 2x2 poolings)", H, W);
    KB_REQUIRE(base_channels >= 16 && base_channels % 16 == 0 && base_channels <= 128,
               "kb_surrogate_create: base_channels=%d must be a multiple of 16 in [16, 128]",
               base_channels);
    // the elementwise kernels index 8-channel chunks of an activation with 32
    // bits: no tensor has more than 12 base_channels channels
    KB_REQUIRE((double)max_batch * H * W * (12.0 * base_channels / 8) < 2147483647.0,
               "kb_surrogate_create: max_batch x H x W = %d x %d x %d too large for %d base channels",
               max_batch, H, W, base_channels);
    cudaStream_t st = kb::as_stream(stream);
    kb_surrogate *s = new kb_surrogate();
    s->Bmax = max_batch;
    s->H = H;
    s->W = W;
    s->C = base_channels;
    for (int t = 0; t < T_COUNT; ++t)
        s->tch[t] = kTensors[t].mult < 0 ? -kTensors[t].mult : kTensors[t].mult * base_channels;
    long long off = 0;
    for (int i = 0; i < N_LAYERS; ++i) {
        const LayerSpec &sp = kLayers[i];
        Layer l;
        l.in1 = sp.in1;
        l.in2 = sp.in2;
        l.out = sp.out;
        l.relu = sp.relu;
        l.pooled_in = sp.pooled_in;
        l.cin1 = s->tch[sp.in1];
        l.cin2 = sp.in2 >= 0 ? s->tch[sp.in2] : 0;
        l.up1 = sp.in2 >= 0 ? 1 : 0;
        l.cin = l.cin1 + l.cin2;
        l.cout = s->tch[sp.out];
        l.level = kTensors[sp.out].level;
        l.Kp = round_up(9 * l.cin, kb::umma::BK);
        l.Kpt = round_up(9 * l.cout, kb::umma::BK);
        l.bn_f = kb::umma::pick_bn(l.cout);
        l.bn_w = l.bn_f;
        l.bn_d = kb::umma::pick_bn(l.cin);
        l.w_off = off;
        off += (long long)l.cout * 9 * l.cin;
        l.b_off = off;
        off += l.cout;
        s->L.push_back(l);
    }
    s->n_params = off;
    int rc = 0;
    auto A = [&](void **p, size_t bytes) {
        if (!rc) rc = alloc(s, p, bytes);
    };
    const size_t pix0 = (size_t)max_batch * H * W;
    for (int t = 1; t < T_COUNT - 1; ++t) {
        const size_t px = pix0 >> (2 * kTensors[t].level);
        A((void **)&s->act[t], px * s->tch[t] * sizeof(bf16));
        A((void **)&s->grad[t], px * s->tch[t] * sizeof(bf16));
    }
    A((void **)&s->out_f32, pix0 * OUT_CH * sizeof(float));
    A((void **)&s->grad[T_OUT], pix0 * OUT_CH * sizeof(bf16));
    size_t part = 0, tmp = 0;
    for (int i = 0; i < N_LAYERS && !rc; ++i) {
        Layer &l = s->L[i];
        A((void **)&l.wb, (size_t)l.cout * l.Kp * sizeof(bf16));
        if (i > 0) A((void **)&l.wt, (size_t)l.cin * l.Kpt * sizeof(bf16));
        const size_t px = pix0 >> (2 * l.level);
        if (i > 0) {
            if (l.in2 >= 0) A((void **)&l.dx, px * l.cin * sizeof(bf16));
            else l.dx = s->grad[l.in1];
        }
        if (l.in2 >= 0) A((void **)&l.up, px * l.cin1 * sizeof(bf16));
        const int cin1 = (l.in1 == T_IN && l.cin1 % 16) ? PAD_CH : l.cin1;
        const size_t E = (size_t)(9 * (cin1 + l.cin2) + 1) * l.cout;
        size_t need = (size_t)max_wgrad_splits(l) * E;
        StripWgradPlan sp{};
        if (plan_strip_wgrad(l, W >> l.level, cin1, sp))
            need = std::max(need, (size_t)kb::sm_count() * kb::umma::TM_MAX_CPS * E);
        // every layer's partials and grouped sums have their own region, so
        // the reductions of all layers run together after the backward pass
        l.part_off = part;
        part += (need + 63) & ~(size_t)63;
        l.tmp_off = tmp;
        tmp += (300000 + E + 63) & ~(size_t)63;
    }
    s->part_floats = part;
    A((void **)&s->part, part * sizeof(float));
    s->tmp_floats = tmp;
    A((void **)&s->tmp, s->tmp_floats * sizeof(float));
    A((void **)&s->params, (size_t)s->n_params * sizeof(float));
    A((void **)&s->grads, (size_t)s->n_params * sizeof(float));
    A((void **)&s->adam_m, (size_t)s->n_params * sizeof(float));
    A((void **)&s->adam_v, (size_t)s->n_params * sizeof(float));
    A((void **)&s->err, sizeof(int));
    A((void **)&s->loss, sizeof(float));
    A((void **)&s->ones, 72 * 64 * sizeof(bf16));
    s->Kp_pad = round_up(9 * PAD_CH, kb::umma::BK);
    A((void **)&s->in_pad, pix0 * PAD_CH * sizeof(bf16));
    A((void **)&s->wb_pad, (size_t)s->L[0].cout * s->Kp_pad * sizeof(bf16));
    s->tp.resize(N_LAYERS);
    if (rc) {
        for (void *p : s->allocs) cudaFree(p);
        delete s;
        return rc;
    }
    // He-normal initialisation on the host (deterministic in `seed`), zero biases
    std::vector<float> h((size_t)s->n_params, 0.f);
    uint64_t x = seed;
    for (int i = 0; i < N_LAYERS; ++i) {
        const Layer &l = s->L[i];
        const double sd = std::sqrt(2.0 / (9.0 * l.cin)) * (l.out == T_OUT ? 0.1 : 1.0);
        for (long long k = 0; k < (long long)l.cout * 9 * l.cin; ++k) {
            const double u1 = ((splitmix(x) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
            const double u2 = ((splitmix(x) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
            h[l.w_off + k] = (float)(sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
        }
    }
    cudaMemcpyAsync(s->params, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice, st);
    static const std::vector<unsigned short> ones = [] {
        std::vector<unsigned short> o(72 * 64, 0);
        for (int k = 0; k < 72; ++k) o[k * 64] = 0x3F80u;  // BF16 1.0
        return o;
    }();
    cudaMemcpyAsync(s->ones, ones.data(), ones.size() * sizeof(unsigned short), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(s->adam_m, 0, (size_t)s->n_params * sizeof(float), st);
    cudaMemsetAsync(s->adam_v, 0, (size_t)s->n_params * sizeof(float), st);
    cudaMemsetAsync(s->grads, 0, (size_t)s->n_params * sizeof(float), st);
    cudaMemsetAsync(s->err, 0, sizeof(int), st);
    repack(s, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        rc = kb::check_launch("kb_surrogate_create");
        for (void *p : s->allocs) cudaFree(p);
        delete s;
        return rc ? rc : KB_ERR_CUDA;
    }
    *out = s;
    return 0;
}

int kb_surrogate_destroy(kb_surrogate *s) {
    if (!s) return 0;
    cudaDeviceSynchronize();
    for (void *p : s->allocs) cudaFree(p);
    delete s;
    return kb::check_launch("kb_surrogate_destroy");
}

int kb_surrogate_num_params(const kb_surrogate *s, long long *n) {
    KB_REQUIRE(s && n, "kb_surrogate_num_params: null argument");
    *n = s->n_params;
    return 0;
}

int kb_surrogate_layer(const kb_surrogate *s, int layer, int *cin, int *cout, int *level,
                       long long *w_off, long long *b_off) {
    KB_REQUIRE(s, "kb_surrogate_layer: null handle");
    KB_REQUIRE(layer >= 0 && layer < N_LAYERS, "kb_surrogate_layer: layer %d out of [0, %d)", layer,
               N_LAYERS);
    const Layer &l = s->L[layer];
    if (cin) *cin = l.cin;
    if (cout) *cout = l.cout;
    if (level) *level = l.level;
    if (w_off) *w_off = l.w_off;
    if (b_off) *b_off = l.b_off;
    return 0;
}

int kb_surrogate_set_normalisation(kb_surrogate *s, const float *scale, const float *offset) {
    KB_REQUIRE(s && scale && offset, "kb_surrogate_set_normalisation: null argument");
    for (int c = 0; c < 3; ++c) {
        KB_REQUIRE(scale[c] != 0.f && std::isfinite(scale[c]) && std::isfinite(offset[c]),
                   "kb_surrogate_set_normalisation: scale %d must be finite and non-zero", c);
        s->norm.scale[c] = scale[c];
        s->norm.offset[c] = offset[c];
    }
    return 0;
}

int kb_surrogate_set_grad_weight(kb_surrogate *s, float weight) {
    KB_REQUIRE(s, "kb_surrogate_set_grad_weight: null handle");
    KB_REQUIRE(weight >= 0.f && std::isfinite(weight),
               "kb_surrogate_set_grad_weight: weight must be finite and >= 0");
    s->grad_weight = weight;
    return 0;
}

int kb_surrogate_params(kb_surrogate *s, float *get, const float *set, void *stream) {
    KB_REQUIRE(s, "kb_surrogate_params: null handle");
    cudaStream_t st = kb::as_stream(stream);
    const size_t bytes = (size_t)s->n_params * sizeof(float);
    if (get) cudaMemcpyAsync(get, s->params, bytes, cudaMemcpyDeviceToDevice, st);
    if (set) {
        cudaMemcpyAsync(s->params, set, bytes, cudaMemcpyDeviceToDevice, st);
        if (int rc = repack(s, st)) return rc;
    }
    return kb::check_launch("kb_surrogate_params");
}

int kb_surrogate_grads(kb_surrogate *s, float *get, void *stream) {
    KB_REQUIRE(s && get, "kb_surrogate_grads: null argument");
    cudaMemcpyAsync(get, s->grads, (size_t)s->n_params * sizeof(float), cudaMemcpyDeviceToDevice,
                    kb::as_stream(stream));
    return kb::check_launch("kb_surrogate_grads");
}

int kb_surrogate_cavity_inputs(const kb_surrogate *s, void *input, const float *re, int n,
                               int n_nodes, void *stream) {
    KB_REQUIRE(s && input && re, "kb_surrogate_cavity_inputs: null argument");
    KB_REQUIRE(n > 0 && n <= s->Bmax, "kb_surrogate_cavity_inputs: n=%d out of [1, %d]", n, s->Bmax);
    cavity_inputs_k<<<ew_grid((long long)n * s->H * s->W), 256, 0, kb::as_stream(stream)>>>(
        (bf16 *)input, re, n, s->H, s->W, (float)n_nodes / 512.f);
    return kb::check_launch("kb_surrogate_cavity_inputs");
}

int kb_surrogate_infer(kb_surrogate *s, const void *input, int n, float *out, void *stream) {
    KB_REQUIRE(s && input, "kb_surrogate_infer: null argument");
    KB_REQUIRE(n > 0 && n <= s->Bmax, "kb_surrogate_infer: n=%d out of [1, %d]", n, s->Bmax);
    KB_REQUIRE(((uintptr_t)input % 16) == 0, "kb_surrogate_infer: input must be 16-byte aligned");
    cudaStream_t st = kb::as_stream(stream);
    if (int rc = forward(s, input, n, st)) return rc;
    if (out) {
        const int M = n * s->H * s->W;
        unpack_k<<<ew_grid(M), 256, 0, st>>>(out, s->out_f32, s->norm, M, s->H * s->W);
    }
    return kb::check_launch("kb_surrogate_infer");
}

int kb_surrogate_loss_backward(kb_surrogate *s, const void *input, const float *target, int n,
                               float *loss_out, void *stream) {
    KB_REQUIRE(s && input && target, "kb_surrogate_loss_backward: null argument");
    KB_REQUIRE(n > 0 && n <= s->Bmax, "kb_surrogate_loss_backward: n=%d out of [1, %d]", n, s->Bmax);
    KB_REQUIRE(((uintptr_t)input % 16) == 0, "kb_surrogate_loss_backward: input must be 16-byte aligned");
    cudaStream_t st = kb::as_stream(stream);
    if (int rc = forward(s, input, n, st)) return rc;
    const int M = n * s->H * s->W;
    cudaMemsetAsync(s->loss, 0, sizeof(float), st);
    const dim3 lg((s->W + LTX - 1) / LTX, (s->H + LTY - 1) / LTY, n);
    loss_k<<<lg, LTX * LTY, 0, st>>>(s->grad[T_OUT], s->loss, s->out_f32, target, s->norm, M, s->H, s->W,
                                     s->grad_weight);
    if (int rc = backward(s, n, st)) return rc;
    if (loss_out) cudaMemcpyAsync(loss_out, s->loss, sizeof(float), cudaMemcpyDeviceToDevice, st);
    return kb::check_launch("kb_surrogate_loss_backward");
}

int kb_surrogate_adam(kb_surrogate *s, float lr, float beta1, float beta2, float eps, int step,
                      void *stream) {
    KB_REQUIRE(s, "kb_surrogate_adam: null handle");
    KB_REQUIRE(step >= 1, "kb_surrogate_adam: step=%d must be >= 1", step);
    KB_REQUIRE(lr >= 0.f && beta1 >= 0.f && beta1 < 1.f && beta2 >= 0.f && beta2 < 1.f && eps > 0.f,
               "kb_surrogate_adam: bad hyper-parameters");
    cudaStream_t st = kb::as_stream(stream);
    const double c1 = 1.0 - std::pow((double)beta1, step), c2 = 1.0 - std::pow((double)beta2, step);
    const float lr_t = (float)(lr * std::sqrt(c2) / c1);
    const float eps_t = (float)(eps * std::sqrt(c2));
    adam_k<<<ew_grid(s->n_params), 256, 0, st>>>(s->params, s->adam_m, s->adam_v, s->grads,
                                                  s->n_params, lr_t, beta1, beta2, eps_t);
    if (int rc = repack(s, st)) return rc;
    return kb::check_launch("kb_surrogate_adam");
}

int kb_surrogate_train_step(kb_surrogate *s, const void *input, const float *target, int n,
                            float lr, int step, float *loss_out, void *stream) {
    if (int rc = kb_surrogate_loss_backward(s, input, target, n, loss_out, stream)) return rc;
    return kb_surrogate_adam(s, lr, 0.9f, 0.999f, 1e-8f, step, stream);
}

int kb_surrogate_status(kb_surrogate *s, int *timed_out, void *stream) {
    KB_REQUIRE(s && timed_out, "kb_surrogate_status: null argument");
    cudaStream_t st = kb::as_stream(stream);
    cudaMemcpyAsync(timed_out, s->err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return kb::check_launch("kb_surrogate_status");
    return 0;
}

int kb_surrogate_flops(const kb_surrogate *s, int n, double *forward_flops, double *train_flops) {
    KB_REQUIRE(s, "kb_surrogate_flops: null handle");
    double f = 0.0, t = 0.0;
    for (int i = 0; i < N_LAYERS; ++i) {
        const Layer &l = s->L[i];
        const double px = (double)n * s->H_at(l.level) * s->W_at(l.level);
        const double one = 2.0 * px * l.cout * 9.0 * l.cin;
        f += one;
        t += one * (i == 0 ? 2.0 : 3.0);
    }
    if (forward_flops) *forward_flops = f;
    if (train_flops) *train_flops = t;
    return 0;
}

}  // extern "C"

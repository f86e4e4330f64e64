// Absorbed-map denoiser network: a 3-level 3-D U-Net (16/32/64 channels) over the MC grid, run
// forward for inference and forward + backward + Adam for training, entirely on the device.
//
//   level 0 (nx, ny, nz):  x16 -> a1 = relu(conv9)  -> s0 = relu(conv)          ... t9 -> head
//   level 1 (/2):          p0 = pool(s0) -> a3 -> s1                             ... t7 -> a8 -> u9
//   level 2 (/4):          p1 = pool(s1) -> a5 -> a6 -> u7
//   decoder: t7 = up(u7) + s1, t9 = up(u9) + s0 (the convolution runs at the coarse level and its
//   epilogue writes the upsampled sum), head: pred = (noisy*scale + w.relu(conv(t9)) + b) * mask.
//
// The flat FP32 parameter vector is, per layer, W[taps][cout][cin] then b[cout], and finally the
// 16 head weights and the head bias. Every convolution reads a bf16 shared-memory image of its
// weights, re-packed after each parameter update.
#include <cuda_bf16.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "conv3d.cuh"

namespace bd {

namespace {

struct LayerSpec {
    int taps, cin, cout;
};
constexpr LayerSpec kLayers[10] = {{9, 16, 16},  {27, 16, 16}, {27, 16, 32}, {27, 32, 32}, {27, 32, 64},
                                   {27, 64, 64}, {27, 64, 32}, {27, 32, 32}, {27, 32, 16}, {27, 16, 16}};
constexpr int kHead = 16;

long long param_count() {
    long long n = 0;
    for (const auto& l : kLayers) n += (long long)l.taps * l.cin * l.cout + l.cout;
    return n + kHead + 1;
}

struct Level {
    int nx, ny, nz;
    long long rows() const { return bd_conv_plane_rows(nx, ny, nz); }   // per 8-channel plane
};

__device__ __forceinline__ int padded_row(int x, int y, int z, int ny, int nz) {
    return ((x + 1) * (ny + 2) + (y + 1)) * (nz + 2) + (z + 1);
}

// 16-byte group of channels [8*plane, 8*plane + 8) of row v in plane-layout storage with R rows.
template <class T>
__device__ __forceinline__ T* plane_at(T* base, long long R, int plane, int v) {
    return base + ((size_t)plane * R + v) * 8;
}

// Input features of voxel (x, y, z): scaled noisy map, log1p(mu_a), log1p(mu_s)/4, tissue state.
__device__ __forceinline__ void voxel_features(const float* a_noisy, const float4* props, const uint8_t* flags,
                                               float scale, size_t u, float* f) {
    const float4 p = props[u];
    const float mu_a = p.x * p.y, mu_s = fmaxf(p.x - mu_a, 0.f);
    const uint8_t fl = flags ? flags[u] : 0;
    f[0] = a_noisy[u] * scale;
    f[1] = log1pf(mu_a);
    f[2] = 0.25f * log1pf(mu_s);
    f[3] = (fl & (BD_FLAG_ABLATED | BD_FLAG_VOID)) ? 0.f : ((fl & BD_FLAG_DRY) ? 0.5f : 1.f);
}

__global__ void k_unet_input(int nx, int ny, int nz, long long R, const float* a_noisy, const float4* props,
                             const uint8_t* flags, float scale, __nv_bfloat16* x16, uint8_t* mask) {
    const long long n = (long long)nx * ny * nz;
    for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < n; u += (long long)gridDim.x * blockDim.x) {
        const int z = (int)(u % nz);
        const long long r = u / nz;
        const int y = (int)(r % ny), x = (int)(r / ny);
        float v[16];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int zz = z + j - 1;
            if (zz >= 0 && zz < nz) {
                voxel_features(a_noisy, props, flags, scale, (size_t)(u + j - 1), v + 4 * j);
            } else {
#pragma unroll
                for (int f = 0; f < 4; ++f) v[4 * j + f] = 0.f;
            }
        }
#pragma unroll
        for (int f = 12; f < 16; ++f) v[f] = 0.f;
        const float4 p = props[u];
        mask[u] = p.x * p.y > 0.f ? 1 : 0;
        uint4 q[2];
        __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(q);
#pragma unroll
        for (int f = 0; f < 8; ++f) h[f] = __floats2bfloat162_rn(v[2 * f], v[2 * f + 1]);
        const int row = padded_row(x, y, z, ny, nz);
        *reinterpret_cast<uint4*>(plane_at(x16, R, 0, row)) = q[0];
        *reinterpret_cast<uint4*>(plane_at(x16, R, 1, row)) = q[1];
    }
}

// Average (sum_mask == false) of the 8 children, or their sum gated by gate(coarse) > 0.
__global__ void k_pool(int nxc, int nyc, int nzc, long long Rc, long long Rf, int C, const __nv_bfloat16* fine,
                       const __nv_bfloat16* gate, __nv_bfloat16* coarse, int sum_mask) {
    const int chunks = C / 8;
    const long long n = (long long)nxc * nyc * nzc * chunks;
    const int nyf = 2 * nyc, nzf = 2 * nzc;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int ch = (int)(i % chunks);
        long long r = i / chunks;
        const int z = (int)(r % nzc);
        r /= nzc;
        const int y = (int)(r % nyc), x = (int)(r / nyc);
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int c8 = 0; c8 < 8; ++c8) {
            const int fx = 2 * x + (c8 >> 2), fy = 2 * y + ((c8 >> 1) & 1), fz = 2 * z + (c8 & 1);
            const uint4 q = *reinterpret_cast<const uint4*>(plane_at(fine, Rf, ch, padded_row(fx, fy, fz, nyf, nzf)));
            const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&q);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float2 f = __bfloat1622float2(h[j]);
                acc[2 * j] += f.x;
                acc[2 * j + 1] += f.y;
            }
        }
        const int vc = padded_row(x, y, z, nyc, nzc);
        if (sum_mask) {
            const uint4 q = *reinterpret_cast<const uint4*>(plane_at(gate, Rc, ch, vc));
            const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&q);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float2 f = __bfloat1622float2(h[j]);
                if (!(f.x > 0.f)) acc[2 * j] = 0.f;
                if (!(f.y > 0.f)) acc[2 * j + 1] = 0.f;
            }
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) acc[j] *= 0.125f;
        }
        uint4 o;
        __nv_bfloat162* ho = reinterpret_cast<__nv_bfloat162*>(&o);
#pragma unroll
        for (int j = 0; j < 4; ++j) ho[j] = __floats2bfloat162_rn(acc[2 * j], acc[2 * j + 1]);
        *reinterpret_cast<uint4*>(plane_at(coarse, Rc, ch, vc)) = o;
    }
}

// out[8*plane + j] += sum over the rows of plane blockIdx.y (pad and margin rows are zero).
__global__ void k_bias_grad(long long R, const __nv_bfloat16* g, float* out) {
    __shared__ float part[8];
    if (threadIdx.x < 8) part[threadIdx.x] = 0.f;
    __syncthreads();
    const int plane = blockIdx.y;
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < R; r += (long long)gridDim.x * blockDim.x) {
        const uint4 q = *reinterpret_cast<const uint4*>(plane_at(g, R, plane, (int)r));
        const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&q);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float2 f = __bfloat1622float2(h[j]);
            acc[2 * j] += f.x;
            acc[2 * j + 1] += f.y;
        }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float v = acc[j];
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&part[j], v);
    }
    __syncthreads();
    if (threadIdx.x < 8) atomicAdd(&out[plane * 8 + threadIdx.x], part[threadIdx.x]);
}

__global__ void k_adam(long long n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

int blocks_for(long long n, int per_block = 256) {
    return (int)std::max(1LL, std::min((n + per_block - 1) / per_block, 148LL * 16));
}

}  // namespace

struct UnetImpl {
    Level lv[3];
    bool training = false;
    long long n_params = 0;
    std::vector<long long> w_off, b_off;
    long long head_off = 0;
    float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    long long adam_t = 0;
    double* loss = nullptr;
    int* err = nullptr;
    uint8_t* mask = nullptr;
    // activations (bf16 padded rows)
    __nv_bfloat16 *x16, *a1, *s0, *t9, *p0, *a3, *s1, *t7, *a8, *u9, *p1, *a5, *a6, *u7;
    // gradients
    __nv_bfloat16 *g0a, *d0, *g9, *g1a, *d1, *g7, *g6, *g5;
    // weight images: fwd[layer][slice], bwd[layer][slice]
    void* fwd_img[10][2] = {};
    void* bwd_img[10][2] = {};
    std::vector<void*> allocs;

    int alloc(void** p, size_t bytes) {
        cudaError_t e = cudaMalloc(p, bytes);
        if (e != cudaSuccess) return cuda_status(e, "bd_unet_create: cudaMalloc");
        allocs.push_back(*p);
        e = cudaMemset(*p, 0, bytes);
        if (e != cudaSuccess) return cuda_status(e, "bd_unet_create: cudaMemset");
        return BD_OK;
    }
    int act(__nv_bfloat16** p, int level, int C) { return alloc((void**)p, (size_t)lv[level].rows() * C * 2); }
    ~UnetImpl() {
        for (void* p : allocs) cudaFree(p);
    }
    static int n_slices(int k, int n) { return (k == 64 && n == 64) ? 2 : 1; }

    int repack(cudaStream_t st) {
        for (int l = 0; l < 10; ++l) {
            const LayerSpec& s = kLayers[l];
            const float* w = params + w_off[l];
            const int fs = n_slices(s.cin, s.cout), fn = s.cout / fs;
            for (int i = 0; i < fs; ++i)
                if (int rc = pack_weights_launch(s.taps, s.cin, s.cout, i * fn, fn, 0, w, fwd_img[l][i], st)) return rc;
            if (training && l > 0) {
                const int bs = n_slices(s.cout, s.cin), bn = s.cin / bs;
                for (int i = 0; i < bs; ++i)
                    if (int rc = pack_weights_launch(s.taps, s.cin, s.cout, i * bn, bn, 1, w, bwd_img[l][i], st)) return rc;
            }
        }
        return BD_OK;
    }

    BdConvCall call(int level, int l, int mode, const void* in, void* out, int slice = 0, bool bwd = false) const {
        const LayerSpec& s = kLayers[l];
        BdConvCall c{};
        c.nx = lv[level].nx; c.ny = lv[level].ny; c.nz = lv[level].nz;
        c.cin = bwd ? s.cout : s.cin;
        c.cout_total = bwd ? s.cin : s.cout;
        const int ns = bwd ? n_slices(s.cout, s.cin) : n_slices(s.cin, s.cout);
        c.n_slice = c.cout_total / ns;
        c.n_off = slice * c.n_slice;
        c.taps = s.taps;
        c.mode = mode;
        c.input = in;
        c.wimage = bwd ? bwd_img[l][slice] : fwd_img[l][slice];
        c.bias = bwd ? nullptr : params + b_off[l] + c.n_off;
        c.out = out;
        return c;
    }

    int conv(const BdConvCall& c, cudaStream_t st) { return conv_launch(c, st, err); }

    int conv_all_slices(BdConvCall c, int l, bool bwd, cudaStream_t st) {
        const LayerSpec& s = kLayers[l];
        const int ns = bwd ? n_slices(s.cout, s.cin) : n_slices(s.cin, s.cout);
        for (int i = 0; i < ns; ++i) {
            BdConvCall ci = c;
            ci.n_off = i * c.n_slice;
            ci.wimage = bwd ? bwd_img[l][i] : fwd_img[l][i];
            if (!bwd) ci.bias = params + b_off[l] + ci.n_off;
            if (int rc = conv(ci, st)) return rc;
        }
        return BD_OK;
    }

    int pool(int coarse, int C, const __nv_bfloat16* fine, const __nv_bfloat16* gate, __nv_bfloat16* out, bool sum_mask,
             cudaStream_t st) {
        const Level& L = lv[coarse];
        const long long n = (long long)L.nx * L.ny * L.nz * (C / 8);
        k_pool<<<blocks_for(n), 256, 0, st>>>(L.nx, L.ny, L.nz, L.rows(), lv[coarse - 1].rows(), C, fine, gate, out,
                                              sum_mask ? 1 : 0);
        BD_CHECK_LAUNCH("k_pool");
        return BD_OK;
    }

    int forward(const float* a_noisy, const float4* props, const uint8_t* flags, float scale, float* pred,
                const float* target, float loss_norm, cudaStream_t st) {
        const Level& L0 = lv[0];
        const long long n0 = (long long)L0.nx * L0.ny * L0.nz;
        k_unet_input<<<blocks_for(n0), 256, 0, st>>>(L0.nx, L0.ny, L0.nz, L0.rows(), a_noisy, props, flags, scale, x16,
                                                     mask);
        BD_CHECK_LAUNCH("k_unet_input");
        int rc;
        if ((rc = conv(call(0, 0, BD_CONV_FWD_RELU, x16, a1), st))) return rc;
        if ((rc = conv(call(0, 1, BD_CONV_FWD_RELU, a1, s0), st))) return rc;
        if ((rc = pool(1, 16, s0, nullptr, p0, false, st))) return rc;
        if ((rc = conv(call(1, 2, BD_CONV_FWD_RELU, p0, a3), st))) return rc;
        if ((rc = conv(call(1, 3, BD_CONV_FWD_RELU, a3, s1), st))) return rc;
        if ((rc = pool(2, 32, s1, nullptr, p1, false, st))) return rc;
        if ((rc = conv(call(2, 4, BD_CONV_FWD_RELU, p1, a5), st))) return rc;
        if ((rc = conv_all_slices(call(2, 5, BD_CONV_FWD_RELU, a5, a6), 5, false, st))) return rc;
        BdConvCall c7 = call(2, 6, BD_CONV_FWD_UPADD, a6, t7);
        c7.aux = s1;
        c7.out_coarse = training ? u7 : nullptr;
        if ((rc = conv(c7, st))) return rc;
        if ((rc = conv(call(1, 7, BD_CONV_FWD_RELU, t7, a8), st))) return rc;
        BdConvCall c9 = call(1, 8, BD_CONV_FWD_UPADD, a8, t9);
        c9.aux = s0;
        c9.out_coarse = training ? u9 : nullptr;
        if ((rc = conv(c9, st))) return rc;
        BdConvCall ch = call(0, 9, BD_CONV_FWD_HEAD, t9, nullptr);
        ch.head = params + head_off;
        ch.a_noisy = a_noisy;
        ch.mask = mask;
        ch.scale = scale;
        ch.loss_norm = loss_norm;
        ch.pred = pred;
        if (target) {
            ch.target = target;
            ch.head_grad = grads + head_off;
            ch.loss = loss;
            ch.grad_out = g0a;
        }
        return conv(ch, st);
    }

    int wgrad(int level, int l, const __nv_bfloat16* g, const __nv_bfloat16* x, cudaStream_t st) {
        const LayerSpec& s = kLayers[l];
        const Level& L = lv[level];
        if (int rc = wgrad_launch(L.nx, L.ny, L.nz, s.cin, s.cout, s.taps, g, x, grads + w_off[l], st, err)) return rc;
        const dim3 bg(std::max(1, std::min(blocks_for(L.rows()), 296)), s.cout / 8);
        k_bias_grad<<<bg, 256, 0, st>>>(L.rows(), g, grads + b_off[l]);
        BD_CHECK_LAUNCH("k_bias_grad");
        return BD_OK;
    }

    int backward(cudaStream_t st) {
        int rc;
        // head gradient g10 (level 0, 16) is in g0a
        if ((rc = wgrad(0, 9, g0a, t9, st))) return rc;
        if ((rc = conv(call(0, 9, BD_CONV_BWD_RAW, g0a, d0, 0, true), st))) return rc;          // dt9
        if ((rc = pool(1, 16, d0, u9, g9, true, st))) return rc;                                  // g9
        if ((rc = wgrad(1, 8, g9, a8, st))) return rc;
        BdConvCall c8 = call(1, 8, BD_CONV_BWD_MASK, g9, g1a, 0, true);                          // g8
        c8.aux = a8;
        if ((rc = conv(c8, st))) return rc;
        if ((rc = wgrad(1, 7, g1a, t7, st))) return rc;
        if ((rc = conv(call(1, 7, BD_CONV_BWD_RAW, g1a, d1, 0, true), st))) return rc;          // dt7
        if ((rc = pool(2, 32, d1, u7, g7, true, st))) return rc;                                  // g7
        if ((rc = wgrad(2, 6, g7, a6, st))) return rc;
        BdConvCall c6 = call(2, 6, BD_CONV_BWD_MASK, g7, g6, 0, true);                           // g6
        c6.aux = a6;
        if ((rc = conv(c6, st))) return rc;
        if ((rc = wgrad(2, 5, g6, a5, st))) return rc;
        BdConvCall c5 = call(2, 5, BD_CONV_BWD_MASK, g6, g5, 0, true);                           // g5
        c5.aux = a5;
        if ((rc = conv_all_slices(c5, 5, true, st))) return rc;
        if ((rc = wgrad(2, 4, g5, p1, st))) return rc;
        BdConvCall c4 = call(2, 4, BD_CONV_BWD_UPADD, g5, g1a, 0, true);                         // g4 (level 1)
        c4.aux = d1;
        c4.aux2 = s1;
        if ((rc = conv(c4, st))) return rc;
        if ((rc = wgrad(1, 3, g1a, a3, st))) return rc;
        BdConvCall c3 = call(1, 3, BD_CONV_BWD_MASK, g1a, d1, 0, true);                          // g3
        c3.aux = a3;
        if ((rc = conv(c3, st))) return rc;
        if ((rc = wgrad(1, 2, d1, p0, st))) return rc;
        BdConvCall c2 = call(1, 2, BD_CONV_BWD_UPADD, d1, g0a, 0, true);                         // g2 (level 0)
        c2.aux = d0;
        c2.aux2 = s0;
        if ((rc = conv(c2, st))) return rc;
        if ((rc = wgrad(0, 1, g0a, a1, st))) return rc;
        BdConvCall c1 = call(0, 1, BD_CONV_BWD_MASK, g0a, d0, 0, true);                          // g1
        c1.aux = a1;
        if ((rc = conv(c1, st))) return rc;
        return wgrad(0, 0, d0, x16, st);
    }
};

}  // namespace bd

using namespace bd;

struct BdUnet {
    UnetImpl impl;
};

extern "C" int64_t bd_unet_param_count(void) { return param_count(); }

extern "C" int bd_unet_create(int nx, int ny, int nz, int training, BdUnet** out) {
    BD_REQUIRE(out != nullptr, "bd_unet_create: out is NULL");
    BD_REQUIRE(nx >= 4 && ny >= 4 && nz >= 4 && nx % 4 == 0 && ny % 4 == 0 && nz % 4 == 0,
               "bd_unet_create: grid dims must be positive multiples of 4 (two 2x poolings)");
    BD_REQUIRE((long long)(nx + 2) * (ny + 2) * (nz + 2) * 64 < (1LL << 31), "bd_unet_create: grid too large");
    *out = nullptr;
    BdUnet* net = new BdUnet();
    UnetImpl& u = net->impl;
    u.training = training != 0;
    for (int i = 0; i < 3; ++i) u.lv[i] = Level{nx >> i, ny >> i, nz >> i};
    long long o = 0;
    for (const auto& l : kLayers) {
        u.w_off.push_back(o);
        o += (long long)l.taps * l.cin * l.cout;
        u.b_off.push_back(o);
        o += l.cout;
    }
    u.head_off = o;
    u.n_params = o + kHead + 1;
    int rc = BD_OK;
    auto A = [&](void** p, size_t b) { if (!rc) rc = u.alloc(p, b); };
    auto ACT = [&](__nv_bfloat16** p, int lvl, int C) { if (!rc) rc = u.act(p, lvl, C); };
    A((void**)&u.params, u.n_params * 4);
    A((void**)&u.grads, u.n_params * 4);
    A((void**)&u.loss, sizeof(double));
    A((void**)&u.err, sizeof(int));
    A((void**)&u.mask, (size_t)nx * ny * nz);
    ACT(&u.x16, 0, 16); ACT(&u.a1, 0, 16); ACT(&u.s0, 0, 16); ACT(&u.t9, 0, 16);
    ACT(&u.p0, 1, 16); ACT(&u.a3, 1, 32); ACT(&u.s1, 1, 32); ACT(&u.t7, 1, 32); ACT(&u.a8, 1, 32);
    ACT(&u.p1, 2, 32); ACT(&u.a5, 2, 64); ACT(&u.a6, 2, 64);
    if (u.training) {
        A((void**)&u.adam_m, u.n_params * 4);
        A((void**)&u.adam_v, u.n_params * 4);
        ACT(&u.u9, 1, 16); ACT(&u.u7, 2, 32);
        ACT(&u.g0a, 0, 16); ACT(&u.d0, 0, 16);
        ACT(&u.g9, 1, 16); ACT(&u.g1a, 1, 32); ACT(&u.d1, 1, 32);
        ACT(&u.g7, 2, 32); ACT(&u.g6, 2, 64); ACT(&u.g5, 2, 64);
    }
    for (int l = 0; l < 10 && !rc; ++l) {
        const LayerSpec& s = kLayers[l];
        const int fs = UnetImpl::n_slices(s.cin, s.cout);
        for (int i = 0; i < fs; ++i) A(&u.fwd_img[l][i], (size_t)bd_conv_image_bytes(s.taps, s.cin, s.cout / fs));
        if (u.training && l > 0) {
            const int bs = UnetImpl::n_slices(s.cout, s.cin);
            for (int i = 0; i < bs; ++i) A(&u.bwd_img[l][i], (size_t)bd_conv_image_bytes(s.taps, s.cout, s.cin / bs));
        }
    }
    if (rc) {
        delete net;
        return rc;
    }
    *out = net;
    return BD_OK;
}

extern "C" int bd_unet_destroy(BdUnet* net) {
    if (net) {
        cudaDeviceSynchronize();
        delete net;
    }
    return BD_OK;
}

extern "C" int bd_unet_set_params(BdUnet* net, const float* params, void* stream) {
    BD_REQUIRE(net && params, "bd_unet_set_params: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    UnetImpl& u = net->impl;
    BD_CUDA(cudaMemcpyAsync(u.params, params, u.n_params * 4, cudaMemcpyDeviceToDevice, st));
    if (u.training) {
        BD_CUDA(cudaMemsetAsync(u.adam_m, 0, u.n_params * 4, st));
        BD_CUDA(cudaMemsetAsync(u.adam_v, 0, u.n_params * 4, st));
        u.adam_t = 0;
    }
    return u.repack(st);
}

extern "C" int bd_unet_get_params(BdUnet* net, float* params, void* stream) {
    BD_REQUIRE(net && params, "bd_unet_get_params: NULL argument");
    BD_CUDA(cudaMemcpyAsync(params, net->impl.params, net->impl.n_params * 4, cudaMemcpyDeviceToDevice,
                            (cudaStream_t)stream));
    return BD_OK;
}

extern "C" int bd_unet_get_grads(BdUnet* net, float* grads, void* stream) {
    BD_REQUIRE(net && grads, "bd_unet_get_grads: NULL argument");
    BD_REQUIRE(net->impl.training, "bd_unet_get_grads: network created without training buffers");
    BD_CUDA(cudaMemcpyAsync(grads, net->impl.grads, net->impl.n_params * 4, cudaMemcpyDeviceToDevice,
                            (cudaStream_t)stream));
    return BD_OK;
}

extern "C" int bd_unet_forward(BdUnet* net, const float* a_noisy, const float* props, const uint8_t* flags,
                               float scale, float* pred, void* stream) {
    BD_REQUIRE(net && a_noisy && props && pred, "bd_unet_forward: NULL argument");
    BD_REQUIRE(scale > 0.f, "bd_unet_forward: scale must be positive");
    return net->impl.forward(a_noisy, reinterpret_cast<const float4*>(props), flags, scale, pred, nullptr, 1.f,
                             (cudaStream_t)stream);
}

extern "C" int bd_unet_forward_backward(BdUnet* net, const float* a_noisy, const float* props, const uint8_t* flags,
                                        const float* target, float scale, float loss_norm, float* pred, void* stream) {
    BD_REQUIRE(net && a_noisy && props && target && pred, "bd_unet_forward_backward: NULL argument");
    BD_REQUIRE(net->impl.training, "bd_unet_forward_backward: network created without training buffers");
    BD_REQUIRE(scale > 0.f, "bd_unet_forward_backward: scale must be positive");
    UnetImpl& u = net->impl;
    cudaStream_t st = (cudaStream_t)stream;
    BD_CUDA(cudaMemsetAsync(u.grads, 0, u.n_params * 4, st));
    BD_CUDA(cudaMemsetAsync(u.loss, 0, sizeof(double), st));
    if (int rc = u.forward(a_noisy, reinterpret_cast<const float4*>(props), flags, scale, pred, target, loss_norm, st))
        return rc;
    return u.backward(st);
}

extern "C" int bd_unet_adam(BdUnet* net, float lr, float beta1, float beta2, float eps, void* stream) {
    BD_REQUIRE(net && net->impl.training, "bd_unet_adam: network created without training buffers");
    BD_REQUIRE(lr >= 0.f && beta1 >= 0.f && beta1 < 1.f && beta2 >= 0.f && beta2 < 1.f && eps > 0.f,
               "bd_unet_adam: bad hyper-parameters");
    UnetImpl& u = net->impl;
    cudaStream_t st = (cudaStream_t)stream;
    u.adam_t += 1;
    const float c1 = 1.f - powf(beta1, (float)u.adam_t), c2 = 1.f - powf(beta2, (float)u.adam_t);
    k_adam<<<blocks_for(u.n_params), 256, 0, st>>>(u.n_params, u.params, u.grads, u.adam_m, u.adam_v, lr, beta1, beta2,
                                                   eps, c1, c2);
    BD_CHECK_LAUNCH("k_adam");
    return u.repack(st);
}

extern "C" int bd_unet_read_loss(BdUnet* net, double* loss, void* stream) {
    BD_REQUIRE(net, "bd_unet_read_loss: NULL network");
    cudaStream_t st = (cudaStream_t)stream;
    UnetImpl& u = net->impl;
    double l = 0.0;
    int e = 0;
    BD_CUDA(cudaMemcpyAsync(&l, u.loss, sizeof(double), cudaMemcpyDeviceToHost, st));
    BD_CUDA(cudaMemcpyAsync(&e, u.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    BD_CUDA(cudaStreamSynchronize(st));
    if (e) return fail(BD_ERR_TIMEOUT, "bd_unet: a bounded convolution pipeline wait timed out");
    if (loss) *loss = l;
    return BD_OK;
}

// 3-D convolutions of the absorbed-map denoiser on the fifth-generation tensor cores.
//
// Volumes are bf16 with a one-voxel zero pad, stored as "8-channel planes": channel c of padded row
// v lives at ((c/8)*R + v)*8 + c%8, with R = padded rows + a zero margin. The neighbour (dx, dy, dz)
// of row v is row v + dx*nyp*nzp + dy*nzp + dz for every interior voxel, so a 3x3x3 convolution is
// 27 row-shifted GEMMs [128 voxels x cin] x [cin x cout] accumulated in TMEM (implicit GEMM), and
// every operand tile is a run of contiguous 16-byte rows: one bulk copy per 8 channels.
//
// Forward / data-gradient kernel (k_conv): persistent CTAs walk tiles of 128 consecutive rows. For
// each of the 9 (dx, dy) pairs, cin/8 bulk copies bring the tile's rows shifted by (dx, dy) into
// shared memory, which is exactly the K-major, no-swizzle UMMA layout. The three z taps are stacked
// along N: one 128 x (3*cout) x 16 MMA per K step accumulates D[u][(dz, co)], and the epilogue
// forms out[v] = D[v-1][dz=-1] + D[v][dz=0] + D[v+1][dz=+1] with warp shuffles (shared memory
// across warp edges), so a tile yields 126 outputs (rows 1..126). A pipeline stage holds 9, 3 or 1
// of a tile's runs (as shared memory allows), so the single MMA-issuing thread waits on one barrier
// per stage, not per run; few, wide MMAs keep the tensor pipe's issue rate off the critical path
// for the 16-channel layers. Weights of all taps stay resident in shared memory. Warp 0 issues the
// copies, warp 1 owns TMEM and issues tcgen05.mma, warps 2-9 (two groups, one per accumulator)
// drain the double-buffered accumulators and run the fused epilogue (bias, ReLU, nearest
// upsampling with the skip add, gradient gating, the 1x1 head).
//
// Weight-gradient kernel (k_conv_wgrad): dW[t][co][ci] = sum_v g[v - off_t][co] x[v][ci]. Taps are
// stacked along M (128/cout taps per MMA): 64-row plane chunks of the shifted gradient are the
// MN-major, no-swizzle A operand (8 channels per 1 KB core-matrix column) and the activation chunks
// are MN-major B; each CTA reduces a contiguous range of 64-voxel chunks in TMEM and adds its
// partial weights with FP32 atomics.
//
// Every mbarrier wait is bounded; a timeout sets the error flag, the roles drain what they issued
// and the CTA frees its TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"
#include "conv3d.cuh"
#include "tma.cuh"
#include "umma.cuh"

namespace bd {

namespace {

constexpr int kTileM = 128;
constexpr int kPlaneBytes = kTileM * 16;   // one 8-channel plane of a tile: 128 rows x 16 B
constexpr int kSmemLimit = 232448;     // 227 KB opt-in dynamic shared memory per CTA
constexpr int kWgradKv = 64;           // voxels per weight-gradient K chunk
constexpr int kRowMargin = 256;        // zero rows after the padded volume (tile copies overrun it)
constexpr int kEpiGroups = 2;          // epilogue warp groups (4 warps each), one per accumulator
constexpr int kConvThreads = 64 + kEpiGroups * 128;

struct Geom {
    int nxp, nyp, nzp;
    int v_lo, v_hi;       // interior rows lie in [v_lo, v_hi)
    int plane;            // nyp * nzp
    int R;                // rows per 8-channel plane (padded rows + margin)
};

__host__ __device__ inline Geom make_geom(int nx, int ny, int nz) {
    Geom g;
    g.nxp = nx + 2; g.nyp = ny + 2; g.nzp = nz + 2;
    g.plane = g.nyp * g.nzp;
    g.v_lo = g.plane + g.nzp + 1;
    g.v_hi = nx * g.plane + ny * g.nzp + nz + 1;
    g.R = g.nxp * g.plane + kRowMargin;
    return g;
}

__device__ __forceinline__ size_t prow(const Geom& g, int chunk, int v) { return ((size_t)chunk * g.R + v) * 8; }

__device__ __forceinline__ int tap_offset(const Geom& g, int t, int taps) {
    if (taps == 27) {
        const int dx = t / 9 - 1, dy = (t / 3) % 3 - 1, dz = t % 3 - 1;
        return dx * g.plane + dy * g.nzp + dz;
    }
    const int dx = t / 3 - 1, dy = t % 3 - 1;
    return dx * g.plane + dy * g.nzp;
}

struct ConvArgs {
    Geom g;        // level of the convolution
    Geom gf;       // finer level (UPADD modes)
    int taps, mode, cout_total, n_off, n_tiles;
    const __nv_bfloat16* input;
    const __nv_bfloat16* wimage;
    int wbytes;
    const float* bias;
    __nv_bfloat16* out;
    __nv_bfloat16* out_coarse;
    const __nv_bfloat16* aux;
    const __nv_bfloat16* aux2;
    const float* head;
    const float* a_noisy;
    const uint8_t* mask;
    float scale, loss_norm;
    float* pred;
    const float* target;
    float* head_grad;
    double* loss;
    __nv_bfloat16* grad_out;
    int* err;
};

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}

// N channels of row v, starting at 8-channel plane c0, from / to plane-layout storage.
template <int N>
__device__ __forceinline__ void store_row(__nv_bfloat16* base, const Geom& g, int c0, int v, const float* val) {
#pragma unroll
    for (int c = 0; c < N; c += 8) {
        uint4 q;
        q.x = pack_bf16x2(val[c + 0], val[c + 1]);
        q.y = pack_bf16x2(val[c + 2], val[c + 3]);
        q.z = pack_bf16x2(val[c + 4], val[c + 5]);
        q.w = pack_bf16x2(val[c + 6], val[c + 7]);
        *reinterpret_cast<uint4*>(base + prow(g, c0 + c / 8, v)) = q;
    }
}

template <int N>
__device__ __forceinline__ void load_row(const __nv_bfloat16* base, const Geom& g, int c0, int v, float* val) {
#pragma unroll
    for (int c = 0; c < N; c += 8) {
        const uint4 q = *reinterpret_cast<const uint4*>(base + prow(g, c0 + c / 8, v));
        const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&q);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float2 f = __bfloat1622float2(h[j]);
            val[c + 2 * j] = f.x;
            val[c + 2 * j + 1] = f.y;
        }
    }
}

struct SharedCtl {
    unsigned long long full[32], empty[32];
    unsigned long long wfull, acc_full[2], acc_empty[2], done;
    uint32_t tmem;
    volatile int abort;
};

__device__ __forceinline__ bool wait_or_abort(unsigned long long* bar, unsigned parity, SharedCtl* ctl, int* err) {
    if (mbar_wait(bar, parity)) return true;
    ctl->abort = 1;
    if (err) atomicExch(err, 1);
    return false;
}

constexpr int pow2_at_least(int x) { return x <= 32 ? 32 : x <= 64 ? 64 : x <= 128 ? 128 : x <= 256 ? 256 : 512; }

template <int CIN, int N>
struct ConvCfg {
    static constexpr int KP = CIN / 8;
    static constexpr int RUN = KP * kPlaneBytes;   // one (dx, dy)-shifted run of a tile
    static constexpr int WMAX = 27 * CIN * N * 2;
    static constexpr int XB = 2 * 2 * 2 * 4 * N;  // floats: edge exchange [group][parity][side][quad][N]
    static constexpr int CTL = 1024 + ((XB * 4 + 256 + 1023) / 1024) * 1024;  // SharedCtl + exchange + bias
    static constexpr int AVAIL = kSmemLimit - 1024 - CTL - WMAX;
    // runs per pipeline stage: as many of the 9 as keep >= 3 stages, so the single MMA-issuing
    // thread waits on few barriers per tile
    static constexpr int RPS = AVAIL / (9 * RUN) >= 3 ? 9 : AVAIL / (3 * RUN) >= 3 ? 3 : 1;
    static constexpr int STAGE = RPS * RUN;
    static constexpr int NST_FIT = AVAIL / STAGE;
    static constexpr int NST = NST_FIT > 32 ? 32 : NST_FIT;
    static constexpr int SMEM = 1024 + CTL + WMAX + NST * STAGE;
    static constexpr int TMEM_COLS = pow2_at_least(2 * 3 * N);   // two accumulators of 3N columns
    static_assert(NST >= 3, "conv: not enough shared memory for a 3-stage pipeline");
    static_assert(SMEM <= kSmemLimit, "conv: shared memory over the limit");
};

// Fused epilogue for the voxel in row v of the level; acc holds its N accumulator values.
template <int N>
__device__ __forceinline__ void conv_epilogue(const ConvArgs& a, int v, float* acc, float* head_acc, double& loss_acc) {
    const Geom& g = a.g;
    const int x = v / g.plane, r = v - x * g.plane, y = r / g.nzp, z = r - y * g.nzp;
    if (v >= g.v_hi || y < 1 || y > g.nyp - 2 || z < 1 || z > g.nzp - 2) return;
    const int mode = a.mode;
    if (mode <= BD_CONV_FWD_HEAD) {
#pragma unroll
        for (int c = 0; c < N; ++c) acc[c] = fmaxf(acc[c], 0.f);
    }
    const int c0 = a.n_off / 8;
    if (mode == BD_CONV_FWD_RELU || mode == BD_CONV_BWD_RAW) {
        store_row<N>(a.out, g, c0, v, acc);
    } else if (mode == BD_CONV_BWD_MASK) {
#pragma unroll
        for (int c = 0; c < N; c += 8) {
            float m[8];
            load_row<8>(a.aux, g, c0 + c / 8, v, m);
#pragma unroll
            for (int j = 0; j < 8; ++j) acc[c + j] = m[j] > 0.f ? acc[c + j] : 0.f;
        }
        store_row<N>(a.out, g, c0, v, acc);
    } else if (mode == BD_CONV_FWD_UPADD || mode == BD_CONV_BWD_UPADD) {
        if (mode == BD_CONV_FWD_UPADD && a.out_coarse) store_row<N>(a.out_coarse, g, c0, v, acc);
        const Geom& f = a.gf;
        for (int ch = 0; ch < 8; ++ch) {
            const int fx = 2 * x - 1 + (ch >> 2), fy = 2 * y - 1 + ((ch >> 1) & 1), fz = 2 * z - 1 + (ch & 1);
            const int vf = fx * f.plane + fy * f.nzp + fz;
#pragma unroll
            for (int c = 0; c < N; c += 8) {
                float s[8], o[8];
                load_row<8>(a.aux, f, c0 + c / 8, vf, s);
                if (mode == BD_CONV_FWD_UPADD) {
#pragma unroll
                    for (int j = 0; j < 8; ++j) o[j] = acc[c + j] + s[j];
                } else {
                    float m[8];
                    load_row<8>(a.aux2, f, c0 + c / 8, vf, m);
#pragma unroll
                    for (int j = 0; j < 8; ++j) o[j] = m[j] > 0.f ? s[j] + 0.125f * acc[c + j] : 0.f;
                }
                store_row<8>(a.out, f, c0 + c / 8, vf, o);
            }
        }
    } else if constexpr (N == 16) {
        if (mode != BD_CONV_FWD_HEAD) return;
        const int nz = g.nzp - 2, ny = g.nyp - 2;
        const size_t u = ((size_t)(x - 1) * ny + (y - 1)) * nz + (z - 1);
        float yv = a.head[N];
#pragma unroll
        for (int c = 0; c < N; ++c) yv = fmaf(a.head[c], acc[c], yv);
        const float m = a.mask[u] ? 1.f : 0.f;
        const float p = (a.a_noisy[u] * a.scale + yv) * m;
        a.pred[u] = p / a.scale;
        if (a.target) {
            const float res = (p - a.target[u] * a.scale) * m;
            loss_acc += (double)res * res;
            const float dy = 2.f * res * a.loss_norm;
            float gr[N];
#pragma unroll
            for (int c = 0; c < N; ++c) {
                gr[c] = acc[c] > 0.f ? dy * a.head[c] : 0.f;
                head_acc[c] = fmaf(dy, acc[c], head_acc[c]);
            }
            head_acc[N] += dy;
            store_row<N>(a.grad_out, g, 0, v, gr);
        }
    }
}

template <int CIN, int N>
__global__ void __launch_bounds__(kConvThreads, 1) k_conv(const ConvArgs a) {
    using C = ConvCfg<CIN, N>;
    extern __shared__ unsigned char smem_raw[];
    const uint32_t base_addr = smem_addr(smem_raw);
    unsigned char* smem = smem_raw + ((1024 - (base_addr & 1023)) & 1023);
    SharedCtl* ctl = reinterpret_cast<SharedCtl*>(smem);
    unsigned char* wsm = smem + C::CTL;
    unsigned char* stages = wsm + C::WMAX;

    float* xbuf = reinterpret_cast<float*>(smem + 1024);
    float* sbias = xbuf + C::XB;                    // [N] bias of the slice (forward modes), else 0
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kz = a.taps == 27 ? 3 : 1;
    const int NN = kz * N;                          // MMA N: z taps stacked along N
    const int out_per_tile = kz == 3 ? kTileM - 2 : kTileM;
    const int u_base = a.g.v_lo - (kz == 3 ? 1 : 0);

    if (threadIdx.x == 0) {
        for (int s = 0; s < C::NST; ++s) {
            mbar_init(&ctl->full[s], 1);
            mbar_init(&ctl->empty[s], 1);
        }
        mbar_init(&ctl->wfull, 1);
        for (int i = 0; i < 2; ++i) {
            mbar_init(&ctl->acc_full[i], 1);
            mbar_init(&ctl->acc_empty[i], 128);
        }
        mbar_init(&ctl->done, 1);
        ctl->abort = 0;
        mbar_init_fence();
    }
    for (int c = threadIdx.x; c < N; c += blockDim.x)
        sbias[c] = (a.mode <= BD_CONV_FWD_HEAD && a.bias) ? a.bias[c] : 0.f;
    if (warp == 1) tmem_alloc(&ctl->tmem, C::TMEM_COLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = ctl->tmem;

    if (warp == 0) {
        if (lane == 0) {
            // ---- producer: resident weights, then 9 (dx, dy)-shifted row runs per tile ----
            mbar_expect_tx(&ctl->wfull, a.wbytes);
            for (int off = 0; off < a.wbytes; off += 32768)
                bulk_load(wsm + off, reinterpret_cast<const unsigned char*>(a.wimage) + off,
                          min(32768, a.wbytes - off), &ctl->wfull);
            int s = 0;
            unsigned ph = 0;
            long long issued = 0;
            for (int tile = blockIdx.x; tile < a.n_tiles && !ctl->abort; tile += gridDim.x) {
                const int u0 = u_base + tile * out_per_tile;
                for (int q0 = 0; q0 < 9; q0 += C::RPS) {
                    if (!wait_or_abort(&ctl->empty[s], ph ^ 1, ctl, a.err)) break;
                    unsigned char* st = stages + s * C::STAGE;
                    mbar_expect_tx(&ctl->full[s], C::STAGE);
#pragma unroll
                    for (int r = 0; r < C::RPS; ++r) {
                        const int q = q0 + r;
                        const int row0 = u0 + (q / 3 - 1) * a.g.plane + (q % 3 - 1) * a.g.nzp;
#pragma unroll
                        for (int p = 0; p < C::KP; ++p)
                            bulk_load(st + r * C::RUN + p * kPlaneBytes, a.input + prow(a.g, p, row0), kPlaneBytes,
                                      &ctl->full[s]);
                    }
                    ++issued;
                    if (++s == C::NST) { s = 0; ph ^= 1; }
                }
            }
            // drain: every issued load has landed before the CTA leaves
            const long long n_drain = issued < C::NST ? issued : C::NST;
            for (long long i = 0; i < n_drain; ++i) {
                if (--s < 0) { s = C::NST - 1; ph ^= 1; }
                mbar_wait(&ctl->full[s], ph);
            }
            mbar_wait(&ctl->wfull, 0);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issuer: per (dx, dy) stage, CIN/16 MMAs of 128 x NN x 16 ----
            const uint32_t idesc = umma_idesc_bf16(kTileM, NN, false, false);
            const uint32_t wbase = smem_addr(wsm), sbase = smem_addr(stages);
            const uint32_t wq = C::KP * NN * 16;    // weight image bytes per (dx, dy) pair
            bool ok = wait_or_abort(&ctl->wfull, 0, ctl, a.err);
            int s = 0, acc = 0;
            unsigned ph = 0, aph = 0;
            for (int tile = blockIdx.x; ok && tile < a.n_tiles && !ctl->abort; tile += gridDim.x) {
                if (!wait_or_abort(&ctl->acc_empty[acc], aph ^ 1, ctl, a.err)) break;
                tc_fence_after();
                const uint32_t d = tmem + acc * NN;
                for (int q0 = 0; q0 < 9 && ok; q0 += C::RPS) {
                    if (!wait_or_abort(&ctl->full[s], ph, ctl, a.err)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t st = sbase + s * C::STAGE;
#pragma unroll
                    for (int r = 0; r < C::RPS; ++r) {
                        const int q = q0 + r;
#pragma unroll
                        for (int kk = 0; kk < CIN / 16; ++kk) {
                            const uint64_t ad = umma_desc(st + r * C::RUN + kk * 2 * kPlaneBytes, kPlaneBytes, 128,
                                                          UMMA_NONE);
                            const uint64_t bd = umma_desc(wbase + q * wq + kk * 2 * (NN * 16), NN * 16, 128, UMMA_NONE);
                            umma_bf16(d, ad, bd, idesc, (q | kk) != 0);
                        }
                    }
                    umma_commit(&ctl->empty[s]);
                    if (++s == C::NST) { s = 0; ph ^= 1; }
                }
                if (!ok) break;
                umma_commit(&ctl->acc_full[acc]);
                acc ^= 1;
                if (acc == 0) aph ^= 1;
            }
            umma_commit(&ctl->done);
            mbar_wait(&ctl->done, 0);
        }
    } else {
        // ---- epilogue: two groups of 4 warps (2..5, 6..9); group g drains accumulator g, i.e.
        // every other tile of this CTA. Warp w reads TMEM lanes 32*(w % 4) .. +31; row = TMEM lane.
        const int grp = (warp - 2) >> 2;
        const int quad = warp & 3;
        const int row = quad * 32 + lane;
        const int acc = grp;
        unsigned aph = 0;
        constexpr int HA = N == 16 ? 17 : 1;        // head gradient accumulators (16-channel head only)
        float head_acc[HA];
#pragma unroll
        for (int c = 0; c < HA; ++c) head_acc[c] = 0.f;
        double loss_acc = 0.0;
        int par = 0;
        for (int tile = blockIdx.x + grp * gridDim.x; tile < a.n_tiles; tile += kEpiGroups * gridDim.x) {
            // a timed-out wait still takes part in the group's named barrier below, so its four
            // warps stay in step; the tile is then skipped
            const bool okw = !ctl->abort && wait_or_abort(&ctl->acc_full[acc], aph, ctl, a.err);
            float v[N];
            float* xb0 = xbuf + (((grp * 2 + par) * 2 + 0) * 4) * N;   // lane 31's dz=-1 block, per quad
            float* xb2 = xbuf + (((grp * 2 + par) * 2 + 1) * 4) * N;   // lane 0's dz=+1 block, per quad
            if (okw) {
                tc_fence_after();
                const uint32_t tb = tmem + ((uint32_t)(quad * 32) << 16) + acc * NN;
                if (kz == 3) {
#pragma unroll
                    for (int c = 0; c < N; c += 16) {
                        float t0[16], t1[16], t2[16];
                        tmem_ld16(tb + c, t0);
                        tmem_ld16(tb + N + c, t1);
                        tmem_ld16(tb + 2 * N + c, t2);
                        tmem_ld_wait();
#pragma unroll
                        for (int j = 0; j < 16; ++j) {
                            const float up = __shfl_up_sync(0xffffffffu, t0[j], 1);
                            const float dn = __shfl_down_sync(0xffffffffu, t2[j], 1);
                            v[c + j] = t1[j] + (lane > 0 ? up : 0.f) + (lane < 31 ? dn : 0.f);
                        }
                        if (lane == 31) {
#pragma unroll
                            for (int j = 0; j < 16; ++j) xb0[quad * N + c + j] = t0[j];
                        }
                        if (lane == 0) {
#pragma unroll
                            for (int j = 0; j < 16; ++j) xb2[quad * N + c + j] = t2[j];
                        }
                    }
                } else {
#pragma unroll
                    for (int c = 0; c < N; c += 16) tmem_ld16(tb + c, v + c);
                    tmem_ld_wait();
                }
                tc_fence_before();
            }
            mbar_arrive(&ctl->acc_empty[acc]);
            asm volatile("bar.sync %0, 128;" ::"r"(1 + grp) : "memory");
            if (okw && kz == 3) {
                if (lane == 0 && quad > 0) {
#pragma unroll
                    for (int c = 0; c < N; ++c) v[c] += xb0[(quad - 1) * N + c];
                }
                if (lane == 31 && quad < 3) {
#pragma unroll
                    for (int c = 0; c < N; ++c) v[c] += xb2[(quad + 1) * N + c];
                }
            }
            const int u0 = u_base + tile * out_per_tile;
            const bool out_row = kz == 1 || (row >= 1 && row <= kTileM - 2);
            if (okw && out_row && !ctl->abort) {
#pragma unroll
                for (int c = 0; c < N; ++c) v[c] += sbias[c];
                conv_epilogue<N>(a, u0 + row, v, head_acc, loss_acc);
            }
            aph ^= 1;
            par ^= 1;
        }
        if (a.mode == BD_CONV_FWD_HEAD && a.target) {
#pragma unroll
            for (int c = 0; c < HA; ++c) {
                float h = head_acc[c];
                for (int o = 16; o; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
                if (lane == 0) atomicAdd(&a.head_grad[c], h);
            }
            for (int o = 16; o; o >>= 1) loss_acc += __shfl_xor_sync(0xffffffffu, loss_acc, o);
            if (lane == 0) atomicAdd(a.loss, loss_acc);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, C::TMEM_COLS);
    }
}

// ------------------------------------------------------------------ weight gradient

struct WgradArgs {
    Geom g;
    int taps, g0, g1, chunks_total, chunks_per_cta;
    const __nv_bfloat16* grad;
    const __nv_bfloat16* act;
    float* dw;
    int* err;
};

template <int COUT, int CIN>
struct WgradCfg {
    static constexpr int TPG = kTileM / COUT;               // taps per group (stacked along M)
    static constexpr int CHUNK = kWgradKv * 16;             // 64 rows of one 8-channel plane (1 KB)
    static constexpr int ABOX = (COUT / 8) * CHUNK;         // one tap's gradient tile
    static constexpr int BBOX = (CIN / 8) * CHUNK;          // activation tile
    static constexpr int STAGE = TPG * ABOX + BBOX;
    static constexpr int CTL = 1024;
    static constexpr int NST_FIT = (kSmemLimit - 1024 - CTL) / STAGE;
    static constexpr int NST = NST_FIT > 12 ? 12 : NST_FIT;
    static constexpr int SMEM = 1024 + CTL + NST * STAGE;
    static constexpr int GMAX = (512 / CIN) < 14 ? (512 / CIN) : 14;   // groups per launch (TMEM columns)
    static_assert(SMEM <= kSmemLimit, "wgrad: shared memory over the limit");
    static_assert(STAGE % 1024 == 0, "wgrad: stage must keep 1024-byte alignment");
};

template <int COUT, int CIN>
__global__ void __launch_bounds__(192, 1) k_conv_wgrad(const WgradArgs a) {
    using C = WgradCfg<COUT, CIN>;
    extern __shared__ unsigned char smem_raw[];
    const uint32_t base_addr = smem_addr(smem_raw);
    unsigned char* smem = smem_raw + ((1024 - (base_addr & 1023)) & 1023);
    SharedCtl* ctl = reinterpret_cast<SharedCtl*>(smem);
    unsigned char* stages = smem + C::CTL;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ng = a.g1 - a.g0;
    uint32_t tcols = 32;
    while (tcols < (uint32_t)(ng * CIN)) tcols <<= 1;

    const int c_begin = blockIdx.x * a.chunks_per_cta;
    const int c_end = min(a.chunks_total, c_begin + a.chunks_per_cta);

    if (threadIdx.x == 0) {
        for (int s = 0; s < C::NST; ++s) {
            mbar_init(&ctl->full[s], 1);
            mbar_init(&ctl->empty[s], 1);
        }
        mbar_init(&ctl->acc_full[0], 1);
        mbar_init(&ctl->done, 1);
        ctl->abort = 0;
        mbar_init_fence();
    }
    if (warp == 1) tmem_alloc(&ctl->tmem, tcols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = ctl->tmem;

    if (warp == 0) {
        if (lane == 0) {
            int s = 0;
            unsigned ph = 0;
            long long issued = 0;
            for (int c = c_begin; c < c_end && !ctl->abort; ++c) {
                const int v0 = a.g.v_lo + c * kWgradKv;
                for (int gi = a.g0; gi < a.g1; ++gi) {
                    if (!wait_or_abort(&ctl->empty[s], ph ^ 1, ctl, a.err)) { c = c_end; break; }
                    unsigned char* st = stages + s * C::STAGE;
                    mbar_expect_tx(&ctl->full[s], C::STAGE);
#pragma unroll
                    for (int j = 0; j < C::TPG; ++j) {
                        const int t = min(gi * C::TPG + j, a.taps - 1);
                        const int row = v0 - tap_offset(a.g, t, a.taps);
#pragma unroll
                        for (int cb = 0; cb < COUT / 8; ++cb)
                            bulk_load(st + j * C::ABOX + cb * C::CHUNK, a.grad + prow(a.g, cb, row), C::CHUNK,
                                      &ctl->full[s]);
                    }
#pragma unroll
                    for (int cb = 0; cb < CIN / 8; ++cb)
                        bulk_load(st + C::TPG * C::ABOX + cb * C::CHUNK, a.act + prow(a.g, cb, v0), C::CHUNK,
                                  &ctl->full[s]);
                    ++issued;
                    if (++s == C::NST) { s = 0; ph ^= 1; }
                }
            }
            const long long n_drain = issued < C::NST ? issued : C::NST;
            for (long long i = 0; i < n_drain; ++i) {
                if (--s < 0) { s = C::NST - 1; ph ^= 1; }
                mbar_wait(&ctl->full[s], ph);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // MN-major, no swizzle: 8 M (or N) elements x 8 K rows per 128-byte core matrix; K groups
            // 128 B apart (LBO), 8-element M/N blocks one 1 KB chunk apart (SBO)
            const uint32_t idesc = umma_idesc_bf16(kTileM, CIN, true, true);
            const uint32_t sbase = smem_addr(stages);
            int s = 0;
            unsigned ph = 0;
            bool ok = true;
            for (int c = c_begin; ok && c < c_end && !ctl->abort; ++c) {
                for (int gi = a.g0; gi < a.g1; ++gi) {
                    if (!wait_or_abort(&ctl->full[s], ph, ctl, a.err)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t st = sbase + s * C::STAGE;
                    const uint32_t d = tmem + (gi - a.g0) * CIN;
#pragma unroll
                    for (int kk = 0; kk < kWgradKv / 16; ++kk) {
                        const uint64_t ad = umma_desc(st + kk * 256, 128, C::CHUNK, UMMA_NONE);
                        const uint64_t bd = umma_desc(st + C::TPG * C::ABOX + kk * 256, 128, C::CHUNK, UMMA_NONE);
                        umma_bf16(d, ad, bd, idesc, (c != c_begin) || kk != 0);
                    }
                    umma_commit(&ctl->empty[s]);
                    if (++s == C::NST) { s = 0; ph ^= 1; }
                }
            }
            umma_commit(&ctl->acc_full[0]);
            mbar_wait(&ctl->acc_full[0], 0);
        }
    } else if (c_begin < c_end) {
        const int quad = warp & 3;
        const int row = quad * 32 + lane;
        if (wait_or_abort(&ctl->acc_full[0], 0, ctl, a.err) && !ctl->abort) {
            tc_fence_after();
            const int j = row / COUT, co = row % COUT;
            for (int gi = a.g0; gi < a.g1; ++gi) {
                float v[CIN];
#pragma unroll
                for (int c = 0; c < CIN; c += 16)
                    tmem_ld16(tmem + ((uint32_t)(quad * 32) << 16) + (gi - a.g0) * CIN + c, v + c);
                tmem_ld_wait();
                const int t = gi * C::TPG + j;
                if (t < a.taps) {
                    float* dst = a.dw + ((size_t)t * COUT + co) * CIN;
#pragma unroll
                    for (int c = 0; c < CIN; ++c) atomicAdd(dst + c, v[c]);
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, tcols);
    }
}

__global__ void k_pack_weights(int taps, int cin, int cout, int n_off, int n_slice, int transpose, const float* w,
                               __nv_bfloat16* img) {
    // image[q][kp][dz][n][8]: for each (dx, dy) pair q, K-major planes of 8 input channels whose
    // rows are the (z tap, output) pairs the stacked MMA computes (kz = 3 z taps, or 1)
    const int K = transpose ? cout : cin;
    const int kz = taps == 27 ? 3 : 1;
    const long long total = (long long)taps * K * n_slice;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(i & 7);
        long long r = i >> 3;
        const int n = (int)(r % n_slice);
        r /= n_slice;
        const int dz = (int)(r % kz);
        r /= kz;
        const int kp = (int)(r % (K / 8));
        const int q = (int)(r / (K / 8));
        const int t = q * kz + dz;
        const int k = kp * 8 + j;
        float val;
        if (!transpose) val = w[((size_t)t * cout + (n_off + n)) * cin + k];
        else val = w[((size_t)(taps - 1 - t) * cout + k) * cin + (n_off + n)];
        img[i] = __float2bfloat16_rn(val);
    }
}

template <int CIN, int N>
int launch_conv_t(const BdConvCall& c, cudaStream_t st, int* err, int sms) {
    using C = ConvCfg<CIN, N>;
    const Geom g = make_geom(c.nx, c.ny, c.nz);
    ConvArgs a{};
    a.g = g;
    a.gf = make_geom(2 * c.nx, 2 * c.ny, 2 * c.nz);
    a.taps = c.taps; a.mode = c.mode; a.cout_total = c.cout_total; a.n_off = c.n_off;
    const int per_tile = c.taps == 27 ? kTileM - 2 : kTileM;
    a.n_tiles = (g.v_hi - g.v_lo + per_tile - 1) / per_tile;
    a.input = static_cast<const __nv_bfloat16*>(c.input);
    a.wimage = static_cast<const __nv_bfloat16*>(c.wimage);
    a.wbytes = (int)bd_conv_image_bytes(c.taps, CIN, N);
    a.bias = c.bias;
    a.out = static_cast<__nv_bfloat16*>(c.out);
    a.out_coarse = static_cast<__nv_bfloat16*>(c.out_coarse);
    a.aux = static_cast<const __nv_bfloat16*>(c.aux);
    a.aux2 = static_cast<const __nv_bfloat16*>(c.aux2);
    a.head = c.head; a.a_noisy = c.a_noisy; a.mask = c.mask; a.scale = c.scale; a.loss_norm = c.loss_norm;
    a.pred = c.pred; a.target = c.target; a.head_grad = c.head_grad; a.loss = c.loss;
    a.grad_out = static_cast<__nv_bfloat16*>(c.grad_out);
    a.err = err;
    BD_CUDA(cudaFuncSetAttribute(k_conv<CIN, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM));
    int occ = 1;
    BD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_conv<CIN, N>, kConvThreads, C::SMEM));
    const int grid = std::max(1, std::min(a.n_tiles, sms * std::max(1, occ)));
    k_conv<CIN, N><<<grid, kConvThreads, C::SMEM, st>>>(a);
    BD_CHECK_LAUNCH("k_conv");
    return BD_OK;
}

template <int COUT, int CIN>
int launch_wgrad_t(int nx, int ny, int nz, int taps, const void* grad, const void* act, float* dw, cudaStream_t st,
                   int* err, int sms) {
    using C = WgradCfg<COUT, CIN>;
    BD_CUDA(cudaFuncSetAttribute(k_conv_wgrad<COUT, CIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM));
    WgradArgs a{};
    a.g = make_geom(nx, ny, nz);
    a.taps = taps;
    a.chunks_total = (a.g.v_hi - a.g.v_lo + kWgradKv - 1) / kWgradKv;
    a.grad = static_cast<const __nv_bfloat16*>(grad);
    a.act = static_cast<const __nv_bfloat16*>(act);
    a.dw = dw;
    a.err = err;
    const int groups = (taps + C::TPG - 1) / C::TPG;
    // split the voxels over the SMs; small levels keep at least 32 chunks per CTA
    const int ctas = std::max(1, std::min(sms, (a.chunks_total + 31) / 32));
    a.chunks_per_cta = (a.chunks_total + ctas - 1) / ctas;
    const int grid = (a.chunks_total + a.chunks_per_cta - 1) / a.chunks_per_cta;
    for (int g0 = 0; g0 < groups; g0 += C::GMAX) {
        a.g0 = g0;
        a.g1 = std::min(groups, g0 + C::GMAX);
        k_conv_wgrad<COUT, CIN><<<grid, 192, C::SMEM, st>>>(a);
        BD_CHECK_LAUNCH("k_conv_wgrad");
    }
    return BD_OK;
}

int sm_count() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

}  // namespace

int conv_check(const BdConvCall& c) {
    BD_REQUIRE(c.nx > 0 && c.ny > 0 && c.nz > 0, "bd_conv3d: dims must be positive");
    BD_REQUIRE(c.cin == 16 || c.cin == 32 || c.cin == 64, "bd_conv3d: cin must be 16, 32 or 64");
    BD_REQUIRE(c.n_slice == 16 || c.n_slice == 32 || c.n_slice == 64, "bd_conv3d: n_slice must be 16, 32 or 64");
    BD_REQUIRE(!(c.cin == 64 && c.n_slice == 64), "bd_conv3d: cin 64 x n_slice 64 exceeds shared memory; split the slice");
    BD_REQUIRE(c.n_off >= 0 && c.n_off + c.n_slice <= c.cout_total && c.n_off % 8 == 0, "bd_conv3d: bad output slice");
    BD_REQUIRE(c.taps == 27 || c.taps == 9, "bd_conv3d: taps must be 27 or 9");
    BD_REQUIRE(c.mode >= BD_CONV_FWD_RELU && c.mode <= BD_CONV_BWD_UPADD, "bd_conv3d: unknown mode");
    BD_REQUIRE(c.input && c.wimage && (c.out || c.mode == BD_CONV_FWD_HEAD),
               "bd_conv3d: in, wimage and out are required");
    const long long vp = (long long)(c.nx + 2) * (c.ny + 2) * (c.nz + 2);
    const long long vpf = (long long)(2 * c.nx + 2) * (2 * c.ny + 2) * (2 * c.nz + 2);
    BD_REQUIRE(vp * c.cout_total < (1LL << 31) && vpf < (1LL << 31), "bd_conv3d: volume too large for 32-bit rows");
    if (c.mode == BD_CONV_FWD_UPADD || c.mode == BD_CONV_BWD_UPADD)
        BD_REQUIRE(c.aux != nullptr && (c.mode == BD_CONV_FWD_UPADD || c.aux2 != nullptr),
                   "bd_conv3d: the upsampling modes need aux (and aux2)");
    if (c.mode == BD_CONV_BWD_MASK) BD_REQUIRE(c.aux != nullptr, "bd_conv3d: BWD_MASK needs aux");
    BD_REQUIRE(((uintptr_t)c.input | (uintptr_t)c.wimage | (uintptr_t)c.out | (uintptr_t)c.aux | (uintptr_t)c.aux2 |
                (uintptr_t)c.out_coarse | (uintptr_t)c.grad_out) % 16 == 0,
               "bd_conv3d: volumes and weight images must be 16-byte aligned");
    if (c.mode == BD_CONV_FWD_HEAD) {
        BD_REQUIRE(c.n_slice == 16 && c.cout_total == 16 && c.n_off == 0, "bd_conv3d: the head takes 16 channels");
        BD_REQUIRE(c.head && c.a_noisy && c.mask && c.pred && c.scale > 0.f, "bd_conv3d: head inputs missing");
        BD_REQUIRE(!c.target || (c.head_grad && c.loss && c.grad_out), "bd_conv3d: training head needs gradients");
    }
    return BD_OK;
}

int conv_launch(const BdConvCall& c, cudaStream_t st, int* err) {
    const int sms = sm_count();
#define BD_CONV_CASE(CI, NN) \
    if (c.cin == CI && c.n_slice == NN) return launch_conv_t<CI, NN>(c, st, err, sms);
    BD_CONV_CASE(16, 16) BD_CONV_CASE(16, 32) BD_CONV_CASE(16, 64)
    BD_CONV_CASE(32, 16) BD_CONV_CASE(32, 32) BD_CONV_CASE(32, 64)
    BD_CONV_CASE(64, 16) BD_CONV_CASE(64, 32)
#undef BD_CONV_CASE
    return fail(BD_ERR_INVALID_ARG, "bd_conv3d: unsupported channel combination");
}

int wgrad_launch(int nx, int ny, int nz, int cin, int cout, int taps, const void* grad, const void* act, float* dw,
                 cudaStream_t st, int* err) {
    const int sms = sm_count();
#define BD_WG_CASE(CO, CI) \
    if (cout == CO && cin == CI) return launch_wgrad_t<CO, CI>(nx, ny, nz, taps, grad, act, dw, st, err, sms);
    BD_WG_CASE(16, 16) BD_WG_CASE(16, 32) BD_WG_CASE(16, 64)
    BD_WG_CASE(32, 16) BD_WG_CASE(32, 32) BD_WG_CASE(32, 64)
    BD_WG_CASE(64, 16) BD_WG_CASE(64, 32) BD_WG_CASE(64, 64)
#undef BD_WG_CASE
    return fail(BD_ERR_INVALID_ARG, "bd_conv3d_wgrad: unsupported channel combination");
}

int pack_weights_launch(int taps, int cin, int cout, int n_off, int n_slice, int transpose, const float* w, void* img,
                        cudaStream_t st) {
    const long long total = (long long)taps * (transpose ? cout : cin) * n_slice;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 4096);
    k_pack_weights<<<blocks, 256, 0, st>>>(taps, cin, cout, n_off, n_slice, transpose, w,
                                           static_cast<__nv_bfloat16*>(img));
    BD_CHECK_LAUNCH("k_pack_weights");
    return BD_OK;
}

// Synchronous wrapper with a transient device error flag, for the standalone entry points.
template <class F>
static int run_checked(cudaStream_t st, const char* what, F launch) {
    int* err = nullptr;
    BD_CUDA(cudaMallocAsync((void**)&err, sizeof(int), st));
    int host_err = 0;
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), st);
    int rc = e == cudaSuccess ? launch(err) : BD_OK;
    if (e == cudaSuccess && rc == BD_OK) e = cudaMemcpyAsync(&host_err, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t e2 = cudaFreeAsync(err, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_status(e, what);
    if (e2 != cudaSuccess) return cuda_status(e2, what);
    if (host_err) return fail(BD_ERR_TIMEOUT, "%s: a bounded pipeline wait timed out", what);
    return BD_OK;
}

}  // namespace bd

using namespace bd;

extern "C" int64_t bd_conv_plane_rows(int nx, int ny, int nz) {
    return (int64_t)(nx + 2) * (ny + 2) * (nz + 2) + kRowMargin;
}

extern "C" int64_t bd_conv_image_bytes(int taps, int k_channels, int n_slice) {
    return (int64_t)taps * k_channels * n_slice * 2;
}

extern "C" int bd_conv_pack_weights(int taps, int cin, int cout, int n_off, int n_slice, int transpose, const float* w,
                                    void* wimage, void* stream) {
    BD_REQUIRE(w && wimage, "bd_conv_pack_weights: NULL pointer");
    BD_REQUIRE(taps == 27 || taps == 9, "bd_conv_pack_weights: taps must be 27 or 9");
    BD_REQUIRE(cin % 8 == 0 && cout % 8 == 0 && n_slice > 0 && n_off >= 0, "bd_conv_pack_weights: bad channels");
    BD_REQUIRE(n_off + n_slice <= (transpose ? cin : cout), "bd_conv_pack_weights: slice out of range");
    return pack_weights_launch(taps, cin, cout, n_off, n_slice, transpose, w, wimage, (cudaStream_t)stream);
}

extern "C" int bd_conv3d(const BdConvCall* c, void* stream) {
    BD_REQUIRE(c != nullptr, "bd_conv3d: call is NULL");
    if (int rc = conv_check(*c)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    return run_checked(st, "bd_conv3d", [&](int* err) { return conv_launch(*c, st, err); });
}

extern "C" int bd_conv3d_wgrad(int nx, int ny, int nz, int cin, int cout, int taps, const void* grad, const void* act,
                               float* dw, void* stream) {
    BD_REQUIRE(grad && act && dw, "bd_conv3d_wgrad: NULL pointer");
    BD_REQUIRE(nx > 0 && ny > 0 && nz > 0, "bd_conv3d_wgrad: dims must be positive");
    BD_REQUIRE((cin == 16 || cin == 32 || cin == 64) && (cout == 16 || cout == 32 || cout == 64),
               "bd_conv3d_wgrad: channels must be 16, 32 or 64");
    BD_REQUIRE(taps == 27 || taps == 9, "bd_conv3d_wgrad: taps must be 27 or 9");
    BD_REQUIRE((long long)(nx + 2) * (ny + 2) * (nz + 2) * 64 < (1LL << 31), "bd_conv3d_wgrad: volume too large");
    BD_REQUIRE(((uintptr_t)grad | (uintptr_t)act) % 16 == 0, "bd_conv3d_wgrad: volumes must be 16-byte aligned");
    cudaStream_t st = (cudaStream_t)stream;
    return run_checked(st, "bd_conv3d_wgrad",
                       [&](int* err) { return wgrad_launch(nx, ny, nz, cin, cout, taps, grad, act, dw, st, err); });
}

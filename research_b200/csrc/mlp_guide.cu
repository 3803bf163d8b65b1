// mlp_guide.cu — learned path guide: a BF16 multilayer perceptron on the
// sm_100a tensor cores that maps a surface point to a mixture of 8 vMF lobes.
//
// Network: inputs (80) = 12-band sin/cos encoding of the position normalised
// to the guide bounds (72), shading normal (3), view direction (3), 2 zeros;
// four hidden layers of 64 with ReLU; 48 outputs = 8 lobes x (direction 3,
// concentration 1, weight logit 1) + 8 unused. Lobe j: mu = v/|v|,
// kappa = softplus(k) + 0.1 (at most 1000), pi = softmax(logits).
//
// Kernels (all hand-written):
//  - mlp_forward_kernel: one CTA of 128 threads per 128-sample tile; every
//    layer is a chain of tcgen05.mma (M=128, N=out, K=16 steps) from the
//    activation tile and the weight tile in shared memory into a TMEM
//    accumulator; the epilogue reads the accumulator (tcgen05.ld), adds the
//    bias, applies ReLU and writes the next BF16 activation tile. Inference
//    writes the mixture of each query; training also keeps the activations
//    and evaluates the weighted negative log-likelihood and its gradient.
//  - mlp_backward_kernel: dX_l = dZ_l W_l on the tensor cores (M=128,
//    N=64, K=out), dZ_{l-1} = dX_l * [X_l > 0].
//  - mlp_wgrad_kernel / mlp_reduce_kernel: dW_l = dZ_l^T X_l, db_l = sum dZ_l
//    on the CUDA cores in FP32, per-block partials reduced in a fixed order.
//  - mlp_adam_kernel: Adam on FP32 master weights (gradients carry a static
//    loss scale), refreshing the BF16 copy used by the tensor cores.

#include "rr_guide.h"
#include "rr_vmf.cuh"
#include "rr_tc.cuh"

#include <cmath>
#include <cstring>

namespace rr {
namespace {

constexpr int kIn = 80, kHid = 64, kOut = 48, kLayers = 5, kTile = 128;
constexpr float kLossScale = 1024.0f;
__host__ __device__ constexpr int lin(int l) { return l == 0 ? kIn : kHid; }
__host__ __device__ constexpr int lout(int l) { return l == kLayers - 1 ? kOut : kHid; }
// FP32 master parameters: for each layer W[out][in] then b[out].
__host__ __device__ constexpr int woff(int l) {
    return l == 0 ? 0 : woff(l - 1) + lout(l - 1) * lin(l - 1) + lout(l - 1);
}
__host__ __device__ constexpr int boff(int l) { return woff(l) + lout(l) * lin(l); }
constexpr int kParams = woff(kLayers);
// BF16 weights: W[out][in] per layer, contiguous.
__host__ __device__ constexpr int hoff(int l) { return l == 0 ? 0 : hoff(l - 1) + lout(l - 1) * lin(l - 1); }
constexpr int kWeightsBf16 = hoff(kLayers);
// activation / gradient columns per layer input (X_l) and output (dZ_l)
__host__ __device__ constexpr int xoff(int l) { return l == 0 ? 0 : xoff(l - 1) + lin(l - 1); }
constexpr int kXCols = xoff(kLayers);            // 80 + 4*64 = 336
__host__ __device__ constexpr int zoff(int l) { return l == 0 ? 0 : zoff(l - 1) + lout(l - 1); }
constexpr int kZCols = zoff(kLayers);            // 4*64 + 48 = 304

// shared memory map of the forward / backward kernels
constexpr int kSmWf = 0;                         // forward weight tiles
constexpr int kSmWt = kSmWf + 2 * kWeightsBf16;  // transposed weight tiles
constexpr int kSmAct = kSmWt + 2 * kWeightsBf16; // 128 x 80 BF16 activation tile
constexpr int kSmBias = kSmAct + kTile * kIn * 2;
constexpr int kSmBar = kSmBias + 4 * 320;
constexpr int kSmTotal = kSmBar + 64;

__device__ __forceinline__ uint32_t wtile(int l) { return uint32_t(kSmWf + 2 * hoff(l)); }
__device__ __forceinline__ uint32_t ttile(int l) { return uint32_t(kSmWt + 2 * hoff(l)); }

struct MlpView {
    const __nv_bfloat16* w16;     // kWeightsBf16
    const float* params;          // kParams (biases read from here)
    float3 bmin, inv_ext;
    int* error;                   // set when an mbarrier wait gave up
};

// Loads both weight layouts and the biases into shared memory.
__device__ void load_weights(unsigned char* sm, const MlpView& V) {
    for (int l = 0; l < kLayers; ++l) {
        const int I = lin(l), O = lout(l);
        const unsigned short* src = reinterpret_cast<const unsigned short*>(V.w16 + hoff(l));
        for (int e = threadIdx.x; e < I * O; e += blockDim.x) {
            const int o = e / I, i = e % I;
            const unsigned short v = src[e];
            *reinterpret_cast<unsigned short*>(sm + wtile(l) + tc::tile_offset(o, i, O)) = v;
            *reinterpret_cast<unsigned short*>(sm + ttile(l) + tc::tile_offset(i, o, I)) = v;
        }
    }
    float* bias = reinterpret_cast<float*>(sm + kSmBias);
    for (int l = 0; l < kLayers; ++l)
        for (int o = threadIdx.x; o < lout(l); o += blockDim.x) bias[l * 64 + o] = V.params[boff(l) + o];
}

__device__ void encode(const MlpView& V, float3 p, float3 n, float3 wo, float* f) {
    const float x[3] = {fminf(fmaxf((p.x - V.bmin.x) * V.inv_ext.x, 0.0f), 1.0f),
                        fminf(fmaxf((p.y - V.bmin.y) * V.inv_ext.y, 0.0f), 1.0f),
                        fminf(fmaxf((p.z - V.bmin.z) * V.inv_ext.z, 0.0f), 1.0f)};
    #pragma unroll
    for (int a = 0; a < 3; ++a) {
        float fr = 3.14159265358979f;
        #pragma unroll
        for (int k = 0; k < 12; ++k) {
            float s, c;
            sincosf(fr * x[a], &s, &c);
            f[a * 24 + k] = s;
            f[a * 24 + 12 + k] = c;
            fr *= 2.0f;
        }
    }
    f[72] = n.x; f[73] = n.y; f[74] = n.z;
    f[75] = wo.x; f[76] = wo.y; f[77] = wo.z;
    f[78] = 0.0f; f[79] = 0.0f;
}

__device__ __forceinline__ float softplus(float x) { return x > 20.0f ? x : log1pf(expf(x)); }
__device__ __forceinline__ float sigmoid(float x) { return 1.0f / (1.0f + expf(-x)); }

// Raw outputs -> mixture (mu, kappa, pi).
__device__ void head_mixture(const float* r, float4* lobe, float* pi) {
    float mxl = -1e30f;
    for (int j = 0; j < kMaxLobes; ++j) mxl = fmaxf(mxl, r[5 * j + 4]);
    float z = 0.0f;
    for (int j = 0; j < kMaxLobes; ++j) { pi[j] = expf(r[5 * j + 4] - mxl); z += pi[j]; }
    for (int j = 0; j < kMaxLobes; ++j) {
        pi[j] /= z;
        const float vx = r[5 * j], vy = r[5 * j + 1], vz = r[5 * j + 2];
        const float len = fmaxf(sqrtf(vx * vx + vy * vy + vz * vz), 1e-6f);
        const float kappa = fminf(softplus(r[5 * j + 3]) + 0.1f, 1000.0f);
        lobe[j] = make_float4(vx / len, vy / len, vz / len, kappa);
    }
}

// Weighted NLL of direction om under the mixture and its gradient w.r.t.
// the 48 raw outputs (scaled by scale). Returns -log p.
__device__ float head_grad(const float* r, float3 om, float scale, float* g) {
    float4 lobe[kMaxLobes];
    float pi[kMaxLobes], lq[kMaxLobes];
    head_mixture(r, lobe, pi);
    float lmax = -1e30f;
    for (int j = 0; j < kMaxLobes; ++j) {
        const float k = lobe[j].w;
        const float cosw = lobe[j].x * om.x + lobe[j].y * om.y + lobe[j].z * om.z;
        const float lognorm = logf(k) - logf(6.28318530718f) - log1pf(-expf(-2.0f * k));
        lq[j] = logf(fmaxf(pi[j], 1e-30f)) + lognorm + k * (cosw - 1.0f);
        lmax = fmaxf(lmax, lq[j]);
    }
    float s = 0.0f;
    for (int j = 0; j < kMaxLobes; ++j) s += expf(lq[j] - lmax);
    const float logp = lmax + logf(s);
    for (int q = 0; q < kOut; ++q) g[q] = 0.0f;
    for (int j = 0; j < kMaxLobes; ++j) {
        const float gam = expf(lq[j] - logp);
        const float k = lobe[j].w;
        const float cosw = lobe[j].x * om.x + lobe[j].y * om.y + lobe[j].z * om.z;
        const float vx = r[5 * j], vy = r[5 * j + 1], vz = r[5 * j + 2];
        const float len = fmaxf(sqrtf(vx * vx + vy * vy + vz * vz), 1e-6f);
        // d(-log p)/dv = -(gam kappa / |v|) (om - (mu.om) mu)
        const float cv = -gam * k / len;
        g[5 * j + 0] = scale * cv * (om.x - cosw * lobe[j].x);
        g[5 * j + 1] = scale * cv * (om.y - cosw * lobe[j].y);
        g[5 * j + 2] = scale * cv * (om.z - cosw * lobe[j].z);
        // d(-log p)/dkappa = -gam (1/kappa - 2 e^{-2k}/(1 - e^{-2k}) + cos - 1)
        const float e2 = expf(-2.0f * k);
        float dk = -gam * (1.0f / k - 2.0f * e2 / (1.0f - e2) + cosw - 1.0f);
        if (softplus(r[5 * j + 3]) + 0.1f > 1000.0f) dk = 0.0f;
        g[5 * j + 3] = scale * dk * sigmoid(r[5 * j + 3]);
        g[5 * j + 4] = scale * (pi[j] - gam);
    }
    return -logp;
}

struct FwdArgs {
    MlpView V;
    // inference: per queue slot surfaces -> mixtures
    const float4* surf;
    float4* mix;
    const uint32_t* count_ptr;
    uint32_t count;
    // training
    GuideSamples S;
    const uint32_t* sel;          // batch -> sample index
    const double* wnorm;          // [0] = clamp value, [1] = 1 / (sum of clamped weights)
    __nv_bfloat16* X;             // [batch][kXCols]
    float* dout;                  // [batch][kOut]
    float* loss_partial;          // per block
};

template <bool Train>
__global__ void __launch_bounds__(kTile) mlp_forward_kernel(FwdArgs A) {
    extern __shared__ __align__(1024) unsigned char sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kSmBar);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kSmBar + 8);
    const float* bias = reinterpret_cast<const float*>(sm + kSmBias);
    unsigned char* act = sm + kSmAct;
    const int t = threadIdx.x, warp = t >> 5;
    load_weights(sm, A.V);
    if (warp == 0) tc::tmem_alloc(tslot, 128);
    if (t == 0) tc::mbar_init(bar, 1);
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t count = Train ? A.count : *A.count_ptr;
    const uint32_t tiles = (count + kTile - 1) / kTile;
    const uint32_t act_addr = tc::smem_addr(act);
    const uint32_t sm_base = tc::smem_addr(sm);
    uint32_t phase = 0;
    float loss_acc = 0.0f;
    bool ok = true;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t row = tile * kTile + t;
        const bool valid = row < count;
        float f[kIn];
        float3 om = f3(0, 0, 0);
        float wgt = 0.0f;
        bool active = false;
        if (valid) {
            if (Train) {
                const uint32_t si = A.sel[row];
                const float4 s0 = A.S.s0[si], s1 = A.S.s1[si], s2 = A.S.s2[si], s3 = A.S.s3[si];
                encode(A.V, xyz(s0), xyz(s2), xyz(s3), f);
                om = xyz(s1);
                wgt = float(double(fminf(s0.w, float(A.wnorm[0]))) * A.wnorm[1]);
                active = true;
            } else {
                const float4 a = A.surf[size_t(row) * 3], b = A.surf[size_t(row) * 3 + 1], c = A.surf[size_t(row) * 3 + 2];
                active = b.w > 0.0f;
                encode(A.V, xyz(a), xyz(b), xyz(c), f);
            }
        } else {
            for (int k = 0; k < kIn; ++k) f[k] = 0.0f;
        }
        for (int k = 0; k < kIn; k += 8) tc::st_row8(act, kTile, t, k, f + k);
        if (Train && valid) {
            uint4* dst = reinterpret_cast<uint4*>(A.X + size_t(row) * kXCols);
            for (int k = 0; k < kIn; k += 8)
                dst[k / 8] = make_uint4(tc::pack_bf16(f[k], f[k + 1]), tc::pack_bf16(f[k + 2], f[k + 3]),
                                        tc::pack_bf16(f[k + 4], f[k + 5]), tc::pack_bf16(f[k + 6], f[k + 7]));
        }
        float out[kHid];
        for (int l = 0; l < kLayers; ++l) {
            const int I = lin(l), O = lout(l);
            tc::fence_proxy_async();
            tc::fence_before_sync();
            __syncthreads();
            if (t == 0) {
                tc::fence_after_sync();
                const uint32_t idesc = tc::idesc_bf16(kTile, O);
                for (int s = 0; s < I / 16; ++s) {
                    const uint64_t ad = tc::smem_desc(act_addr + s * 2 * (kTile / 8) * 128, (kTile / 8) * 128, 128);
                    const uint64_t bd = tc::smem_desc(sm_base + wtile(l) + s * 2 * (O / 8) * 128, (O / 8) * 128, 128);
                    tc::mma_bf16(tmem, ad, bd, idesc, s > 0);
                }
                tc::mma_commit(bar);
            }
            ok = tc::mbar_wait(bar, phase) && ok;
            phase ^= 1u;
            tc::fence_after_sync();
            for (int c = 0; c < O; c += 16) tc::tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + c, out + c);
            tc::tmem_wait_ld();
            for (int o = 0; o < O; ++o) out[o] += bias[l * 64 + o];
            if (l + 1 < kLayers) {
                for (int o = 0; o < O; ++o) out[o] = fmaxf(out[o], 0.0f);
                for (int k = 0; k < O; k += 8) tc::st_row8(act, kTile, t, k, out + k);
                if (Train && valid) {
                    uint4* dst = reinterpret_cast<uint4*>(A.X + size_t(row) * kXCols + xoff(l + 1));
                    for (int k = 0; k < O; k += 8)
                        dst[k / 8] = make_uint4(tc::pack_bf16(out[k], out[k + 1]), tc::pack_bf16(out[k + 2], out[k + 3]),
                                                tc::pack_bf16(out[k + 4], out[k + 5]), tc::pack_bf16(out[k + 6], out[k + 7]));
                }
            }
        }
        if (valid) {
            if (Train) {
                float g[kOut];
                const float nll = head_grad(out, om, wgt * kLossScale, g);
                loss_acc += wgt * nll;
                float4* d = reinterpret_cast<float4*>(A.dout + size_t(row) * kOut);
                for (int q = 0; q < kOut; q += 4) d[q / 4] = make_float4(g[q], g[q + 1], g[q + 2], g[q + 3]);
                (void)active;
            } else {
                float4 lobe[kMaxLobes];
                float pi[kMaxLobes];
                float4* m = A.mix + size_t(row) * (kMaxLobes + 2);
                if (active) {
                    head_mixture(out, lobe, pi);
                    for (int j = 0; j < kMaxLobes; ++j) m[j] = lobe[j];
                    m[kMaxLobes] = make_float4(pi[0], pi[1], pi[2], pi[3]);
                    m[kMaxLobes + 1] = make_float4(pi[4], pi[5], pi[6], pi[7]);
                } else {
                    m[kMaxLobes] = make_float4(0, 0, 0, 0);
                    m[kMaxLobes + 1] = make_float4(0, 0, 0, 0);
                }
            }
        }
    }
    if (Train) {
        __shared__ float red[kTile];
        red[t] = loss_acc;
        __syncthreads();
        for (int s = kTile / 2; s > 0; s >>= 1) {
            if (t < s) red[t] += red[t + s];
            __syncthreads();
        }
        if (t == 0) A.loss_partial[blockIdx.x] = red[0];
    }
    if (!ok && t == 0) atomicExch(A.V.error, 1);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_free(tmem, 128);
    }
}

struct BwdArgs {
    MlpView V;
    uint32_t count;
    const __nv_bfloat16* X;       // [batch][kXCols]
    const float* dout;            // [batch][kOut]
    __nv_bfloat16* dZ;            // [batch][kZCols]
};

// dZ_4 = dout; dX_l = dZ_l W_l (tensor cores), dZ_{l-1} = dX_l * [X_l > 0].
__global__ void __launch_bounds__(kTile) mlp_backward_kernel(BwdArgs A) {
    extern __shared__ __align__(1024) unsigned char sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kSmBar);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kSmBar + 8);
    unsigned char* act = sm + kSmAct;
    const int t = threadIdx.x, warp = t >> 5;
    load_weights(sm, A.V);
    if (warp == 0) tc::tmem_alloc(tslot, 128);
    if (t == 0) tc::mbar_init(bar, 1);
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t tiles = (A.count + kTile - 1) / kTile;
    const uint32_t act_addr = tc::smem_addr(act);
    const uint32_t sm_base = tc::smem_addr(sm);
    uint32_t phase = 0;
    bool ok = true;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t row = tile * kTile + t;
        const bool valid = row < A.count;
        float dz[kHid];
        for (int q = 0; q < kOut; ++q) dz[q] = valid ? A.dout[size_t(row) * kOut + q] : 0.0f;
        for (int q = kOut; q < kHid; ++q) dz[q] = 0.0f;
        for (int l = kLayers - 1; l >= 0; --l) {
            const int I = lin(l), O = lout(l);
            // dZ_l: keep it for the weight gradient and stage it as the A operand
            if (valid) {
                uint4* dst = reinterpret_cast<uint4*>(A.dZ + size_t(row) * kZCols + zoff(l));
                for (int k = 0; k < O; k += 8)
                    dst[k / 8] = make_uint4(tc::pack_bf16(dz[k], dz[k + 1]), tc::pack_bf16(dz[k + 2], dz[k + 3]),
                                            tc::pack_bf16(dz[k + 4], dz[k + 5]), tc::pack_bf16(dz[k + 6], dz[k + 7]));
            }
            if (l == 0) break;
            for (int k = 0; k < O; k += 8) tc::st_row8(act, kTile, t, k, dz + k);
            tc::fence_proxy_async();
            tc::fence_before_sync();
            __syncthreads();
            if (t == 0) {
                tc::fence_after_sync();
                const uint32_t idesc = tc::idesc_bf16(kTile, I);
                for (int s = 0; s < O / 16; ++s) {
                    const uint64_t ad = tc::smem_desc(act_addr + s * 2 * (kTile / 8) * 128, (kTile / 8) * 128, 128);
                    const uint64_t bd = tc::smem_desc(sm_base + ttile(l) + s * 2 * (I / 8) * 128, (I / 8) * 128, 128);
                    tc::mma_bf16(tmem, ad, bd, idesc, s > 0);
                }
                tc::mma_commit(bar);
            }
            ok = tc::mbar_wait(bar, phase) && ok;
            phase ^= 1u;
            tc::fence_after_sync();
            float dx[kHid];
            for (int c = 0; c < I; c += 16) tc::tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + c, dx + c);
            tc::tmem_wait_ld();
            tc::fence_before_sync();
            __syncthreads();  // every lane has read the accumulator before the next chain
            // X_l (input of layer l, l >= 1) is ReLU(Z_{l-1}): its mask gates dZ_{l-1}
            for (int k = 0; k < I; ++k) {
                float xv = 0.0f;
                if (valid) xv = __bfloat162float(A.X[size_t(row) * kXCols + xoff(l) + k]);
                dz[k] = xv > 0.0f ? dx[k] : 0.0f;
            }
        }
    }
    if (!ok && t == 0) atomicExch(A.V.error, 1);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_free(tmem, 128);
    }
}

// Weight gradients on the CUDA cores: block (layer, chunk) accumulates
// dW[o][i] (and db[o] as column I) over its sample chunk.
constexpr int kWgChunk = 2048;
__global__ void __launch_bounds__(256) mlp_wgrad_kernel(const __nv_bfloat16* __restrict__ X,
                                                        const __nv_bfloat16* __restrict__ dZ, uint32_t count,
                                                        float* __restrict__ partial, uint32_t chunks) {
    const int l = blockIdx.y;
    const int I = lin(l), O = lout(l);
    const uint32_t b0 = blockIdx.x * kWgChunk;
    const uint32_t b1 = min(count, b0 + kWgChunk);
    __shared__ float sx[32][kIn + 1];
    __shared__ float sz[32][kHid];
    const int t = threadIdx.x;
    const int o = t >> 2;                 // 0..63
    const int iq = t & 3;                 // columns iq, iq+4, ... (I+1 columns incl. bias)
    float acc[21];
    for (int j = 0; j < 21; ++j) acc[j] = 0.0f;
    for (uint32_t bb = b0; bb < b1; bb += 32) {
        for (int e = t; e < 32 * (I + 1); e += 256) {
            const int r = e / (I + 1), c = e % (I + 1);
            const uint32_t b = bb + r;
            sx[r][c] = (b < b1) ? (c < I ? __bfloat162float(X[size_t(b) * kXCols + xoff(l) + c]) : 1.0f) : 0.0f;
        }
        for (int e = t; e < 32 * O; e += 256) {
            const int r = e / O, c = e % O;
            const uint32_t b = bb + r;
            sz[r][c] = (b < b1) ? __bfloat162float(dZ[size_t(b) * kZCols + zoff(l) + c]) : 0.0f;
        }
        __syncthreads();
        if (o < O) {
            for (int r = 0; r < 32; ++r) {
                const float z = sz[r][o];
                for (int j = 0, i = iq; i <= I; ++j, i += 4) acc[j] += z * sx[r][i];
            }
        }
        __syncthreads();
    }
    if (o < O) {
        float* dst = partial + (size_t(l) * chunks + blockIdx.x) * (kHid * (kIn + 1));
        for (int j = 0, i = iq; i <= I; ++j, i += 4) dst[o * (kIn + 1) + i] = acc[j];
    }
}

__global__ void __launch_bounds__(256) mlp_reduce_kernel(const float* __restrict__ partial, uint32_t chunks,
                                                         float* __restrict__ grad) {
    const int l = blockIdx.y;
    const int I = lin(l), O = lout(l);
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= O * (I + 1)) return;
    const int o = e / (I + 1), i = e % (I + 1);
    float s = 0.0f;
    for (uint32_t c = 0; c < chunks; ++c) s += partial[(size_t(l) * chunks + c) * (kHid * (kIn + 1)) + o * (kIn + 1) + i];
    if (i < I) grad[woff(l) + o * I + i] = s;
    else grad[boff(l) + o] = s;
}

__global__ void __launch_bounds__(256) mlp_adam_kernel(float* __restrict__ params, const float* __restrict__ grad,
                                                       float* __restrict__ m, float* __restrict__ v,
                                                       __nv_bfloat16* __restrict__ w16, float lr, float bc1,
                                                       float bc2) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    const float g = grad[p] / kLossScale;
    const float mm = 0.9f * m[p] + 0.1f * g;
    const float vv = 0.999f * v[p] + 0.001f * g * g;
    m[p] = mm;
    v[p] = vv;
    const float th = params[p] - lr * (mm / bc1) / (sqrtf(vv / bc2) + 1e-8f);
    params[p] = th;
    // refresh the BF16 copy of weights (biases stay FP32)
    for (int l = 0; l < kLayers; ++l)
        if (p >= woff(l) && p < boff(l)) w16[hoff(l) + (p - woff(l))] = __float2bfloat16_rn(th);
}

// Sum of clamped weights of the batch (clamp = 20 x mean), fixed order.
__global__ void __launch_bounds__(256) mlp_weight_norm_kernel(GuideSamples S, const uint32_t* sel, uint32_t n,
                                                              double* out) {
    __shared__ double red[256];
    const int t = threadIdx.x;
    double s = 0.0;
    for (uint32_t i = t; i < n; i += 256) s += double(S.s0[sel[i]].w);
    red[t] = s;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) { if (t < k) red[t] += red[t + k]; __syncthreads(); }
    const double mean = red[0] / double(n > 0 ? n : 1);
    const double clampv = 20.0 * mean;
    __syncthreads();
    s = 0.0;
    for (uint32_t i = t; i < n; i += 256) s += fmin(double(S.s0[sel[i]].w), clampv);
    red[t] = s;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) { if (t < k) red[t] += red[t + k]; __syncthreads(); }
    if (t == 0) { out[0] = clampv; out[1] = red[0] > 0.0 ? 1.0 / red[0] : 0.0; }
}

__global__ void mlp_select_kernel(uint32_t* sel, uint32_t batch, uint32_t n, uint32_t offset) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= batch) return;
    sel[i] = uint32_t((uint64_t(i) * n) / batch + offset) % n;
}

// deterministic uniform init (hash), He-uniform for hidden layers
__global__ void mlp_init_kernel(float* params, __nv_bfloat16* w16, uint32_t seed) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    float v = 0.0f;
    for (int l = 0; l < kLayers; ++l) {
        if (p >= woff(l) && p < boff(l)) {
            uint32_t h = pcg_hash(uint32_t(p) * 2654435761u ^ seed);
            const float u = float(h >> 8) * (1.0f / 16777216.0f) * 2.0f - 1.0f;
            const float a = l == kLayers - 1 ? 0.05f : sqrtf(6.0f / float(lin(l)));
            v = u * a;
            w16[hoff(l) + (p - woff(l))] = __float2bfloat16_rn(v);
        }
    }
    params[p] = v;
}

} // namespace
} // namespace rr

using namespace rr;

struct rr_mlp_state {
    float* params = nullptr;
    float* grad = nullptr;
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    __nv_bfloat16* w16 = nullptr;
    int* error = nullptr;
    uint32_t* sel = nullptr;
    double* wnorm = nullptr;
    __nv_bfloat16* X = nullptr;
    __nv_bfloat16* dZ = nullptr;
    float* dout = nullptr;
    float* loss_partial = nullptr;
    float* wpartial = nullptr;
    uint32_t batch_cap = 0;
    uint32_t steps = 0;
    int grid = 0;
    double last_loss = 0.0;
    float* loss_host = nullptr;
};

rr_guide::~rr_guide() {
    for (int k = 0; k < 4; ++k) cudaFree(rec[k]);
    cudaFree(mlp_surf);
    cudaFree(mlp_mix);
    if (mlp) cudaFreeHost(mlp->loss_host);
    delete mlp;
}

static MlpView mlp_view(rr_guide* g) {
    MlpView V;
    V.w16 = g->mlp->w16;
    V.params = g->mlp->params;
    V.bmin = make_float3(g->desc.bounds_min[0], g->desc.bounds_min[1], g->desc.bounds_min[2]);
    V.inv_ext = make_float3(1.0f / (g->desc.bounds_max[0] - g->desc.bounds_min[0]),
                            1.0f / (g->desc.bounds_max[1] - g->desc.bounds_min[1]),
                            1.0f / (g->desc.bounds_max[2] - g->desc.bounds_min[2]));
    V.error = g->mlp->error;
    return V;
}

rr_status rr_mlp_guide_init(rr_ctx* ctx, rr_guide* g) {
    g->mlp = new rr_mlp_state;
    rr_mlp_state& M = *g->mlp;
    const uint32_t B = std::max(128u, g->desc.mlp_batch ? g->desc.mlp_batch : (1u << 18));
    M.batch_cap = B;
    auto al = [&](void** p, size_t bytes) -> rr_status {
        RR_TRY_CUDA(ctx, cudaMalloc(p, bytes));
        g->allocations.push_back(*p);
        return RR_OK;
    };
    rr_status st;
    if ((st = al(reinterpret_cast<void**>(&M.params), kParams * 4)) != RR_OK) return st;
    if ((st = al(reinterpret_cast<void**>(&M.grad), kParams * 4)) != RR_OK) return st;
    if ((st = al(reinterpret_cast<void**>(&M.adam_m), kParams * 4)) != RR_OK) return st;
    if ((st = al(reinterpret_cast<void**>(&M.adam_v), kParams * 4)) != RR_OK) return st;
    if ((st = al(reinterpret_cast<void**>(&M.w16), kWeightsBf16 * 2)) != RR_OK) return st;
    if ((st = al(reinterpret_cast<void**>(&M.error), 16)) != RR_OK) return st;
    if ((st = al(reinterpret_cast<void**>(&M.sel), size_t(B) * 4)) != RR_OK) return st;
    if ((st = al(reinterpret_cast<void**>(&M.wnorm), 16)) != RR_OK) return st;
    if ((st = al(reinterpret_cast<void**>(&M.X), size_t(B) * kXCols * 2)) != RR_OK) return st;
    if ((st = al(reinterpret_cast<void**>(&M.dZ), size_t(B) * kZCols * 2)) != RR_OK) return st;
    if ((st = al(reinterpret_cast<void**>(&M.dout), size_t(B) * kOut * 4)) != RR_OK) return st;
    M.grid = ctx->sm_count;
    if ((st = al(reinterpret_cast<void**>(&M.loss_partial), size_t(M.grid) * 4 * 4)) != RR_OK) return st;
    const uint32_t chunks = (B + kWgChunk - 1) / kWgChunk;
    if ((st = al(reinterpret_cast<void**>(&M.wpartial), size_t(kLayers) * chunks * kHid * (kIn + 1) * 4)) != RR_OK)
        return st;
    RR_TRY_CUDA(ctx, cudaMallocHost(&M.loss_host, size_t(M.grid) * 4 * 4));
    for (auto k : {mlp_forward_kernel<true>, mlp_forward_kernel<false>})
        RR_TRY_CUDA(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmTotal));
    RR_TRY_CUDA(ctx, cudaFuncSetAttribute(mlp_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmTotal));
    return RR_OK;
}

rr_status rr_mlp_guide_reset(rr_ctx* ctx, rr_guide* g, cudaStream_t stream) {
    rr_mlp_state& M = *g->mlp;
    mlp_init_kernel<<<(kParams + 255) / 256, 256, 0, stream>>>(M.params, M.w16, g->desc.seed * 0x9E3779B9u + 1u);
    RR_CHECK_LAUNCH(ctx);
    RR_TRY_CUDA(ctx, cudaMemsetAsync(M.adam_m, 0, kParams * 4, stream));
    RR_TRY_CUDA(ctx, cudaMemsetAsync(M.adam_v, 0, kParams * 4, stream));
    RR_TRY_CUDA(ctx, cudaMemsetAsync(M.grad, 0, kParams * 4, stream));
    RR_TRY_CUDA(ctx, cudaMemsetAsync(M.error, 0, 16, stream));
    M.steps = 0;
    M.last_loss = 0.0;
    return RR_OK;
}

rr_status rr_mlp_guide_ensure(rr_ctx* ctx, rr_guide* g, size_t slots) {
    if (g->mlp_slots >= slots) return RR_OK;
    cudaFree(g->mlp_surf);
    cudaFree(g->mlp_mix);
    g->mlp_surf = nullptr;
    g->mlp_mix = nullptr;
    g->mlp_slots = 0;
    RR_TRY_CUDA(ctx, cudaMalloc(&g->mlp_surf, slots * 3 * sizeof(float4)));
    RR_TRY_CUDA(ctx, cudaMalloc(&g->mlp_mix, slots * (kMaxLobes + 2) * sizeof(float4)));
    g->mlp_slots = slots;
    return RR_OK;
}

rr_status rr_mlp_guide_infer(rr_ctx* ctx, rr_guide* g, const uint32_t* count_dev, uint32_t max_count,
                             cudaStream_t stream) {
    FwdArgs A{};
    A.V = mlp_view(g);
    A.surf = g->mlp_surf;
    A.mix = g->mlp_mix;
    A.count_ptr = count_dev;
    const uint32_t tiles = (max_count + kTile - 1) / kTile;
    const int grid = int(std::min<uint32_t>(tiles, uint32_t(2 * ctx->sm_count)));
    mlp_forward_kernel<false><<<std::max(grid, 1), kTile, kSmTotal, stream>>>(A);
    RR_CHECK_LAUNCH(ctx);
    g->mlp_infer_launches = 1;
    return RR_OK;
}

// Runs the network on caller-provided surfaces (rr_guide_eval for MLP guides).
rr_status rr_mlp_guide_eval(rr_ctx* ctx, rr_guide* g, const float4* surf, float4* mix, const uint32_t* count_dev,
                            uint32_t count, cudaStream_t stream) {
    FwdArgs A{};
    A.V = mlp_view(g);
    A.surf = surf;
    A.mix = mix;
    A.count_ptr = count_dev;
    const uint32_t tiles = (count + kTile - 1) / kTile;
    const int grid = int(std::min<uint32_t>(tiles, uint32_t(2 * ctx->sm_count)));
    mlp_forward_kernel<false><<<std::max(grid, 1), kTile, kSmTotal, stream>>>(A);
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}

rr_status rr_mlp_guide_train(rr_ctx* ctx, rr_guide* g, uint32_t n, cudaStream_t stream) {
    rr_mlp_state& M = *g->mlp;
    if (n == 0) return RR_OK;
    const uint32_t B = std::min(n, M.batch_cap);
    mlp_select_kernel<<<(B + 255) / 256, 256, 0, stream>>>(M.sel, B, n, (M.steps * 7919u) % n);
    RR_CHECK_LAUNCH(ctx);
    mlp_weight_norm_kernel<<<1, 256, 0, stream>>>(g->samples, M.sel, B, M.wnorm);
    RR_CHECK_LAUNCH(ctx);
    FwdArgs A{};
    A.V = mlp_view(g);
    A.count = B;
    A.S = g->samples;
    A.sel = M.sel;
    A.wnorm = M.wnorm;
    A.X = M.X;
    A.dout = M.dout;
    A.loss_partial = M.loss_partial;
    const uint32_t tiles = (B + kTile - 1) / kTile;
    const int grid = int(std::min<uint32_t>(tiles, uint32_t(M.grid)));
    RR_TRY_CUDA(ctx, cudaMemsetAsync(M.loss_partial, 0, size_t(M.grid) * 4, stream));
    mlp_forward_kernel<true><<<grid, kTile, kSmTotal, stream>>>(A);
    RR_CHECK_LAUNCH(ctx);
    BwdArgs Bw{};
    Bw.V = A.V;
    Bw.count = B;
    Bw.X = M.X;
    Bw.dout = M.dout;
    Bw.dZ = M.dZ;
    mlp_backward_kernel<<<grid, kTile, kSmTotal, stream>>>(Bw);
    RR_CHECK_LAUNCH(ctx);
    const uint32_t chunks = (B + kWgChunk - 1) / kWgChunk;
    mlp_wgrad_kernel<<<dim3(chunks, kLayers), 256, 0, stream>>>(M.X, M.dZ, B, M.wpartial, chunks);
    RR_CHECK_LAUNCH(ctx);
    mlp_reduce_kernel<<<dim3((kHid * (kIn + 1) + 255) / 256, kLayers), 256, 0, stream>>>(M.wpartial, chunks, M.grad);
    RR_CHECK_LAUNCH(ctx);
    M.steps += 1;
    const float bc1 = 1.0f - std::pow(0.9f, float(M.steps));
    const float bc2 = 1.0f - std::pow(0.999f, float(M.steps));
    mlp_adam_kernel<<<(kParams + 255) / 256, 256, 0, stream>>>(M.params, M.grad, M.adam_m, M.adam_v, M.w16,
                                                               g->desc.learning_rate, bc1, bc2);
    RR_CHECK_LAUNCH(ctx);
    RR_TRY_CUDA(ctx, cudaMemcpyAsync(M.loss_host, M.loss_partial, size_t(M.grid) * 4, cudaMemcpyDeviceToHost, stream));
    ctx->launches += 8;
    return RR_OK;
}

double rr_mlp_guide_last_loss(rr_guide* g) {
    rr_mlp_state& M = *g->mlp;
    double s = 0.0;
    for (int i = 0; i < M.grid; ++i) s += M.loss_host[i];
    M.last_loss = s;
    return s;
}

extern "C" rr_status rr_guide_mlp_params(rr_ctx* ctx, rr_guide* g, float* params_out, float* grad_out,
                                         float* params_in, uint32_t count, int* error_flag) {
    if (!ctx || !g) return RR_ERR_INVALID_ARGUMENT;
    if (g->desc.kind != RR_GUIDE_MLP || !g->mlp) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "not an MLP guide");
    if (count != uint32_t(kParams))
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "parameter count is %d, not %u", kParams, count);
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    RR_TRY_CUDA(ctx, cudaDeviceSynchronize());
    rr_mlp_state& M = *g->mlp;
    if (params_out) RR_TRY_CUDA(ctx, cudaMemcpy(params_out, M.params, kParams * 4, cudaMemcpyDeviceToHost));
    if (grad_out) RR_TRY_CUDA(ctx, cudaMemcpy(grad_out, M.grad, kParams * 4, cudaMemcpyDeviceToHost));
    if (error_flag) RR_TRY_CUDA(ctx, cudaMemcpy(error_flag, M.error, 4, cudaMemcpyDeviceToHost));
    if (params_in) {
        RR_TRY_CUDA(ctx, cudaMemcpy(M.params, params_in, kParams * 4, cudaMemcpyHostToDevice));
        std::vector<__nv_bfloat16> h(kWeightsBf16);
        for (int l = 0; l < kLayers; ++l)
            for (int e = 0; e < lout(l) * lin(l); ++e) h[hoff(l) + e] = __float2bfloat16_rn(params_in[woff(l) + e]);
        RR_TRY_CUDA(ctx, cudaMemcpy(M.w16, h.data(), kWeightsBf16 * 2, cudaMemcpyHostToDevice));
    }
    return RR_OK;
}

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
//  - mlp_backward_kernel: per 128-sample tile and layer l = 4 .. 1,
//    dX_l = dZ_l W_l (M=128, N=64, K=out) and dW_l^T += X_l^T dZ_l (M=128
//    features, N=out, K=128 samples) on the tensor cores, then
//    dZ_{l-1} = dX_l * [X_l > 0] in place in shared memory; dW_0^T last.
//    X_l and dZ_4 arrive by tensor copies (TMA); every CTA accumulates its
//    tiles' weight gradients in TMEM and writes one FP32 partial;
//    mlp_reduce_kernel sums the partials in CTA order.
//  - mlp_adam_kernel: Adam on FP32 master weights and biases (gradients carry
//    a static loss scale), refreshing the BF16 copy used by the tensor cores;
//    the forward kernel adds the biases inside the MMA (a constant-1 input
//    column against a BF16 bias column of the weight tile).

#include "rr_guide.h"

#include <cuda.h>
#include <cudaTypedefs.h>

// cuTensorMapEncodeTiled from the driver (atrous.cu).
PFN_cuTensorMapEncodeTiled_v12000 rr_tensor_map_encoder();
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
// Offsets are closed forms (not recursions), so they also fold or stay cheap
// where the layer index is only known at run time.
// FP32 master parameters: for each layer W[out][in] then b[out].
__host__ __device__ constexpr int woff(int l) {
    return l == 0 ? 0
                  : (kHid * kIn + kHid) + (l - 1) * (kHid * kHid + kHid) -
                        (l == kLayers ? kHid * kHid + kHid - (kOut * kHid + kOut) : 0);
}
__host__ __device__ constexpr int boff(int l) { return woff(l) + lout(l) * lin(l); }
constexpr int kParams = woff(kLayers);
// BF16 weights: W[out][in] per layer, contiguous.
__host__ __device__ constexpr int hoff(int l) {
    return l == 0 ? 0 : kHid * kIn + (l - 1) * kHid * kHid - (l == kLayers ? kHid * kHid - kOut * kHid : 0);
}
constexpr int kWeightsBf16 = hoff(kLayers);
// activation / gradient columns per layer input (X_l) and output (dZ_l)
__host__ __device__ constexpr int xoff(int l) { return l == 0 ? 0 : kIn + (l - 1) * kHid; }
constexpr int kXCols = xoff(kLayers);            // 80 + 4*64 = 336
__host__ __device__ constexpr int zoff(int l) { return l * kHid - (l == kLayers ? kHid - kOut : 0); }
constexpr int kZCols = zoff(kLayers);            // 4*64 + 48 = 304
static_assert(kParams == 80 * 64 + 64 + 3 * (64 * 64 + 64) + 48 * 64 + 48, "parameter count");
static_assert(kWeightsBf16 == 80 * 64 + 3 * 64 * 64 + 48 * 64 && kXCols == 336 && kZCols == 304, "layouts");

// shared memory maps: the forward kernel keeps W (B operand N = out, K = in),
// the backward kernel W^T (N = in, K = out); each has one 128-row BF16
// activation tile (the A operand) and one mbarrier
// Forward weight tiles carry the bias: every layer runs with K = 80, the
// activation tile holds a constant 1 in column kBiasCol(l) (78 for layer 0,
// whose inputs 78 and 79 are zero padding; 64 after the 64 hidden values) and
// the weight tile holds the bias in that column, so the epilogue adds nothing.
__host__ __device__ constexpr int kBiasCol(int l) { return l == 0 ? 78 : kHid; }
__host__ __device__ constexpr int fwd_wtile(int l) { return l == 0 ? 0 : l * kHid * kIn * 2; }  // bytes
constexpr int kSmFwdW = 0;
constexpr int kSmFwdAct = kSmFwdW + fwd_wtile(kLayers - 1) + kOut * kIn * 2;
constexpr int kSmFwdBar = kSmFwdAct + kTile * kIn * 2;
constexpr int kSmFwd = kSmFwdBar + 64;
// Forward CTAs of NW warpgroups (128 threads each) share one copy of the
// weights; each warpgroup owns an activation tile, an mbarrier and 64 TMEM
// columns, and runs its own stream of tiles.
__host__ __device__ constexpr int fwd_act(int wg) { return kSmFwdAct + wg * kTile * kIn * 2; }
__host__ __device__ constexpr int fwd_bar(int nw) { return fwd_act(nw); }
__host__ __device__ constexpr int fwd_smem(int nw) { return fwd_bar(nw) + 64; }
__host__ __device__ constexpr uint32_t tmem_cols(int nw) { return nw <= 2 ? 128u : (nw <= 4 ? 256u : 512u); }
constexpr int kInferWG = 5;   // inference: 640 threads, 96 registers each, 149 KB of shared memory
constexpr int kTrainWG = 4;   // training forward: 512 threads at 128 registers (94.1 against 98.9 us with 3 warpgroups at 167)
static_assert(kSmFwdAct % 128 == 0 && (kTile * kIn * 2) % 128 == 0, "operand tiles 128-byte aligned");

// Backward CTAs: kBwdWG warpgroups, each with its own tile stream, a dZ tile
// and three X buffers (each 128 samples x 64 features, 128-byte rows with
// the 128-byte swizzle); then W^T of layers 1..4 (the B operand of dX, N =
// in, K = out, K-major without swizzle), a block of 16 rows whose feature 0
// is 1 (the bias rows of the weight gradients), the mbarriers and the TMEM
// address. TMEM: 64 columns of dX per warpgroup, then the five dW^T
// accumulators at kDwCol + zoff(l).
constexpr int kBwdWG = 3;
constexpr int kBwdBlk = kTile * 128;                            // 16 KB
constexpr int kBwdWGBytes = 4 * kBwdBlk;                        // dZ tile + three X buffers
__host__ __device__ constexpr int hoff1(int l) { return hoff(l) - hoff(1); }
constexpr int kBwdWt = kBwdWG * kBwdWGBytes;
constexpr int kBwdOnes = kBwdWt + 2 * hoff1(kLayers);
constexpr int kBwdBar = kBwdOnes + 16 * 128;
constexpr int kBwdBars = 5 + kLayers;                           // mbarriers per warpgroup
constexpr int kBwdSmem = kBwdBar + kBwdWG * kBwdBars * 8 + 16 + 1024;   // + 1024-byte alignment of the base
constexpr int kDwCol = kBwdWG * 64;
static_assert(kBwdOnes % 1024 == 0, "the ones block keeps the 1024-byte swizzle alignment");
static_assert(kBwdSmem <= 227 * 1024, "backward shared memory");
static_assert(kDwCol + kZCols <= 512, "backward TMEM columns");
static_assert(kHid == 64 && kIn > 64 && kIn <= 128 && kBiasCol(0) < kIn, "block plan");

// W of every layer as the forward's B operand (out x 80), with the BF16 bias
// in column kBiasCol(l) and zeros in the other columns past the inputs. Each
// thread issues 8 global loads before its 8 shared stores.
__device__ void load_weights_fwd(unsigned char* sm, const MlpView& V) {
    #pragma unroll
    for (int l = 0; l < kLayers; ++l) {
        const int I = lin(l), O = lout(l);
        const unsigned short* src = reinterpret_cast<const unsigned short*>(V.w16 + hoff(l));
        for (int e0 = threadIdx.x; e0 < O * kIn; e0 += 8 * blockDim.x) {
            unsigned short v[8];
            #pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int e = e0 + u * blockDim.x, o = e / kIn, k = e % kIn;
                v[u] = 0;
                if (e < O * kIn) {
                    if (k == kBiasCol(l)) v[u] = __bfloat16_as_ushort(__float2bfloat16_rn(V.params[boff(l) + o]));
                    else if (k < I) v[u] = src[o * I + k];
                }
            }
            #pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int e = e0 + u * blockDim.x, o = e / kIn, k = e % kIn;
                if (e < O * kIn)
                    *reinterpret_cast<unsigned short*>(sm + kSmFwdW + fwd_wtile(l) + tc::tile_offset(o, k, O)) = v[u];
            }
        }
    }
}

// W^T of layers 1..4 as the backward's B operand (8 loads in flight per thread).
__device__ void load_weights_bwd(unsigned char* sm, const MlpView& V) {
    #pragma unroll
    for (int l = 1; l < kLayers; ++l) {
        const int I = lin(l), O = lout(l);
        const unsigned short* src = reinterpret_cast<const unsigned short*>(V.w16 + hoff(l));
        for (int e0 = threadIdx.x; e0 < I * O; e0 += 8 * blockDim.x) {
            unsigned short v[8];
            #pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int e = e0 + u * blockDim.x;
                v[u] = e < I * O ? src[e] : 0;
            }
            #pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int e = e0 + u * blockDim.x, o = e / I, i = e % I;
                if (e < I * O)
                    *reinterpret_cast<unsigned short*>(sm + kBwdWt + 2 * hoff1(l) + tc::tile_offset(i, o, I)) = v[u];
            }
        }
    }
}

// Input encoding. Band k of axis a is (sin, cos)(pi 2^k x_a): sincospif gives
// band 0 with an exact argument, and each further band follows from the
// double-angle identities sin 2t = 2 sin t cos t, cos 2t = (cos t - sin t)
// (cos t + sin t). The error doubles per band, to about 1e-4 at band 11,
// well under the BF16 rounding (2^-9) the tensor cores apply to the inputs.
__device__ void encode(const MlpView& V, float3 p, float3 n, float3 wo, float* f) {
    const float x[3] = {fminf(fmaxf((p.x - V.bmin.x) * V.inv_ext.x, 0.0f), 1.0f),
                        fminf(fmaxf((p.y - V.bmin.y) * V.inv_ext.y, 0.0f), 1.0f),
                        fminf(fmaxf((p.z - V.bmin.z) * V.inv_ext.z, 0.0f), 1.0f)};
    #pragma unroll
    for (int a = 0; a < 3; ++a) {
        float s, c;
        sincospif(x[a], &s, &c);
        #pragma unroll
        for (int k = 0; k < 12; ++k) {
            f[a * 24 + k] = s;
            f[a * 24 + 12 + k] = c;
            const float s2 = 2.0f * s * c;
            c = (c - s) * (c + s);
            s = s2;
        }
    }
    f[72] = n.x; f[73] = n.y; f[74] = n.z;
    f[75] = wo.x; f[76] = wo.y; f[77] = wo.z;
    f[78] = 0.0f; f[79] = 0.0f;
}

// The head uses the fast intrinsics (__expf, __logf, rsqrtf, __fdividef):
// the mixture only has to be the one the tracer samples and evaluates (its
// pdf is computed from these same parameters), and the training gradient is
// compared with the FP64 reference at BF16-level tolerances; IEEE-exact
// exp/log/sqrt/division here cost thousands of instructions per query.
__device__ __forceinline__ float softplus(float x) { return x > 20.0f ? x : __logf(1.0f + __expf(x)); }
__device__ __forceinline__ float sigmoid(float x) {
    return __fdividef(1.0f, 1.0f + __expf(-fminf(fmaxf(x, -80.0f), 80.0f)));
}

// Raw outputs -> mixture (mu, kappa, pi).
__device__ __forceinline__ void head_mixture(const float* r, float4* lobe, float* pi) {
    float mxl = r[4];
    #pragma unroll
    for (int j = 1; j < kMaxLobes; ++j) mxl = fmaxf(mxl, r[5 * j + 4]);
    float z = 0.0f;
    #pragma unroll
    for (int j = 0; j < kMaxLobes; ++j) { pi[j] = __expf(r[5 * j + 4] - mxl); z += pi[j]; }
    const float iz = __fdividef(1.0f, z);   // z in [1, 8]
    #pragma unroll
    for (int j = 0; j < kMaxLobes; ++j) {
        pi[j] *= iz;
        const float vx = r[5 * j], vy = r[5 * j + 1], vz = r[5 * j + 2];
        const float il = rsqrtf(fmaxf(vx * vx + vy * vy + vz * vz, 1e-12f));   // 1 / max(|v|, 1e-6)
        const float kappa = fminf(softplus(r[5 * j + 3]) + 0.1f, 1000.0f);
        lobe[j] = make_float4(vx * il, vy * il, vz * il, kappa);
    }
}

// Weighted NLL of direction om under the mixture and its gradient w.r.t.
// the 48 raw outputs (scaled by scale). Returns -log p.
__device__ __forceinline__ float head_grad(const float* r, float3 om, float scale, float* g) {
    float4 lobe[kMaxLobes];
    float pi[kMaxLobes], lq[kMaxLobes];
    head_mixture(r, lobe, pi);
    float lmax = -1e30f;
    #pragma unroll
    for (int j = 0; j < kMaxLobes; ++j) {
        const float k = lobe[j].w;
        const float cosw = lobe[j].x * om.x + lobe[j].y * om.y + lobe[j].z * om.z;
        // log vMF normaliser: log k - log 2pi - log(1 - e^{-2k})   (k >= 0.1)
        const float lognorm = __logf(k) - 1.83787706641f - __logf(1.0f - __expf(-2.0f * k));
        lq[j] = __logf(fmaxf(pi[j], 1e-30f)) + lognorm + k * (cosw - 1.0f);
        lmax = fmaxf(lmax, lq[j]);
    }
    float s = 0.0f;
    #pragma unroll
    for (int j = 0; j < kMaxLobes; ++j) s += __expf(lq[j] - lmax);
    const float logp = lmax + __logf(s);
    #pragma unroll
    for (int q = 0; q < kOut; ++q) g[q] = 0.0f;
    #pragma unroll
    for (int j = 0; j < kMaxLobes; ++j) {
        const float gam = __expf(lq[j] - logp);
        const float k = lobe[j].w;
        const float cosw = lobe[j].x * om.x + lobe[j].y * om.y + lobe[j].z * om.z;
        const float vx = r[5 * j], vy = r[5 * j + 1], vz = r[5 * j + 2];
        const float il = rsqrtf(fmaxf(vx * vx + vy * vy + vz * vz, 1e-12f));
        // d(-log p)/dv = -(gam kappa / |v|) (om - (mu.om) mu)
        const float cv = -gam * k * il;
        g[5 * j + 0] = scale * cv * (om.x - cosw * lobe[j].x);
        g[5 * j + 1] = scale * cv * (om.y - cosw * lobe[j].y);
        g[5 * j + 2] = scale * cv * (om.z - cosw * lobe[j].z);
        // d(-log p)/dkappa = -gam (1/kappa - 2 e^{-2k}/(1 - e^{-2k}) + cos - 1); zero where kappa is clamped
        const float e2 = __expf(-2.0f * k);
        float dk = -gam * (__fdividef(1.0f, k) - __fdividef(2.0f * e2, 1.0f - e2) + cosw - 1.0f);
        if (r[5 * j + 3] > 999.9f) dk = 0.0f;   // softplus(x) + 0.1 > 1000
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
    __nv_bfloat16* X;             // [batch][kXCols], inputs of every layer
    __nv_bfloat16* dZ;            // [batch][kZCols], the forward writes the output layer's block
    float* loss_partial;          // per block
    // grouped inference: group g's rows are slots group_base[g] + [0, group_count[g]) of surf/mix,
    // its tiles [tile_prefix[g], tile_prefix[g + 1]), its network nets[g]
    const MlpView* nets;
    uint32_t groups;
    const uint32_t* group_base;
    const uint32_t* group_count;
    const uint32_t* tile_prefix;
};

__device__ __forceinline__ void store_row_bf16(__nv_bfloat16* dst, const float* v, int n) {
    uint4* d = reinterpret_cast<uint4*>(dst);
    #pragma unroll
    for (int k = 0; k < n; k += 8)
        d[k / 8] = make_uint4(tc::pack_bf16(v[k], v[k + 1]), tc::pack_bf16(v[k + 2], v[k + 3]),
                              tc::pack_bf16(v[k + 4], v[k + 5]), tc::pack_bf16(v[k + 6], v[k + 7]));
}

// Issues the MMA chain D = A(128 x K) * B(N x K)^T from two K-major tiles and
// commits it to bar (one thread).
__device__ __forceinline__ void mma_chain(uint32_t tmem, uint32_t a_addr, uint32_t b_addr, int K, int N,
                                          uint64_t* bar) {
    const uint32_t idesc = tc::idesc_bf16(kTile, uint32_t(N));
    for (int s = 0; s < K / 16; ++s) {
        const uint64_t ad = tc::smem_desc(a_addr + s * 2 * (kTile / 8) * 128, (kTile / 8) * 128, 128);
        const uint64_t bd = tc::smem_desc(b_addr + s * 2 * (N / 8) * 128, (N / 8) * 128, 128);
        tc::mma_bf16(tmem, ad, bd, idesc, s > 0);
    }
    tc::mma_commit(bar);
}

// Waits for the chain committed to bar: the issuing thread polls the mbarrier
// (bounded), the rest of the CTA waits at the barrier instruction, which
// takes no issue slots (128 polling threads per CTA would crowd out the other
// CTAs' epilogues on the SM).
__device__ __forceinline__ void wait_chain(uint64_t* bar, uint32_t phase, bool& ok) {
    if (threadIdx.x == 0) ok = tc::mbar_wait(bar, phase) && ok;
    __syncthreads();
    tc::fence_after_sync();
}

// Grouped (inference only, one warpgroup per CTA): the CTA takes a
// contiguous range of the groups' tiles and loads a group's weights when its
// range enters that group. Otherwise warpgroup g of CTA b takes tiles
// b * NW + g, + gridDim.x * NW, ...; the warpgroups synchronise only among
// themselves (named barrier 1 + g) inside the tile loop, so one warpgroup's
// epilogue runs while another's MMA chain is on the tensor cores.
template <bool Train, bool Grouped = false, int NW = 1>
__global__ void __launch_bounds__(kTile * NW, Grouped ? 3 : 1) mlp_forward_kernel(FwdArgs A) {
    static_assert(!(Train && Grouped), "grouped forward is inference only");
    static_assert(!Grouped || NW == 1, "grouped forward runs one warpgroup per CTA");
    static_assert(NW >= 1 && NW <= 7, "warpgroups per CTA");
    extern __shared__ __align__(1024) unsigned char sm[];
    const int wg = int(threadIdx.x) / kTile;
    const int t = int(threadIdx.x) % kTile, warp = t >> 5;
    constexpr int kBar = fwd_bar(NW);
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kBar) + wg;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kBar + 56);
    unsigned char* act = sm + fwd_act(wg);
    MlpView V = A.V;
    if constexpr (!Grouped) load_weights_fwd(sm, V);
    if (threadIdx.x < 32) tc::tmem_alloc(tslot, tmem_cols(NW));
    if (t == 0) tc::mbar_init(bar, 1);
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot + uint32_t(wg * 64);
    uint32_t count = 0, tile_first, tile_end, tile_step;
    if constexpr (Grouped) {
        const uint32_t tiles = A.tile_prefix[A.groups];
        const uint32_t per = (tiles + gridDim.x - 1) / gridDim.x;
        tile_first = blockIdx.x * per;
        tile_end = min(tiles, tile_first + per);
        tile_step = 1;
    } else {
        count = Train ? A.count : *A.count_ptr;
        tile_first = blockIdx.x * NW + wg;
        tile_end = (count + kTile - 1) / kTile;
        tile_step = gridDim.x * NW;
    }
    auto wg_sync = [&]() {
        if constexpr (NW == 1) __syncthreads();
        else asm volatile("bar.sync %0, %1;" ::"r"(1 + wg), "r"(kTile) : "memory");
    };
    const uint32_t act_addr = tc::smem_addr(act);
    const uint32_t w_addr = tc::smem_addr(sm + kSmFwdW);
    uint32_t phase = 0;
    float loss_acc = 0.0f;
    bool ok = true;
    uint32_t loaded = ~0u;
    for (uint32_t tile = tile_first; tile < tile_end; tile += tile_step) {
        uint32_t row;
        bool valid;
        if constexpr (Grouped) {
            // the tile's group: the last g with tile_prefix[g] <= tile (empty groups are skipped)
            uint32_t lo = 0, hi = A.groups - 1;
            while (lo < hi) {
                const uint32_t mid = (lo + hi + 1) >> 1;
                if (A.tile_prefix[mid] <= tile) lo = mid; else hi = mid - 1;
            }
            if (lo != loaded) {
                // the previous tile's chains have completed: the weight tiles are free
                if (!ok && t == 0) atomicExch(V.error, 1);
                ok = true;
                V = A.nets[lo];
                load_weights_fwd(sm, V);
                loaded = lo;
            }
            const uint32_t local = (tile - A.tile_prefix[lo]) * kTile + t;
            valid = local < A.group_count[lo];
            row = A.group_base[lo] + local;
        } else {
            row = tile * kTile + t;
            valid = row < count;
        }
        float3 om = f3(0, 0, 0);
        float wgt = 0.0f;
        bool active = false;
        {
            float f[kIn];
            if (valid) {
                if (Train) {
                    const uint32_t si = A.sel[row];
                    const float4 s0 = A.S.s0[si], s1 = A.S.s1[si], s2 = A.S.s2[si], s3 = A.S.s3[si];
                    encode(V, xyz(s0), xyz(s2), xyz(s3), f);
                    om = xyz(s1);
                    wgt = float(double(fminf(s0.w, float(A.wnorm[0]))) * A.wnorm[1]);
                    active = true;
                } else {
                    const float4 a = A.surf[size_t(row) * 3], b = A.surf[size_t(row) * 3 + 1],
                                 c = A.surf[size_t(row) * 3 + 2];
                    active = b.w > 0.0f;
                    encode(V, xyz(a), xyz(b), xyz(c), f);
                }
            } else {
                #pragma unroll
                for (int k = 0; k < kIn; ++k) f[k] = 0.0f;
            }
            f[kBiasCol(0)] = 1.0f;   // X_0 keeps it too (the backward's bias row of dW_0)
            #pragma unroll
            for (int k = 0; k < kIn; k += 8) tc::st_row8(act, kTile, t, k, f + k);
        }
        float out[kHid];
        #pragma unroll
        for (int l = 0; l < kLayers; ++l) {
            const int I = lin(l), O = lout(l);
            tc::fence_proxy_async();
            tc::fence_before_sync();
            wg_sync();
            if (t == 0) {
                tc::fence_after_sync();
                mma_chain(tmem, act_addr, w_addr + fwd_wtile(l), kIn, O, bar);
            }
            if constexpr (Train) {
                // X_l (this layer's input, now complete in the tile) to global
                // memory while the chain runs, by the warpgroup together: a
                // warp store covers 8 rows x 4 chunks of 16 bytes (64
                // contiguous bytes per row); chunk c of row r is at
                // c * 2048 + r * 16 in the tile, so a warp's reads touch
                // every bank once per chunk.
                constexpr int kRowBlocks = kTile / 8;
                const int chunks = l == 0 ? kIn / 8 : kHid / 8;
                const int groups = kRowBlocks * ((chunks + 3) / 4);
                const int lane = t & 31;
                for (int g = warp; g < groups; g += kTile / 32) {
                    const int r = (g % kRowBlocks) * 8 + (lane & 7);
                    const int c = (g / kRowBlocks) * 4 + (lane >> 3);
                    const uint32_t xr = tile * kTile + uint32_t(r);
                    if (c < chunks && xr < count) {
                        const uint4 v = *reinterpret_cast<const uint4*>(act + tc::tile_offset(r, c * 8, kTile));
                        *reinterpret_cast<uint4*>(A.X + size_t(xr) * kXCols + xoff(l) + c * 8) = v;
                    }
                }
            }
            if (t == 0) ok = tc::mbar_wait(bar, phase) && ok;
            wg_sync();
            tc::fence_after_sync();
            phase ^= 1u;
            (void)I;
            const uint32_t trow = tmem + (uint32_t(warp * 32) << 16);
            tc::tmem_ld32_wait(trow, out);
            if (O == 64) tc::tmem_ld32_wait(trow + 32, out + 32);
            else tc::tmem_ld16_wait(trow + 32, out + 32);
            if (l == 0) {  // the hidden layers' constant columns: 1 at kBiasCol, zeros after it
                uint4* cst = reinterpret_cast<uint4*>(act + tc::tile_offset(t, kHid, kTile));
                *cst = make_uint4(0x3F80u, 0u, 0u, 0u);
                *reinterpret_cast<uint4*>(act + tc::tile_offset(t, kHid + 8, kTile)) = make_uint4(0u, 0u, 0u, 0u);
            }
            if (l + 1 < kLayers) {
                // ReLU in the BF16 conversion, into the activation tile. The
                // chain that read the tile has completed (mbarrier), so each
                // thread may overwrite its row; the barrier before the next
                // chain orders every thread's TMEM reads before that chain's
                // writes.
                #pragma unroll
                for (int k = 0; k < O; k += 8) {
                    const uint4 q = make_uint4(tc::pack_bf16_relu(out[k], out[k + 1]),
                                               tc::pack_bf16_relu(out[k + 2], out[k + 3]),
                                               tc::pack_bf16_relu(out[k + 4], out[k + 5]),
                                               tc::pack_bf16_relu(out[k + 6], out[k + 7]));
                    *reinterpret_cast<uint4*>(act + tc::tile_offset(t, k, kTile)) = q;
                }
            }
        }
        if (valid) {
            if (Train) {
                float g[kOut];
                const float nll = head_grad(out, om, wgt * kLossScale, g);
                loss_acc += wgt * nll;
                store_row_bf16(A.dZ + size_t(row) * kZCols + zoff(kLayers - 1), g, kOut);
                (void)active;
            } else {
                float4 lobe[kMaxLobes];
                float pi[kMaxLobes];
                float4* m = A.mix + size_t(row) * (kMaxLobes + 2);
                if (active) {
                    head_mixture(out, lobe, pi);
                    #pragma unroll
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
        __shared__ float red[kTile * NW];
        red[threadIdx.x] = loss_acc;
        __syncthreads();
        if (threadIdx.x < kTile) {
            for (int g = 1; g < NW; ++g) red[threadIdx.x] += red[threadIdx.x + g * kTile];
        }
        __syncthreads();
        for (int s = kTile / 2; s > 0; s >>= 1) {
            if (int(threadIdx.x) < s) red[threadIdx.x] += red[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) A.loss_partial[blockIdx.x] = red[0];
    }
    if (!ok && t == 0 && V.error) atomicExch(V.error, 1);
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) {
        tc::fence_after_sync();
        tc::tmem_free(*tslot, tmem_cols(NW));
    }
}

struct BwdArgs {
    MlpView V;
    uint32_t count;
    float* partial;               // per CTA: kParams FP32 (weights and biases of every layer)
};

// kind::f16 instruction descriptor with both operands MN-major.
__host__ __device__ constexpr uint32_t idesc_bf16_mn(uint32_t M, uint32_t N) {
    return tc::idesc_bf16(M, N) | (1u << 15) | (1u << 16);
}

// Shared-memory descriptor with the 128-byte swizzle (layout type 2). The
// operand's 8-row groups are 1024 bytes apart (SBO); for an MN-major operand
// LBO is the distance to its next block of 64 features.
__device__ __forceinline__ uint64_t desc_sw128(uint32_t addr, uint32_t lbo) {
    return tc::smem_desc(addr, lbo, 1024) | (uint64_t(2) << 61);
}

// One 2-D tensor copy (box of 64 features x 128 samples) into shared memory,
// completing `bar` with its bytes.
__device__ __forceinline__ void tma_tile(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_addr(bar)),
                 "r"(uint32_t(kBwdBlk))
                 : "memory");
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(tc::smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(tc::smem_addr(bar))
        : "memory");
}

// Byte offset of 16-byte chunk c (features 8c .. 8c+7) of row r in a tile
// with 128-byte rows and the 128-byte swizzle.
__device__ __forceinline__ uint32_t sw_chunk(uint32_t r, uint32_t c) { return r * 128u + ((c ^ (r & 7u)) << 4); }

// Backward pass and weight gradients of one training batch. Warpgroup g of
// CTA b takes tiles b * kBwdWG + g, + gridDim.x * kBwdWG, ...; thread t of
// a warpgroup owns sample t of the tile (TMEM lane t). Per tile:
//   layer l = 4 .. 1: dX_l = dZ_l W_l into the warpgroup's TMEM columns and
//     dW_l^T += X_l^T dZ_l into the CTA's accumulator; once both have
//     completed, thread t forms dZ_{l-1} = dX_l * [X_l > 0] of its sample in
//     place of dZ_l in the dZ tile;
//   dW_0^T += X_0^T dZ_0.
// Operands in shared memory (128-byte swizzle, rows of 128 bytes): the dZ
// tile is the K-major A operand of dX (M = samples, K = out) and the
// MN-major B operand of dW (N = out, K = samples); an X tile is the MN-major
// A operand of dW (M = features, K = samples), its second block of 64
// features the ones block (row 64 of the product is db_l); X_0's two blocks
// give rows 0..127 with its constant-1 column 78 (db_0). X_l and dZ_4 come
// by tensor copies: the tile's X_4 once the previous tile's layer-1 step is
// done with buffer 0, its dZ_4, X_3, X_2 when the previous tile's last
// product has completed, X_1 and X_0 into buffers the tile has finished
// with. The CTA's dW accumulators are shared by its warpgroups;
// their products are issued in tile order (warpgroup g's k-th tile is the
// CTA's tile k * kBwdWG + g, and it waits until the product of the tile
// before it has completed), so the sums do not depend on timing.
// kTile * kBwdWG threads, one CTA per SM (its shared memory and TMEM);
// registers capped at 128 (no spills).
__global__ void __maxnreg__(128) mlp_backward_kernel(const __grid_constant__ CUtensorMap mx,
                                                     const __grid_constant__ CUtensorMap mz, BwdArgs A) {
    extern __shared__ unsigned char sm_raw[];
    unsigned char* sm = sm_raw + ((1024u - (tc::smem_addr(sm_raw) & 1023u)) & 1023u);
    const int wg = int(threadIdx.x) / kTile;
    const int t = int(threadIdx.x) % kTile, warp = t >> 5;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + kBwdBar);
    uint64_t* act_full = bars + wg * kBwdBars;   // dZ_4 copied
    uint64_t* buf_full = act_full + 1;           // X buffer 0..2 copied
    uint64_t* mma_done = act_full + 4;           // the warpgroup's products completed
    uint64_t* dw_done = act_full + 5;            // per layer: the warpgroup's dW product completed
    // the warpgroup whose dW products come just before this one's
    const int pred = (wg + kBwdWG - 1) % kBwdWG;
    uint64_t* dw_pred = bars + pred * kBwdBars + 5;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + kBwdWG * kBwdBars);
    unsigned char* act = sm + wg * kBwdWGBytes;
    unsigned char* buf[3] = {act + kBwdBlk, act + 2 * kBwdBlk, act + 3 * kBwdBlk};
    unsigned char* ones = sm + kBwdOnes;
    load_weights_bwd(sm, A.V);
    for (int e = threadIdx.x; e < 16 * 8; e += blockDim.x) {   // 16 rows x 8 chunks of 16 bytes
        const int r = e / 8, c = e % 8;
        reinterpret_cast<uint4*>(ones)[e] = make_uint4(c == (r & 7) ? 0x3F80u : 0u, 0u, 0u, 0u);
    }
    if (threadIdx.x < 32) tc::tmem_alloc(tslot, 512);
    if (threadIdx.x == 0) {
        for (int k = 0; k < kBwdWG * kBwdBars; ++k) tc::mbar_init(bars + k, 1);
    }
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t tdx = tmem + uint32_t(wg * 64) + (uint32_t(warp * 32) << 16);
    const uint32_t tiles = (A.count + kTile - 1) / kTile;
    const uint32_t act_a = tc::smem_addr(act), ones_a = tc::smem_addr(ones);
    const uint32_t buf_a[3] = {tc::smem_addr(buf[0]), tc::smem_addr(buf[1]), tc::smem_addr(buf[2])};
    const uint32_t wt_a = tc::smem_addr(sm + kBwdWt);
    auto wg_sync = [&]() { asm volatile("bar.sync %0, %1;" ::"r"(1 + wg), "r"(kTile) : "memory"); };
    uint32_t ph_act = 0, ph_buf[3] = {0, 0, 0}, ph_mma = 0;
    bool ok = true;
    const uint32_t first = blockIdx.x * kBwdWG + wg, stride = gridDim.x * kBwdWG;
    // the copies that open a tile: dZ_4, X_3, X_2 (X_4 goes ahead, as soon
    // as buffer 0 is free)
    auto open_tile = [&](uint32_t tile) {
        const int y = int(tile * kTile);
        tma_tile(act, &mz, zoff(kLayers - 1), y, act_full);
        tma_tile(buf[1], &mx, xoff(3), y, buf_full + 1);
        tma_tile(buf[2], &mx, xoff(2), y, buf_full + 2);
    };
    auto wait_buf = [&](int b) {
        ok = tc::mbar_wait(buf_full + b, ph_buf[b]) && ok;
        ph_buf[b] ^= 1u;
    };
    // the dW_l products of the warpgroup's k-th tile (the CTA's tile
    // j = k kBwdWG + wg), after the CTA's tile j - 1 ones have completed: the
    // predecessor's k-th (wg > 0) or (k-1)-th (wg = 0) completion. Each
    // barrier gets one completion per tile of its warpgroup and a waiter has
    // seen the one before, so a parity names exactly one completion.
    auto issue_dw = [&](int l, uint32_t k, uint32_t j, uint32_t a0, uint32_t lbo_fixed) {
        if (j > 0) ok = tc::mbar_wait(dw_pred + l, (wg > 0 ? k : k - 1) & 1u) && ok;
        tc::fence_after_sync();
        const uint32_t idesc = idesc_bf16_mn(kTile, uint32_t(lout(l)));
        #pragma unroll
        for (int ks = 0; ks < kTile / 16; ++ks) {
            const uint32_t a = a0 + uint32_t(ks) * 2048u;
            const uint32_t lbo = lbo_fixed ? lbo_fixed : ones_a - a;
            tc::mma_bf16(tmem + uint32_t(kDwCol + zoff(l)), desc_sw128(a, lbo),
                         desc_sw128(act_a + uint32_t(ks) * 2048u, 16u), idesc, j > 0 || ks > 0);
        }
    };
    if (t == 0 && first < tiles) {
        tma_tile(buf[0], &mx, xoff(4), int(first * kTile), buf_full + 0);
        open_tile(first);
    }
    uint32_t k = 0;
    for (uint32_t tile = first; tile < tiles; tile += stride, ++k) {
        const uint32_t j = k * kBwdWG + uint32_t(wg);
        const int y = int(tile * kTile);
        #pragma unroll
        for (int l = kLayers - 1; l >= 1; --l) {
            const int b = l == 4 ? 0 : (l == 3 ? 1 : (l == 2 ? 2 : 0));
            tc::fence_proxy_async();
            tc::fence_before_sync();
            wg_sync();
            if (t == 0) {
                tc::fence_after_sync();
                // buffers this tile has finished with take X_1 and X_0
                if (l == 3) tma_tile(buf[0], &mx, xoff(1), y, buf_full + 0);
                if (l == 2) tma_tile(buf[1], &mx, 0, y, buf_full + 1);
                if (l == 1) tma_tile(buf[2], &mx, 64, y, buf_full + 2);
                if (l == kLayers - 1) {
                    ok = tc::mbar_wait(act_full, ph_act) && ok;
                    ph_act ^= 1u;
                }
                wait_buf(b);
                tc::fence_after_sync();
                const int O = lout(l);
                const uint32_t idesc = tc::idesc_bf16(kTile, uint32_t(kHid));
                const uint32_t wt = wt_a + uint32_t(2 * hoff1(l));
                for (int s = 0; s < O / 16; ++s) {
                    const uint64_t bd = tc::smem_desc(wt + s * 2 * (kHid / 8) * 128, (kHid / 8) * 128, 128);
                    tc::mma_bf16(tmem + uint32_t(wg * 64), desc_sw128(act_a + uint32_t(s) * 32u, 16u), bd, idesc,
                                 s > 0);
                }
                issue_dw(l, k, j, buf_a[b], 0u);
                tc::mma_commit(mma_done);
                tc::mma_commit(dw_done + l);
                ok = tc::mbar_wait(mma_done, ph_mma) && ok;
            }
            ph_mma ^= 1u;
            wg_sync();
            tc::fence_after_sync();
            // dZ_{l-1} of sample t, eight features at a time, in place of dZ_l
            const unsigned char* xrow = buf[b];
            #pragma unroll
            for (int h = 0; h < 2; ++h) {
                float dx[32];
                tc::tmem_ld32_wait(tdx + uint32_t(h * 32), dx);
                #pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const uint32_t off = sw_chunk(uint32_t(t), uint32_t(h * 4 + c));
                    const uint4 xw = *reinterpret_cast<const uint4*>(xrow + off);
                    const uint32_t w[4] = {xw.x, xw.y, xw.z, xw.w};
                    uint32_t q[4];
                    #pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const float x0 = __uint_as_float(w[e] << 16), x1 = __uint_as_float(w[e] & 0xFFFF0000u);
                        const float d0 = x0 > 0.0f ? dx[c * 8 + 2 * e] : 0.0f;
                        const float d1 = x1 > 0.0f ? dx[c * 8 + 2 * e + 1] : 0.0f;
                        q[e] = tc::pack_bf16(d0, d1);
                    }
                    *reinterpret_cast<uint4*>(act + off) = make_uint4(q[0], q[1], q[2], q[3]);
                }
            }
        }
        // dW_0^T += X_0^T dZ_0 (X_0 in buffers 1 and 2)
        tc::fence_proxy_async();
        tc::fence_before_sync();
        wg_sync();
        if (t == 0) {
            tc::fence_after_sync();
            // buffer 0 (X_1) is done with: the next tile's X_4
            if (tile + stride < tiles) tma_tile(buf[0], &mx, xoff(4), int((tile + stride) * kTile), buf_full + 0);
            wait_buf(1);
            wait_buf(2);
            issue_dw(0, k, j, buf_a[1], buf_a[2] - buf_a[1]);
            tc::mma_commit(mma_done);
            tc::mma_commit(dw_done + 0);
            ok = tc::mbar_wait(mma_done, ph_mma) && ok;
            // every buffer of this warpgroup is free: the next tile's copies
            if (tile + stride < tiles) open_tile(tile + stride);
        }
        ph_mma ^= 1u;
    }
    // every product has completed (each warpgroup waited for its last one,
    // and each dW product waited for the one before it); warpgroup g writes
    // the partial gradient of layers g, g + kBwdWG
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    float* dst = A.partial + size_t(blockIdx.x) * kParams;
    const int r = t;   // TMEM lane = row of dW^T = input feature
    const uint32_t lanes = uint32_t(warp * 32) << 16;
    #pragma unroll
    for (int l = 0; l < kLayers; ++l) {
        if (l % kBwdWG != wg) continue;
        const int I = lin(l), O = lout(l), bias = kBiasCol(l);
        #pragma unroll
        for (int c = 0; c < O; c += 16) {
            float v[16];
            tc::tmem_ld16_wait(tmem + lanes + uint32_t(kDwCol + zoff(l) + c), v);
            #pragma unroll
            for (int q = 0; q < 16; ++q) {
                if (r == bias) dst[boff(l) + c + q] = v[q];
                // layer 0's column kBiasCol(0) is the bias's place in the weight tile: no weight
                if (r < I) dst[woff(l) + (c + q) * I + r] = r == bias ? 0.0f : v[q];
            }
        }
    }
    if (!ok && t == 0) atomicExch(A.V.error, 1);
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) {
        tc::fence_after_sync();
        tc::tmem_free(tmem, 512);
    }
}

// grad = sum of the CTA partials in CTA order.
__global__ void __launch_bounds__(256) mlp_reduce_kernel(const float* __restrict__ partial, uint32_t parts,
                                                         float* __restrict__ grad) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    float s = 0.0f;
    for (uint32_t c = 0; c < parts; ++c) s += partial[size_t(c) * kParams + p];
    grad[p] = s;
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

// Batch weight normalisation (clamp = 20 x mean, then 1 / sum of clamped
// weights), as two fixed-order reductions: block b sums the batch slice
// [b n / G, (b+1) n / G) in FP64, then one warp adds the G partials in a
// fixed order.
constexpr int kWnBlocks = 148;
__global__ void __launch_bounds__(256) mlp_wsum_kernel(GuideSamples S, const uint32_t* __restrict__ sel, uint32_t n,
                                                       const double* __restrict__ wnorm, bool clamped,
                                                       double* __restrict__ partial) {
    __shared__ double red[256];
    const int t = threadIdx.x;
    const uint32_t b0 = uint32_t((uint64_t(blockIdx.x) * n) / gridDim.x);
    const uint32_t b1 = uint32_t((uint64_t(blockIdx.x + 1) * n) / gridDim.x);
    const double cv = clamped ? wnorm[0] : 0.0;
    double s = 0.0;
    for (uint32_t i = b0 + t; i < b1; i += 256) {
        const double w = double(S.s0[sel[i]].w);
        s += clamped ? fmin(w, cv) : w;
    }
    red[t] = s;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if (t < k) red[t] += red[t + k];
        __syncthreads();
    }
    if (t == 0) partial[blockIdx.x] = red[0];
}

// One warp: lane l adds partials l, l + 32, ... in order, then the lanes'
// sums are combined by a fixed butterfly (the same order every run).
__global__ void __launch_bounds__(32) mlp_wfinish_kernel(const double* __restrict__ partial, uint32_t parts,
                                                         uint32_t n, bool clamped, double* __restrict__ wnorm) {
    double s = 0.0;
    for (uint32_t c = threadIdx.x; c < parts; c += 32) s += partial[c];
    #pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (threadIdx.x != 0) return;
    if (!clamped) wnorm[0] = 20.0 * (s / double(n > 0 ? n : 1));
    else wnorm[1] = s > 0.0 ? 1.0 / s : 0.0;
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
    float* loss_partial = nullptr;
    float* wpartial = nullptr;    // per backward CTA: kParams FP32
    double* wn_partial = nullptr; // per weight-norm block
    int wg_grid = 0;
    uint32_t batch_cap = 0;
    uint32_t steps = 0;
    int grid = 0;
    double last_loss = 0.0;
    float* loss_host = nullptr;
};

rr_guide::~rr_guide() {
    for (int k = 0; k < 4; ++k) cudaFree(rec[k]);
    cudaFree(resolve_first);
    cudaFree(resolve_sums);
    cudaFree(mlp_surf);
    cudaFree(mlp_mix);
    if (mlp) cudaFreeHost(mlp->loss_host);
    delete mlp;
}

MlpView rr_mlp_guide_view(rr_guide* g) {
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
    M.grid = 3 * ctx->sm_count;
    if ((st = al(reinterpret_cast<void**>(&M.loss_partial), size_t(M.grid) * 4)) != RR_OK) return st;
    M.wg_grid = ctx->sm_count;
    if ((st = al(reinterpret_cast<void**>(&M.wpartial), size_t(M.wg_grid) * kParams * 4)) != RR_OK) return st;
    if ((st = al(reinterpret_cast<void**>(&M.wn_partial), size_t(kWnBlocks) * 8)) != RR_OK) return st;
    RR_TRY_CUDA(ctx, cudaMallocHost(&M.loss_host, size_t(M.grid) * 4));
    RR_TRY_CUDA(ctx, cudaFuncSetAttribute(mlp_forward_kernel<true, false, kTrainWG>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, fwd_smem(kTrainWG)));
    RR_TRY_CUDA(ctx, cudaFuncSetAttribute(mlp_forward_kernel<false, false, kInferWG>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, fwd_smem(kInferWG)));
    RR_TRY_CUDA(ctx, cudaFuncSetAttribute(mlp_forward_kernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          kSmFwd));
    RR_TRY_CUDA(ctx, cudaFuncSetAttribute(mlp_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          kBwdSmem));
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
    A.V = rr_mlp_guide_view(g);
    A.surf = g->mlp_surf;
    A.mix = g->mlp_mix;
    A.count_ptr = count_dev;
    const uint32_t tiles = (max_count + kTile - 1) / kTile;
    const int grid = int(std::min<uint32_t>((tiles + kInferWG - 1) / kInferWG, uint32_t(ctx->sm_count)));
    mlp_forward_kernel<false, false, kInferWG><<<std::max(grid, 1), kTile * kInferWG, fwd_smem(kInferWG), stream>>>(A);
    RR_CHECK_LAUNCH(ctx);
    g->mlp_infer_launches = 1;
    return RR_OK;
}

namespace rr {
namespace {
// Per group: its first inference tile (one thread; groups are the scenes of
// one batch).
__global__ void group_tiles_kernel(const uint32_t* __restrict__ group_count, uint32_t groups,
                                   uint32_t* __restrict__ tile_prefix) {
    uint32_t acc = 0;
    for (uint32_t g = 0; g < groups; ++g) {
        tile_prefix[g] = acc;
        acc += (group_count[g] + kTile - 1) / kTile;
    }
    tile_prefix[groups] = acc;
}
} // namespace
} // namespace rr

rr_status rr_mlp_guide_infer_grouped(rr_ctx* ctx, const MlpView* nets, uint32_t groups, const float4* surf,
                                     float4* mix, const uint32_t* group_base, const uint32_t* group_count,
                                     uint32_t* tile_prefix, cudaStream_t stream) {
    if (groups == 0) return RR_OK;
    group_tiles_kernel<<<1, 1, 0, stream>>>(group_count, groups, tile_prefix);
    RR_CHECK_LAUNCH(ctx);
    FwdArgs A{};
    A.surf = surf;
    A.mix = mix;
    A.nets = nets;
    A.groups = groups;
    A.group_base = group_base;
    A.group_count = group_count;
    A.tile_prefix = tile_prefix;
    mlp_forward_kernel<false, true><<<3 * ctx->sm_count, kTile, kSmFwd, stream>>>(A);
    RR_CHECK_LAUNCH(ctx);
    return RR_OK;
}

// Runs the network on caller-provided surfaces (rr_guide_eval for MLP guides).
rr_status rr_mlp_guide_eval(rr_ctx* ctx, rr_guide* g, const float4* surf, float4* mix, const uint32_t* count_dev,
                            uint32_t count, cudaStream_t stream) {
    FwdArgs A{};
    A.V = rr_mlp_guide_view(g);
    A.surf = surf;
    A.mix = mix;
    A.count_ptr = count_dev;
    const uint32_t tiles = (count + kTile - 1) / kTile;
    const int grid = int(std::min<uint32_t>((tiles + kInferWG - 1) / kInferWG, uint32_t(ctx->sm_count)));
    mlp_forward_kernel<false, false, kInferWG><<<std::max(grid, 1), kTile * kInferWG, fwd_smem(kInferWG), stream>>>(A);
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}

// A [rows][cols] BF16 row-major array as a 2-D tensor for the backward's
// copies: box of 64 columns x 128 rows with the 128-byte swizzle; columns
// and rows past the array read as zeros.
static bool operand_map(CUtensorMap* m, const void* base, uint32_t cols, uint32_t rows) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = rr_tensor_map_encoder();
    if (!enc || (reinterpret_cast<uintptr_t>(base) & 15u) != 0 || rows == 0) return false;
    const cuuint64_t dims[2] = {cols, rows};
    const cuuint64_t strides[1] = {cuuint64_t(cols) * 2};
    const cuuint32_t box[2] = {64, kTile};
    const cuuint32_t estr[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

rr_status rr_mlp_guide_train(rr_ctx* ctx, rr_guide* g, uint32_t n, cudaStream_t stream) {
    rr_mlp_state& M = *g->mlp;
    if (n == 0) return RR_OK;
    const uint32_t B = std::min(n, M.batch_cap);
    mlp_select_kernel<<<(B + 255) / 256, 256, 0, stream>>>(M.sel, B, n, (M.steps * 7919u) % n);
    RR_CHECK_LAUNCH(ctx);
    mlp_wsum_kernel<<<kWnBlocks, 256, 0, stream>>>(g->samples, M.sel, B, M.wnorm, false, M.wn_partial);
    mlp_wfinish_kernel<<<1, 32, 0, stream>>>(M.wn_partial, kWnBlocks, B, false, M.wnorm);
    mlp_wsum_kernel<<<kWnBlocks, 256, 0, stream>>>(g->samples, M.sel, B, M.wnorm, true, M.wn_partial);
    mlp_wfinish_kernel<<<1, 32, 0, stream>>>(M.wn_partial, kWnBlocks, B, true, M.wnorm);
    RR_CHECK_LAUNCH(ctx);
    FwdArgs A{};
    A.V = rr_mlp_guide_view(g);
    A.count = B;
    A.S = g->samples;
    A.sel = M.sel;
    A.wnorm = M.wnorm;
    A.X = M.X;
    A.dZ = M.dZ;
    A.loss_partial = M.loss_partial;
    const uint32_t tiles = (B + kTile - 1) / kTile;
    const int fgrid = int(std::min<uint32_t>((tiles + kTrainWG - 1) / kTrainWG, uint32_t(ctx->sm_count)));
    RR_TRY_CUDA(ctx, cudaMemsetAsync(M.loss_partial, 0, size_t(M.grid) * 4, stream));
    mlp_forward_kernel<true, false, kTrainWG><<<fgrid, kTile * kTrainWG, fwd_smem(kTrainWG), stream>>>(A);
    RR_CHECK_LAUNCH(ctx);
    // The backward's copies are boxes of kTile rows; a batch of fewer rows
    // is mapped as kTile rows whose tail is zeroed here (the buffers hold
    // at least kTile rows), larger ones read zeros past the batch.
    const uint32_t map_rows = std::max(B, uint32_t(kTile));
    if (B < map_rows) {
        RR_TRY_CUDA(ctx, cudaMemsetAsync(M.X + size_t(B) * kXCols, 0, size_t(map_rows - B) * kXCols * 2, stream));
        RR_TRY_CUDA(ctx, cudaMemsetAsync(M.dZ + size_t(B) * kZCols, 0, size_t(map_rows - B) * kZCols * 2, stream));
    }
    CUtensorMap mx, mz;
    if (!operand_map(&mx, M.X, kXCols, map_rows) || !operand_map(&mz, M.dZ, kZCols, map_rows))
        return rr_fail(ctx, RR_ERR_CUDA, "rr_mlp_guide_train: tensor map encoding failed");
    BwdArgs Bw{};
    Bw.V = A.V;
    Bw.count = B;
    Bw.partial = M.wpartial;
    const int bgrid = int(std::min<uint32_t>((tiles + kBwdWG - 1) / kBwdWG, uint32_t(M.wg_grid)));
    mlp_backward_kernel<<<bgrid, kTile * kBwdWG, kBwdSmem, stream>>>(mx, mz, Bw);
    RR_CHECK_LAUNCH(ctx);
    mlp_reduce_kernel<<<(kParams + 255) / 256, 256, 0, stream>>>(M.wpartial, uint32_t(bgrid), M.grad);
    RR_CHECK_LAUNCH(ctx);
    M.steps += 1;
    const float bc1 = 1.0f - std::pow(0.9f, float(M.steps));
    const float bc2 = 1.0f - std::pow(0.999f, float(M.steps));
    mlp_adam_kernel<<<(kParams + 255) / 256, 256, 0, stream>>>(M.params, M.grad, M.adam_m, M.adam_v, M.w16,
                                                               g->desc.learning_rate, bc1, bc2);
    RR_CHECK_LAUNCH(ctx);
    RR_TRY_CUDA(ctx, cudaMemcpyAsync(M.loss_host, M.loss_partial, size_t(M.grid) * 4, cudaMemcpyDeviceToHost, stream));
    ctx->launches += 10;
    return RR_OK;
}

namespace rr {
namespace {
// Self-test of the bounded mbarrier wait used by the tensor-core kernels:
// a barrier that receives its one arrival completes; a barrier that nothing
// arrives on makes the wait give up after `limit` tries, and the kernel
// returns normally with the outcome recorded.
__global__ void tc_wait_selftest_kernel(uint32_t limit, int* out) {
    __shared__ __align__(8) uint64_t bars[2];
    if (threadIdx.x == 0) {
        tc::mbar_init(&bars[0], 1);
        tc::mbar_init(&bars[1], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(
                         tc::smem_addr(&bars[1]))
                     : "memory");
        out[1] = tc::mbar_wait(&bars[1], 0, limit) ? 1 : 0;
        out[0] = tc::mbar_wait(&bars[0], 0, limit) ? 1 : 0;
    }
}
} // namespace
} // namespace rr

extern "C" rr_status rr_tc_wait_selftest(rr_ctx* ctx, uint32_t limit, int* completed_out) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!completed_out || limit == 0 || limit > (1u << 22))
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_tc_wait_selftest: bad argument");
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    int* d = nullptr;
    RR_TRY_CUDA(ctx, cudaMalloc(&d, 2 * sizeof(int)));
    rr::tc_wait_selftest_kernel<<<1, 32>>>(limit, d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(completed_out, d, 2 * sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return rr_fail(ctx, RR_ERR_CUDA, "rr_tc_wait_selftest: %s", cudaGetErrorString(e));
    ctx->launches += 1;
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
